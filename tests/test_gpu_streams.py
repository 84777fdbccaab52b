"""num_streams: radius-0 frames lease one of num_streams slots (a stream and a
set of frame buffers each), so frames requested from several host threads
overlap -- one frame's host copies with another frame's kernels -- as the
reference's slot pool does (src/cuda/runtime/stream_pool.hpp:62-140,
src/cuda/runtime/context.hpp:17-23). The output must not depend on it.
"""
import importlib
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


@pytest.fixture(scope="module")
def clip_frames():
    synth = importlib.import_module("vapoursynth-nssfactory_b200.synth")
    return synth.yuv420_clip(77, 320, 240, frames=8, sigma=8)


def render(nssb, frames, threads, **kw):
    node = nssb.BM3D(nssb.Clip.from_frames(frames, nssb.YUV, 1, 1), sigma=8, final=1, **kw)
    try:
        with ThreadPoolExecutor(threads) as ex:
            return list(ex.map(lambda n: [p.clone() if hasattr(p, "clone") else np.array(p, copy=True)
                                          for p in node.get_frame(n)], range(len(frames))))
    finally:
        node.close()


@pytest.mark.parametrize("streams", [1, 2, 3, 4])
def test_output_does_not_depend_on_num_streams(nssb, dev, clip_frames, streams):
    want = render(nssb, clip_frames, 1)
    got = render(nssb, clip_frames, 4, num_streams=streams)
    for a, b in zip(want, got):
        assert all(np.array_equal(x, y) for x, y in zip(a, b))


def test_device_frames_from_threads(nssb, dev, clip_frames):
    d = [tuple(torch.from_numpy(p).to(dev) for p in f) for f in clip_frames]
    want = [[p.cpu().numpy() for p in f] for f in render(nssb, d, 1)]
    got = [[p.cpu().numpy() for p in f] for f in render(nssb, d, 4, num_streams=3)]
    for a, b in zip(want, got):
        assert all(np.array_equal(x, y) for x, y in zip(a, b))


def test_memory_limit_counts_every_stream(nssb, dev, clip_frames):
    vi_clip = nssb.Clip.from_frames(clip_frames, nssb.YUV, 1, 1)
    with pytest.raises(nssb.Error, match=r"each of the 4 stream\(s\) needs at least"):
        nssb.BM3D(vi_clip, sigma=8, final=1, num_streams=4, memory_limit_mb=1)
