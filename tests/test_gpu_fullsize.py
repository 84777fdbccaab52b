"""Full-size parity: benchmark-sized frames through the C ABI against the CPU
oracle, not crops.

- C2's shape: one 1920x1080 YUV420 frame, two-stage (final=1), sigma 5,
  radius 0, default arguments, through the per-frame drop-in;
- C3's shape: a 5-frame 1920x1080 YUV420 clip of the panning sequence,
  radius 2, two-stage, sigma 10, with the tensor-core precision matcher.

Bar: PSNR >= 60 dB against the oracle (the reference's contract floor,
tests/data/cuda_tolerances_v1.json; measured: ~92-98 dB). At these sizes a
few hard-threshold decisions at |c| = 2.7 sigma fall the other way under FP32
rounding, which moves a handful of pixels by up to ~1e-2, so the per-pixel
bound is on the share of pixels off by more than 1e-3 (< 1e-3 of them), not
on the maximum. The oracle runs plane by plane on a thread pool (its C calls
release the GIL).
"""
import importlib
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

MIN_PSNR = 60.0
OFF = 1e-3           # a pixel "off" by more than this ...
MAX_OFF_SHARE = 1e-3  # ... in at most this share of all pixels


@pytest.fixture(scope="module")
def dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


@pytest.fixture(scope="module")
def synth():
    return importlib.import_module("vapoursynth-nssfactory_b200.synth")


def oracle_clip(O, frames, sigma, radius):
    st = O.stage(O.effective_sigma(sigma))

    def plane(i):
        ps = [f[i] for f in frames]
        if radius == 0:
            return [O.bm3d_plane_two_stage(p, st, st)[0] for p in ps]
        basic = O.bm3d_clip_plane(ps, st, radius)
        return O.bm3d_clip_plane(ps, st, radius, ref_frames=basic)

    with ThreadPoolExecutor(len(frames[0])) as ex:
        per_plane = list(ex.map(plane, range(len(frames[0]))))
    return [tuple(per_plane[i][n] for i in range(len(frames[0]))) for n in range(len(frames))]


def check(O, got, want, label):
    p = O.psnr([x for f in got for x in f], [x for f in want for x in f])
    diffs = [np.abs(a.astype(np.float64) - b) for fg, fw in zip(got, want) for a, b in zip(fg, fw)]
    worst = max(float(d.max()) for d in diffs)
    off = sum(int((d > OFF).sum()) for d in diffs) / sum(d.size for d in diffs)
    print(f"{label}: {p:.1f} dB, max |diff| {worst:.2e}, share off by > {OFF:g}: {off:.2e}")
    assert p >= MIN_PSNR and off < MAX_OFF_SHARE


def test_c2_1080p_yuv420_two_stage_vs_oracle(nssb, oracle, dev, synth):
    frames = synth.yuv420_clip(1000, 1920, 1080, frames=1, sigma=5)
    d = [tuple(torch.from_numpy(p).to(dev) for p in f) for f in frames]
    node = nssb.BM3D(nssb.Clip.from_frames(d, nssb.YUV, 1, 1), sigma=5, final=1)
    got = [[p.cpu().numpy() for p in node.get_frame(0)]]
    node.close()
    check(oracle, got, oracle_clip(oracle, frames, 5.0, 0), "C2 1920x1080 YUV420 two-stage")


def test_c3_1080p_yuv420_temporal_precision_vs_oracle(nssb, oracle, dev, synth):
    frames = synth.panning_clip(3100, 1920, 1080, frames=5, sigma=10.0)
    d = [tuple(torch.from_numpy(p).to(dev) for p in f) for f in frames]
    node = nssb.BM3D(nssb.Clip.from_frames(d, nssb.YUV, 1, 1), sigma=10.0, radius=2, final=1)
    node.set_matcher(1)
    got = [[p.cpu().numpy() for p in node.get_frame(n)] for n in range(5)]
    node.close()
    check(oracle, got, oracle_clip(oracle, frames, 10.0, 2), "C3 1920x1080 YUV420 radius 2, 5 frames")
