"""The batched form (nssb_batch_*): many radius-0 frames of different nodes --
resolutions, formats, sigmas, one- and two-stage, ref clips, CBM3D, sigma-0
planes, non-default block shapes -- in one call.

Every output must be bit-identical to the same node's own get_frame (which
test_gpu_parity.py pins to the oracle), whatever launch shape the batch uses
(matcher column split 1/2/4, grid or persistent tile queue; 2/4/8 groups per
CTA) and whether it replays a captured graph; a small mixed batch is also
checked against the oracle directly (>= 60 dB).
"""
import importlib

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

MIN_PSNR = 60.0


@pytest.fixture(scope="module")
def dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


@pytest.fixture(scope="module")
def synth():
    return importlib.import_module("vapoursynth-nssfactory_b200.synth")


def gray_clip(nssb, synth, w, h, n, sigma, seed):
    return nssb.Clip.from_frames([(synth.gray_frame(seed + i, w, h, sigma)[0],) for i in range(n)], nssb.GRAY)


def to_device(nssb, clip, dev, family, ssw=0, ssh=0):
    frames = [tuple(torch.from_numpy(p).to(dev) for p in f) for f in clip.frames]
    return nssb.Clip.from_frames(frames, family, ssw, ssh)


@pytest.fixture(scope="module")
def nodes(nssb, synth, dev):
    out = []
    g = gray_clip(nssb, synth, 96, 64, 2, 10, 1)
    out.append(nssb.BM3D(g, sigma=10, final=1))
    y = nssb.Clip.from_frames(synth.yuv420_clip(3, 128, 72, 2, 5), nssb.YUV, 1, 1)
    out.append(nssb.BM3D(y, sigma=[5, 3, 3], final=1))
    out.append(nssb.BM3D(gray_clip(nssb, synth, 80, 48, 2, 20, 5), sigma=20))
    y444 = nssb.Clip.from_frames([tuple(synth.gray_frame(40 + 3 * i + p, 64, 48, 8)[0] for p in range(3))
                                  for i in range(2)], nssb.YUV)
    out.append(nssb.BM3D(y444, sigma=8, chroma=1, final=1))
    noisy = gray_clip(nssb, synth, 72, 56, 2, 12, 9)
    out.append(nssb.BM3D(noisy, ref=gray_clip(nssb, synth, 72, 56, 2, 4, 9), sigma=12))
    out.append(nssb.BM3D(nssb.Clip.from_frames(synth.yuv420_clip(11, 96, 64, 2, 8), nssb.YUV, 1, 1),
                         sigma=[8, 0, 0], final=1))
    out.append(nssb.BM3D(gray_clip(nssb, synth, 64, 40, 2, 15, 13), sigma=15, block_size=4, final=1))
    out.append(nssb.BM3D(gray_clip(nssb, synth, 88, 72, 2, 10, 17), sigma=10, group_size=16, final=1))
    dclip = to_device(nssb, nssb.Clip.from_frames(synth.yuv420_clip(21, 160, 96, 2, 10), nssb.YUV, 1, 1), dev,
                      nssb.YUV, 1, 1)
    out.append(nssb.BM3D(dclip, sigma=10, final=1))
    return out


def as_np(planes):
    return [p.cpu().numpy() if hasattr(p, "cpu") else np.asarray(p) for p in planes]


def expected(nodes, reqs):
    return [as_np(n.get_frame(f)) for n, f in reqs]


def assert_same(got, want):
    for g, w in zip(got, want):
        g = as_np(g)
        assert len(g) == len(w)
        for a, b in zip(g, w):
            assert a.shape == b.shape
            assert np.array_equal(a, b)


def test_mixed_batch_equals_per_frame(nssb, nodes):
    reqs = [(n, f) for f in (0, 1) for n in nodes]
    want = expected(nodes, reqs)
    b = nssb.Batch(chunk_frames=len(reqs))
    assert_same(b.run(reqs), want)
    info = b.info()
    assert info.tunings == 1 and info.graphs == 1 and info.graph_builds == 1 and info.chunks == 1
    assert info.kernel_launches > 0 and info.frames == len(reqs)
    # graph replay on the same layout, then a different layout
    assert_same(b.run(reqs), want)
    assert b.info().graph_builds == 1 and b.info().tunings == 1
    sub = reqs[::3]
    assert_same(b.run(sub), [want[i] for i in range(0, len(reqs), 3)])
    assert b.info().tunings == 2
    b.close()


@pytest.mark.parametrize("chunk", [0, 1, 4])
def test_chunked_two_stream_runs(nssb, nodes, chunk):
    # host items split into chunks on three streams (0: automatic), repeated
    reqs = [(n, f) for f in (0, 1) for n in nodes]
    want = expected(nodes, reqs)
    b = nssb.Batch(chunk_frames=chunk)
    for _ in range(2):
        assert_same(b.run(reqs), want)
    info = b.info()
    assert info.chunks == (len(reqs) + chunk - 1) // chunk if chunk else info.chunks >= 2
    b.close()


@pytest.mark.parametrize("shape", [
    dict(match_parts=1, match_persistent=0, group_warps=2, group_ctas_per_sm=32),
    dict(match_parts=2, match_persistent=1, group_warps=4, group_ctas_per_sm=8),
    dict(match_parts=4, match_persistent=1, group_warps=8, group_ctas_per_sm=16),
    dict(match_parts=4, match_persistent=0, group_warps=8, group_ctas_per_sm=1),
    dict(match_form=1, match_parts=2, match_persistent=0, group_warps=4, group_ctas_per_sm=16),
])
@pytest.mark.parametrize("graph", [False, True])
def test_launch_shapes_identical(nssb, synth, nodes, shape, graph):
    # a 1080p frame: more matcher tiles than resident CTAs, so the persistent queue cycles
    big = nssb.BM3D(nssb.Clip.from_frames(synth.yuv420_clip(31, 1920, 1080, 1, 5), nssb.YUV, 1, 1), sigma=5,
                    final=1)
    reqs = [(n, 0) for n in nodes] + [(big, 0)]
    want = expected(nodes, reqs)
    b = nssb.Batch(autotune=False, graph=graph, **shape)
    assert_same(b.run(reqs), want)
    info = b.info()
    assert (info.match_parts, info.match_persistent, info.group_warps, info.group_ctas_per_sm) == (
        shape["match_parts"], shape["match_persistent"], shape["group_warps"], shape["group_ctas_per_sm"])
    assert info.match_form == shape.get("match_form", 0)
    b.close()
    big.close()


def test_batch_vs_oracle(nssb, oracle, synth, dev):
    y = synth.yuv420_clip(5, 96, 64, 1, 10)
    g = synth.gray_frame(6, 80, 56, 20)[0]
    ny = nssb.BM3D(nssb.Clip.from_frames(y, nssb.YUV, 1, 1), sigma=10, final=1)
    ng = nssb.BM3D(nssb.Clip.from_frames([(g,)], nssb.GRAY), sigma=20)
    got = nssb.Batch().run([(ny, 0), (ng, 0)])
    s10, s20 = oracle.stage(oracle.effective_sigma(10.0)), oracle.stage(oracle.effective_sigma(20.0))
    for p in range(3):
        want = oracle.bm3d_plane_two_stage(y[0][p], s10, s10)[0]
        assert oracle.psnr(got[0][p], want) >= MIN_PSNR
    want = oracle.bm3d_plane(g, s20)
    assert oracle.psnr(got[1][0], want) >= MIN_PSNR


def test_batch_rejects(nssb, synth, dev):
    t = nssb.BM3D(gray_clip(nssb, synth, 64, 48, 3, 10, 2), sigma=10, radius=1)
    b = nssb.Batch()
    with pytest.raises(nssb.Error, match="radius-0"):
        b.run([(t, 1)])
    b.close()


def test_plan_reused_for_other_nodes_of_equal_arguments(nssb, synth, dev):
    # A batch plan laid out for one node serves any later node with the same
    # arguments; the first node may be gone by then (the serving form retires
    # requests every tick), so the plan must take every stage parameter from
    # the items of the run in hand, not from the node it was laid out for.
    frames = [(synth.gray_frame(70 + i, 96, 64, 10)[0],) for i in range(2)]
    batch = nssb.Batch()
    first = nssb.BM3D(nssb.Clip.from_frames(frames, nssb.GRAY), sigma=10, final=1)
    batch.run([(first, 0)])
    first.close()
    # other nodes (other block sizes, ranges, groups) take the memory the first one released
    others = [nssb.BM3D(nssb.Clip.from_frames(frames, nssb.GRAY), sigma=s, block_size=b, bm_range=r,
                        group_size=g) for s, b, r, g in ((3, 4, 5, 4), (20, 16, 7, 16), (7, 12, 4, 2), (9, 8, 3, 32))]
    second = nssb.BM3D(nssb.Clip.from_frames(frames, nssb.GRAY), sigma=10, final=1)
    for n in range(2):
        got = batch.run([(second, n)])[0]
        want = second.get_frame(n)
        assert all(np.array_equal(a, b) for a, b in zip(got, want))
    for o in others:
        o.close()
    second.close()
    batch.close()
