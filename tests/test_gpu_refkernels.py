"""This build against the reference's OWN CUDA BM3D kernels on the same GPU.

oracle/_ref/libref_bm3d_gpu.so is the reference's src/cuda/bm3d/kernels.cu and
src/cuda/common/{match,match_window,match_square,match_column,aggregate}.cu,
compiled unchanged for sm_100a and driven the way its per-frame driver does
(filter_center, src/cuda/common/group_driver.cpp:760-856). These tests pin
this build's outputs and match lists to reference code rather than to a
restatement:

- match lists: the same positions as the reference kernels' except at near
  ties, by the reference's own rule |a - b| <= 2e-5 max(1, |a|, |b|)
  (tests/cuda/test_cuda_match.cpp:49-51); the share of references with a
  near-tie flip is printed;
- stages and two-stage frames, up to a full 1920x1080 YUV420 frame: PSNR of
  this build's output against the reference kernels' >= 60 dB, the contract
  floor of tests/data/cuda_tolerances_v1.json (both sides sum in 2^32 fixed
  point; the remaining differences are the transforms' rounding and near-tie
  matches).

Skipped where the library was not built (it needs the reference sources).
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
def refgpu():
    import refgpu as R

    if not R.available():
        pytest.skip("oracle/_ref/libref_bm3d_gpu.so not built (make -C oracle refgpu needs the reference sources)")
    return R


@pytest.fixture(scope="module")
def ctx(refgpu, dev):
    c = refgpu.RefGpu()
    yield c
    c.close()


@pytest.fixture(scope="module")
def synth():
    return importlib.import_module("vapoursynth-nssfactory_b200.synth")


def psnr(a, b):
    a = np.concatenate([np.ravel(x) for x in a]).astype(np.float64)
    b = np.concatenate([np.ravel(x) for x in b]).astype(np.float64)
    mse = float(np.mean((a - b) ** 2))
    return float("inf") if mse == 0 else 10 * np.log10(1.0 / mse)


def grid(n, block, step):
    return (n - block + step - 1) // step + 1


def ours_match(nssb, d, w, h, block, step, rng_, group):
    n = grid(w, block, step) * grid(h, block, step)
    pos = torch.full((n, group), -1, dtype=torch.int32, device=d.device)
    dist = torch.zeros((n, group), dtype=torch.float32, device=d.device)
    cnt = torch.zeros(n, dtype=torch.int32, device=d.device)
    nssb.check(nssb.lib().nssb_match_spatial(d.data_ptr(), w, w, h, block, step, rng_, group, pos.data_ptr(),
                                             dist.data_ptr(), cnt.data_ptr(), None))
    torch.cuda.synchronize()
    return pos.cpu().numpy(), dist.cpu().numpy(), cnt.cpu().numpy()


def ref_match(refgpu, ctx, d, w, h, block, step, rng_, group):
    n = grid(w, block, step) * grid(h, block, step)
    rec = torch.zeros((n, group, 4), dtype=torch.int32, device=d.device)
    cnt = torch.zeros(n, dtype=torch.int32, device=d.device)
    ctx.match(d.data_ptr(), w, h, block, step, rng_, group, rec.data_ptr(), cnt.data_ptr())
    torch.cuda.synchronize()
    r = rec.cpu().numpy()
    pos = (r[..., 1] << 16) | r[..., 0]
    dist = r[..., 3].copy().view(np.float32)
    return pos, dist, cnt.cpu().numpy()


def compare_lists(ours, theirs):
    """Positions equal slot by slot, or the two distances at the slot are a
    near tie. Returns (references with a flip, total references)."""
    import refgpu as R

    pos_a, dist_a, cnt_a = ours
    pos_b, dist_b, cnt_b = theirs
    assert np.array_equal(cnt_a, cnt_b)
    n, g = pos_a.shape
    valid = np.arange(g)[None, :] < cnt_a[:, None]
    differ = valid & (pos_a != pos_b)
    assert np.all(R.near_tie(dist_a[differ], dist_b[differ])), "a match differs beyond a near tie"
    same = valid & (pos_a == pos_b)
    assert np.all(R.near_tie(dist_a[same], dist_b[same])), "the same match with distances beyond rounding"
    return int(np.any(differ, axis=1).sum()), n


# (block, step, group, bm_range, the reference matcher the shape takes)
MATCH_SHAPES = [
    (8, 8, 8, 9, "window/lane"),   # the default shape
    (8, 8, 16, 9, "window/lane"),
    (8, 4, 8, 9, "square"),        # block = 2 x step
    (8, 3, 16, 19, "column"),      # the "heavy" preset's basic stage
    (8, 3, 32, 19, "column"),      # and its final stage
    (8, 8, 8, 25, "tensor"),       # a window side of 51: the mma.sync matcher
    (4, 4, 16, 6, None),
    (16, 8, 8, 7, None),
]


@pytest.mark.parametrize("block,step,group,rng_,kind", MATCH_SHAPES)
def test_match_lists_vs_reference_kernels(nssb, refgpu, ctx, dev, synth, block, step, group, rng_, kind):
    w, h = 640, 360
    noisy, _ = synth.gray_frame(71 + block + step, w, h, sigma=10)
    taken = refgpu.matcher_kind(w, h, block, step, rng_, group)
    d = torch.from_numpy(noisy).to(dev)
    flips, n = compare_lists(ours_match(nssb, d, w, h, block, step, rng_, group),
                             ref_match(refgpu, ctx, d, w, h, block, step, rng_, group))
    print(f"block {block} step {step} group {group} range {rng_} (reference matcher: {taken}, expected {kind}): "
          f"{flips} of {n} references with a near-tie flip")
    assert flips <= max(2, n // 100)


def test_match_lists_1080p_luma_vs_reference_kernels(nssb, refgpu, ctx, dev, synth):
    y = synth.yuv420_clip(5, 1920, 1080, frames=1, sigma=5)[0][0]
    d = torch.from_numpy(y).to(dev)
    flips, n = compare_lists(ours_match(nssb, d, 1920, 1080, 8, 8, 9, 8),
                             ref_match(refgpu, ctx, d, 1920, 1080, 8, 8, 9, 8))
    print(f"1080p luma, defaults: {flips} of {n} references with a near-tie flip")
    assert flips <= n // 100


def stage_pair(nssb, ctx, src, ref, sigma, block, step, group, rng_):
    h, w = src.shape
    ours = torch.empty_like(src)
    theirs = torch.empty_like(src)
    rp = ref[0].data_ptr() if ref is not None else None
    nssb.check(nssb.lib().nssb_bm3d_plane_stage(src.data_ptr(), rp, ours.data_ptr(), w, w, h, sigma, block, group,
                                                step, rng_, None))
    rp2 = ref[1].data_ptr() if ref is not None else None
    ctx.stage(src.data_ptr(), rp2, theirs.data_ptr(), w, h, sigma, block=block, step=step, bm_range=rng_,
              group=group)
    torch.cuda.synchronize()
    return ours, theirs


@pytest.mark.parametrize("block,step,group,rng_", [(8, 8, 8, 9), (8, 8, 16, 9), (8, 3, 16, 19), (4, 4, 8, 6),
                                                   (16, 8, 8, 7), (8, 4, 32, 9)])
def test_two_stage_plane_vs_reference_kernels(nssb, refgpu, ctx, dev, synth, block, step, group, rng_):
    noisy, _ = synth.gray_frame(90 + group, 384, 256, sigma=10)
    sigma = 10 / 255 * 0.75
    src = torch.from_numpy(noisy).to(dev)
    b_ours, b_theirs = stage_pair(nssb, ctx, src, None, sigma, block, step, group, rng_)
    p_basic = psnr([b_ours.cpu().numpy()], [b_theirs.cpu().numpy()])
    f_ours, f_theirs = stage_pair(nssb, ctx, src, (b_ours, b_theirs), sigma, block, step, group, rng_)
    p_final = psnr([f_ours.cpu().numpy()], [f_theirs.cpu().numpy()])
    print(f"block {block} step {step} group {group} range {rng_}: basic {p_basic:.1f} dB, final {p_final:.1f} dB")
    assert p_basic >= MIN_PSNR and p_final >= MIN_PSNR


def test_c1_512_gray_vs_reference_kernels(nssb, refgpu, ctx, dev, synth):
    noisy, _ = synth.gray_frame(1, 512, 512, sigma=10)
    src = torch.from_numpy(noisy).to(dev)
    ours, theirs = stage_pair(nssb, ctx, src, None, 10 / 255 * 0.75, 8, 8, 8, 9)
    p = psnr([ours.cpu().numpy()], [theirs.cpu().numpy()])
    print(f"C1 512x512 gray, hard threshold: {p:.1f} dB")
    assert p >= MIN_PSNR


def test_c2_1080p_yuv420_two_stage_vs_reference_kernels(nssb, refgpu, ctx, dev, synth):
    """A full C2 frame (1920x1080 YUV420, sigma 5, final=1) through this
    build's per-frame drop-in against the reference kernels plane by plane."""
    frame = synth.yuv420_clip(3, 1920, 1080, frames=1, sigma=5)[0]
    planes = [torch.from_numpy(p).to(dev) for p in frame]
    node = nssb.BM3D(nssb.Clip.from_frames([tuple(planes)], nssb.YUV, 1, 1), sigma=5, final=1)
    ours = [p.cpu().numpy() for p in node.get_frame(0)]
    node.close()
    sigma = 5 / 255 * 0.75
    theirs = []
    for p in planes:
        h, w = p.shape
        basic = torch.empty_like(p)
        out = torch.empty_like(p)
        ctx.stage(p.data_ptr(), None, basic.data_ptr(), w, h, sigma)
        ctx.stage(p.data_ptr(), basic.data_ptr(), out.data_ptr(), w, h, sigma)
        torch.cuda.synchronize()
        theirs.append(out.cpu().numpy())
    p = psnr(ours, theirs)
    print(f"C2 1080p YUV420 two-stage: {p:.1f} dB against the reference kernels")
    assert p >= MIN_PSNR


@pytest.mark.parametrize("radius,group,rng_,ps_num,ps_range", [(2, 8, 9, 2, 4), (1, 16, 9, 2, 4), (2, 4, 7, 1, 4),
                                                               (1, 8, 5, 3, 3)])
def test_temporal_match_lists_vs_reference_kernels(nssb, refgpu, ctx, dev, synth, radius, group, rng_, ps_num,
                                                   ps_range):
    """Predictive temporal matching of the centre frame over 2r+1 frames of a
    panning sequence: this build's lists against the reference's own
    predictive kernels (square / window / lane, its filter_center choice)."""
    import ctypes as C

    ntemp = 2 * radius + 1
    w, h = 480, 272
    frames = [f[0] for f in synth.panning_clip(40 + radius, w, h, frames=ntemp, sigma=10.0, yuv420=False)]
    d = [torch.from_numpy(np.ascontiguousarray(f)).to(dev) for f in frames]
    step = 8
    n = grid(w, 8, step) * grid(h, 8, step)
    pos = torch.full((n, group), -1, dtype=torch.int32, device=dev)
    slot = torch.full((n, group), -1, dtype=torch.int32, device=dev)
    dist = torch.zeros((n, group), dtype=torch.float32, device=dev)
    cnt = torch.zeros(n, dtype=torch.int32, device=dev)
    ptrs = (C.c_void_p * ntemp)(*[t.data_ptr() for t in d])
    strides = (C.c_int64 * ntemp)(*([w] * ntemp))
    nssb.check(nssb.lib().nssb_match_temporal(ptrs, strides, ntemp, radius, 0, ntemp, w, h, 8, step, rng_, group,
                                              ps_num, ps_range, pos.data_ptr(), slot.data_ptr(), dist.data_ptr(),
                                              cnt.data_ptr(), None))
    rec = torch.zeros((n, group, 4), dtype=torch.int32, device=dev)
    rcnt = torch.zeros(n, dtype=torch.int32, device=dev)
    refgpu.match_temporal(ctx, [t.data_ptr() for t in d], radius, 0, ntemp, w, h, 8, step, rng_, group, ps_num,
                          ps_range, rec.data_ptr(), rcnt.data_ptr())
    torch.cuda.synchronize()
    r = rec.cpu().numpy()
    theirs_pos = (r[..., 1] << 16) | r[..., 0]
    theirs_slot = r[..., 2]
    theirs_dist = r[..., 3].copy().view(np.float32)
    ours_pos, ours_slot, ours_dist, ours_cnt = pos.cpu().numpy(), slot.cpu().numpy(), dist.cpu().numpy(), cnt.cpu().numpy()
    assert np.array_equal(ours_cnt, rcnt.cpu().numpy())
    valid = np.arange(group)[None, :] < ours_cnt[:, None]
    differ = valid & ((ours_pos != theirs_pos) | (ours_slot != theirs_slot))
    assert np.all(refgpu.near_tie(ours_dist[differ], theirs_dist[differ])), "a temporal match differs beyond a near tie"
    same = valid & ~differ
    assert np.all(refgpu.near_tie(ours_dist[same], theirs_dist[same]))
    flips = int(np.any(differ, axis=1).sum())
    print(f"temporal radius {radius} group {group} range {rng_} ps {ps_num}/{ps_range}: {flips} of {n} "
          f"references with a near-tie flip")
    assert flips <= max(2, n // 100)
