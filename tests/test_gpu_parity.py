"""GPU parity of the CUDA path against the CPU oracle (through the C ABI).

- Matching: the device groups equal the oracle's exactly (positions, order,
  counts) and the distances are bit-identical: both use one FMA chain per
  candidate in row-major order. Near-ties therefore cannot flip.
- Stages and frames: PSNR of the device output against the oracle's, with
  the reference's own contract floor of 60 dB (tests/data/cuda_tolerances_v1.json)
  and a max-abs bound; run-to-run bit identity (fixed-point sums).
"""
import ctypes as C
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


def to_dev(a, dev):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def gpu_match(nssb, plane_np, block, step, rng_, group, dev):
    h, w = plane_np.shape
    d = to_dev(plane_np, dev)
    nx = (w - block + step - 1) // step + 1
    ny = (h - block + step - 1) // step + 1
    pos = torch.full((nx * ny, group), -7, dtype=torch.int32, device=dev)
    dist = torch.zeros((nx * ny, group), dtype=torch.float32, device=dev)
    cnt = torch.zeros(nx * ny, dtype=torch.int32, device=dev)
    nssb.check(nssb.lib().nssb_match_spatial(d.data_ptr(), w, w, h, block, step, rng_, group, pos.data_ptr(),
                                             dist.data_ptr(), cnt.data_ptr(), None))
    torch.cuda.synchronize()
    return pos.cpu().numpy(), dist.cpu().numpy(), cnt.cpu().numpy()


SHAPES = [(8, 8, 8, 9), (8, 4, 16, 9), (4, 4, 8, 6), (8, 8, 32, 5), (16, 8, 16, 7), (12, 6, 8, 5),
          (2, 2, 4, 4), (1, 1, 2, 3), (32, 16, 4, 3), (8, 3, 64, 7), (8, 8, 1, 9), (4, 3, 16, 12),
          # the 8x8 fast path at its other ranges
          (8, 8, 8, 4), (8, 8, 16, 5), (8, 5, 4, 6), (8, 8, 8, 7), (8, 2, 2, 8), (8, 6, 8, 12), (8, 8, 16, 15),
          # ranges served by the kernel of the next larger built range (10-11 on 12,
          # 13-14 on 15, 17-24 on 25, 26-31 on 31)
          (8, 8, 8, 10), (8, 5, 4, 11), (8, 8, 16, 13), (8, 7, 8, 20), (8, 8, 2, 24), (8, 8, 8, 28),
          (8, 4, 16, 31),
          # large windows (bm_range 16 and up: the window spans most of the test image);
          # the 8x8 fast path covers up to 31
          (8, 8, 8, 25), (8, 4, 4, 25), (8, 8, 16, 16), (8, 6, 2, 16), (8, 4, 16, 32), (4, 3, 8, 40),
          (16, 8, 8, 64),
          # groups of 32 on the 8x8 matcher (the list split over a reference's two lanes),
          # the "heavy" preset's range 19 (its own kernel) among them
          (8, 3, 32, 19), (8, 4, 32, 9), (8, 8, 32, 25), (8, 2, 32, 12), (8, 5, 16, 19), (8, 1, 32, 6),
          # steps 1-4 on the column-reuse matcher (the last grid column clamped at W = 61
          # for steps 2-4 goes to the direct one)
          (8, 1, 8, 9), (8, 2, 16, 16), (8, 3, 8, 25), (8, 4, 8, 31), (8, 3, 4, 12), (8, 1, 16, 19),
          (8, 2, 4, 10), (8, 4, 32, 19),
          # ranges 32-64 on the 8x8 matcher, in bands of 63 x 63 candidates
          (8, 8, 8, 40), (8, 8, 16, 64), (8, 6, 32, 45), (8, 3, 8, 33)]


@pytest.mark.parametrize("block,step,group,rng_", SHAPES)
def test_match_spatial_exact(nssb, oracle, synth, dev, block, step, group, rng_):
    noisy, _ = synth.gray_frame(5, 61, 47, sigma=10)
    pos, dist, cnt = gpu_match(nssb, noisy, block=block, step=step, rng_=rng_, group=group, dev=dev)
    st = oracle.stage(oracle.effective_sigma(10.0), block=block, group=group, step=step, bm_range=rng_)
    _, want, wcnt = oracle.bm3d_plane(noisy, st, want_matches=True)
    assert np.array_equal(cnt, wcnt)
    assert np.array_equal(pos, want)
    # distances bit-identical with the oracle's SSD
    nx = (61 - block + step - 1) // step + 1
    for j in range(0, pos.shape[0], max(1, pos.shape[0] // 23)):
        bx, by = min((j % nx) * step, 61 - block), min((j // nx) * step, 47 - block)
        om = oracle.spatial_match(noisy, bx, by, block, rng_, group)
        assert [m[3] for m in om] == [float(v) for v in dist[j, :len(om)]]


@pytest.mark.parametrize("rng_,group,step", [(16, 8, 8), (25, 16, 8), (20, 8, 8), (30, 4, 8), (11, 8, 8), (19, 32, 8),
                                             (19, 16, 8), (31, 32, 8), (19, 16, 3), (19, 32, 3), (9, 8, 4),
                                             (12, 16, 2), (40, 8, 8), (64, 16, 8), (33, 32, 4)])
def test_match_large_window_whole(nssb, oracle, synth, dev, rng_, group, step):
    # windows well inside a larger plane (most references see the whole window)
    noisy, _ = synth.gray_frame(17, 256, 160, sigma=10)
    pos, dist, cnt = gpu_match(nssb, noisy, block=8, step=step, rng_=rng_, group=group, dev=dev)
    st = oracle.stage(oracle.effective_sigma(10.0), block=8, group=group, step=step, bm_range=rng_)
    _, want, wcnt = oracle.bm3d_plane(noisy, st, want_matches=True)
    assert np.array_equal(cnt, wcnt)
    assert np.array_equal(pos, want)


def test_match_exact_ties(nssb, oracle, dev):
    # piecewise-constant image: exact distance ties resolve by (y, x) (test_cuda_match.cpp:33-46)
    img = np.kron(np.array([[0.25, 0.5], [0.75, 0.25]], np.float32), np.ones((16, 20), np.float32))
    pos, _, cnt = gpu_match(nssb, img, block=8, step=4, rng_=9, group=16, dev=dev)
    st = oracle.stage(0.01, block=8, group=16, step=4, bm_range=9)
    _, want, wcnt = oracle.bm3d_plane(img, st, want_matches=True)
    assert np.array_equal(pos, want) and np.array_equal(cnt, wcnt)


def test_match_nonfinite(nssb, oracle, dev):
    rng = np.random.default_rng(1)
    img = rng.uniform(0, 1, (40, 48)).astype(np.float32)
    img[10, 11] = np.nan
    img[30, 40] = np.inf
    pos, _, cnt = gpu_match(nssb, img, block=8, step=8, rng_=9, group=8, dev=dev)
    with np.errstate(all="ignore"):
        st = oracle.stage(0.01)
        _, want, wcnt = oracle.bm3d_plane(img, st, want_matches=True)
    assert np.array_equal(cnt, wcnt)
    assert np.array_equal(pos, want)


def gpu_stage(nssb, src, ref, st, dev):
    h, w = src.shape
    s = to_dev(src, dev)
    r = to_dev(ref, dev) if ref is not None else None
    out = torch.empty_like(s)
    nssb.check(nssb.lib().nssb_bm3d_plane_stage(s.data_ptr(), r.data_ptr() if r is not None else None,
                                                out.data_ptr(), w, w, h, st.sigma, st.block, st.group, st.step,
                                                st.bm_range, None))
    torch.cuda.synchronize()
    return out.cpu().numpy()


STAGES = [(8, 8, 8, 9), (8, 4, 16, 9), (4, 4, 8, 6), (16, 8, 16, 7), (12, 6, 8, 5), (2, 2, 4, 4), (1, 1, 2, 3),
          (32, 16, 8, 3), (8, 3, 32, 7), (16, 8, 64, 5), (32, 16, 32, 4), (8, 8, 16, 25), (8, 4, 8, 32),
          (8, 8, 8, 16), (8, 3, 32, 19), (8, 8, 32, 9), (8, 3, 16, 19)]


@pytest.mark.parametrize("block,step,group,rng_", STAGES)
@pytest.mark.parametrize("wiener", [False, True])
def test_stage_vs_oracle(nssb, oracle, synth, dev, block, step, group, rng_, wiener):
    noisy, clean = synth.gray_frame(9, 96, 80, sigma=20)
    st = oracle.stage(oracle.effective_sigma(20.0), block=block, group=group, step=step, bm_range=rng_)
    ref = oracle.bm3d_plane(noisy, st) if wiener else None
    want = oracle.bm3d_plane(noisy, st, ref=ref)
    got = gpu_stage(nssb, noisy, ref, st, dev)
    p = oracle.psnr(got, want)
    assert p >= MIN_PSNR, p
    assert np.max(np.abs(got - want)) < 1e-3
    assert np.array_equal(got, gpu_stage(nssb, noisy, ref, st, dev))  # run-to-run identical


def stage_at(nssb, src, ref, dev, pitch, offset, sigma):
    """nssb_bm3d_plane_stage (8x8 blocks, groups of 8, step 8, bm_range 9) on
    planes laid out at `pitch` floats per row, `offset` floats into their
    allocation."""
    h, w = src.shape

    def place(a):
        buf = torch.zeros(offset + h * pitch, dtype=torch.float32, device=dev)
        if a is not None:
            buf[offset:].view(h, pitch)[:, :w] = to_dev(a, dev)
        return buf

    s, o = place(src), place(None)
    r = place(ref) if ref is not None else None
    ptr = lambda t: t.data_ptr() + 4 * offset
    nssb.check(nssb.lib().nssb_bm3d_plane_stage(ptr(s), ptr(r) if r is not None else None, ptr(o), pitch, w, h,
                                                sigma, 8, 8, 8, 9, None))
    torch.cuda.synchronize()
    return o[offset:].view(h, pitch)[:, :w].cpu().numpy()


@pytest.mark.parametrize("w,h", [(96, 64), (240, 136), (1920, 1080)])
def test_staged_rows_equal_plane_reads(nssb, oracle, synth, dev, w, h):
    """The group filter reads patch rows as aligned 16-byte chunks when the
    plane's rows start on 16 bytes and one float at a time otherwise (an odd
    pitch, a base 4 bytes off); the matcher and the finish take any pitch:
    the same bits for every layout, in both stages."""
    noisy, _ = synth.gray_frame(17, w, h, sigma=10)
    sigma = oracle.effective_sigma(10.0)
    basic = stage_at(nssb, noisy, None, dev, w, 0, sigma)
    for pitch, offset in ((w + 1, 0), (w, 1), (w + 4, 0)):
        assert np.array_equal(basic, stage_at(nssb, noisy, None, dev, pitch, offset, sigma)), (pitch, offset)
    final = stage_at(nssb, noisy, basic, dev, w, 0, sigma)
    for pitch, offset in ((w + 1, 0), (w, 1), (w + 4, 0)):
        assert np.array_equal(final, stage_at(nssb, noisy, basic, dev, pitch, offset, sigma)), (pitch, offset)


def test_frame_api_two_stage_yuv420(nssb, oracle, synth, dev):
    frames = synth.yuv420_clip(3, 128, 96, frames=2, sigma=5)
    clip = nssb.Clip.from_frames(frames, nssb.YUV, 1, 1)
    node = nssb.BM3D(clip, sigma=5, final=1)
    s = oracle.stage(oracle.effective_sigma(5.0))
    for n in range(2):
        got = node.get_frame(n)
        want = [oracle.bm3d_plane_two_stage(p, s, s)[0] for p in frames[n]]
        assert oracle.psnr(list(got), want) >= MIN_PSNR
    node.close()


def test_frame_api_device_resident_equals_host(nssb, synth, dev):
    frames = synth.yuv420_clip(4, 96, 64, frames=1, sigma=10)
    host = nssb.BM3D(nssb.Clip.from_frames(frames, nssb.YUV, 1, 1), sigma=10, final=1).get_frame(0)
    dframes = [tuple(to_dev(p, dev) for p in f) for f in frames]
    devout = nssb.BM3D(nssb.Clip.from_frames(dframes, nssb.YUV, 1, 1), sigma=10, final=1).get_frame(0)
    for a, b in zip(host, devout):
        assert np.array_equal(a, b.cpu().numpy())


def test_frame_api_ref_and_sigma_zero(nssb, oracle, synth, dev):
    frames = synth.yuv420_clip(6, 96, 64, frames=1, sigma=10)
    clip = nssb.Clip.from_frames(frames, nssb.YUV, 1, 1)
    basic = nssb.BM3D(clip, sigma=[10, 0, 7]).get_frame(0)
    assert np.array_equal(basic[1], frames[0][1])  # sigma 0 copies the plane
    refclip = nssb.Clip.from_frames([basic], nssb.YUV, 1, 1)
    final = nssb.BM3D(clip, ref=refclip, sigma=[10, 0, 7]).get_frame(0)
    both = nssb.BM3D(clip, sigma=[10, 0, 7], final=1).get_frame(0)
    for a, b in zip(final, both):  # final=1 is the two calls (bm3d_args.cpp:161-196)
        assert np.array_equal(a, b)
    s = oracle.stage(oracle.effective_sigma(10.0))
    want = oracle.bm3d_plane_two_stage(frames[0][0], s, s)[0]
    assert oracle.psnr(final[0], want) >= MIN_PSNR


def test_frame_api_chroma(nssb, oracle, synth, dev):
    rng = np.random.default_rng(2)
    y, _ = synth.gray_frame(8, 64, 48, sigma=10)
    u = (y * 0.3 + rng.normal(0, 0.02, y.shape)).astype(np.float32)
    v = (0.5 - y * 0.2 + rng.normal(0, 0.02, y.shape)).astype(np.float32)
    clip = nssb.Clip.from_frames([(y, u, v)], nssb.YUV, 0, 0)
    got = nssb.BM3D(clip, sigma=[10, 6, 6], chroma=1).get_frame(0)
    # plane 0 exactly as without chroma; every plane filtered with the plane-0 groups
    alone = nssb.BM3D(nssb.Clip.from_frames([(y,)], nssb.GRAY), sigma=10).get_frame(0)
    assert np.array_equal(got[0], alone[0])
    stages = [oracle.stage(oracle.effective_sigma(sg)) for sg in (10.0, 6.0, 6.0)]
    want = oracle.bm3d_planes_chroma([y, u, v], stages)
    for c in range(3):
        assert oracle.psnr(got[c], want[c]) >= MIN_PSNR
    # two-stage CBM3D: plane 0 of the basic estimate guides the Wiener stage
    both = nssb.BM3D(clip, sigma=[10, 6, 6], chroma=1, final=1).get_frame(0)
    basic = oracle.bm3d_planes_chroma([y, u, v], stages)
    want = oracle.bm3d_planes_chroma([y, u, v], stages, refs=basic)
    for c in range(3):
        assert oracle.psnr(both[c], want[c]) >= MIN_PSNR


def test_frame_api_rgb(nssb, oracle, synth, dev):
    # RGB: three full-resolution planes, each matched and filtered on its own,
    # per-plane sigma; one and two stages against the oracle
    planes = [synth.gray_frame(40 + c, 96, 72, sigma=8)[0] for c in range(3)]
    clip = nssb.Clip.from_frames([tuple(planes)], nssb.RGB)
    sig = [8.0, 5.0, 11.0]
    one = nssb.BM3D(clip, sigma=sig).get_frame(0)
    two = nssb.BM3D(clip, sigma=sig, final=1).get_frame(0)
    for c in range(3):
        st = oracle.stage(oracle.effective_sigma(sig[c]))
        assert oracle.psnr(one[c], oracle.bm3d_plane(planes[c], st)) >= MIN_PSNR
        assert oracle.psnr(two[c], oracle.bm3d_plane_two_stage(planes[c], st, st)[0]) >= MIN_PSNR


def test_stage_errors_vs_fp64(nssb, oracle, dev):
    """Each stage against an FP64 host recomputation of the same groups."""
    import importlib

    synth = importlib.import_module("vapoursynth-nssfactory_b200.synth")
    img = synth.gray_frame(33, 200, 136, 10)[0]
    h, w = img.shape
    st = oracle.stage(oracle.effective_sigma(10.0))
    src = torch.from_numpy(img).to(dev)
    basic, final = torch.empty_like(src), torch.empty_like(src)
    for dst, ref in ((basic, None), (final, basic)):
        nssb.check(nssb.lib().nssb_bm3d_plane_stage(src.data_ptr(), ref.data_ptr() if ref is not None else None,
                                                    dst.data_ptr(), w, w, h, st.sigma, 8, 8, 8, 9, None))
    torch.cuda.synchronize()
    b, f = basic.cpu().numpy(), final.cpu().numpy()
    for got, want in ((b, oracle.bm3d_plane_f64(img, st)), (f, oracle.bm3d_plane_f64(img, st, ref=b))):
        d = got.astype(np.float64) - want
        assert np.abs(d).max() < 1e-4 and np.sqrt(np.mean(d * d)) < 1e-5


def test_memory_limit_fits_or_fails_at_creation(nssb, dev):
    """memory_limit_mb is a creation error when the plan does not fit, and never changes the output."""
    import importlib

    synth = importlib.import_module("vapoursynth-nssfactory_b200.synth")
    frames = [(synth.gray_frame(40 + i, 256, 160, 10)[0],) for i in range(3)]
    clip = nssb.Clip.from_frames(frames, nssb.GRAY)
    with pytest.raises(nssb.Error, match=r"nss_cuda.BM3D: memory_limit_mb is too small for this clip: each of the 1 "
                                         r"stream\(s\) needs at least \d+ MiB"):
        nssb.BM3D(clip, sigma=10, radius=1, final=1, memory_limit_mb=1)
    a = nssb.BM3D(clip, sigma=10, final=1)
    b = nssb.BM3D(clip, sigma=10, final=1, memory_limit_mb=4096)
    for n in range(3):
        assert np.array_equal(a.get_frame(n)[0], b.get_frame(n)[0])


def test_c1_config_512_gray_hard_threshold(nssb, oracle, dev):
    """The CPU-runnable benchmark case: one Gray 512x512 frame, sigma 10, final=0, radius 0, defaults."""
    import importlib

    synth = importlib.import_module("vapoursynth-nssfactory_b200.synth")
    noisy, clean = synth.gray_frame(2024, 512, 512, 10)
    node = nssb.BM3D(nssb.Clip.from_frames([(noisy,)], nssb.GRAY), sigma=10)
    got = node.get_frame(0)[0]
    st = oracle.stage(oracle.effective_sigma(10.0))
    want = oracle.bm3d_plane(noisy, st)
    assert oracle.psnr(got, want) >= 60.0
    assert oracle.psnr(got, clean) > oracle.psnr(noisy, clean)  # it denoises
