"""Precision form of the 8x8 matcher (tensor-core distances + exact re-rank):
its lists must equal the FP32 matcher's bit for bit -- positions, distances
and counts -- on textured, noisy, flat (all ties) and non-finite images, at
every step and group size it covers, and its re-rank margin must hold
(largest |approximate - exact| / margin below 1)."""
import ctypes as C
import importlib

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
def synth():
    return importlib.import_module("vapoursynth-nssfactory_b200.synth")


def grid(n, b, s):
    return (n - b + s - 1) // s + 1


def run_both(nssb, img, dev, step=8, group=8, bm_range=9):
    h, w = img.shape
    plane = torch.from_numpy(np.ascontiguousarray(img, np.float32)).to(dev)
    jobs = grid(w, 8, step) * grid(h, 8, step)
    out = []
    stats = nssb.TcStats()
    for tc in (False, True):
        pos = torch.full((jobs, group), -7, dtype=torch.int32, device=dev)
        dist = torch.full((jobs, group), -7.0, dtype=torch.float32, device=dev)
        cnt = torch.zeros(jobs, dtype=torch.int32, device=dev)
        if tc:
            rc = nssb.lib().nssb_match_spatial_tc(plane.data_ptr(), w, w, h, step, bm_range, group, pos.data_ptr(),
                                                  dist.data_ptr(), cnt.data_ptr(), C.byref(stats), None)
        else:
            rc = nssb.lib().nssb_match_spatial(plane.data_ptr(), w, w, h, 8, step, bm_range, group, pos.data_ptr(),
                                               dist.data_ptr(), cnt.data_ptr(), None)
        nssb.check(rc)
        torch.cuda.synchronize()
        out.append((pos.cpu().numpy(), dist.cpu().numpy(), cnt.cpu().numpy()))
    return out, stats


def assert_equal_lists(out):
    (p0, d0, c0), (p1, d1, c1) = out
    assert np.array_equal(c0, c1)
    assert np.array_equal(p0, p1)
    assert np.array_equal(d0.view(np.uint32), d1.view(np.uint32))


def test_small_plane_first(nssb, synth, dev):
    img = synth.gray_frame(3, 64, 48, 10)[0]
    out, st = run_both(nssb, img, dev)
    assert st.timeouts == 0
    assert_equal_lists(out)
    assert st.refs == 8 * 6 and 0 <= st.max_error_ratio < 1.0


@pytest.mark.parametrize("w,h,step,group,sigma", [
    (160, 96, 8, 8, 10), (200, 120, 4, 8, 5), (131, 77, 8, 16, 20), (96, 64, 3, 4, 10), (256, 40, 8, 2, 3),
    (150, 90, 1, 8, 10), (513, 61, 7, 16, 5),
])
def test_equals_fp32_matcher(nssb, synth, dev, w, h, step, group, sigma):
    img = synth.gray_frame(w * 7 + h, w, h, sigma)[0]
    out, st = run_both(nssb, img, dev, step, group)
    assert st.timeouts == 0 and st.flagged_tiles == 0
    assert_equal_lists(out)
    assert st.max_error_ratio < 1.0
    assert st.survivors < 40 * st.refs  # the re-rank stays a small share of the window


def test_flat_image_all_ties(nssb, dev):
    img = np.full((72, 88), 0.25, np.float32)
    out, st = run_both(nssb, img, dev)
    assert_equal_lists(out)


def test_quantised_image_many_ties(nssb, dev):
    rng = np.random.default_rng(5)
    img = (rng.integers(0, 4, (80, 120)) / 4.0).astype(np.float32)
    out, st = run_both(nssb, img, dev, group=16)
    assert_equal_lists(out)


def test_non_finite_pixels_take_the_exact_path(nssb, synth, dev):
    img = synth.gray_frame(11, 96, 64, 10)[0]
    img[10, 20] = np.nan
    img[40, 70] = np.inf
    out, st = run_both(nssb, img, dev)
    assert st.flagged_tiles > 0
    assert_equal_lists(out)


def test_large_values(nssb, synth, dev):
    img = synth.gray_frame(12, 120, 80, 10)[0] * 1000.0 + 500.0
    out, st = run_both(nssb, img, dev)
    assert_equal_lists(out)
    assert st.max_error_ratio < 1.0


def test_1080p_plane(nssb, synth, dev):
    img = synth.yuv420_clip(9, 1920, 1080, 1, 5.0)[0][0]
    out, st = run_both(nssb, img, dev)
    assert_equal_lists(out)
    assert st.max_error_ratio < 1.0


def test_engine_precision_form_same_frames(nssb, synth, dev):
    # spatial two-stage YUV420 and temporal (radius 1 and 2): the precision form gives the same bits
    frames = synth.panning_clip(21, 160, 96, frames=5, sigma=10)
    clip = nssb.Clip.from_frames(frames, nssb.YUV, 1, 1)
    for kw in (dict(sigma=10, final=1), dict(sigma=10, radius=1, final=1), dict(sigma=[10, 6, 6], radius=2)):
        a, b = nssb.BM3D(clip, **kw), nssb.BM3D(clip, **kw)
        b.set_matcher(1)
        for n in range(5):
            for pa, pb in zip(a.get_frame(n), b.get_frame(n)):
                assert np.array_equal(pa, pb)
        st = b.stats(False, False)
        assert st.tc_refs > 0 and st.tc_max_error_ratio < 1.0
        a.close()
        b.close()


# bm_range 10-64: the references on the MMA's M side (match_tcw.cu)
@pytest.mark.parametrize("w,h,step,rng_,group,sigma", [
    (160, 96, 3, 19, 16, 10), (160, 96, 3, 19, 32, 10), (200, 120, 8, 25, 8, 5), (131, 77, 4, 16, 4, 20),
    (300, 90, 8, 31, 8, 10), (96, 200, 2, 12, 2, 10), (257, 130, 5, 40, 32, 5), (150, 90, 1, 10, 16, 10),
    (400, 150, 8, 64, 8, 10), (88, 72, 6, 20, 32, 3),
])
def test_large_window_equals_fp32_matcher(nssb, synth, dev, w, h, step, rng_, group, sigma):
    img = synth.gray_frame(w * 5 + h + rng_, w, h, sigma)[0]
    out, st = run_both(nssb, img, dev, step, group, rng_)
    print(f"{w}x{h} step {step} range {rng_} group {group}: {st.survivors / max(1, st.refs):.1f} survivors "
          f"per reference, max error/margin {st.max_error_ratio:.4f}")
    assert st.timeouts == 0 and st.flagged_tiles == 0
    assert_equal_lists(out)
    assert st.refs == grid(w, 8, step) * grid(h, 8, step)
    assert st.max_error_ratio < 1.0


@pytest.mark.parametrize("rng_,group", [(19, 16), (25, 32)])
def test_large_window_ties_and_non_finite(nssb, synth, dev, rng_, group):
    flat = np.full((72, 136), 0.25, np.float32)
    out, _ = run_both(nssb, flat, dev, 3, group, rng_)
    assert_equal_lists(out)
    rng = np.random.default_rng(rng_)
    quant = (rng.integers(0, 4, (90, 150)) / 4.0).astype(np.float32)
    out, _ = run_both(nssb, quant, dev, 4, group, rng_)
    assert_equal_lists(out)
    img = synth.gray_frame(13, 140, 100, 10)[0]
    img[10, 20] = np.nan
    img[60, 120] = np.inf
    out, st = run_both(nssb, img, dev, 3, group, rng_)
    assert st.flagged_tiles > 0
    assert_equal_lists(out)


def test_heavy_preset_1080p_plane(nssb, synth, dev):
    # the "heavy" preset's matching shapes (block_step 3, bm_range 19, groups 16 and 32) on a 1080p luma plane
    img = synth.yuv420_clip(9, 1920, 1080, 1, 5.0)[0][0]
    for group in (16, 32):
        out, st = run_both(nssb, img, dev, 3, group, 19)
        assert_equal_lists(out)
        assert st.max_error_ratio < 1.0 and st.timeouts == 0


def test_automatic_matcher_form(nssb, synth, dev):
    # the default form takes the precision form from bm_range 32 on at block steps 1-7 and
    # from 63 on at step 8, the FP32 matcher otherwise; the output is the FP32 form's bit
    # for bit either way
    frames = synth.yuv420_clip(31, 256, 144, 1, 10.0)
    clip = nssb.Clip.from_frames(frames, nssb.YUV, 1, 1)
    for rng_, step, tensor in ((40, 8, False), (64, 8, True), (40, 4, True), (16, 4, False)):
        auto, fp32 = (nssb.BM3D(clip, sigma=10, final=1, bm_range=rng_, block_step=step) for _ in range(2))
        fp32.set_matcher(0)
        auto.stats(True, True)
        a, b = auto.get_frame(0), fp32.get_frame(0)
        assert all(np.array_equal(x, y) for x, y in zip(a, b))
        st = auto.stats(False, False)
        assert (st.tc_refs > 0) == tensor
        auto.close()
        fp32.close()
    # temporal: the centre frame's spatial matching takes the same choice
    tclip = nssb.Clip.from_frames(synth.panning_clip(32, 160, 96, frames=3, sigma=10), nssb.YUV, 1, 1)
    auto, fp32 = (nssb.BM3D(tclip, sigma=10, radius=1, final=1, bm_range=64) for _ in range(2))
    fp32.set_matcher(0)
    auto.stats(True, True)
    for n in range(3):
        assert all(np.array_equal(x, y) for x, y in zip(auto.get_frame(n), fp32.get_frame(n)))
    assert auto.stats(False, False).tc_refs > 0
    auto.close()
    fp32.close()


@pytest.mark.parametrize("w,h", [(8, 8), (9, 40), (40, 9), (300, 8), (13, 200), (71, 67)])
@pytest.mark.parametrize("step,rng_,group", [(1, 32, 2), (8, 64, 32), (3, 40, 16)])
def test_large_window_small_and_thin_planes(nssb, synth, dev, w, h, step, rng_, group):
    rs = np.random.default_rng(w * 1000 + h + rng_)
    img = (rs.random((h, w)) * 0.8 + 0.1).astype(np.float32)
    out, st = run_both(nssb, img, dev, step, group, rng_)
    assert st.timeouts == 0
    assert_equal_lists(out)
    assert st.refs == grid(w, 8, step) * grid(h, 8, step)


def test_uncovered_shapes_are_rejected(nssb, dev):
    # the precision entry point covers 8x8 blocks at bm_range 9 (groups 2-16) and 10-64 (groups 2-32)
    w, h = 64, 48
    plane = torch.zeros((h, w), dtype=torch.float32, device=dev)
    pos = torch.empty((grid(w, 8, 8) * grid(h, 8, 8), 32), dtype=torch.int32, device=dev)
    cnt = torch.empty(grid(w, 8, 8) * grid(h, 8, 8), dtype=torch.int32, device=dev)
    for rng_, group in ((65, 8), (9, 32), (40, 3), (5, 8)):
        rc = nssb.lib().nssb_match_spatial_tc(plane.data_ptr(), w, w, h, 8, rng_, group, pos.data_ptr(), None,
                                              cnt.data_ptr(), None, None)
        assert rc != 0
        with pytest.raises(nssb.Error, match="precision matcher covers"):
            nssb.check(rc)


def test_automatic_form_in_cbm3d_batch_and_served(nssb, synth, dev):
    # bm_range 40 takes the tensor form by default in every path that matches:
    # CBM3D (plane 0's groups serve all planes), the batched form and the
    # serving form -- each output equal to the FP32 form's bit for bit
    rng = np.random.default_rng(9)
    y = synth.gray_frame(51, 136, 96, 10)[0]
    u = (y * 0.3 + rng.normal(0, 0.02, y.shape)).astype(np.float32)
    v = (0.5 - y * 0.2 + rng.normal(0, 0.02, y.shape)).astype(np.float32)
    c444 = nssb.Clip.from_frames([(y, u, v)], nssb.YUV, 0, 0)
    auto = nssb.BM3D(c444, sigma=[10, 6, 6], chroma=1, final=1, bm_range=40)
    fp32 = nssb.BM3D(c444, sigma=[10, 6, 6], chroma=1, final=1, bm_range=40)
    fp32.set_matcher(0)
    want = fp32.get_frame(0)
    assert all(np.array_equal(a, b) for a, b in zip(auto.get_frame(0), want))
    # the batched form (its autotuner may pick either matcher form) equals the node
    frames = synth.yuv420_clip(52, 160, 96, 2, 10.0)
    node = nssb.BM3D(nssb.Clip.from_frames(frames, nssb.YUV, 1, 1), sigma=10, final=1, bm_range=40)
    batch = nssb.Batch()
    got = batch.run([(node, 0), (node, 1), (auto, 0)])
    assert all(np.array_equal(a, b) for a, b in zip(got[0], node.get_frame(0)))
    assert all(np.array_equal(a, b) for a, b in zip(got[1], node.get_frame(1)))
    assert all(np.array_equal(a, b) for a, b in zip(got[2], want))
    batch.close()
    # a served request
    srv = nssb.Server(device_id=0, workers=2)
    clip = nssb.Clip.from_frames(frames, nssb.YUV, 1, 1)
    outs = [tuple(np.empty_like(p) for p in f) for f in frames]
    srv.wait(srv.submit(clip, outs=outs, sigma=10, final=1, bm_range=40))
    srv.close()
    for n in range(2):
        assert all(np.array_equal(a, b) for a, b in zip(outs[n], node.get_frame(n)))
    for x in (auto, fp32, node):
        x.close()
