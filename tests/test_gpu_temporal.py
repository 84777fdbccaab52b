"""GPU parity of the temporal path (radius > 0) against the CPU oracle.

- predictive matching (collect_temporal, matcher.hpp:319-373): positions,
  slots and distances identical to the oracle's;
- rolling output (finished frames) vs the oracle's legacy + VAggregate:
  >= 60 dB, in order and out of order (a request out of order restarts the
  ring and must give the same frame, bit for bit);
- legacy output (fat num/den slices of one centre) vs the oracle's;
- final=1 with radius > 0 (rolling basic stage feeding the Wiener stage);
- device-resident and host frames give the same bits.
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


def gray_clip(synth, n, w, h, sigma, seed=4):
    return [f[0] for f in synth.panning_clip(seed, w, h, frames=n, sigma=sigma, yuv420=False)]


@pytest.mark.parametrize("block,group,rng_,radius,ps_num,ps_range,valid", [
    (8, 8, 9, 2, 2, 4, (0, -1)), (8, 16, 5, 1, 3, 3, (1, -1)), (4, 8, 6, 2, 2, 2, (0, 4)),
    (8, 4, 7, 2, 1, 4, (2, 5)), (16, 8, 5, 1, 2, 2, (0, -1)), (12, 32, 4, 1, 4, 3, (0, -1)),
    # the 8x8 fast path at its limits: 8 seeds, wide windows clamped at the edges, radius 3, groups 2 and 16
    (8, 8, 9, 3, 5, 7, (0, -1)), (8, 16, 9, 2, 8, 2, (1, 4)), (8, 2, 9, 1, 1, 12, (0, -1)),
    (8, 16, 6, 2, 4, 12, (0, -1)),
])
def test_match_temporal_exact(nssb, oracle, synth, dev, block, group, rng_, radius, ps_num, ps_range, valid):
    ntemp = 2 * radius + 1
    frames = gray_clip(synth, ntemp, 72, 56, 10, seed=block + group)
    h, w = frames[0].shape
    step = max(1, block // 2)
    dframes = [torch.from_numpy(f).to(dev) for f in frames]
    nx, ny = (w - block + step - 1) // step + 1, (h - block + step - 1) // step + 1
    pos = torch.full((nx * ny, group), -7, dtype=torch.int32, device=dev)
    slot = torch.full((nx * ny, group), -7, dtype=torch.int32, device=dev)
    dist = torch.zeros((nx * ny, group), dtype=torch.float32, device=dev)
    cnt = torch.zeros(nx * ny, dtype=torch.int32, device=dev)
    ptrs = (C.c_void_p * ntemp)(*[f.data_ptr() for f in dframes])
    strides = (C.c_int64 * ntemp)(*([w] * ntemp))
    nssb.check(nssb.lib().nssb_match_temporal(ptrs, strides, ntemp, radius, valid[0], valid[1], w, h, block, step,
                                              rng_, group, ps_num, ps_range, pos.data_ptr(), slot.data_ptr(),
                                              dist.data_ptr(), cnt.data_ptr(), None))
    torch.cuda.synchronize()
    pos, slot, dist, cnt = pos.cpu().numpy(), slot.cpu().numpy(), dist.cpu().numpy(), cnt.cpu().numpy()
    for j in range(nx * ny):
        bx, by = min((j % nx) * step, w - block), min((j // nx) * step, h - block)
        want = oracle.predictive_match(frames, bx, by, radius, block=block, group=group, bm_range=rng_,
                                       radius=radius, ps_num=ps_num, ps_range=ps_range, step=step, valid=valid)
        assert cnt[j] == len(want), (j, cnt[j], len(want))
        got = [(int(p) & 0xFFFF, int(p) >> 16, int(t), float(d)) for p, t, d in zip(pos[j], slot[j], dist[j])]
        assert got[:cnt[j]] == [(m[0], m[1], m[2], m[3]) for m in want], j


def render_all(node, n, order):
    out = {}
    for i in order:
        out[i] = node.get_frame(i)[0].copy()
    return [out[i] for i in range(n)]


@pytest.mark.parametrize("radius", [1, 2])
def test_rolling_vs_oracle(nssb, oracle, synth, dev, radius):
    n = 6
    frames = gray_clip(synth, n, 64, 48, 15)
    clip = nssb.Clip.from_frames([(f,) for f in frames], nssb.GRAY)
    got = render_all(nssb.BM3D(clip, sigma=15, radius=radius), n, range(n))
    st = oracle.stage(oracle.effective_sigma(15.0))
    want = oracle.bm3d_clip_plane(frames, st, radius)
    for g, wv in zip(got, want):
        assert oracle.psnr(g, wv) >= MIN_PSNR
    shuffled = render_all(nssb.BM3D(clip, sigma=15, radius=radius), n, [3, 0, 5, 1, 4, 2])
    for a, b in zip(got, shuffled):
        assert np.array_equal(a, b)


def test_legacy_fat_vs_oracle(nssb, oracle, synth, dev):
    n, radius = 5, 1
    frames = gray_clip(synth, n, 64, 48, 15)
    clip = nssb.Clip.from_frames([(f,) for f in frames], nssb.GRAY)
    node = nssb.BM3D(clip, sigma=15, radius=radius, temporal_mode="legacy")
    assert node.vi.height == 48 * (2 * radius + 1) * 2
    st = oracle.stage(oracle.effective_sigma(15.0))
    for c in (0, 2, 4):
        got = node.get_frame(c)[0]
        want = oracle.bm3d_plane_fat(frames, c, st, radius)
        assert got.shape == want.shape
        assert np.max(np.abs(got - want)) < 2e-3 * max(1.0, float(np.max(np.abs(want))))


def test_two_stage_temporal_vs_oracle(nssb, oracle, synth, dev):
    n, radius = 5, 1
    frames = gray_clip(synth, n, 64, 48, 12)
    clip = nssb.Clip.from_frames([(f,) for f in frames], nssb.GRAY)
    got = render_all(nssb.BM3D(clip, sigma=12, radius=radius, final=1), n, range(n))
    st = oracle.stage(oracle.effective_sigma(12.0))
    basic = oracle.bm3d_clip_plane(frames, st, radius)
    want = oracle.bm3d_clip_plane(frames, st, radius, ref_frames=basic)
    for g, wv in zip(got, want):
        assert oracle.psnr(g, wv) >= MIN_PSNR


def test_temporal_yuv420_device_frames(nssb, oracle, synth, dev):
    n, radius = 4, 1
    frames = synth.panning_clip(7, 96, 64, frames=n, sigma=10)
    dframes = [tuple(torch.from_numpy(p).to(dev) for p in f) for f in frames]
    node = nssb.BM3D(nssb.Clip.from_frames(dframes, nssb.YUV, 1, 1), sigma=[10, 7, 7], radius=radius)
    hnode = nssb.BM3D(nssb.Clip.from_frames(frames, nssb.YUV, 1, 1), sigma=[10, 7, 7], radius=radius)
    host = []
    for i in range(n):
        d = [p.cpu().numpy() for p in node.get_frame(i)]
        hh = [p.copy() for p in hnode.get_frame(i)]
        host.append(hh)
        for a, b in zip(d, hh):
            assert np.array_equal(a, b)
    sts = [oracle.stage(oracle.effective_sigma(s)) for s in (10.0, 7.0, 7.0)]
    for p in range(3):
        want = oracle.bm3d_clip_plane([f[p] for f in frames], sts[p], radius)
        assert oracle.psnr([h[p] for h in host], want) >= MIN_PSNR


def test_frame_props(nssb, synth, dev):
    frames = gray_clip(synth, 3, 64, 48, 10)
    clip = nssb.Clip.from_frames([(f,) for f in frames], nssb.GRAY)
    base = {"_NSSModel": 1, "_NSSModelVersion": 3, "_NSSNoiseProfile": 1}
    assert nssb.BM3D(clip, sigma=10).frame_props(1) == base
    assert nssb.BM3D(clip, sigma=10, radius=1).frame_props(2) == base  # rolling: finished frames
    fat = nssb.BM3D(clip, sigma=10, radius=1, temporal_mode="legacy").frame_props(2)
    assert fat == {**base, "_NSSFatVersion": 2, "_NSSFatRadius": 1, "_NSSFatCenter": 2, "_NSSFatLayout": 1}


def test_temporal_planes_8192_and_wider(nssb, oracle, synth, dev):
    """Planes 8192 and more pixels wide take the generic temporal kernel
    (16-bit coordinates); its match lists equal the oracle's, refs past
    x = 8192 included, and the rolling output of a node keeps the 60 dB bar."""
    radius, block, group, rng_, ps_num, ps_range, step = 1, 8, 8, 9, 2, 4, 8
    ntemp = 2 * radius + 1
    frames = gray_clip(synth, ntemp, 8232, 24, 10, seed=17)
    h, w = frames[0].shape
    dframes = [torch.from_numpy(f).to(dev) for f in frames]
    nx, ny = (w - block + step - 1) // step + 1, (h - block + step - 1) // step + 1
    pos = torch.full((nx * ny, group), -7, dtype=torch.int32, device=dev)
    slot = torch.full((nx * ny, group), -7, dtype=torch.int32, device=dev)
    dist = torch.zeros((nx * ny, group), dtype=torch.float32, device=dev)
    cnt = torch.zeros(nx * ny, dtype=torch.int32, device=dev)
    ptrs = (C.c_void_p * ntemp)(*[f.data_ptr() for f in dframes])
    strides = (C.c_int64 * ntemp)(*([w] * ntemp))
    nssb.check(nssb.lib().nssb_match_temporal(ptrs, strides, ntemp, radius, 0, -1, w, h, block, step, rng_, group,
                                              ps_num, ps_range, pos.data_ptr(), slot.data_ptr(), dist.data_ptr(),
                                              cnt.data_ptr(), None))
    torch.cuda.synchronize()
    pos, slot, dist, cnt = pos.cpu().numpy(), slot.cpu().numpy(), dist.cpu().numpy(), cnt.cpu().numpy()
    rs = np.random.default_rng(3)
    jobs = [j for j in range(nx * ny) if min((j % nx) * step, w - block) >= 8150]
    jobs += list(rs.choice(nx * ny, 120, replace=False))
    assert any(int(p) & 0xFFFF >= 8192 for j in jobs for p in pos[j][:cnt[j]])
    for j in jobs:
        bx, by = min((j % nx) * step, w - block), min((j // nx) * step, h - block)
        want = oracle.predictive_match(frames, bx, by, radius, block=block, group=group, bm_range=rng_,
                                       radius=radius, ps_num=ps_num, ps_range=ps_range, step=step)
        assert cnt[j] == len(want), (j, cnt[j], len(want))
        got = [(int(p) & 0xFFFF, int(p) >> 16, int(t), float(d)) for p, t, d in zip(pos[j], slot[j], dist[j])]
        assert got[:cnt[j]] == [(m[0], m[1], m[2], m[3]) for m in want], j

    clip = nssb.Clip.from_frames([(f,) for f in frames], nssb.GRAY)
    node = nssb.BM3D(clip, sigma=10, radius=radius)
    got = node.get_frame(1)[0]
    node.close()
    st = oracle.stage(oracle.effective_sigma(10.0))
    want = oracle.bm3d_clip_plane(frames, st, radius)[1]
    assert oracle.psnr(got, want) >= MIN_PSNR
