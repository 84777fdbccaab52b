"""Pins of the CPU oracle against the reference's own known answers.

Each test restates a check of the reference's test suite for the BM3D path:
tests/test_bm3d_contract.cpp (FP64 transform oracle, threshold neighbours,
cross-frame SSDs, motion tracking, aggregation identity) and
tests/test_matcher.cpp (tie order, short windows, non-finite distances),
plus the exact agreement of the oracle's matching with the reference's own
header-only matcher (src/cpu/bm/matcher.hpp) when oracle/_ref is built.
"""
import ctypes as C
import math
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


# ---- independent FP64 transforms (test_bm3d_contract.cpp:19-60) ----

def dct_matrix(n):
    k = np.arange(n)[:, None]
    x = np.arange(n)[None, :]
    m = np.sqrt(np.where(k == 0, 1.0, 2.0) / n) * np.cos(np.pi * (x + 0.5) * k / n)
    return m


def haar_matrix(n):
    h = np.array([[1.0]])
    m = 1
    s = 1 / math.sqrt(2)
    while m < n:
        nxt = np.zeros((2 * m, 2 * m))
        for r in range(m):
            for c in range(m):
                nxt[r, 2 * c] = nxt[r, 2 * c + 1] = h[r, c] * s
        for r in range(m):
            nxt[m + r, 2 * r] = s
            nxt[m + r, 2 * r + 1] = -s
        h = nxt
        m *= 2
    return h


def transform(v, b, g, inverse):
    D = dct_matrix(b)
    H = haar_matrix(g)
    v = v.reshape(g, b, b)
    if not inverse:
        v = np.einsum("ki,gri->grk", D, v)  # rows
        v = np.einsum("ki,gic->gkc", D, v)  # columns
        v = np.einsum("hg,gij->hij", H, v)
    else:
        v = np.einsum("hg,hij->gij", H, v)
        v = np.einsum("ki,grk->gri", D, v)
        v = np.einsum("ki,gkc->gic", D, v)
    return v.reshape(-1)


def fp64_oracle(v, ref, b, g, sigma, wiener):
    v = transform(v.astype(np.float64), b, g, False)
    weight = 0.0
    if wiener:
        r = transform(ref.astype(np.float64), b, g, False)
        den = r * r + sigma * sigma
        w = np.where(den > 0, r * r / np.where(den > 0, den, 1), 0.0)
        w[0] = 1.0
        v = v * w
        weight = float(np.sum(w * w))
    else:
        keep = np.abs(v) >= 2.7 * sigma
        keep[0] = True
        v = np.where(keep, v, 0.0)
        weight = float(np.sum(keep))
    return transform(v, b, g, True), 1 / max(weight, 1e-12)


@pytest.mark.parametrize("b", [1, 2, 4, 8, 12, 16, 32])
@pytest.mark.parametrize("g", [1, 2, 4, 8, 16, 32, 64])
@pytest.mark.parametrize("wiener", [False, True])
def test_group_filter_vs_fp64(oracle, b, g, wiener):
    # test_bm3d_contract.cpp:61-71: k = min(g, 3) real patches, sigma 0.015, tolerances as there
    rng = np.random.default_rng(42 + b * 100 + g)
    k, area, sigma = min(g, 3), b * b, 0.015
    cube = np.zeros((g, b, b), np.float32)
    ref = np.zeros((g, b, b), np.float32)
    cube[:k] = rng.uniform(-0.2, 0.8, (k, b, b))
    ref[:k] = rng.uniform(-0.2, 0.8, (k, b, b))
    want, wweight = fp64_oracle(cube.reshape(-1), ref.reshape(-1), b, g, sigma, wiener)
    got, weight = oracle.filter_group(cube, ref if wiener else None, sigma, wiener)
    assert abs(weight - wweight) <= 1e-5
    want = want.reshape(g, b, b)[:k]
    tol = np.minimum(3e-5, 2e-5 + 2e-4 * np.abs(want))
    assert np.all(np.abs(got[:k] - want) <= tol)
    # the FP64 recomputation the per-stage error reports use agrees with the independent one
    got64, w64 = oracle.filter_group_f64(cube, ref if wiener else None, sigma, wiener)
    assert abs(w64 - wweight) <= 1e-9 * max(1.0, wweight)
    assert np.max(np.abs(got64[:k] - want)) < 1e-9


def test_threshold_neighbors(oracle):
    # test_bm3d_contract.cpp:140-161
    sigma = oracle.effective_sigma(3.0)
    thr = np.float32(2.7) * np.float32(sigma)
    basis = np.array([(1.0 if g < 4 else -1.0) / math.sqrt(8) / 8 for g in range(8) for _ in range(64)])
    for coef in (thr * np.float32(0.99), np.nextafter(thr, np.float32(0)), thr,
                 np.nextafter(thr, np.float32(np.inf)), thr * np.float32(1.01)):
        coef = float(coef)
        inp = (0.25 + coef * basis).astype(np.float32)
        out, weight = oracle.filter_group(inp.reshape(8, 8, 8), None, sigma, False)
        rec = float(np.sum((out.reshape(-1).astype(np.float64) - 0.25) * basis))
        retained = abs(rec - coef) < 2e-5
        removed = abs(rec) < 2e-5
        assert retained or removed
        if coef < thr - 2e-5:
            assert removed
        if coef > thr + 2e-5:
            assert retained
        assert abs(weight - (0.5 if retained else 1.0)) <= 1e-6
        assert np.max(np.abs(out.reshape(-1) - (0.25 + (coef * basis if retained else 0)))) <= 2e-5


def test_cross_frame_ssd(oracle):
    # test_bm3d_contract.cpp:96-103: frames of 1, 0, 2 with strides 8, 9, 10
    a = np.ones((8, 8), np.float32)
    b = np.zeros((8, 9), np.float32)
    c = np.full((8, 10), 2.0, np.float32)
    kw = dict(block=8, group=8, radius=1, bm_range=0, ps_range=0, ps_num=2, width=8, height=8)
    out = oracle.predictive_match([a, b, c], 0, 0, 1, **kw)
    assert len(out) == 3
    for x, y, t, d, _ in out:
        assert d == {0: 64.0, 1: 0.0, 2: 256.0}[t]
    out = oracle.predictive_match([a, b, c], 0, 0, 1, valid=(1, -1), **kw)
    assert len(out) == 2


def test_directional_motion(oracle):
    # test_bm3d_contract.cpp:112-117
    w, h = 40, 24
    frames = []
    for t in range(5):
        shift = (t - 2) * 2
        yy, xx = np.mgrid[0:h, 0:w]
        frames.append(np.sin((xx - shift) * 0.91 + yy * 0.73).astype(np.float32))
    out = oracle.predictive_match(frames, 16, 8, 2, block=4, radius=2, bm_range=2, ps_range=2, ps_num=2, group=16)
    seen = set()
    found = [False] * 5
    for x, y, t, d, _ in out:
        assert (t, y, x) not in seen
        seen.add((t, y, x))
        e = frames[2][8:12, 16:20].astype(np.float64) - frames[t][y:y + 4, x:x + 4]
        assert abs(d - float(np.sum(e * e))) <= 1e-4
        if y == 8 and x == 16 + (t - 2) * 2:
            found[t] = True
    assert all(found)


def scalar_spatial(frame, bx, by, block, rng_, group):
    """test_matcher.cpp:53-82: every distance, stable sort by (finite, dist, y, x)."""
    h, w = frame.shape
    cx, cy = min(max(bx, 0), w - block), min(max(by, 0), h - block)
    allm = []
    ordinal = 1
    for y in range(max(0, cy - rng_), min(h - block, cy + rng_) + 1):
        for x in range(max(0, cx - rng_), min(w - block, cx + rng_) + 1):
            if not (x == cx and y == cy):
                d = 0.0
                acc = np.float32(0)
                for i in range(block):
                    for j in range(block):
                        t = np.float32(frame[cy + i, cx + j]) - np.float32(frame[y + i, x + j])
                        acc = np.float32(acc + np.float32(t * t))
                d = float(acc)
                allm.append((x, y, d, ordinal))
            ordinal += 1
    allm.sort(key=lambda m: (not math.isfinite(m[2]), m[2] if math.isfinite(m[2]) else 0.0, m[1], m[0], m[3]))
    allm = allm[: group - 1]
    return [(cx, cy, 0.0, 0)] + allm


def close_distance(a, b):
    if not (math.isfinite(a) and math.isfinite(b)):
        return (math.isnan(a) and math.isnan(b)) or a == b or (not math.isfinite(a) and not math.isfinite(b))
    return abs(a - b) <= 8e-6 * max(1.0, abs(a), abs(b))


def test_matcher_random_vs_scalar(oracle):
    # test_matcher.cpp main: random frame 23x19, every block/group/position
    rng = np.random.default_rng(7)
    frame = rng.uniform(-1, 1, (19, 23)).astype(np.float32)
    for block in (1, 2, 4, 8, 12, 16):
        for group in (1, 2, 4, 8, 16, 32, 64):
            for bx, by in ((0, 0), (3, 5), (11, 7), (22, 18), (-4, 30)):
                if block > 19:
                    continue
                got = oracle.spatial_match(frame, bx, by, block, 7, group)
                want = scalar_spatial(frame, bx, by, block, 7, group)
                assert len(got) == len(want)
                for g_, w_ in zip(got, want):
                    assert (g_[0], g_[1]) == (w_[0], w_[1]) or close_distance(g_[3], w_[2])
                    assert close_distance(g_[3], w_[2])


def test_constant_ties(oracle):
    # test_matcher.cpp:136-160
    frame = np.full((20, 24), 0.5, np.float32)
    got = oracle.spatial_match(frame, 10, 9, 8, 7, 8)
    want = scalar_spatial(frame, 10, 9, 8, 7, 8)
    assert len(got) == 8
    assert [(g[0], g[1]) for g in got] == [(w[0], w[1]) for w in want]


def test_short_window(oracle):
    # test_matcher.cpp:162-177
    frame = np.full((8, 8), 0.25, np.float32)
    got = oracle.spatial_match(frame, 0, 0, 8, 64, 8)
    assert len(got) == 1 and got[0][:2] == (0, 0) and got[0][3] == 0.0


@pytest.mark.parametrize("case", [
    (24, 24, 8, 8, 8, 0, 0, float("nan"), -1, -1, 0.0),
    (24, 24, 8, 8, 8, 15, 15, float("inf"), -1, -1, 0.0),
    (16, 8, 0, 0, 64, 14, 0, float("nan"), -1, -1, 0.0),
    (15, 8, 0, 0, 64, 13, 0, math.sqrt(np.finfo(np.float32).max), 14, 0, math.ldexp(1.0, 52)),
])
def test_nonfinite(oracle, case):
    # test_matcher.cpp:280-330
    w, h, bx, by, rng_, x1, y1, v1, x2, y2, v2 = case
    frame = np.zeros((h, w), np.float32)
    frame[y1, x1] = v1
    if x2 >= 0:
        frame[y2, x2] = v2
    with np.errstate(all="ignore"):
        got = oracle.spatial_match(frame, bx, by, 8, rng_, 8)
        want = scalar_spatial(frame, bx, by, 8, rng_, 8)
    assert len(got) == len(want)
    for g_, w_ in zip(got, want):
        assert (g_[0], g_[1], g_[4]) == (w_[0], w_[1], w_[3])
        assert close_distance(g_[3], w_[2])


def test_vaggregate_identity(oracle):
    # test_bm3d_contract.cpp:118-123: a single unit-weight contribution is exact
    vals = np.full((1, 64), 0.05, np.float32)
    fat = np.concatenate([vals, np.ones((1, 64), np.float32)], 0)
    src = np.full((1, 64), 0.7, np.float32)
    P = C.POINTER(C.c_float)
    dst = np.empty((1, 64), np.float32)
    fats = (P * 1)(oracle._fp(fat))
    sl = (C.c_int * 1)(0)
    oracle.lib().om_vaggregate(fats, 1, oracle._fp(src), 64, 1, 64, 64, 0, sl, oracle._fp(dst), 64)
    assert np.array_equal(dst, vals)


@pytest.mark.parametrize("count", [1, 2, 3, 9, 33])
def test_vaggregate_slices(oracle, count):
    # test_bm3d_contract.cpp:124-130: contributions summed, den 0 falls back to src
    w, h = 19, 3
    P = C.POINTER(C.c_float)
    fats, keep = [], []
    for c in range(count):
        num = np.fromfunction(lambda y, x: (c + 1) * (x + y), (h, w)).astype(np.float32)
        den = np.fromfunction(lambda y, x: np.where(x > 0, c + 1, 0), (h, w)).astype(np.float32)
        fat = np.ascontiguousarray(np.concatenate([num, den], 0))
        keep.append(fat)
    src = np.full((h, w), 0.27, np.float32)
    dst = np.empty((h, w), np.float32)
    arr = (P * count)(*[oracle._fp(f) for f in keep])
    sl = (C.c_int * count)(*([0] * count))
    oracle.lib().om_vaggregate(arr, count, oracle._fp(src), w, h, w, w, 0, sl, oracle._fp(dst), w)
    expect = np.fromfunction(lambda y, x: np.where(x > 0, x + y, np.float32(0.27)), (h, w))
    tol = 2 * np.finfo(np.float32).eps * np.maximum(1.0, np.abs(expect))
    assert np.all(np.abs(dst - expect) <= tol)


def test_plane_pass_matches_filter_group(oracle):
    """One reference's group filtered through the plane pass equals filter_group on its patches."""
    rng = np.random.default_rng(3)
    img = rng.uniform(0, 1, (24, 24)).astype(np.float32)
    st = oracle.stage(oracle.effective_sigma(10.0))
    out, matches, counts = oracle.bm3d_plane(img, st, want_matches=True)
    assert out.shape == img.shape and np.all(np.isfinite(out))
    assert counts.min() == 8
    first = [(int(p) & 0xFFFF, int(p) >> 16) for p in matches[0]]
    assert first[0] == (0, 0)


ref_lib = ROOT / "oracle" / "_ref" / "libref_matcher.so"


@pytest.mark.skipif(not ref_lib.exists(), reason="reference matcher not built (needs the reference tree)")
def test_oracle_selection_equals_reference_header(oracle):
    R = C.CDLL(str(ref_lib))
    P = C.POINTER(C.c_float)
    R.ref_spatial_match.argtypes = [P, C.c_ssize_t, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                    C.POINTER(oracle.Match)]
    R.ref_predictive_match.argtypes = [C.POINTER(P), C.POINTER(C.c_ssize_t), C.c_int, C.c_int, C.c_int, C.c_int,
                                       C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(oracle.Match)]
    rng = np.random.default_rng(11)
    for trial in range(150):
        h, w = (int(v) for v in rng.integers(8, 36, 2))
        b = int(rng.choice([1, 2, 4, 8, 12, 16]))
        if b > min(h, w):
            continue
        quant = trial % 2 == 1
        img = (rng.integers(0, 4, (h, w)) * 0.25).astype(np.float32) if quant else rng.random((h, w), np.float32)
        g = int(rng.choice([1, 2, 4, 8, 16, 32, 64]))
        r = int(rng.integers(0, 12))
        bx, by = int(rng.integers(-3, w)), int(rng.integers(-3, h))
        a = oracle.spatial_match(img, bx, by, b, r, g)
        out = (oracle.Match * 64)()
        n = R.ref_spatial_match(oracle._fp(img), w, w, h, bx, by, b, r, g, out)
        assert a == [(m.x, m.y, m.t, m.dist, m.ordinal) for m in out[:n]]
        T = int(rng.integers(1, 6))
        frames = [rng.random((h, w), np.float32) if not quant else (rng.integers(0, 3, (h, w)) * 0.5).astype(np.float32)
                  for _ in range(T)]
        t0 = int(rng.integers(0, T))
        rad, psn, psr = int(rng.integers(0, 3)), min(int(rng.integers(1, 4)), g), int(rng.integers(0, 5))
        vb = int(rng.integers(0, t0 + 1))
        ve = -1 if rng.random() < 0.5 else int(rng.integers(t0 + 1, T + 1))
        a = oracle.predictive_match(frames, bx, by, t0, block=b, group=g, bm_range=r, radius=rad, ps_num=psn,
                                    ps_range=psr, valid=(vb, ve))
        arr = (P * T)(*[oracle._fp(f) for f in frames])
        st = (C.c_ssize_t * T)(*([w] * T))
        cfg = (C.c_int * 9)(b, 8, g, r, rad, psn, psr, vb, ve)
        n = R.ref_predictive_match(arr, st, T, w, h, bx, by, t0, cfg, out)
        assert a == [(m.x, m.y, m.t, m.dist, m.ordinal) for m in out[:n]]


def test_fp64_stage_agrees_with_fp32_oracle(oracle):
    import importlib

    synth = importlib.import_module("vapoursynth-nssfactory_b200.synth")
    img = synth.gray_frame(31, 96, 72, 10)[0]
    st = oracle.stage(oracle.effective_sigma(10.0))
    ht = oracle.bm3d_plane(img, st)
    ht64 = oracle.bm3d_plane_f64(img, st)
    assert oracle.psnr(ht, ht64.astype(np.float32)) >= 110.0
    wi = oracle.bm3d_plane(img, st, ref=ht)
    wi64 = oracle.bm3d_plane_f64(img, st, ref=ht)
    assert oracle.psnr(wi, wi64.astype(np.float32)) >= 110.0


def test_order_mismatch_rate_is_small(oracle):
    import importlib

    synth = importlib.import_module("vapoursynth-nssfactory_b200.synth")
    img = synth.gray_frame(32, 160, 120, 5)[0]
    bad, refs = oracle.order_mismatch(img, oracle.stage(oracle.effective_sigma(5.0)))
    assert refs == 20 * 15 and bad / refs < 0.05
    flat = np.full((64, 64), 0.5, np.float32)  # exact ties everywhere: both orders sum zeros
    assert oracle.order_mismatch(flat, oracle.stage(oracle.effective_sigma(5.0)))[0] == 0
