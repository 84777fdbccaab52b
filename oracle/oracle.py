"""ctypes front of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Loaded by tests/, __graft_entry__.smoke() and bench.py's CPU legs as the
checker and the timed CPU restatement. The product (the CUDA library and its
Python mirror) never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liboracle.so"


class Match(C.Structure):
    _fields_ = [("x", C.c_int32), ("y", C.c_int32), ("t", C.c_int32), ("dist", C.c_float), ("ordinal", C.c_uint32)]


class Search(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("block", "step", "group", "bm_range", "radius", "ps_num", "ps_range",
                                       "valid_t_begin", "valid_t_end")]


class Stage(C.Structure):
    _fields_ = [("sigma", C.c_float)] + [(n, C.c_int) for n in ("block", "group", "step", "bm_range", "ps_num",
                                                                "ps_range")]


def build() -> None:
    """Compile the oracle library (make in this directory)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = C.CDLL(str(LIB_PATH))
        fp = C.POINTER(C.c_float)
        L.om_ssd.restype = C.c_float
        L.om_ssd.argtypes = [fp, C.c_ssize_t, fp, C.c_ssize_t, C.c_int]
        L.om_bm3d_plane_f64.argtypes = [fp, C.c_ssize_t, fp, C.c_ssize_t, C.c_int, C.c_int, C.POINTER(Stage), C.c_int,
                                        C.POINTER(C.c_double), C.c_ssize_t]
        L.om_order_mismatch.restype = C.c_long
        L.om_order_mismatch.argtypes = [fp, C.c_ssize_t, C.c_int, C.c_int, C.POINTER(Stage), C.POINTER(C.c_long)]
        L.om_ssd_lanes8.restype = C.c_float
        L.om_ssd_lanes8.argtypes = [fp, C.c_ssize_t, fp, C.c_ssize_t]
        L.om_spatial_match.restype = C.c_int
        L.om_spatial_match.argtypes = [fp, C.c_ssize_t, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                       C.c_int, C.POINTER(Match), C.c_int]
        L.om_predictive_match.restype = C.c_int
        L.om_predictive_match.argtypes = [C.POINTER(fp), C.POINTER(C.c_ssize_t), C.c_int, C.c_int, C.c_int, C.c_int,
                                          C.c_int, C.c_int, C.POINTER(Search), C.POINTER(Match)]
        L.om_filter_group.restype = C.c_float
        L.om_filter_group.argtypes = [fp, fp, C.c_int, C.c_int, C.c_float, C.c_int]
        dp = C.POINTER(C.c_double)
        L.om_filter_group_f64.restype = C.c_double
        L.om_filter_group_f64.argtypes = [dp, dp, C.c_int, C.c_int, C.c_double, C.c_int]
        L.om_bm3d_plane.restype = C.c_int
        L.om_bm3d_plane.argtypes = [fp, C.c_ssize_t, fp, C.c_ssize_t, C.c_int, C.c_int, C.POINTER(Stage), C.c_int,
                                    fp, C.c_ssize_t, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
        L.om_bm3d_plane_window.restype = C.c_int
        L.om_bm3d_plane_window.argtypes = [fp, C.c_ssize_t, fp, C.c_ssize_t, C.c_int, C.c_int, C.POINTER(Stage),
                                           C.c_int, fp, fp, C.c_ssize_t]
        L.om_bm3d_plane_matched.restype = C.c_int
        L.om_bm3d_plane_matched.argtypes = [fp, C.c_ssize_t, fp, C.c_ssize_t, fp, C.c_ssize_t, C.c_int, C.c_int,
                                            C.POINTER(Stage), C.c_int, fp, C.c_ssize_t, C.POINTER(C.c_int32),
                                            C.POINTER(C.c_int32)]
        L.om_bm3d_plane_clip.restype = C.c_int
        L.om_bm3d_plane_clip.argtypes = [C.POINTER(fp), C.POINTER(fp), C.c_int, C.c_int, C.c_int, C.c_ssize_t,
                                         C.POINTER(Stage), C.c_int, C.c_int, C.POINTER(fp)]
        L.om_bm3d_plane_fat.restype = C.c_int
        L.om_bm3d_plane_fat.argtypes = [C.POINTER(fp), C.POINTER(fp), C.c_int, C.c_int, C.c_int, C.c_int,
                                        C.c_ssize_t, C.POINTER(Stage), C.c_int, C.c_int, fp, C.c_ssize_t]
        L.om_vaggregate.restype = None
        L.om_vaggregate.argtypes = [C.POINTER(fp), C.c_int, fp, C.c_int, C.c_int, C.c_ssize_t, C.c_ssize_t, C.c_int,
                                    C.POINTER(C.c_int), fp, C.c_ssize_t]
        L.om_bm3d_frames_mt.restype = C.c_int
        L.om_bm3d_frames_mt.argtypes = [C.POINTER(fp), C.POINTER(fp), C.POINTER(fp), C.c_int, C.c_int, C.c_int,
                                        C.c_ssize_t, C.POINTER(Stage), C.POINTER(Stage), C.c_int, C.c_int]
        L.om_noise_effective.restype = C.c_float
        L.om_noise_effective.argtypes = [C.c_float]
        L.om_haar_scale.restype = C.c_float
        L.om_haar_scale.argtypes = [C.c_int, C.c_int]
        L.om_grid_count.restype = C.c_int
        L.om_grid_count.argtypes = [C.c_int, C.c_int, C.c_int]
        _lib = L
    return _lib


def _fp(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def effective_sigma(user_sigma: float) -> float:
    return float(lib().om_noise_effective(user_sigma))


def stage(sigma_eff: float, block=8, group=8, step=None, bm_range=9, ps_num=None, ps_range=4) -> Stage:
    step = min(8, block) if step is None else step
    ps_num = min(2, group) if ps_num is None else ps_num
    return Stage(sigma_eff, block, group, step, bm_range, ps_num, ps_range)


def ssd(a: np.ndarray, b: np.ndarray, lanes8: bool = False) -> float:
    a, b = _f32(a), _f32(b)
    if lanes8:
        return float(lib().om_ssd_lanes8(_fp(a), a.shape[1], _fp(b), b.shape[1]))
    return float(lib().om_ssd(_fp(a), a.shape[1], _fp(b), b.shape[1], a.shape[0]))


def spatial_match(plane, bx, by, block=8, bm_range=9, group=8, lanes8=False):
    """[(x, y, t, dist, ordinal)] of collect_spatial_coords."""
    p = _f32(plane)
    out = (Match * 64)()
    n = lib().om_spatial_match(_fp(p), p.shape[1], p.shape[1], p.shape[0], bx, by, block, bm_range, group, out,
                               int(lanes8))
    return [(m.x, m.y, m.t, m.dist, m.ordinal) for m in out[:n]]


def predictive_match(planes, bx, by, t0, block=8, group=8, bm_range=9, radius=1, ps_num=2, ps_range=4, step=8,
                     valid=(0, -1), strides=None, width=None, height=None):
    ps = [_f32(p) for p in planes]
    arr = (C.POINTER(C.c_float) * len(ps))(*[_fp(p) for p in ps])
    st = (C.c_ssize_t * len(ps))(*(strides or [p.shape[1] for p in ps]))
    cfg = Search(block, step, group, bm_range, radius, ps_num, ps_range, valid[0], valid[1])
    out = (Match * 64)()
    w = width if width is not None else ps[0].shape[1]
    h = height if height is not None else ps[0].shape[0]
    n = lib().om_predictive_match(arr, st, len(ps), w, h, bx, by, t0, C.byref(cfg), out)
    return [(m.x, m.y, m.t, m.dist, m.ordinal) for m in out[:n]]


def filter_group(cube: np.ndarray, ref: np.ndarray | None, sigma_eff: float, wiener: bool):
    """Bm3dFilterGroup on a (group, block, block) cube (zero-padded). Returns (out, weight)."""
    c = _f32(cube).copy()
    g, b, _ = c.shape
    r = _f32(ref) if ref is not None else None
    w = lib().om_filter_group(_fp(c), _fp(r) if r is not None else None, g, b, sigma_eff, int(wiener))
    return c, float(w)


def filter_group_f64(cube: np.ndarray, ref: np.ndarray | None, sigma: float, wiener: bool):
    c = np.ascontiguousarray(cube, dtype=np.float64).copy()
    g, b, _ = c.shape
    r = np.ascontiguousarray(ref, dtype=np.float64) if ref is not None else None
    dp = C.POINTER(C.c_double)
    w = lib().om_filter_group_f64(c.ctypes.data_as(dp), r.ctypes.data_as(dp) if r is not None else None, g, b,
                                  sigma, int(wiener))
    return c, float(w)


def bm3d_plane(src, st: Stage, ref=None, want_matches=False):
    """One stage of one plane at radius 0. ref given = Wiener stage."""
    s = _f32(src)
    h, w = s.shape
    r = _f32(ref) if ref is not None else None
    dst = np.empty_like(s)
    nx = lib().om_grid_count(w, st.block, st.step)
    ny = lib().om_grid_count(h, st.block, st.step)
    matches = counts = None
    mp = cp = None
    if want_matches:
        matches = np.full((ny * nx, st.group), -1, np.int32)
        counts = np.zeros(ny * nx, np.int32)
        mp = matches.ctypes.data_as(C.POINTER(C.c_int32))
        cp = counts.ctypes.data_as(C.POINTER(C.c_int32))
    rc = lib().om_bm3d_plane(_fp(s), w, _fp(r) if r is not None else None, w, w, h, C.byref(st), int(r is not None),
                             _fp(dst), w, mp, cp)
    if rc != 0:
        raise RuntimeError("oracle plane pass failed")
    if want_matches:
        return dst, matches, counts
    return dst


def kaiser_window(block: int, beta: float) -> np.ndarray:
    """block x block Kaiser window (outer product of the 1-D window
    I0(beta sqrt(1 - (2n/(N-1) - 1)^2)) / I0(beta)), float32; ones at beta 0."""
    def i0(x):
        term, s, k = 1.0, 1.0, 1
        while term > 1e-17 * s:
            term *= (x / (2.0 * k)) ** 2
            s += term
            k += 1
        return s
    if block == 1 or beta == 0.0:
        w1 = np.ones(block)
    else:
        n = np.arange(block)
        r = 2.0 * n / (block - 1) - 1.0
        w1 = np.array([i0(beta * np.sqrt(max(0.0, 1.0 - v * v))) / i0(beta) for v in r])
    return np.outer(w1, w1).astype(np.float32)


def bm3d_plane_window(src, st: Stage, win: np.ndarray, ref=None) -> np.ndarray:
    """One radius-0 stage with the opt-in aggregation window (see the C header)."""
    s = _f32(src)
    h, w = s.shape
    r = _f32(ref) if ref is not None else None
    wn = _f32(win)
    dst = np.empty_like(s)
    rc = lib().om_bm3d_plane_window(_fp(s), w, _fp(r) if r is not None else None, w, w, h, C.byref(st),
                                    int(r is not None), _fp(wn), _fp(dst), w)
    if rc != 0:
        raise RuntimeError("oracle windowed pass failed")
    return dst


def bm3d_plane_f64(src, st: Stage, ref=None) -> np.ndarray:
    """One radius-0 stage, group filter and sums in FP64, on the FP32 matcher's
    groups (matched on ref for the Wiener stage)."""
    s = _f32(src)
    h, w = s.shape
    r = _f32(ref) if ref is not None else None
    dst = np.empty((h, w), np.float64)
    rc = lib().om_bm3d_plane_f64(_fp(s), w, _fp(r) if r is not None else None, w, w, h, C.byref(st),
                                 int(r is not None), dst.ctypes.data_as(C.POINTER(C.c_double)), w)
    if rc != 0:
        raise RuntimeError("oracle FP64 plane pass failed")
    return dst


def order_mismatch(plane, st: Stage):
    """(references whose groups differ between this build's SSD order and the
    reference's AVX2 order, references)."""
    p = _f32(plane)
    h, w = p.shape
    refs = C.c_long()
    bad = lib().om_order_mismatch(_fp(p), w, w, h, C.byref(st), C.byref(refs))
    return int(bad), int(refs.value)


def bm3d_planes_chroma(planes, stages, refs=None):
    """CBM3D: groups matched on plane 0 (of refs when given) filter every plane;
    stages: one Stage per plane (its sigma; the shape of plane 0 holds for all)."""
    ps = [_f32(p) for p in planes]
    rs = [_f32(p) for p in refs] if refs is not None else None
    h, w = ps[0].shape
    match = rs[0] if rs is not None else ps[0]
    outs = []
    for c, p in enumerate(ps):
        st = stages[c]
        dst = np.empty_like(p)
        r = rs[c] if rs is not None else None
        if st.sigma == 0.0:
            outs.append(p.copy())
            continue
        rc = lib().om_bm3d_plane_matched(_fp(p), w, _fp(r) if r is not None else None, w, _fp(match), w, w, h,
                                         C.byref(st), int(r is not None), _fp(dst), w, None, None)
        if rc != 0:
            raise RuntimeError("oracle plane pass failed")
        outs.append(dst)
    return outs


def bm3d_plane_two_stage(src, basic: Stage, final: Stage):
    b = bm3d_plane(src, basic)
    return bm3d_plane(src, final, ref=b), b


def bm3d_clip_plane(frames, st: Stage, radius: int, ref_frames=None):
    """Radius > 0 finished frames of one plane (legacy fat + VAggregate)."""
    fs = [_f32(f) for f in frames]
    h, w = fs[0].shape
    rs = [_f32(f) for f in ref_frames] if ref_frames is not None else None
    outs = [np.empty_like(f) for f in fs]
    P = C.POINTER(C.c_float)
    sp = (P * len(fs))(*[_fp(f) for f in fs])
    rp = (P * len(fs))(*[_fp(f) for f in rs]) if rs is not None else None
    op = (P * len(fs))(*[_fp(f) for f in outs])
    rc = lib().om_bm3d_plane_clip(sp, rp, len(fs), w, h, w, C.byref(st), radius, int(rs is not None), op)
    if rc != 0:
        raise RuntimeError("oracle clip pass failed")
    return outs


def bm3d_plane_fat(frames, n: int, st: Stage, radius: int, ref_frames=None):
    fs = [_f32(f) for f in frames]
    h, w = fs[0].shape
    rs = [_f32(f) for f in ref_frames] if ref_frames is not None else None
    P = C.POINTER(C.c_float)
    sp = (P * len(fs))(*[_fp(f) for f in fs])
    rp = (P * len(fs))(*[_fp(f) for f in rs]) if rs is not None else None
    out = np.zeros(((2 * radius + 1) * 2 * h, w), np.float32)
    rc = lib().om_bm3d_plane_fat(sp, rp, len(fs), n, w, h, w, C.byref(st), radius, int(rs is not None), _fp(out), w)
    if rc != 0:
        raise RuntimeError("oracle fat pass failed")
    return out


def frames_mt(frames, basic: Stage | None, final: Stage, threads: int):
    """Frame-parallel radius-0 pass over same-size planes (CPU timing)."""
    fs = [_f32(f) for f in frames]
    h, w = fs[0].shape
    outs = [np.empty_like(f) for f in fs]
    scratch = [np.empty_like(f) for f in fs] if basic is not None else outs
    P = C.POINTER(C.c_float)
    sp = (P * len(fs))(*[_fp(f) for f in fs])
    op = (P * len(fs))(*[_fp(f) for f in outs])
    bp = (P * len(fs))(*[_fp(f) for f in scratch])
    rc = lib().om_bm3d_frames_mt(sp, op, bp, len(fs), w, h, w, C.byref(basic) if basic is not None else None,
                                 C.byref(final), int(basic is not None), threads)
    if rc != 0:
        raise RuntimeError("oracle threaded pass failed")
    return outs


def psnr(a, b) -> float:
    """10*log10(1/MSE) pooled over all samples (test_cuda_bm3d_live.py:204-206)."""
    a = np.concatenate([np.asarray(x, np.float64).ravel() for x in (a if isinstance(a, (list, tuple)) else [a])])
    b = np.concatenate([np.asarray(x, np.float64).ravel() for x in (b if isinstance(b, (list, tuple)) else [b])])
    mse = float(np.mean((a - b) ** 2))
    return float("inf") if mse == 0 else 10.0 * np.log10(1.0 / mse)


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1
