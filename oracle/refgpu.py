"""ctypes front of the reference's own CUDA BM3D kernels -- TEST INFRASTRUCTURE ONLY.

``_ref/libref_bm3d_gpu.so`` is compiled (``make -C oracle refgpu``) from the
reference's unchanged sources -- src/cuda/bm3d/kernels.cu and
src/cuda/common/{match,match_window,match_square,match_column,aggregate}.cu --
for sm_100a, with ``ref_gpu_driver.cu`` driving them the way the reference's
per-frame driver does (filter_center, src/cuda/common/group_driver.cpp:760-856).
The tests use it to pin this build's outputs and match lists to reference code
on the same GPU; bench.py times it beside this build's kernels. The product
never imports this module. Planes are dense float32 (pitch = width).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_ref" / "libref_bm3d_gpu.so"

# DeviceMatch {int x, int y, int t, float dist} (src/cuda/common/match.hpp:21-26)
MATCH_DTYPE = np.dtype([("x", np.int32), ("y", np.int32), ("t", np.int32), ("dist", np.float32)])

_lib = None


def available() -> bool:
    return LIB_PATH.exists()


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise FileNotFoundError(f"{LIB_PATH} is not built (make -C oracle refgpu, needs the reference sources)")
        L = C.CDLL(str(LIB_PATH))
        vp = C.c_void_p
        L.refgpu_last_error.restype = C.c_char_p
        L.refgpu_create.argtypes = [C.POINTER(vp)]
        L.refgpu_destroy.argtypes = [vp]
        L.refgpu_match.argtypes = [vp, vp] + [C.c_int] * 6 + [vp, vp, vp]
        L.refgpu_stage.argtypes = [vp, vp, vp, vp] + [C.c_int] * 6 + [C.c_float, vp]
        L.refgpu_matcher_kind.argtypes = [C.c_int] * 6
        L.refgpu_match_temporal.argtypes = [vp, C.POINTER(vp)] + [C.c_int] * 12 + [vp, vp, vp]
        _lib = L
    return _lib


def _check(rc: int) -> None:
    if rc != 0:
        raise RuntimeError("reference CUDA kernels: " + lib().refgpu_last_error().decode())


class RefGpu:
    """One context of the reference kernels' scratch (matches, sums, finish rows)."""

    def __init__(self):
        h = C.c_void_p()
        _check(lib().refgpu_create(C.byref(h)))
        self._h = h

    def close(self):
        if self._h:
            lib().refgpu_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def stage(self, src_ptr: int, ref_ptr: int | None, dst_ptr: int, width: int, height: int, sigma_eff: float,
              block=8, step=None, bm_range=9, group=8, stream: int | None = None) -> None:
        """One radius-0 stage of one dense plane (device pointers): ref None is
        the hard-threshold stage, else the Wiener stage against ref."""
        step = min(8, block) if step is None else step
        _check(lib().refgpu_stage(self._h, src_ptr, ref_ptr, dst_ptr, width, height, block, step, bm_range, group,
                                  C.c_float(sigma_eff), stream))

    def match(self, plane_ptr: int, width: int, height: int, block=8, step=None, bm_range=9, group=8,
              matches_ptr: int = 0, counts_ptr: int = 0, stream: int | None = None) -> None:
        """Matching only: grid-count x group DeviceMatch records and the counts."""
        step = min(8, block) if step is None else step
        _check(lib().refgpu_match(self._h, plane_ptr, width, height, block, step, bm_range, group, matches_ptr,
                                  counts_ptr, stream))


def match_temporal(ctx: "RefGpu", plane_ptrs, t0: int, valid_begin: int, valid_end: int, width: int, height: int,
                   block=8, step=8, bm_range=9, group=8, ps_num=2, ps_range=4, matches_ptr: int = 0,
                   counts_ptr: int = 0, stream: int | None = None) -> None:
    """The reference's predictive matching of the centre slot t0 over the
    frames (device pointers of dense planes): DeviceMatch records and counts."""
    arr = (C.c_void_p * len(plane_ptrs))(*plane_ptrs)
    _check(lib().refgpu_match_temporal(ctx._h, arr, len(plane_ptrs), t0, valid_begin, valid_end, width, height,
                                       block, step, bm_range, group, ps_num, ps_range, matches_ptr, counts_ptr,
                                       stream))


def matcher_kind(width, height, block=8, step=8, bm_range=9, group=8) -> str:
    """The reference matcher filter_center takes for this plane."""
    k = lib().refgpu_matcher_kind(width, height, block, step, bm_range, group)
    return {0: "window/lane", 1: "column", 2: "square", 3: "tensor"}[k]


def near_tie(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """The reference's GPU-vs-CPU near-tie rule: |a - b| <= 2e-5 max(1, |a|, |b|)
    (tests/cuda/test_cuda_match.cpp:49-51)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b) <= 2e-5 * np.maximum(1.0, np.maximum(np.abs(a), np.abs(b)))
