"""Python mirror of ``core.nss_cuda.BM3D`` over the C ABI of ``libnss_b200.so``.

The reference exposes BM3D as a VapourSynth API4 filter (src/cuda/plugin.cpp:76-98,
src/cuda/bm3d/filter.cpp:19-122). This module offers the same call for users
and tests without VapourSynth: ``BM3D(clip, ref=None, **args)`` with the same
argument names, defaults and creation errors (raised as :class:`Error` with
the filter's exact text), returning a node whose ``get_frame(n)`` renders a
frame on the GPU. Clips are lists of frames; a frame is a tuple of 2-D float32
planes (numpy arrays in host memory, or torch CUDA tensors for device-resident
frames).

There is no CPU path: without the library, or without a B200, calls fail.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from pathlib import Path
from typing import Sequence

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libnss_b200.so"

# kBm3dSignature (src/frontend/bm3d_args.hpp:8-12) + kBackendSignature (src/cuda/runtime/context.hpp:17)
SIGNATURE = (
    "clip:vnode;ref:vnode:opt;sigma:float[]:opt;block_size:int[]:opt;group_size:int[]:opt;"
    "block_step:int[]:opt;bm_range:int[]:opt;radius:int:opt;ps_num:int[]:opt;ps_range:int[]:opt;chroma:int:opt;"
    "final:int:opt;sigma_basic:float[]:opt;block_size_basic:int[]:opt;group_size_basic:int[]:opt;"
    "temporal_mode:data:opt;rolling_chunk:int:opt;rolling_cache_chunks:int:opt;rolling_cache_limit:int:opt;"
    "memory_limit_mb:int:opt;device_id:int:opt;num_streams:int:opt;"
)

GRAY, RGB, YUV = 1, 2, 3
OK, ERR_ARGUMENT, ERR_CUDA, ERR_RESOURCE, ERR_STATE, ERR_TIMEOUT = range(6)
MEM_HOST, MEM_DEVICE = 0, 1
ARG_INT, ARG_FLOAT, ARG_DATA = 1, 2, 3


class Error(Exception):
    """A filter error (the text VapourSynth would report as vs.Error)."""


def parse_signature(sig: str = SIGNATURE):
    out = {}
    for item in filter(None, sig.split(";")):
        name, kind, *flags = item.split(":")
        out[name] = (kind.rstrip("[]"), kind.endswith("[]"), "opt" in flags)
    return out


ARGS = parse_signature()


class VideoInfo(C.Structure):
    _fields_ = [("color_family", C.c_int), ("sample_float", C.c_int), ("bits_per_sample", C.c_int),
                ("subsampling_w", C.c_int), ("subsampling_h", C.c_int), ("width", C.c_int), ("height", C.c_int),
                ("num_frames", C.c_int)]

    def planes(self) -> int:
        return 1 if self.color_family == GRAY else 3

    def plane_shape(self, p: int):
        return (self.height >> (self.subsampling_h if p else 0), self.width >> (self.subsampling_w if p else 0))

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class Arg(C.Structure):
    _fields_ = [("key", C.c_char_p), ("type", C.c_int), ("count", C.c_int), ("ints", C.POINTER(C.c_int64)),
                ("floats", C.POINTER(C.c_double)), ("data", C.c_char_p)]


class Frame(C.Structure):
    _fields_ = [("planes", C.c_void_p * 3), ("strides", C.c_int64 * 3)]


class FrameOut(C.Structure):
    _fields_ = [("planes", C.c_void_p * 3), ("strides", C.c_int64 * 3)]


class KernelStats(C.Structure):
    _fields_ = [("launches", C.c_int64), ("match_launches", C.c_int64), ("group_launches", C.c_int64),
                ("finish_launches", C.c_int64), ("match_ms", C.c_double), ("group_ms", C.c_double),
                ("finish_ms", C.c_double), ("match_flops", C.c_double), ("match_pairs", C.c_double),
                ("tc_survivors", C.c_int64), ("tc_refs", C.c_int64), ("tc_max_error_ratio", C.c_double)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


_lib = None


class Prop(C.Structure):
    _fields_ = [("key", C.c_char_p), ("value", C.c_int64)]


class TcStats(C.Structure):
    _fields_ = [("survivors", C.c_int64), ("refs", C.c_int64), ("max_error_ratio", C.c_float),
                ("flagged_tiles", C.c_int), ("timeouts", C.c_int)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class BatchItem(C.Structure):
    _fields_ = [("node", C.c_void_p), ("clip", C.POINTER(Frame)), ("ref", C.POINTER(Frame)), ("memory", C.c_int),
                ("out", C.POINTER(FrameOut))]


class BatchInfo(C.Structure):
    _fields_ = [("match_parts", C.c_int), ("match_persistent", C.c_int), ("match_form", C.c_int), ("group_warps", C.c_int),
                ("group_ctas_per_sm", C.c_int), ("graphs", C.c_int), ("runs", C.c_int64), ("frames", C.c_int64),
                ("kernel_launches", C.c_int64), ("graph_builds", C.c_int64), ("tunings", C.c_int64),
                ("chunks", C.c_int), ("last_run_ms", C.c_double), ("arena_bytes", C.c_size_t)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class ServeRequest(C.Structure):
    _fields_ = [("vi", VideoInfo), ("args", C.POINTER(Arg)), ("nargs", C.c_int), ("clip", C.POINTER(Frame)),
                ("ref", C.POINTER(Frame)), ("memory", C.c_int), ("out", C.POINTER(FrameOut))]


class ServeResult(C.Structure):
    _fields_ = [("status", C.c_int), ("frames", C.c_int), ("queue_ms", C.c_double), ("latency_ms", C.c_double),
                ("footprint_bytes", C.c_int64), ("error", C.c_char * 192)]


class ServerStats(C.Structure):
    _fields_ = [(f, C.c_int64) for f in (
        "submitted", "completed", "failed", "frames", "ticks", "tick_frames", "temporal_frames", "queued", "active",
        "peak_active", "budget_bytes", "reserved_bytes", "peak_reserved_bytes", "engines_created",
        "engines_reused")]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


def lib():
    """The loaded library; raises if it is missing (no fallback)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: build it with `make -C {HERE}` (or __graft_entry__.build())")
        L = C.CDLL(str(LIB_PATH))
        L.nssb_last_error.restype = C.c_char_p
        L.nssb_version.restype = C.c_char_p
        L.nssb_backend_info.argtypes = [C.c_int, C.c_char_p, C.c_size_t]
        L.nssb_bm3d_check.argtypes = [C.POINTER(VideoInfo), C.POINTER(VideoInfo), C.POINTER(Arg), C.c_int,
                                      C.POINTER(VideoInfo)]
        L.nssb_bm3d_create.argtypes = [C.POINTER(VideoInfo), C.POINTER(VideoInfo), C.POINTER(Arg), C.c_int,
                                       C.POINTER(C.c_void_p)]
        L.nssb_bm3d_free.argtypes = [C.c_void_p]
        L.nssb_bm3d_free.restype = None
        L.nssb_bm3d_output_info.argtypes = [C.c_void_p, C.POINTER(VideoInfo)]
        L.nssb_bm3d_frame_window.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.nssb_bm3d_get_frame.argtypes = [C.c_void_p, C.c_int, C.POINTER(Frame), C.POINTER(Frame), C.c_int, C.c_int,
                                          C.c_int, C.POINTER(FrameOut)]
        L.nssb_bm3d_stats.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(KernelStats)]
        L.nssb_match_spatial.argtypes = [C.c_void_p, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                         C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.nssb_match_temporal.argtypes = [C.POINTER(C.c_void_p), C.POINTER(C.c_int64), C.c_int, C.c_int, C.c_int,
                                          C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                          C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.nssb_bm3d_plane_stage.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int, C.c_int,
                                            C.c_float, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p]
        L.nssb_bm3d_plane_stage_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int, C.c_int,
                                                    C.c_float, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p]
        L.nssb_bm3d_set_matcher.argtypes = [C.c_void_p, C.c_int]
        L.nssb_bm3d_set_window.argtypes = [C.c_void_p, C.c_float]
        L.nssb_bm3d_frame_props.argtypes = [C.c_void_p, C.c_int, C.POINTER(Prop), C.c_int, C.POINTER(C.c_int)]
        L.nssb_match_spatial_tc.argtypes = [C.c_void_p, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                            C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(TcStats), C.c_void_p]
        L.nssb_batch_create.argtypes = [C.c_int, C.POINTER(Arg), C.c_int, C.POINTER(C.c_void_p)]
        L.nssb_batch_run.argtypes = [C.c_void_p, C.POINTER(BatchItem), C.c_int]
        L.nssb_batch_get_info.argtypes = [C.c_void_p, C.POINTER(BatchInfo)]
        L.nssb_batch_free.argtypes = [C.c_void_p]
        L.nssb_batch_free.restype = None
        L.nssb_server_create.argtypes = [C.c_int, C.POINTER(Arg), C.c_int, C.POINTER(C.c_void_p)]
        L.nssb_server_submit.argtypes = [C.c_void_p, C.POINTER(ServeRequest), C.POINTER(C.c_int64)]
        L.nssb_server_wait.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.POINTER(ServeResult)]
        L.nssb_server_get_stats.argtypes = [C.c_void_p, C.POINTER(ServerStats)]
        L.nssb_server_free.argtypes = [C.c_void_p]
        L.nssb_server_free.restype = None
        _lib = L
    return _lib


def last_error() -> str:
    return lib().nssb_last_error().decode()


def check(rc: int) -> None:
    if rc != OK:
        raise Error(last_error())


def video_info(family: int, width: int, height: int, num_frames: int, ss_w: int = 0, ss_h: int = 0) -> VideoInfo:
    return VideoInfo(family, 1, 32, ss_w, ss_h, width, height, num_frames)


FORMATS = {
    "GRAYS": (GRAY, 0, 0),
    "RGBS": (RGB, 0, 0),
    "YUV444PS": (YUV, 0, 0),
    "YUV420PS": (YUV, 1, 1),
    "YUV422PS": (YUV, 1, 0),
}


def format_info(name: str, width: int, height: int, num_frames: int) -> VideoInfo:
    fam, sw, sh = FORMATS[name]
    return video_info(fam, width, height, num_frames, sw, sh)


class _ArgBuffer:
    """The call's arguments as nssb_arg entries (types as VapourSynth coerces them)."""

    def __init__(self, kwargs: dict):
        self.keep = []
        entries = []
        for key, value in kwargs.items():
            if key not in ARGS:
                raise Error(f"BM3D: Function does not take argument(s) named {key}")
            kind, is_array, _ = ARGS[key]
            if value is None:
                continue
            vals = list(value) if isinstance(value, (list, tuple)) else [value]
            if not is_array and len(vals) != 1:
                raise Error(f"BM3D: Argument '{key}' is not an array")
            if kind == "int":
                if any(isinstance(v, float) for v in vals):
                    raise Error(f"BM3D: Argument '{key}' is not of type int")
                arr = (C.c_int64 * len(vals))(*[int(v) for v in vals])
                self.keep.append(arr)
                entries.append(Arg(key.encode(), ARG_INT, len(vals), arr, None, None))
            elif kind == "float":
                arr = (C.c_double * len(vals))(*[float(v) for v in vals])
                self.keep.append(arr)
                entries.append(Arg(key.encode(), ARG_FLOAT, len(vals), None, arr, None))
            elif kind == "data":
                data = vals[0].encode() if isinstance(vals[0], str) else bytes(vals[0])
                self.keep.append(data)
                entries.append(Arg(key.encode(), ARG_DATA, 1, None, None, data))
            else:
                raise Error(f"BM3D: Argument '{key}' has an unsupported type")
        self.array = (Arg * max(1, len(entries)))(*entries)
        self.count = len(entries)


def check_args(clip_vi: VideoInfo, ref_vi: VideoInfo | None = None, **kwargs) -> VideoInfo:
    """Creation checks only (no device): the output video info, or Error."""
    args = _ArgBuffer(kwargs)
    out = VideoInfo()
    check(lib().nssb_bm3d_check(C.byref(clip_vi), C.byref(ref_vi) if ref_vi is not None else None, args.array,
                                args.count, C.byref(out)))
    return out


@dataclass
class Clip:
    """A clip: frames (each a tuple of 2-D float32 planes) and its format."""

    frames: Sequence
    vi: VideoInfo

    @staticmethod
    def from_frames(frames, family: int = GRAY, ss_w: int = 0, ss_h: int = 0) -> "Clip":
        frames = [tuple(f) if isinstance(f, (tuple, list)) else (f,) for f in frames]
        h, w = frames[0][0].shape
        return Clip(frames, video_info(family, w, h, len(frames), ss_w, ss_h))

    @property
    def device(self) -> bool:
        p = self.frames[0][0]
        return hasattr(p, "is_cuda") and p.is_cuda


def _plane_ptr(p):
    if hasattr(p, "data_ptr"):
        assert p.dtype.__str__() == "torch.float32" and p.stride(1) == 1
        return p.data_ptr(), p.stride(0)
    assert p.dtype == np.float32 and p.strides[1] == 4
    return p.ctypes.data, p.strides[0] // 4


class Node:
    """A created BM3D filter; frames render on the GPU."""

    def __init__(self, clip: Clip, ref: Clip | None, kwargs: dict):
        self.clip, self.ref = clip, ref
        args = _ArgBuffer(kwargs)
        h = C.c_void_p()
        check(lib().nssb_bm3d_create(C.byref(clip.vi), C.byref(ref.vi) if ref is not None else None, args.array,
                                     args.count, C.byref(h)))
        self.handle = h
        self.vi = VideoInfo()
        check(lib().nssb_bm3d_output_info(self.handle, C.byref(self.vi)))

    def close(self):
        if getattr(self, "handle", None):
            lib().nssb_bm3d_free(self.handle)
            self.handle = None

    def __del__(self):
        self.close()

    def stats(self, enable_timing: bool, reset: bool) -> KernelStats:
        """Kernel accounting since the last reset; turns event timing on or off."""
        st = KernelStats()
        check(lib().nssb_bm3d_stats(self.handle, int(enable_timing), int(reset), C.byref(st)))
        return st

    def frame_props(self, n: int) -> dict:
        """The properties stamped on output frame n (_NSSModel, ..., _NSSFat* on the legacy intermediate)."""
        arr = (Prop * 8)()
        k = C.c_int()
        check(lib().nssb_bm3d_frame_props(self.handle, n, arr, 8, C.byref(k)))
        return {arr[i].key.decode(): arr[i].value for i in range(k.value)}

    def set_matcher(self, form: int) -> None:
        """0: FP32 matcher; 1: tensor-core precision form; 2: automatic (the default: the precision
        form from bm_range 32 on at block steps 1-7 and from 63 on at step 8, FP32 elsewhere).
        Identical lists whichever runs."""
        check(lib().nssb_bm3d_set_matcher(self.handle, int(form)))

    def set_window(self, beta: float) -> None:
        """Opt-in Kaiser aggregation window (beta > 0); 0 restores the reference's flat weights."""
        check(lib().nssb_bm3d_set_window(self.handle, float(beta)))

    def frame_window(self, n: int):
        a, b = C.c_int(), C.c_int()
        check(lib().nssb_bm3d_frame_window(self.handle, n, C.byref(a), C.byref(b)))
        return a.value, b.value

    def _frames(self, clip: Clip, first: int, last: int):
        arr = (Frame * (last - first + 1))()
        for i, n in enumerate(range(first, last + 1)):
            for p, plane in enumerate(clip.frames[n]):
                ptr, stride = _plane_ptr(plane)
                arr[i].planes[p] = ptr
                arr[i].strides[p] = stride
        return arr

    def get_frame(self, n: int, out=None):
        """Output frame n: a tuple of planes (numpy, or torch CUDA tensors when the clip is device-resident)."""
        first, last = self.frame_window(n)
        device = self.clip.device
        src = self._frames(self.clip, first, last)
        ref = self._frames(self.ref, first, last) if self.ref is not None else None
        if out is None:
            shapes = [self.vi.plane_shape(p) for p in range(self.vi.planes())]
            if device:
                import torch

                out = tuple(torch.empty(s, dtype=torch.float32, device=self.clip.frames[0][0].device) for s in shapes)
            else:
                out = tuple(np.empty(s, np.float32) for s in shapes)
        fo = FrameOut()
        for p, plane in enumerate(out):
            ptr, stride = _plane_ptr(plane)
            fo.planes[p] = ptr
            fo.strides[p] = stride
        check(lib().nssb_bm3d_get_frame(self.handle, n, src, ref, first, last - first + 1,
                                        MEM_DEVICE if device else MEM_HOST, C.byref(fo)))
        return out


def _frame_struct(planes, cls=Frame):
    f = cls()
    for p, plane in enumerate(planes):
        ptr, stride = _plane_ptr(plane)
        f.planes[p] = ptr
        f.strides[p] = stride
    return f


class Batch:
    """The batched form: many radius-0 output frames (of any nodes) per call.

    ``run([(node, n), ...])`` renders frame n of each node and returns the
    output planes in order (numpy, or CUDA tensors for device-resident clips);
    every output is bit-identical to ``node.get_frame(n)``.
    """

    def __init__(self, device_id: int = 0, autotune: bool = True, graph: bool = True, **shape):
        vals = {"autotune": int(autotune), "graph": int(graph), **{k: int(v) for k, v in shape.items()}}
        arrs = [(C.c_int64 * 1)(v) for v in vals.values()]
        args = (Arg * len(vals))(*[Arg(k.encode(), ARG_INT, 1, a, None, None) for k, a in zip(vals, arrs)])
        h = C.c_void_p()
        check(lib().nssb_batch_create(device_id, args, len(vals), C.byref(h)))
        self.handle = h

    def close(self):
        if getattr(self, "handle", None):
            lib().nssb_batch_free(self.handle)
            self.handle = None

    def __del__(self):
        self.close()

    def info(self) -> BatchInfo:
        inf = BatchInfo()
        check(lib().nssb_batch_get_info(self.handle, C.byref(inf)))
        return inf

    def run(self, requests, outs=None):
        n = len(requests)
        items = (BatchItem * n)()
        keep = []
        results = []
        for i, (node, fn) in enumerate(requests):
            device = node.clip.device
            src = _frame_struct(node.clip.frames[fn])
            ref = _frame_struct(node.ref.frames[fn]) if node.ref is not None else None
            if outs is not None:
                out = outs[i]
            else:
                shapes = [node.vi.plane_shape(p) for p in range(node.vi.planes())]
                if device:
                    import torch

                    dev = node.clip.frames[0][0].device
                    out = tuple(torch.empty(s, dtype=torch.float32, device=dev) for s in shapes)
                else:
                    out = tuple(np.empty(s, np.float32) for s in shapes)
            fo = _frame_struct(out, FrameOut)
            keep += [src, ref, fo]
            items[i].node = node.handle
            items[i].clip = C.pointer(src)
            items[i].ref = C.pointer(ref) if ref is not None else None
            items[i].memory = MEM_DEVICE if device else MEM_HOST
            items[i].out = C.pointer(fo)
            results.append(out)
        check(lib().nssb_batch_run(self.handle, items, n))
        return results


def _int_args(vals: dict):
    arrs = [(C.c_int64 * 1)(int(v)) for v in vals.values()]
    return (Arg * max(1, len(vals)))(*[Arg(k.encode(), ARG_INT, 1, a, None, None) for k, a in zip(vals, arrs)]), arrs


class Server:
    """The serving form: ``submit(clip, ref=None, **bm3d_args)`` queues a request
    (a short clip, the arguments of BM3D) and returns a ticket; ``wait(ticket)``
    returns (outputs, result). Requests are admitted by device footprint and
    rendered in continuous batches (radius 0) or on pooled engines (radius > 0)."""

    def __init__(self, device_id: int = 0, **opts):
        args, self._keep = _int_args(opts)
        h = C.c_void_p()
        check(lib().nssb_server_create(device_id, args, len(opts), C.byref(h)))
        self.handle = h
        self._pending = {}

    def close(self):
        if getattr(self, "handle", None):
            lib().nssb_server_free(self.handle)
            self.handle = None

    def __del__(self):
        self.close()

    def submit(self, clip: Clip, ref: Clip | None = None, outs=None, **kwargs) -> int:
        n = clip.vi.num_frames
        device = clip.device
        frames = (Frame * n)(*[_frame_struct(f) for f in clip.frames])
        refs = (Frame * n)(*[_frame_struct(f) for f in ref.frames]) if ref is not None else None
        if outs is None:
            shapes = [clip.vi.plane_shape(p) for p in range(clip.vi.planes())]
            if device:
                import torch

                dev = clip.frames[0][0].device
                outs = [tuple(torch.empty(sh, dtype=torch.float32, device=dev) for sh in shapes) for _ in range(n)]
            else:
                outs = [tuple(np.empty(sh, np.float32) for sh in shapes) for _ in range(n)]
        fouts = (FrameOut * n)(*[_frame_struct(o, FrameOut) for o in outs])
        args = _ArgBuffer(kwargs)
        req = ServeRequest(clip.vi, args.array, args.count, frames, refs, MEM_DEVICE if device else MEM_HOST, fouts)
        ticket = C.c_int64()
        check(lib().nssb_server_submit(self.handle, C.byref(req), C.byref(ticket)))
        self._pending[ticket.value] = (clip, ref, frames, refs, fouts, outs, args)
        return ticket.value

    def wait(self, ticket: int, timeout_ms: int = -1):
        res = ServeResult()
        check(lib().nssb_server_wait(self.handle, ticket, timeout_ms, C.byref(res)))
        outs = self._pending.pop(ticket)[5]
        if res.status != OK:
            raise Error(res.error.decode())
        return outs, res

    def stats(self) -> ServerStats:
        st = ServerStats()
        check(lib().nssb_server_get_stats(self.handle, C.byref(st)))
        return st


def BM3D(clip: Clip, ref: Clip | None = None, **kwargs) -> Node:
    """core.nss_cuda.BM3D(clip, ref, ...) -- see docs/api/cuda/bm3d.md of the reference for the arguments."""
    return Node(clip, ref, kwargs)


def backend(device_id: int = 0) -> str:
    buf = C.create_string_buffer(1024)
    check(lib().nssb_backend_info(device_id, buf, len(buf)))
    return buf.value.decode()


def version() -> str:
    return lib().nssb_version().decode()


def build() -> None:
    import subprocess

    subprocess.run(["make", "-s", "-j8", "-C", str(HERE)], check=True)
