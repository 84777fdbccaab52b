"""Seeded synthetic BM3D inputs (the reference's quality images are not
available; these stand in with the shapes and value ranges of the workloads).

- ``gray_frame``: linear gradient + 20 axis-aligned rectangles of uniform
  intensity in [0, 1] + a 2-D sinusoidal texture (period 8-32 px, amplitude
  0.1), plus i.i.d. Gaussian noise of sigma/255, no clamping.
- ``yuv420_clip``: luma from the same generator per frame, translated by a
  random 0-3 px between frames; chroma planes are half-resolution smooth
  gradients; noise sigma/255 on every plane.
- ``panning_clip``: a textured background panning 1-2 px/frame plus 5
  independently moving rectangles (the temporal workload).
"""
from __future__ import annotations

import numpy as np


def _clean(rng: np.random.Generator, w: int, h: int) -> np.ndarray:
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    gx, gy = rng.uniform(-0.5, 0.5, 2)
    img = 0.5 + gx * (xx / max(w - 1, 1) - 0.5) + gy * (yy / max(h - 1, 1) - 0.5)
    for _ in range(20):
        rw = int(rng.integers(max(2, w // 20), max(3, w // 3)))
        rh = int(rng.integers(max(2, h // 20), max(3, h // 3)))
        x0 = int(rng.integers(0, max(1, w - rw)))
        y0 = int(rng.integers(0, max(1, h - rh)))
        img[y0:y0 + rh, x0:x0 + rw] = rng.uniform(0.0, 1.0)
    px, py = rng.uniform(8.0, 32.0, 2)
    phase = rng.uniform(0, 2 * np.pi)
    img += 0.1 * np.sin(2 * np.pi * (xx / px + yy / py) + phase)
    return img


def gray_frame(seed: int, width: int = 512, height: int = 512, sigma: float = 10.0):
    """(noisy, clean) float32 planes."""
    rng = np.random.default_rng(seed)
    clean = _clean(rng, width, height)
    noisy = clean + rng.normal(0.0, sigma / 255.0, clean.shape)
    return noisy.astype(np.float32), clean.astype(np.float32)


def _chroma(rng, w, h):
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    a, b, c = rng.uniform(-0.2, 0.2, 3)
    return a * xx / max(w - 1, 1) + b * yy / max(h - 1, 1) + c


def yuv420_clip(seed: int, width: int = 1920, height: int = 1080, frames: int = 30, sigma: float = 5.0,
                with_clean: bool = False):
    """List of (Y, U, V) noisy frames; luma translates 0-3 px per frame."""
    rng = np.random.default_rng(seed)
    pad = 3 * frames + 8
    canvas = _clean(rng, width + pad, height + pad)
    u = _chroma(rng, width // 2, height // 2)
    v = _chroma(rng, width // 2, height // 2)
    out, clean = [], []
    ox = oy = 0
    for f in range(frames):
        if f:
            ox = min(ox + int(rng.integers(0, 4)), pad - 1)
            oy = min(oy + int(rng.integers(0, 4)), pad - 1)
        y = canvas[oy:oy + height, ox:ox + width]
        planes = (y, u, v)
        noisy = tuple((p + rng.normal(0.0, sigma / 255.0, p.shape)).astype(np.float32) for p in planes)
        out.append(noisy)
        if with_clean:
            clean.append(tuple(p.astype(np.float32) for p in planes))
    return (out, clean) if with_clean else out


def panning_clip(seed: int, width: int = 1920, height: int = 1080, frames: int = 60, sigma: float = 10.0,
                 yuv420: bool = True):
    """Textured background panning 1-2 px/frame + 5 moving rectangles."""
    rng = np.random.default_rng(seed)
    pad = 2 * frames + 8
    bg = _clean(rng, width + pad, height + pad)
    rects = []
    for _ in range(5):
        rw, rh = int(rng.integers(width // 16, width // 5)), int(rng.integers(height // 16, height // 5))
        rects.append([float(rng.uniform(0, width - rw)), float(rng.uniform(0, height - rh)), rw, rh,
                      float(rng.uniform(-4, 4)), float(rng.uniform(-4, 4)), float(rng.uniform(0, 1))])
    dx, dy = rng.uniform(1, 2), rng.uniform(1, 2)
    u = _chroma(rng, width // 2, height // 2)
    v = _chroma(rng, width // 2, height // 2)
    out = []
    for f in range(frames):
        ox, oy = int(round(f * dx)) % pad, int(round(f * dy)) % pad
        y = bg[oy:oy + height, ox:ox + width].copy()
        for r in rects:
            x0 = int(r[0] + f * r[4]) % max(1, width - r[2])
            y0 = int(r[1] + f * r[5]) % max(1, height - r[3])
            y[y0:y0 + r[3], x0:x0 + r[2]] = r[6]
        planes = (y, u, v) if yuv420 else (y,)
        out.append(tuple((p + rng.normal(0.0, sigma / 255.0, p.shape)).astype(np.float32) for p in planes))
    return out
