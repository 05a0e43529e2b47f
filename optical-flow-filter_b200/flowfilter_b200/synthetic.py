"""Deterministic synthetic image sequences for the flow-filter workloads.

The reference measures on a Blender "monkey" sequence that is not shipped with
it (notebooks/GPU_example.ipynb:298).  These seeded generators stand in for it
with the shapes, sizes and value distributions of the five workloads:

* ``seq_constant``   320x240 u8, blurred noise (sigma 2, seed 0), constant
                     (0.7, -0.4) px/frame translation.
* ``seq_rotzoom``    640x480 u8, blurred noise (sigma 1.5, seed 1), rotation by
                     0.5 deg/frame about the centre plus zoom 1.004/frame.
* ``seq_bumps``      2048x1088 u8, blurred noise (sigma 1, seed 2) + N(0, 3 DN)
                     sensor noise per frame, flow = sum of 8 Gaussian bumps
                     (sigma 150 px, amplitude U[-3, 3] px/frame).
* ``seq_bumps_float`` float32 frames in [0, 1] with a bump flow (sigma 40 px,
                     amplitude U[-2, 2]).

Everything is numpy only (plus a separable Gaussian written here), so the
same frames are produced on any machine with the same numpy version.
"""

from __future__ import annotations

import math
import os

import numpy as np

__all__ = [
    "blurred_noise",
    "warp_bilinear",
    "bump_flow",
    "seq_constant",
    "seq_rotzoom",
    "seq_bumps",
    "iter_bumps",
    "seq_bumps_float",
    "sequence",
]


def _gauss_kernel(sigma: float) -> np.ndarray:
    r = int(math.ceil(4.0 * sigma))
    x = np.arange(-r, r + 1, dtype=np.float64)
    k = np.exp(-0.5 * (x / sigma) ** 2)
    return k / k.sum()


def _blur_axis(img: np.ndarray, k: np.ndarray, axis: int) -> np.ndarray:
    r = (k.size - 1) // 2
    pad = [(0, 0), (0, 0)]
    pad[axis] = (r, r)
    p = np.pad(img, pad, mode="edge")  # border replicate ("nearest")
    out = np.zeros_like(img)
    n = img.shape[axis]
    for i, w in enumerate(k):
        sl = [slice(None), slice(None)]
        sl[axis] = slice(i, i + n)
        out += w * p[tuple(sl)]
    return out


def blurred_noise(height: int, width: int, sigma: float, rng: np.random.Generator) -> np.ndarray:
    """uniform[0,1) noise, Gaussian blur (border replicate), min-max rescale to [0, 255]."""
    noise = rng.uniform(0.0, 1.0, size=(height, width))
    k = _gauss_kernel(sigma)
    b = _blur_axis(_blur_axis(noise, k, 0), k, 1)
    lo, hi = b.min(), b.max()
    return (b - lo) * (255.0 / max(hi - lo, 1e-12))


def warp_bilinear(img: np.ndarray, sx: np.ndarray, sy: np.ndarray) -> np.ndarray:
    """Sample ``img`` at (sx, sy) bilinearly with border replicate."""
    h, w = img.shape
    sx = np.clip(sx, 0.0, w - 1.0)
    sy = np.clip(sy, 0.0, h - 1.0)
    x0 = np.floor(sx).astype(np.int64)
    y0 = np.floor(sy).astype(np.int64)
    x1 = np.minimum(x0 + 1, w - 1)
    y1 = np.minimum(y0 + 1, h - 1)
    fx = sx - x0
    fy = sy - y0
    top = img[y0, x0] * (1.0 - fx) + img[y0, x1] * fx
    bot = img[y1, x0] * (1.0 - fx) + img[y1, x1] * fx
    return top * (1.0 - fy) + bot * fy


def bump_flow(height: int, width: int, n_bumps: int, sigma: float, amp: float,
              rng: np.random.Generator) -> tuple[np.ndarray, np.ndarray]:
    """Smooth random flow: sum of Gaussian bumps with per-component amplitudes U[-amp, amp]."""
    yy, xx = np.mgrid[0:height, 0:width].astype(np.float64)
    u = np.zeros((height, width))
    v = np.zeros((height, width))
    for _ in range(n_bumps):
        au, av = rng.uniform(-amp, amp, size=2)
        cx = rng.uniform(0, width)
        cy = rng.uniform(0, height)
        g = np.exp(-((xx - cx) ** 2 + (yy - cy) ** 2) / (2.0 * sigma * sigma))
        u += au * g
        v += av * g
    return u, v


def _to_u8(x: np.ndarray) -> np.ndarray:
    return np.clip(np.rint(x), 0, 255).astype(np.uint8)


def seq_constant(frames: int = 100, height: int = 240, width: int = 320,
                 sigma: float = 2.0, seed: int = 0, flow=(0.7, -0.4)) -> np.ndarray:
    """Constant translation sequence, uint8 [T, H, W]."""
    rng = np.random.default_rng(seed)
    tex = blurred_noise(height, width, sigma, rng)
    yy, xx = np.mgrid[0:height, 0:width].astype(np.float64)
    out = np.empty((frames, height, width), np.uint8)
    for t in range(frames):
        out[t] = _to_u8(warp_bilinear(tex, xx - t * flow[0], yy - t * flow[1]))
    return out


def seq_rotzoom(frames: int = 300, height: int = 480, width: int = 640,
                sigma: float = 1.5, seed: int = 1, deg_per_frame: float = 0.5,
                zoom_per_frame: float = 1.004) -> np.ndarray:
    """Rotation about the centre plus zoom, uint8 [T, H, W]."""
    rng = np.random.default_rng(seed)
    tex = blurred_noise(height, width, sigma, rng)
    yy, xx = np.mgrid[0:height, 0:width].astype(np.float64)
    cx, cy = (width - 1) / 2.0, (height - 1) / 2.0
    out = np.empty((frames, height, width), np.uint8)
    for t in range(frames):
        a = math.radians(deg_per_frame * t)
        s = zoom_per_frame ** t
        # backward map: source = R(-a) (x - c) / s + c
        dx, dy = xx - cx, yy - cy
        sx = (math.cos(a) * dx + math.sin(a) * dy) / s + cx
        sy = (-math.sin(a) * dx + math.cos(a) * dy) / s + cy
        out[t] = _to_u8(warp_bilinear(tex, sx, sy))
    return out


def iter_bumps(frames: int = 1000, height: int = 1088, width: int = 2048,
               sigma: float = 1.0, seed: int = 2, n_bumps: int = 8,
               bump_sigma: float = 150.0, amp: float = 3.0,
               sensor_noise: float = 3.0, threads: int | None = None):
    """The frames of ``seq_bumps`` one at a time (uint8 [H, W] each), for sequences too long to
    hold.  The warps run on a thread pool a few frames ahead (numpy releases the GIL in them);
    the sensor noise is drawn in frame order from the one generator, so the frames are
    identical to ``seq_bumps``'s."""
    from collections import deque
    from concurrent.futures import ThreadPoolExecutor

    rng = np.random.default_rng(seed)
    tex = blurred_noise(height, width, sigma, rng)
    u, v = bump_flow(height, width, n_bumps, bump_sigma, amp, rng)
    yy, xx = np.mgrid[0:height, 0:width].astype(np.float64)

    def warp(t):
        return warp_bilinear(tex, xx - t * u, yy - t * v)

    threads = threads or min(16, os.cpu_count() or 1)
    with ThreadPoolExecutor(threads) as pool:
        ahead = deque(pool.submit(warp, t) for t in range(min(frames, 2 * threads)))
        for t in range(frames):
            noise = rng.normal(0.0, sensor_noise, size=(height, width)) if sensor_noise > 0 else None
            img = ahead.popleft().result()
            if t + len(ahead) + 1 < frames:
                ahead.append(pool.submit(warp, t + len(ahead) + 1))
            if noise is not None:
                img = img + noise
            yield _to_u8(img)


def seq_bumps(frames: int = 1000, height: int = 1088, width: int = 2048,
              sigma: float = 1.0, seed: int = 2, n_bumps: int = 8,
              bump_sigma: float = 150.0, amp: float = 3.0,
              sensor_noise: float = 3.0) -> np.ndarray:
    """Bump-flow sequence with additive sensor noise, uint8 [T, H, W]."""
    out = np.empty((frames, height, width), np.uint8)
    for t, f in enumerate(iter_bumps(frames, height, width, sigma, seed, n_bumps, bump_sigma, amp, sensor_noise)):
        out[t] = f
    return out


def seq_bumps_float(frames: int = 32, height: int = 256, width: int = 256,
                    sigma: float = 1.5, seed: int = 200, n_bumps: int = 8,
                    bump_sigma: float = 40.0, amp: float = 2.0):
    """float32 frames in [0, 1] and the known per-frame flow (u, v), each [H, W]."""
    rng = np.random.default_rng(seed)
    tex = blurred_noise(height, width, sigma, rng) / 255.0
    u, v = bump_flow(height, width, n_bumps, bump_sigma, amp, rng)
    yy, xx = np.mgrid[0:height, 0:width].astype(np.float64)
    out = np.empty((frames, height, width), np.float32)
    for t in range(frames):
        out[t] = np.clip(warp_bilinear(tex, xx - t * u, yy - t * v), 0.0, 1.0)
    return out, u.astype(np.float32), v.astype(np.float32)


def sequence(name: str, frames: int | None = None, **kw) -> np.ndarray:
    """Named sequence lookup used by the tests and the benchmark."""
    table = {
        "constant": seq_constant,
        "rotzoom": seq_rotzoom,
        "bumps": seq_bumps,
    }
    fn = table[name]
    if frames is not None:
        kw["frames"] = frames
    return fn(**kw)
