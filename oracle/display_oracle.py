"""ORACLE of the flow colour encoding — TEST INFRASTRUCTURE ONLY.

A numpy restatement of the reference's FlowToColor lookup (src/gpu/device/display_k.cu:14-43;
texture set up in src/gpu/display.cu:64-75 as normalised-coordinate, point-sampled,
clamp-addressed, element-type reads, src/gpu/image.cu:241-247) and of the Middlebury
colour code that the library uses as its default wheel (Baker et al., IJCV 2011).  tests/
use it to check ff_flow_to_color and ff_color_wheel_default; the product never imports it.
The texel choice is pinned against the reference kernel run on a B200 with an
index-encoding wheel (tests/golden/ref_flow_to_color.npz).
"""

from __future__ import annotations

import math

import numpy as np

WHEEL = 256


def wheel_texel(f: np.ndarray, maxflow: float) -> np.ndarray:
    """Texel index along one axis for float32 flow components f (display_k.cu:34-35, then
    clamp + point sampling over 256 texels)."""
    f = np.asarray(f, np.float32)
    m = np.float32(maxflow)
    with np.errstate(invalid="ignore", over="ignore"):
        u = (f + m) / (np.float32(2.0) * m)
        idx = np.zeros(f.shape, np.int64)
        inside = (u > 0) & (u < 1)
        idx[inside] = (u[inside] * np.float32(WHEEL)).astype(np.int64)
        idx[u >= 1] = WHEEL - 1
    return idx


def flow_to_color(flow: np.ndarray, maxflow: float, wheel: np.ndarray) -> np.ndarray:
    """(H, W, 2) float32 flow -> (H, W, 4) uint8 through a (256, 256, 4) wheel (row = y)."""
    ix = wheel_texel(flow[..., 0], maxflow)
    iy = wheel_texel(flow[..., 1], maxflow)
    return wheel[iy, ix]


def middlebury_wheel() -> np.ndarray:
    """The Middlebury colour code at texel centres: 55-colour hue cycle (RY 15, YG 6, GC 4,
    CB 11, BM 13, MR 6, integer RGB), saturation from the radius, 0.75 outside |flow| = 1."""
    seg = [15, 6, 4, 11, 13, 6]
    cyc = []
    cyc += [(255, 255 * i // seg[0], 0) for i in range(seg[0])]
    cyc += [(255 - 255 * i // seg[1], 255, 0) for i in range(seg[1])]
    cyc += [(0, 255, 255 * i // seg[2]) for i in range(seg[2])]
    cyc += [(0, 255 - 255 * i // seg[3], 255) for i in range(seg[3])]
    cyc += [(255 * i // seg[4], 0, 255) for i in range(seg[4])]
    cyc += [(255, 0, 255 - 255 * i // seg[5]) for i in range(seg[5])]
    cyc = np.array(cyc, np.float64)
    n = len(cyc)
    c = (np.arange(WHEEL) + 0.5) / (WHEEL // 2) - 1.0
    u, v = np.meshgrid(c, c)
    rad = np.sqrt(u * u + v * v)
    # the C library's atan2 (as the library computes it), not numpy's vectorised one
    a = np.vectorize(math.atan2, otypes=[np.float64])(-v, -u) / np.pi
    fk = (a + 1.0) / 2.0 * (n - 1)
    k0 = np.floor(fk).astype(np.int64)
    k1 = np.where(k0 + 1 == n, 0, k0 + 1)
    f = fk - k0
    out = np.empty((WHEEL, WHEEL, 4), np.uint8)
    for ch in range(3):
        col = (1.0 - f) * cyc[k0, ch] / 255.0 + f * cyc[k1, ch] / 255.0
        col = np.where(rad <= 1.0, 1.0 - rad * (1.0 - col), col * 0.75)
        out[..., ch] = np.floor(255.0 * col).astype(np.int64)
    out[..., 3] = 255
    return out


def index_wheel() -> np.ndarray:
    """A wheel whose texel (row i, column j) holds (j, i, 0, 255): the lookup's output names
    the texel it read."""
    j, i = np.meshgrid(np.arange(WHEEL), np.arange(WHEEL))
    w = np.zeros((WHEEL, WHEEL, 4), np.uint8)
    w[..., 0], w[..., 1], w[..., 3] = j, i, 255
    return w


def probe_flows(maxflow: float, seed: int) -> np.ndarray:
    """(64, 96, 2) float32 flows for pinning the lookup: uniform over +-1.3 maxflow, every
    texel boundary and its float neighbours, +-maxflow, 0, and non-finite values."""
    rng = np.random.default_rng(seed)
    m = np.float32(maxflow)
    flow = rng.uniform(-1.3, 1.3, (64, 96, 2)).astype(np.float32) * m
    k = np.arange(WHEEL + 1, dtype=np.float32)
    edge = (k / np.float32(WHEEL) * np.float32(2.0) - np.float32(1.0)) * m
    edges = np.concatenate([edge, np.nextafter(edge, np.float32(np.inf)), np.nextafter(edge, np.float32(-np.inf))])
    special = np.array([0.0, m, -m, np.nextafter(m, np.float32(0)), np.nextafter(-m, np.float32(0)), 2 * m, -2 * m,
                        1e30, -1e30, np.inf, -np.inf, np.nan, 1e-30, -1e-30], np.float32)
    vals = np.concatenate([edges, special])
    flat = flow.reshape(-1, 2)
    flat[:len(vals), 0] = vals
    flat[:len(vals), 1] = rng.permutation(vals)
    flat[len(vals):2 * len(vals), 1] = vals
    flat[len(vals):2 * len(vals), 0] = rng.permutation(vals)
    return flow
