"""ORACLE of the flow colour encoding — TEST INFRASTRUCTURE ONLY.

A numpy restatement of the reference's FlowToColor lookup (src/gpu/device/display_k.cu:14-43;
texture set up in src/gpu/display.cu:64-75 as normalised-coordinate, point-sampled,
clamp-addressed, element-type reads, src/gpu/image.cu:241-247) and the
reference's colour wheel table that the library uses as its default wheel.  tests/
use it to check ff_flow_to_color and ff_color_wheel_default; the product never imports it.
The texel choice is pinned against the reference kernel run on a B200 with an
index-encoding wheel (tests/golden/ref_flow_to_color.npz).
"""

from __future__ import annotations

import math
import os

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


def reference_wheel() -> np.ndarray:
    """The reference's colour wheel table (src/colorwheel.cpp), as the package keeps it
    (optical-flow-filter_b200/csrc/colorwheel.z, decoded by colorwheel_asset.py)."""
    import importlib.util

    csrc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "optical-flow-filter_b200", "csrc")
    spec = importlib.util.spec_from_file_location("colorwheel_asset", os.path.join(csrc, "colorwheel_asset.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.load(os.path.join(csrc, "colorwheel.z"))


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
