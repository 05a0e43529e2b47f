"""Flow colour encoding on the GPU (ff_flow_to_color, flowfilter_b200.FlowToColor) against
the reference's own lookup (index-wheel fixture) and the oracle."""

from __future__ import annotations

import ctypes
import os

import numpy as np
import pytest

from conftest import ROOT
from oracle import display_oracle as D

pytestmark = pytest.mark.gpu

FIXTURE = os.path.join(ROOT, "tests", "golden", "ref_flow_to_color.npz")


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def run_c_abi(cuda, flow_np, maxflow, wheel_np=None, pad=0):
    """ff_flow_to_color on a (H, W, 2) float32 array, rows padded by `pad` float2."""
    from flowfilter_b200 import lib

    h, w = flow_np.shape[:2]
    fbuf = cuda.zeros((h, w + pad, 2), dtype=cuda.float32, device="cuda")
    fbuf[:, :w] = cuda.from_numpy(flow_np)
    out = cuda.zeros((h, w + pad, 4), dtype=cuda.uint8, device="cuda")
    wheel = cuda.from_numpy(np.ascontiguousarray(wheel_np)).cuda() if wheel_np is not None else None
    st = lib().ff_flow_to_color(_p(fbuf), fbuf.stride(0) * 4, h, w, maxflow, _p(wheel) if wheel is not None else None,
                                _p(out), out.stride(0), None)
    assert st == 0, lib().ff_last_error()
    cuda.cuda.synchronize()
    return out[:, :w].cpu().numpy()


def test_texels_equal_the_reference_lookup(cuda):
    """The index-encoding wheel makes the output name the texel read: bit-exact with the
    reference's flowToColor_k on every probe (texel edges, +-maxflow, non-finite values)."""
    g = np.load(FIXTURE)
    for k, (m, seed) in enumerate(zip(g["maxflow"], g["seed"])):
        flow = D.probe_flows(float(m), int(seed))
        got = run_c_abi(cuda, flow, float(m), D.index_wheel(), pad=3)
        np.testing.assert_array_equal(got[..., 0], g["col"][k])
        np.testing.assert_array_equal(got[..., 1], g["row"][k])
        assert (got[..., 2] == 0).all() and (got[..., 3] == 255).all()


def test_default_colours_equal_the_reference_lookup(cuda):
    """With its default wheel, ff_flow_to_color gives the reference FlowToColor's bytes: the
    reference's table at the texel the reference kernel read for every probe pixel."""
    g = np.load(FIXTURE)
    w = D.reference_wheel()
    for k, (m, seed) in enumerate(zip(g["maxflow"], g["seed"])):
        flow = D.probe_flows(float(m), int(seed))
        np.testing.assert_array_equal(run_c_abi(cuda, flow, float(m)), w[g["row"][k], g["col"][k]])


@pytest.mark.parametrize("h,w,maxflow", [(1, 1, 1.0), (7, 5, 2.0), (53, 70, 4.0), (480, 640, 4.0)])
def test_default_wheel_matches_oracle(cuda, h, w, maxflow):
    rng = np.random.default_rng(h * w)
    flow = rng.normal(0, maxflow * 0.7, (h, w, 2)).astype(np.float32)
    got = run_c_abi(cuda, flow, maxflow)
    np.testing.assert_array_equal(got, D.flow_to_color(flow, maxflow, D.reference_wheel()))


def test_flow_to_color_class_on_filter_flow(cuda):
    """FlowToColor over a filter's device flow (a pitched view), as the reference's demos do."""
    from flowfilter_b200 import FlowToColor, PyramidalFlowFilter, synthetic

    frames = synthetic.seq_rotzoom(frames=4, height=96, width=128, seed=3)
    f = PyramidalFlowFilter(96, 128, 2)
    f.maxflow = 4.0
    for k in range(frames.shape[0]):
        f.loadImage(frames[k])
        f.compute()
    dev = f.getFlowDevice()
    c = FlowToColor(dev, 3.0)
    c.compute()
    assert c.elapsedTime() > 0.0
    got = c.download()
    np.testing.assert_array_equal(got, D.flow_to_color(f.getFlow(), 3.0, D.reference_wheel()))
    # another wheel, given as a host table
    wheel = np.random.default_rng(9).integers(0, 256, (256, 256, 4), dtype=np.uint8)
    c.setColorWheel(wheel)
    c.maxflow = 2.5
    c.compute()
    np.testing.assert_array_equal(c.download(), D.flow_to_color(f.getFlow(), 2.5, wheel))
    c.setColorWheel(None)
    c.compute()
    np.testing.assert_array_equal(c.download(), D.flow_to_color(f.getFlow(), 2.5, D.reference_wheel()))


def test_flow_to_color_errors(cuda):
    from flowfilter_b200 import FFLogicError, FlowToColor, lib

    flow = cuda.zeros((8, 8, 2), dtype=cuda.float32, device="cuda")
    with pytest.raises(ValueError):
        FlowToColor(flow, 0.0)
    c = FlowToColor()
    with pytest.raises(FFLogicError):
        c.compute()
    with pytest.raises(FFLogicError):
        c.configure()
    with pytest.raises(ValueError):
        c.setInputFlow(cuda.zeros((8, 8), dtype=cuda.float32, device="cuda"))
    with pytest.raises(ValueError):
        c.setInputFlow(flow.cpu())
    with pytest.raises(ValueError):
        c.maxflow = -1.0
    with pytest.raises(ValueError):
        c.setColorWheel(np.zeros((255, 256, 4), np.uint8))
    out = cuda.zeros((8, 8, 4), dtype=cuda.uint8, device="cuda")
    # C ABI: maxflow <= 0, a misaligned flow pitch and empty sizes are refused before any launch
    assert lib().ff_flow_to_color(_p(flow), 64, 8, 8, 0.0, None, _p(out), 32, None) != 0
    assert lib().ff_flow_to_color(_p(flow), 66, 8, 8, 1.0, None, _p(out), 32, None) != 0
    assert lib().ff_flow_to_color(_p(flow), 64, 0, 8, 1.0, None, _p(out), 32, None) != 0
