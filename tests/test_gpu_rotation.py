"""Rotational predictor and Lax-Wendroff propagation on the GPU (ff_rotational_predict,
ff_lax_wendroff and the Python classes) against the reference's outputs and the oracle."""

from __future__ import annotations

import ctypes
import os

import numpy as np
import pytest

import oracle as O
from conftest import GOLDEN
from make_reference_fixtures import LW_CASES, ROT_CASES, lw_inputs, rot_image

pytestmark = pytest.mark.gpu


def dev(cuda, a, pad=0):
    """A CUDA tensor view of `a` whose rows are `pad` pixels longer than the image."""
    h, w = a.shape[:2]
    full = cuda.zeros((h, w + pad) + a.shape[2:], dtype=cuda.float32, device="cuda")
    full[:, :w] = cuda.from_numpy(np.ascontiguousarray(a))
    return full[:, :w]


@pytest.fixture(scope="module")
def golden():
    return np.load(os.path.join(GOLDEN, "ref_rotation.npz"))


def test_lax_wendroff_equals_reference(cuda, golden):
    from flowfilter_b200 import LaxWendroffPropagator

    for k, (h, w, d, it, seed) in enumerate(LW_CASES):
        flow, img = lw_inputs(h, w, d, seed)
        lw = LaxWendroffPropagator(dev(cuda, flow, pad=3), dev(cuda, img, pad=5))
        if it > 0:
            lw.iterations = it
        lw.compute()
        got = lw.getPropagatedImage().cpu().numpy()
        np.testing.assert_array_equal(got.view(np.uint32), golden[f"lw_out_{k}"].view(np.uint32))
        assert lw.elapsedTime() > 0.0


def test_rotational_predictor_equals_reference(cuda, golden):
    from flowfilter_b200 import RotationalFlowImagePredictor, createPerspectiveCamera

    for k, (h, w, d, focal, sh, sw, wx, wy, wz, it, seed) in enumerate(ROT_CASES):
        cam = createPerspectiveCamera(focal, h, w, sh, sw)
        p = RotationalFlowImagePredictor(cam, dev(cuda, rot_image(h, w, d, seed), pad=7))
        p.setAngularVelocity(wx, wy, wz)
        if it > 0:
            p.iterations = it
        p.compute()
        np.testing.assert_array_equal(p.getOpticalFlow().cpu().numpy().view(np.uint32),
                                      golden[f"rot_flow_{k}"].view(np.uint32))
        np.testing.assert_array_equal(p.getPredictedImage().cpu().numpy().view(np.uint32),
                                      golden[f"rot_pred_{k}"].view(np.uint32))


@pytest.mark.parametrize("h,w,d,it", [(480, 640, 1, 3), (101, 77, 4, 17), (70, 90, 1, 40), (64, 64, 4, 33),
                                      (1, 1, 1, 2), (3, 200, 4, 5), (300, 2, 1, 9)])
def test_lax_wendroff_matches_oracle(cuda, h, w, d, it):
    """Sizes the fixture does not cover: a VGA frame, ragged and degenerate sizes, and more
    iterations than one launch covers (the chained launches through the workspace)."""
    from flowfilter_b200 import LaxWendroffPropagator

    flow, img = lw_inputs(h, w, d, h * 7 + w + it)
    lw = LaxWendroffPropagator(dev(cuda, flow), dev(cuda, img, pad=2))
    lw.iterations = it
    lw.compute()
    np.testing.assert_array_equal(lw.getPropagatedImage().cpu().numpy(), O.lax_wendroff(flow, img, it))


def test_rotational_predictor_chained_and_reconfigured(cuda):
    from flowfilter_b200 import RotationalFlowImagePredictor, createPerspectiveCamera

    h, w = 90, 120
    img = rot_image(h, w, 4, 77)
    cam = createPerspectiveCamera(0.004, h, w, 0.003, 0.004)
    p = RotationalFlowImagePredictor(cam, dev(cuda, img))
    p.setAngularVelocity(0.01, 0.02, -0.03)
    p.iterations = 20  # two launches
    p.compute()
    cam4 = np.array([cam.alphaX, cam.alphaY, cam.centerX, cam.centerY], np.float32)
    flow = O.rotational_flow(cam4, 0.01, 0.02, -0.03, h, w)
    np.testing.assert_array_equal(p.getOpticalFlow().cpu().numpy(), flow)
    np.testing.assert_array_equal(p.getPredictedImage().cpu().numpy(), O.lax_wendroff(flow, img, 20))
    # configure() starts a new propagator: iterations back to 0, the image passes unchanged
    p.configure()
    assert p.iterations == 0
    p.compute()
    np.testing.assert_array_equal(p.getPredictedImage().cpu().numpy(), O.lax_wendroff(flow, img, 0))


def test_rotation_errors(cuda):
    from flowfilter_b200 import (FFLogicError, LaxWendroffPropagator, RotationalFlowImagePredictor,
                                 createPerspectiveCamera, lib)

    flow = cuda.zeros((8, 8, 2), dtype=cuda.float32, device="cuda")
    img = cuda.zeros((8, 8), dtype=cuda.float32, device="cuda")
    with pytest.raises(ValueError):
        LaxWendroffPropagator(flow, cuda.zeros((8, 8, 2), dtype=cuda.float32, device="cuda"))
    with pytest.raises(ValueError):
        LaxWendroffPropagator(flow, cuda.zeros((9, 8), dtype=cuda.float32, device="cuda"))
    lw = LaxWendroffPropagator()
    with pytest.raises(FFLogicError):
        lw.compute()
    with pytest.raises(FFLogicError):
        lw.configure()
    lw = LaxWendroffPropagator(flow, img)
    with pytest.raises(ValueError):
        lw.iterations = 0
    p = RotationalFlowImagePredictor()
    with pytest.raises(FFLogicError):
        p.configure()
    cam = createPerspectiveCamera(0.004, 8, 8, 0.003, 0.003)
    p = RotationalFlowImagePredictor(cam, img)
    with pytest.raises(ValueError):
        p.iterations = -2
    # C ABI: more iterations than one launch without a workspace, and output == input
    out = cuda.zeros_like(img)
    vp = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    n = lib().ff_lax_wendroff_max_fused() + 1
    assert lib().ff_lax_wendroff(vp(flow), 64, vp(img), 32, 1, 8, 8, n, vp(out), 32, None, 0, None) != 0
    assert lib().ff_lax_wendroff(vp(flow), 64, vp(img), 32, 1, 8, 8, 2, vp(img), 32, None, 0, None) != 0
    assert lib().ff_lax_wendroff(vp(flow), 64, vp(img), 32, 2, 8, 8, 2, vp(out), 32, None, 0, None) != 0
