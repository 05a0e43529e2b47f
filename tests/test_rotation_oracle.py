"""Rotational predictor and Lax-Wendroff propagation, CPU side: the oracle (and the
library's host camera function) against the reference's own outputs on a B200
(tests/golden/ref_rotation.npz, made by oracle/make_reference_fixtures.py)."""

from __future__ import annotations

import hashlib
import json
import os

import numpy as np

import oracle as O
from conftest import GOLDEN
from make_reference_fixtures import LW_CASES, ROT_CASES, lw_inputs, rot_image


def fixture():
    g = np.load(os.path.join(GOLDEN, "ref_rotation.npz"))
    return g, json.loads(bytes(g["inputs_sha256"]).decode())


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def test_lax_wendroff_oracle_equals_reference():
    g, shas = fixture()
    for k, (h, w, d, it, seed) in enumerate(LW_CASES):
        flow, img = lw_inputs(h, w, d, seed)
        assert [sha(flow), sha(img)] == shas[f"lw_{k}"]
        ref = g[f"lw_out_{k}"]
        np.testing.assert_array_equal(O.lax_wendroff(flow, img, it).view(np.uint32), ref.view(np.uint32))


def test_rotational_predictor_oracle_equals_reference():
    g, shas = fixture()
    for k, (h, w, d, focal, sh, sw, wx, wy, wz, it, seed) in enumerate(ROT_CASES):
        img = rot_image(h, w, d, seed)
        assert [sha(img)] == shas[f"rot_{k}"]
        cam = O.camera_perspective(focal, h, w, sh, sw)
        np.testing.assert_array_equal(cam, g[f"rot_cam_{k}"])
        flow = O.rotational_flow(cam, wx, wy, wz, h, w)
        np.testing.assert_array_equal(flow.view(np.uint32), g[f"rot_flow_{k}"].view(np.uint32))
        pred = O.lax_wendroff(flow, img, it)
        np.testing.assert_array_equal(pred.view(np.uint32), g[f"rot_pred_{k}"].view(np.uint32))


def test_library_camera_equals_reference():
    from flowfilter_b200 import createPerspectiveCamera

    g, _ = fixture()
    for k, (h, w, d, focal, sh, sw, *_rest) in enumerate(ROT_CASES):
        c = createPerspectiveCamera(focal, h, w, sh, sw)
        got = np.array([c.alphaX, c.alphaY, c.centerX, c.centerY], np.float32)
        np.testing.assert_array_equal(got, g[f"rot_cam_{k}"])
