"""Flow colour encoding, CPU side: the oracle's texel choice against the reference's own
lookup kernel (fixture made on a B200 by oracle/make_reference_fixtures.py), and the
library's default colour wheel against the oracle's Middlebury colour code."""

from __future__ import annotations

import ctypes
import hashlib
import json
import os

import numpy as np

from conftest import ROOT
from oracle import display_oracle as D

FIXTURE = os.path.join(ROOT, "tests", "golden", "ref_flow_to_color.npz")


def test_oracle_texels_match_the_reference_lookup():
    g = np.load(FIXTURE)
    shas = json.loads(bytes(g["flows_sha256"]).decode())
    for k, (m, seed) in enumerate(zip(g["maxflow"], g["seed"])):
        flow = D.probe_flows(float(m), int(seed))
        assert hashlib.sha256(flow.tobytes()).hexdigest() == shas[k]
        np.testing.assert_array_equal(D.wheel_texel(flow[..., 0], float(m)), g["col"][k])
        np.testing.assert_array_equal(D.wheel_texel(flow[..., 1], float(m)), g["row"][k])


def test_probe_flows_cover_the_edges():
    flow = D.probe_flows(4.0, 32)
    assert np.isnan(flow).any() and np.isinf(flow).any()
    ix = D.wheel_texel(flow[..., 0], 4.0)
    assert ix.min() == 0 and ix.max() == 255 and len(np.unique(ix)) == 256


def test_default_wheel_is_the_middlebury_code():
    from flowfilter_b200 import color_wheel, lib

    w = color_wheel()
    assert w.shape == (256, 256, 4) and w.dtype == np.uint8
    np.testing.assert_array_equal(w, D.middlebury_wheel())
    assert (w[..., 3] == 255).all()
    # NULL output buffer is refused
    assert lib().ff_color_wheel_default(ctypes.c_void_p(0)) != 0
