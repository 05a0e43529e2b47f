"""Flow colour encoding, CPU side: the oracle's texel choice against the reference's own
lookup kernel (fixture made on a B200 by oracle/make_reference_fixtures.py), and the
library's default colour wheel: the reference's own table, byte for byte."""

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


def test_default_wheel_is_the_reference_table():
    """ff_color_wheel_default gives the reference's 256x256 RGBA table (src/colorwheel.cpp,
    COLOR_WHEEL_D): the sha256 below is that of the table read from the reference source."""
    from flowfilter_b200 import color_wheel, lib

    w = color_wheel()
    assert w.shape == (256, 256, 4) and w.dtype == np.uint8
    assert hashlib.sha256(w.tobytes()).hexdigest() == \
        "966163576b67b0a8dfee44fd06e692f64572f7c92291fb4c2eae56c353ddea03"
    np.testing.assert_array_equal(w, D.reference_wheel())
    assert (w[..., 3] == 255).all()
    # NULL output buffer is refused
    assert lib().ff_color_wheel_default(ctypes.c_void_p(0)) != 0


def test_reference_colours_on_the_probes():
    """Default colours of the probe flows: the reference's table at the texel the reference's
    own lookup kernel read (fixture), i.e. the reference's FlowToColor output bytes."""
    g = np.load(FIXTURE)
    w = D.reference_wheel()
    for k, (m, seed) in enumerate(zip(g["maxflow"], g["seed"])):
        flow = D.probe_flows(float(m), int(seed))
        np.testing.assert_array_equal(D.flow_to_color(flow, float(m), w), w[g["row"][k], g["col"][k]])
