"""The CPU oracle against outputs of the reference library itself (golden fixtures).

The fixtures were produced by running the reference's own stages and filters, built
from its sources for sm_100a, on a B200 (oracle/make_reference_fixtures.py).  The
oracle must reproduce them bit for bit.
"""

from __future__ import annotations

import json
import os

import numpy as np
import pytest

import oracle as O
from conftest import GOLDEN, golden_case, golden_stages
from make_reference_fixtures import CASES, case_frames, sha, stage_inputs, subsample_rows_cols


@pytest.fixture(scope="module")
def stage_data():
    ins = stage_inputs()
    outs = golden_stages()
    recorded = json.loads(bytes(outs.pop("inputs_sha256")).decode())
    assert {k: sha(v) for k, v in ins.items()} == recorded, "stage-input generator drifted"
    return ins, outs


def bits_equal(a, b):
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    return a.shape == b.shape and a.dtype == b.dtype and a.tobytes() == b.tobytes()


def test_norm_table_matches_texture_reads():
    ref = np.load(os.path.join(GOLDEN, "ref_norm_u8.npy"))
    assert bits_equal(O.norm_table(), ref)
    assert bits_equal(ref, np.arange(256, dtype=np.float32) / np.float32(255.0))


def test_upmap_index_matches_texture_unit():
    d = np.load(os.path.join(GOLDEN, "ref_upmap_detail.npy"))
    i = 0
    n = 0
    while i < len(d):
        _, w, wc = int(d[i]), int(d[i + 1]), int(d[i + 2])
        idx = d[i + 3:i + 3 + w]
        i += 3 + w
        got = np.array([O.upmap_index(x, w, wc) for x in range(w)])
        assert np.array_equal(got, idx), (w, wc)
        n += 1
    assert n >= 50


@pytest.mark.parametrize("level", [1, 2, 3])
@pytest.mark.parametrize("kind", ["u8", "f32"])
def test_pyramid(stage_data, level, kind):
    ins, outs = stage_data
    x = ins["img_u8" if kind == "u8" else "img_f32"]
    for _ in range(level):
        x = O.pyramid_down(x)
    assert bits_equal(x, outs[f"pyr_{kind}_l{level}"])


@pytest.mark.parametrize("kind", ["u8", "f32"])
def test_image_model(stage_data, kind):
    ins, outs = stage_data
    a0, g = O.image_model(ins["img_u8" if kind == "u8" else "img_f32"])
    assert bits_equal(a0, outs[f"model_{kind}_a0"])
    assert bits_equal(g, outs[f"model_{kind}_grad"])


@pytest.mark.parametrize("n", [1, 2, 3, 4])
@pytest.mark.parametrize("border", [3, 0])
def test_propagate(stage_data, n, border):
    ins, outs = stage_data
    assert bits_equal(O.propagate(ins["flow"], n, border), outs[f"prop_n{n}_b{border}"])


@pytest.mark.parametrize("n", [1, 2, 3, 4])
def test_propagate_payload(stage_data, n):
    ins, outs = stage_data
    f, s, v = O.propagate_payload(ins["flow"], ins["scalar"], ins["vector"], n, 3)
    assert bits_equal(f, outs[f"prop_payload_n{n}_flow"])
    assert bits_equal(s, outs[f"prop_payload_n{n}_scalar"])
    assert bits_equal(v, outs[f"prop_payload_n{n}_vector"])


GAMMAS = [np.float32(10.0) / np.float32(255.0 * 255.0), 1.0, 0.05]
MAXFLOWS = [4.0, 1.0, 0.5]


@pytest.mark.parametrize("k", [0, 1, 2])
def test_update(stage_data, k):
    ins, outs = stage_data
    f, im = O.update(ins["a0"], ins["grad"], ins["a0old"], ins["flow"], GAMMAS[k], MAXFLOWS[k])
    assert bits_equal(f, outs[f"update_k{k}_flow"])
    assert bits_equal(im, outs[f"update_k{k}_image"])


@pytest.mark.parametrize("k", [0, 1, 2])
def test_delta_update(stage_data, k):
    ins, outs = stage_data
    f, d, im = O.delta_update(ins["a0"], ins["grad"], ins["a0old"], ins["vector"], ins["coarse"], GAMMAS[k], MAXFLOWS[k])
    assert bits_equal(f, outs[f"dupdate_k{k}_flow"])
    assert bits_equal(d, outs[f"dupdate_k{k}_delta"])
    assert bits_equal(im, outs[f"dupdate_k{k}_image"])


@pytest.mark.parametrize("s", [1, 2, 3])
def test_smooth(stage_data, s):
    ins, outs = stage_data
    assert bits_equal(O.smooth(ins["flow"], s), outs[f"smooth_s{s}"])


@pytest.mark.parametrize("name", list(CASES))
def test_sequence_bit_exact(name):
    """Whole filters over multi-frame sequences: FlowFilter and PyramidalFlowFilter."""
    case = CASES[name]
    meta, arr = golden_case(name)
    frames = case_frames(case)
    assert sha(frames) == meta["frames_sha256"], "sequence generator drifted"
    O.set_threads(8)
    try:
        flows = O.run_case(case, frames)
    finally:
        O.set_threads(0)
    assert [sha(f) for f in flows] == meta["flow_sha256"]
    if meta["layout"] == "full":
        assert np.array_equal(flows, arr["flow"])
    else:
        rows, cols = subsample_rows_cols(*frames.shape[1:])
        assert np.array_equal(flows[:, rows][:, :, cols], arr["flow"])
