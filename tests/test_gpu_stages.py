"""Stage kernels through the C ABI against the oracle and the reference's own outputs."""

from __future__ import annotations

import json

import numpy as np
import pytest

import oracle as O
from conftest import golden_stages
from make_reference_fixtures import sha, stage_inputs

pytestmark = pytest.mark.gpu

SIZES = [(1, 1), (1, 7), (7, 1), (2, 3), (5, 7), (33, 65), (48, 64), (53, 70)]


def bits_equal(a, b):
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    return a.shape == b.shape and a.dtype == b.dtype and a.tobytes() == b.tobytes()


def rand_inputs(h, w, seed):
    rng = np.random.default_rng(seed)
    return dict(
        img_u8=rng.integers(0, 256, (h, w), dtype=np.uint8),
        img_f32=rng.uniform(0, 1, (h, w)).astype(np.float32),
        flow=rng.normal(0, 1.5, (h, w, 2)).astype(np.float32),
        scalar=rng.uniform(0, 1, (h, w)).astype(np.float32),
        vector=rng.normal(0, 0.8, (h, w, 2)).astype(np.float32),
        a0=rng.uniform(0, 1, (h, w)).astype(np.float32),
        grad=rng.normal(0, 0.05, (h, w, 2)).astype(np.float32),
        a0old=rng.uniform(0, 1, (h, w)).astype(np.float32),
        coarse=rng.normal(0, 1.0, (max(h // 2, 1), max(w // 2, 1), 2)).astype(np.float32),
    )


@pytest.fixture(scope="module")
def st(cuda):
    from flowfilter_b200 import stages

    return stages


def dev(cuda, a):
    return cuda.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("h,w", SIZES)
def test_pyramid_down(cuda, st, h, w):
    x = rand_inputs(h, w, 1)
    for k in ("img_u8", "img_f32"):
        if h < 2 or w < 2:
            assert st.pyramid_down(dev(cuda, x[k])).numel() == 0
            continue
        got = st.pyramid_down(dev(cuda, x[k])).cpu().numpy()
        assert bits_equal(got, O.pyramid_down(x[k]))


@pytest.mark.parametrize("h,w", SIZES)
def test_image_model(cuda, st, h, w):
    x = rand_inputs(h, w, 2)
    for k in ("img_u8", "img_f32"):
        a0, g = st.image_model(dev(cuda, x[k]))
        ra0, rg = O.image_model(x[k])
        assert bits_equal(a0.cpu().numpy(), ra0)
        assert bits_equal(g.cpu().numpy(), rg)


@pytest.mark.parametrize("h,w", SIZES)
@pytest.mark.parametrize("n,border", [(1, 3), (2, 0), (3, 3), (5, 1), (2, 40)])
def test_propagate(cuda, st, h, w, n, border):
    x = rand_inputs(h, w, 3)
    got = st.propagate(dev(cuda, x["flow"]), n, border).cpu().numpy()
    assert bits_equal(got, O.propagate(x["flow"], n, border))
    f, s, v = st.propagate_payload(dev(cuda, x["flow"]), dev(cuda, x["scalar"]), dev(cuda, x["vector"]), n, border)
    rf, rs, rv = O.propagate_payload(x["flow"], x["scalar"], x["vector"], n, border)
    assert bits_equal(f.cpu().numpy(), rf)
    assert bits_equal(s.cpu().numpy(), rs)
    assert bits_equal(v.cpu().numpy(), rv)


@pytest.mark.parametrize("h,w", SIZES)
@pytest.mark.parametrize("gamma,maxflow", [(10 / 65025, 4.0), (1.0, 1.0), (0.05, 0.5)])
def test_updates(cuda, st, h, w, gamma, maxflow):
    x = rand_inputs(h, w, 4)
    f, im = st.update(*(dev(cuda, x[k]) for k in ("a0", "grad", "a0old", "flow")), gamma, maxflow)
    rf, ri = O.update(x["a0"], x["grad"], x["a0old"], x["flow"], gamma, maxflow)
    assert bits_equal(f.cpu().numpy(), rf)
    assert bits_equal(im.cpu().numpy(), ri)
    f, d, im = st.delta_update(*(dev(cuda, x[k]) for k in ("a0", "grad", "a0old", "vector", "coarse")), gamma, maxflow)
    rf, rd, ri = O.delta_update(x["a0"], x["grad"], x["a0old"], x["vector"], x["coarse"], gamma, maxflow)
    assert bits_equal(f.cpu().numpy(), rf)
    assert bits_equal(d.cpu().numpy(), rd)
    assert bits_equal(im.cpu().numpy(), ri)


def test_update_non_finite_inputs(cuda, st):
    """inf/NaN solutions are zeroed (update_k.cu:70-71, 137-138); clamps follow fminf/fmaxf."""
    x = rand_inputs(16, 24, 5)
    x["grad"][0, :5] = [[np.inf, 0], [np.nan, 1], [0, np.inf], [1e30, 1e30], [-np.inf, np.nan]]
    x["a0"][1, :3] = [np.nan, np.inf, -np.inf]
    x["flow"][2, :2] = [[np.nan, 0], [np.inf, -np.inf]]
    x["vector"][2, :2] = [[np.nan, 0], [np.inf, -np.inf]]
    x["coarse"][0, 0] = [np.nan, np.inf]
    for gamma in (1e-30, 1.0):
        f, im = st.update(*(dev(cuda, x[k]) for k in ("a0", "grad", "a0old", "flow")), gamma, 2.0)
        rf, ri = O.update(x["a0"], x["grad"], x["a0old"], x["flow"], gamma, 2.0)
        assert bits_equal(f.cpu().numpy(), rf)
        np.testing.assert_array_equal(im.cpu().numpy(), ri)
        f, d, im = st.delta_update(*(dev(cuda, x[k]) for k in ("a0", "grad", "a0old", "vector", "coarse")), gamma, 2.0)
        rf, rd, ri = O.delta_update(x["a0"], x["grad"], x["a0old"], x["vector"], x["coarse"], gamma, 2.0)
        assert bits_equal(f.cpu().numpy(), rf)
        assert bits_equal(d.cpu().numpy(), rd)
        assert np.all(np.isfinite(f.cpu().numpy()))


@pytest.mark.parametrize("h,w", SIZES)
@pytest.mark.parametrize("s", [1, 2, 4])
def test_smooth(cuda, st, h, w, s):
    x = rand_inputs(h, w, 6)
    assert bits_equal(st.smooth(dev(cuda, x["flow"]), s).cpu().numpy(), O.smooth(x["flow"], s))


def test_stages_match_reference_library(cuda, st):
    """The same inputs the reference library ran on (tests/golden/ref_stages.npz)."""
    ins = stage_inputs()
    outs = golden_stages()
    assert {k: sha(v) for k, v in ins.items()} == json.loads(bytes(outs.pop("inputs_sha256")).decode())
    d = {k: dev(cuda, v) for k, v in ins.items()}
    for kind in ("u8", "f32"):
        a0, g = st.image_model(d["img_" + kind])
        assert bits_equal(a0.cpu().numpy(), outs[f"model_{kind}_a0"])
        assert bits_equal(g.cpu().numpy(), outs[f"model_{kind}_grad"])
        x = d["img_" + kind]
        for lv in range(1, 4):
            x = st.pyramid_down(x)
            assert bits_equal(x.cpu().numpy(), outs[f"pyr_{kind}_l{lv}"])
    for n in range(1, 5):
        for b in (3, 0):
            assert bits_equal(st.propagate(d["flow"], n, b).cpu().numpy(), outs[f"prop_n{n}_b{b}"])
        f, s, v = st.propagate_payload(d["flow"], d["scalar"], d["vector"], n, 3)
        assert bits_equal(f.cpu().numpy(), outs[f"prop_payload_n{n}_flow"])
        assert bits_equal(s.cpu().numpy(), outs[f"prop_payload_n{n}_scalar"])
        assert bits_equal(v.cpu().numpy(), outs[f"prop_payload_n{n}_vector"])
    gammas = [np.float32(10.0) / np.float32(255.0 * 255.0), 1.0, 0.05]
    maxflows = [4.0, 1.0, 0.5]
    for k in range(3):
        f, im = st.update(d["a0"], d["grad"], d["a0old"], d["flow"], float(gammas[k]), maxflows[k])
        assert bits_equal(f.cpu().numpy(), outs[f"update_k{k}_flow"])
        f, dd, im = st.delta_update(d["a0"], d["grad"], d["a0old"], d["vector"], d["coarse"], float(gammas[k]),
                                    maxflows[k])
        assert bits_equal(f.cpu().numpy(), outs[f"dupdate_k{k}_flow"])
        assert bits_equal(dd.cpu().numpy(), outs[f"dupdate_k{k}_delta"])
    for s in range(1, 4):
        assert bits_equal(st.smooth(d["flow"], s).cpu().numpy(), outs[f"smooth_s{s}"])


def test_stage_input_validation(cuda, st):
    with pytest.raises(ValueError):
        st.image_model(cuda.zeros((4, 4), dtype=cuda.int32, device="cuda"))
    with pytest.raises(ValueError):
        st.propagate(cuda.zeros((4, 4, 3), device="cuda"), 1)
    with pytest.raises(ValueError):
        st.propagate(cuda.zeros((4, 4, 2), device="cuda"), 0)
    with pytest.raises(ValueError):
        st.smooth(cuda.zeros((4, 4, 2)), 1)  # host tensor
