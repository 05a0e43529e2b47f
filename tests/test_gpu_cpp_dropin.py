"""The C++ drop-in classes (include/flowfilter/gpu/*.h, libflowfilter_gpu.so) driven by a
C++ program the way the reference's demos use the reference classes, against the oracle."""

from __future__ import annotations

import os
import subprocess

import numpy as np
import pytest

import oracle as O
from oracle import display_oracle as D
from conftest import ROOT
from make_reference_fixtures import case_frames

pytestmark = pytest.mark.gpu

PKG = os.path.join(ROOT, "optical-flow-filter_b200", "flowfilter_b200")


@pytest.fixture(scope="module")
def program(cuda, tmp_path_factory):
    out = str(tmp_path_factory.mktemp("dropin") / "dropin_sequence")
    cmd = ["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "dropin_sequence.cpp"), "-o", out,
           "-L", PKG, "-lflowfilter_gpu", "-Wl,-rpath," + PKG]
    subprocess.run(cmd, check=True)
    return out


@pytest.mark.parametrize("h,w,levels", [(45, 61, 0), (96, 128, 2), (98, 150, 3)])
def test_cpp_dropin_sequence_matches_oracle(program, tmp_path, h, w, levels):
    t = 6
    frames = case_frames(dict(seq="bumps", frames=t, kw=dict(height=h, width=w, sigma=1.0, seed=h + w, n_bumps=2,
                                                              bump_sigma=max(h, w) / 3, amp=2.0)))
    fin, fout, fcol = tmp_path / "frames.u8", tmp_path / "out.f32", tmp_path / "colour.u8"
    frames.tofile(fin)
    r = subprocess.run([program, str(fin), str(h), str(w), str(t), str(levels), str(fout), str(fcol)],
                       capture_output=True, text=True)
    assert r.returncode == 0, (r.returncode, r.stderr)
    got = np.fromfile(fout, np.float32)
    if levels == 0:
        of = O.Filter.flowfilter(h, w, 2, 4.0, 10.0)
    else:
        of = O.Filter.pyramidal(h, w, levels)
        of.set_gammas([5.0 * 2 ** l for l in range(levels)])
        of.set_smooths([1 + l % 3 for l in range(levels)])
        of.set_max_flow(4.0)
    n2, n1 = h * w * 2, h * w
    off = 0
    for k in range(t):
        of.load(frames[k])
        of.compute()
        np.testing.assert_array_equal(got[off:off + n2].reshape(h, w, 2), of.flow()); off += n2
        np.testing.assert_array_equal(got[off:off + n2].reshape(h, w, 2), of.get_flow()); off += n2
        np.testing.assert_array_equal(got[off:off + n1].reshape(h, w), of.image()); off += n1
    a0, grad = O.image_model(frames[-1])
    np.testing.assert_array_equal(got[off:off + n1].reshape(h, w), a0); off += n1
    np.testing.assert_array_equal(got[off:off + n2].reshape(h, w, 2), grad); off += n2
    assert off == got.size
    # FlowToColor(filter.getFlow(), 4) with the library's wheel
    colour = np.fromfile(fcol, np.uint8).reshape(h, w, 4)
    np.testing.assert_array_equal(colour, D.flow_to_color(of.get_flow(), 4.0, D.reference_wheel()))


@pytest.mark.parametrize("h,w,d,n", [(45, 61, 1, 3), (50, 70, 4, 18)])
def test_cpp_dropin_rotation_matches_oracle(cuda, tmp_path, h, w, d, n):
    """The C++ camera, RotationalFlowImagePredictor and LaxWendroffPropagator classes."""
    prog = str(tmp_path / "dropin_rotation")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "dropin_rotation.cpp"), "-o", prog, "-L", PKG,
                    "-lflowfilter_gpu", "-Wl,-rpath," + PKG], check=True)
    img = np.random.default_rng(h + w + d).random((h, w) if d == 1 else (h, w, d)).astype(np.float32)
    fin, fout = tmp_path / "img.f32", tmp_path / "out.f32"
    img.tofile(fin)
    r = subprocess.run([prog, str(fin), str(h), str(w), str(d), str(n), str(fout)], capture_output=True, text=True)
    assert r.returncode == 0, (r.returncode, r.stderr)
    got = np.fromfile(fout, np.float32)
    cam = O.camera_perspective(0.004, h, w, 0.003, 0.004)
    np.testing.assert_array_equal(got[:4], cam)
    flow = O.rotational_flow(cam, 0.01, -0.02, 0.03, h, w)
    pred = O.lax_wendroff(flow, img, n)
    n2, nd = h * w * 2, h * w * d
    np.testing.assert_array_equal(got[4:4 + n2].reshape(flow.shape), flow)
    np.testing.assert_array_equal(got[4 + n2:4 + n2 + nd].reshape(img.shape), pred)
    np.testing.assert_array_equal(got[4 + n2 + nd:].reshape(img.shape), pred)


@pytest.fixture(scope="module")
def stages_program(cuda, tmp_path_factory):
    out = str(tmp_path_factory.mktemp("dropin") / "dropin_stages")
    cmd = ["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "dropin_stages.cpp"), "-o", out,
           "-L", PKG, "-lflowfilter_gpu", "-Wl,-rpath," + PKG]
    subprocess.run(cmd, check=True)
    return out


@pytest.mark.parametrize("name", ["constant_320x240_L1", "small_96x64_L2", "odd_150x98_L3"])
def test_cpp_stage_classes_rebuild_the_reference_filters(stages_program, tmp_path, name):
    """FlowSmoother, ImagePyramid, FlowPropagator[Payload], [Delta]FlowUpdate and ImageModel
    wired into the reference's filters by a C++ program: the flows of the reference library,
    bit for bit (sha256 per dumped frame)."""
    from conftest import golden_case
    from make_reference_fixtures import CASES, sha

    case = CASES[name]
    meta, _ = golden_case(name)
    frames = case_frames(case)
    t, h, w = frames.shape
    fin, fout = tmp_path / "frames.u8", tmp_path / "flows.f32"
    frames.tofile(fin)
    r = subprocess.run([stages_program, str(fin), str(h), str(w), str(t), str(case["levels"]), repr(case["maxflow"]),
                        ",".join(repr(g) for g in case["gamma"]), ",".join(str(s) for s in case["smooth"]), str(fout)],
                       capture_output=True, text=True)
    assert r.returncode == 0, (r.returncode, r.stderr)
    flows = np.fromfile(fout, np.float32).reshape(t, h, w, 2)
    assert [sha(flows[k]) for k in sorted(set(case["dump"]))] == meta["flow_sha256"]
