"""bench.py --config: every configuration selectable on its own; the reference arm's lines
for them on CPU (the oracle port), and the inputs of the 320x240 configuration pinned to the
parity fixture's frames (runs without a GPU)."""

from __future__ import annotations

import hashlib
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT

sys.path.insert(0, ROOT)
import bench  # noqa: E402


def run_reference(config, steps=3):
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    env.pop("RANK", None)
    env.pop("WORLD_SIZE", None)
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--config",
                        str(config), "--steps", str(steps), "--warmup", "3"],
                       env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_every_config_names_a_workload_or_leg():
    assert sorted(bench.CONFIGS) == [0, 1, 2, 3, 4]
    assert bench.CONFIGS[2] == bench.PRIMARY
    for c in (0, 1, 2):
        assert bench.CONFIGS[c] in bench.WORKLOADS
    assert bench.metric_of("constant_320x240_L1").startswith("frames/s (FlowFilter forward")
    assert bench.metric_of(bench.PRIMARY) == bench.METRIC


def test_config0_frames_are_the_parity_fixture_frames():
    """The 320x240 workload's 100-frame ring is the sequence the reference library's
    golden flows (tests/golden/ref_case_constant_320x240_L1.npz) were computed on."""
    w = bench.WORKLOADS["constant_320x240_L1"]
    frames = bench.make_frames(w)
    meta = json.loads(bytes(np.load(os.path.join(ROOT, "tests", "golden",
                                                  "ref_case_constant_320x240_L1.npz"))["meta"]).decode())
    assert frames.shape == (meta["frames"], 240, 320)
    assert hashlib.sha256(np.ascontiguousarray(frames).tobytes()).hexdigest() == meta["frames_sha256"]
    assert (meta["gamma"], meta["smooth"], meta["maxflow"]) == (w["gamma"], w["smooth"], w["maxflow"])


@pytest.mark.parametrize("config", [0, 1])
def test_reference_arm_times_the_selected_workload(config):
    name = bench.CONFIGS[config]
    line = run_reference(config, steps=3 if config == 0 else 2)
    assert line["impl"] == "reference"
    assert line["config"] == bench.bench_config(name)
    assert line["metric"] == bench.metric_of(name)
    assert line["value"] > 0 and line["cpu_baseline"]["kind"] == "port"
    assert line["e2e"]["value"] == line["value"]


@pytest.mark.parametrize("config", [3, 4])
def test_reference_arm_has_no_batched_or_gradient_path(config):
    line = run_reference(config)
    assert line["impl"] == "reference" and "unavailable" in line


@pytest.mark.gpu
def test_config0_line_on_the_gpu():
    """--config 0 on the GPU: a complete line for the 320x240 FlowFilter (device value,
    level-0 roofline, end-to-end, CPU port), launches counted."""
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--config", "0", "--steps", "50",
                        "--warmup", "3"], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-3000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["config"] == bench.bench_config("constant_320x240_L1")
    assert line["value"] > 0 and line["e2e"]["value"] > 0 and line["cpu_baseline"]["value"] > 0
    assert line["gpu_launches"] >= 50 and line["gpu_launches"] % 50 == 0  # the frame's launches x 50
    assert line["roofline"]["algorithmic_bytes"] == 240 * 320 * 25
    assert "batched" not in line and "extra" not in line
