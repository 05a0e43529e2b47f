"""The 2048x1088 three-level throughput workload over its full 1000-frame sequence, bit for bit
against the reference library run on the same frames (every frame's flow hashed by sha256).

A long recurrence with discontinuous branches (upwind selects, clamps, the pyramid's uint8
truncation) is where a one-ulp difference would show up late, so every frame is compared,
with the streaming and the tile-fused level-0 kernels."""

from __future__ import annotations

import hashlib
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN
from make_reference_fixtures import LONG_CASES, long_frames

pytestmark = pytest.mark.gpu


def long_golden(name):
    path = os.path.join(GOLDEN, f"ref_long_{name}.npz")
    if not os.path.exists(path):
        pytest.skip(f"no reference fixture {os.path.basename(path)}")
    z = np.load(path)
    meta = json.loads(bytes(z["meta"]).decode())
    return meta, {k: z[k] for k in z.files if k != "meta"}


@pytest.mark.parametrize("name", list(LONG_CASES))
def test_long_sequence_bit_exact_every_frame(cuda, name):
    import flowfilter_b200 as ffb

    case = LONG_CASES[name]
    meta, arr = long_golden(name)
    filters = {}
    for mode in (1, 3):  # streaming and tile-fused kernels
        f = ffb.PyramidalFlowFilter(1088, 2048, case["levels"])
        f.gamma = case["gamma"]
        f.smoothIterations = case["smooth"]
        f.maxflow = case["maxflow"]
        f.setFused(mode)
        filters[mode] = f
    frames_sha = hashlib.sha256()
    first_bad = {m: None for m in filters}
    rows, cols = arr["rows"], arr["cols"]
    keep = [int(k) for k in arr["keep"]]
    flow = np.empty((1088, 2048, 2), np.float32)
    keep_err = {}
    n = 0
    for t, frame in enumerate(long_frames(case)):
        frames_sha.update(frame.tobytes())
        for mode, f in filters.items():
            f.loadImage(frame)
            f.compute()
            f.getFlow(flow)
            if first_bad[mode] is None and hashlib.sha256(flow.tobytes()).digest() != arr["digests"][t].tobytes():
                first_bad[mode] = t
            if t in keep:
                err = float(np.max(np.abs(flow[rows][:, cols] - arr["flow"][keep.index(t)])))
                keep_err[(mode, t)] = err
        n += 1
    assert n == case["frames"] == arr["digests"].shape[0]
    assert frames_sha.hexdigest() == meta["frames_sha256"], "the frame generator drifted"
    assert all(e <= 1e-4 for e in keep_err.values()), keep_err  # the stated tolerance ...
    assert first_bad == {1: None, 3: None}, f"first frame whose flow differs, per kernel mode: {first_bad}"
