"""Time the reference's own NumPy/SciPy CPU path (test infrastructure, for information only).

The reference ships a pure-NumPy filter (python/flowfilter/flowfilter.py: SimpleFlowFilter
:91-221, PyramidalFlowFilter :381-575) beside its CUDA library.  It is a different algorithm
from the CUDA path (SciPy 'reflect' borders against clamp-to-edge, a '>=' dominant-flow test
in propagation.py:88 against '>' in propagation_k.cu:40, a truncation to +-propIterations in
place of the +-maxflow clamp, a 3x3 binomial pyramid with bilinear upsampling), so it is not
a parity oracle; this script reports its speed and how far its flow lies from the reference
CUDA library's on the same frames (the committed fixtures tests/golden/ref_case_*.npz).

It imports the reference package from its checkout, named by FLOWFILTER_REFERENCE (the
directory holding python/flowfilter), with three import-time shims for names that current
Python and NumPy removed: collections.Iterable, numpy.float and time.clock.  The reference's
files are not modified.  It cannot run where the checkout is absent.

    FLOWFILTER_REFERENCE=<checkout> python oracle/time_numpy_reference.py [--frames-rotzoom N]

Configurations (the same sequences as the parity fixtures):
  constant_320x240_L1   SimpleFlowFilter(propIterations=4, gamma=10, smoothIterations=1), 100 frames
  rotzoom_640x480_L2    PyramidalFlowFilter(levels=2, propIterations=4, gamma=[10, 50],
                        smoothIterations=[2, 4], maxflow=2), 300 frames
Images are passed as float32 in 0..255 (the CUDA path's u8 normalisation and gamma/255^2
scaling are the same solve in those units).
"""

from __future__ import annotations

import argparse
import collections
import collections.abc
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "optical-flow-filter_b200"))

from flowfilter_b200 import synthetic  # noqa: E402


def import_reference():
    ref = os.environ.get("FLOWFILTER_REFERENCE", "")
    pkg = os.path.join(ref, "python")
    if not ref or not os.path.isdir(os.path.join(pkg, "flowfilter")):
        raise SystemExit("set FLOWFILTER_REFERENCE to the reference checkout (the directory holding python/flowfilter)")
    # names removed from Python 3.10 / NumPy 1.24 / Python 3.8 that the module still uses
    collections.Iterable = collections.abc.Iterable
    np.float = float
    time.clock = time.perf_counter
    sys.path.insert(0, pkg)
    from flowfilter import flowfilter as ff  # noqa: E402
    return ff


def run(ff, name, frames):
    fixture = np.load(os.path.join(ROOT, "tests", "golden", f"ref_case_{name}.npz"))
    meta = json.loads(bytes(fixture["meta"]).decode())
    dump = list(meta["dump"])
    if name == "constant_320x240_L1":
        seq = synthetic.sequence("constant", frames=frames)
        filt = ff.SimpleFlowFilter(propIterations=4, gamma=10.0, smoothIterations=1)
    else:
        seq = synthetic.sequence("rotzoom", frames=frames)
        filt = ff.PyramidalFlowFilter(levels=2, propIterations=4, gamma=[10.0, 50.0],
                                      smoothIterations=[2, 4], maxflow=2.0)
    rows, cols = fixture["rows"], fixture["cols"]
    times, diffs = [], []
    for t in range(frames):
        img = seq[t].astype(np.float32)
        t0 = time.perf_counter()
        filt.loadImage(img)
        filt.compute()
        times.append(time.perf_counter() - t0)
        if t in dump:
            flow = np.asarray(filt.getFlow(), np.float32)[np.ix_(rows, cols)]
            ref = fixture["flow"][dump.index(t)]
            d = flow - ref
            diffs.append({"frame": t, "max_abs_px": float(np.abs(d).max()),
                          "mean_epe_px": float(np.sqrt((d ** 2).sum(-1)).mean())})
    H, W = seq.shape[1:]
    steady = np.asarray(times[1:]) if frames > 1 else np.asarray(times)
    ms = float(np.median(steady) * 1e3)
    return {"workload": name, "frames": frames, "ms_per_frame_median": ms, "fps": 1e3 / ms,
            "mpix_per_s": H * W / ms / 1e3, "threads": 1,
            "vs_reference_cuda": diffs}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--frames-rotzoom", type=int, default=300)
    args = ap.parse_args()
    ff = import_reference()
    out = {"path": "reference NumPy/SciPy filter (python/flowfilter/flowfilter.py), one process",
           "cases": [run(ff, "constant_320x240_L1", 100),
                     run(ff, "rotzoom_640x480_L2", args.frames_rotzoom)]}
    print(json.dumps(out))


if __name__ == "__main__":
    main()
