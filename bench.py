#!/usr/bin/env python
"""Throughput benchmark of the flow-filter hot path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl {b200,reference}] [--config {0,1,2,3,4}]
    python bench.py --profile WORKLOAD --steps K --warmup W     (profiler target only)
    python bench.py --profile-next --steps K --warmup W         (profiler target: FlowToColor, rotation)
    python bench.py --profile-batched --steps K --warmup W      (profiler target: the 64-stream batched step)
    python bench.py --profile-diff --steps K --warmup W         (profiler target: the differentiable filter)

A step is one frame of the PyramidalFlowFilter: the frame (already resident in HBM) is
loaded into the filter and one compute() runs (pyramid, then one fused kernel per
level; CUDA-graph replay).  The primary workload is the throughput run: 2048x1088 uint8
frames (the camera-sensor size), 3 levels, gamma [5, 20, 50], smoothing [1, 2, 4],
maxflow 4, on a seeded synthetic sequence (blurred noise plus sensor noise, moved by a
smooth field of Gaussian bumps).  The reference's published configuration (640x480,
2 levels, gamma [10, 50], smoothing [2, 4], on a seeded rotation+zoom sequence standing in
for the reference's Blender sequence) is reported beside it under "extra", the 64-stream
mixed-size batched step (BatchFlowFilter, against the same 64 streams looped as single
filters) under "batched", and the differentiable filter's forward and forward+backward
time under "differentiable".

Timing: every step is bracketed by CUDA events on the filter's stream and the L2 is
flushed (a 256 MiB write) between steps outside those events, so every frame reads its
state from HBM.  value = frames of all ranks / max over ranks of the summed step time.
--gpus N runs N independent replicas (one process per GPU, torch.distributed for the
barrier and the max over ranks); the path does not shard.

--config N prints one configuration's line alone: 0 the single-level FlowFilter at 320x240
(gamma 10, smoothing 1, maxflow 4, a constant translation of (0.7, -0.4) px/frame), 1 the
reference's published 640x480 configuration, 2 the default run above, 3 the batched step,
4 the differentiable filter (forward+backward frames/s).

--impl reference times the reference's CPU path restated in C++ (oracle/, the same
arithmetic as the reference kernels) on all host cores: the reference has no CPU
implementation of its CUDA path, and its NumPy module is a different algorithm.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "optical-flow-filter_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

WORKLOADS = {
    # single-level FlowFilter on a constant translation (the reference's CPU-runnable case)
    "constant_320x240_L1": dict(seq="constant", H=240, W=320, levels=1, gamma=[10.0], smooth=[1], maxflow=4.0,
                                ring=100, filter="FlowFilter"),
    # the reference's published notebook configuration (notebooks/GPU_example.ipynb)
    "rotzoom_640x480_L2": dict(seq="rotzoom", H=480, W=640, levels=2, gamma=[10.0, 50.0], smooth=[2, 4],
                               maxflow=4.0, ring=96),
    # camera-sensor size, 3 levels (throughput / roofline run)
    "bumps_2048x1088_L3": dict(seq="bumps", H=1088, W=2048, levels=3, gamma=[5.0, 20.0, 50.0], smooth=[1, 2, 4],
                               maxflow=4.0, ring=24),
}
# the throughput and roofline workload: camera-sensor size, 3 levels
PRIMARY = "bumps_2048x1088_L3"
# the reference's published configuration, reported beside it
EXTRA = "rotzoom_640x480_L2"
METRIC = "frames/s (PyramidalFlowFilter forward, flow err <= 1e-4 px vs reference)"
# --config N: 0-2 one filter workload each, 3 the 64-stream batched step, 4 the differentiable filter
CONFIGS = {0: "constant_320x240_L1", 1: "rotzoom_640x480_L2", 2: "bumps_2048x1088_L3", 3: "batched", 4: "differentiable"}


def metric_of(name):
    w = WORKLOADS[name]
    return METRIC.replace("PyramidalFlowFilter", w.get("filter", "PyramidalFlowFilter"))
# reference notebook: 1.172 ms/frame on its textured sequence for the 640x480 2-level
# configuration (notebooks/GPU_example.ipynb:292); 0.996 ms/frame on all-zero frames (:400).
# Nothing is published for 2048x1088.
PUBLISHED_FPS = {"rotzoom_640x480_L2": 1000.0 / 1.172}
FLUSH_BYTES = 256 << 20
L2_NOTE = "flushed between steps (256 MiB write outside the step events)"
SEQUENCE = {
    "constant": "seeded blurred noise (sigma 2, seed 0) translated by (0.7, -0.4) px/frame",
    "rotzoom": "seeded blurred noise (sigma 1.5, seed 1), rotation 0.5 deg + zoom 1.004 per frame",
    "bumps": "seeded blurred noise (sigma 1, seed 2) + N(0, 3 DN) sensor noise, flow = 8 Gaussian bumps "
             "(sigma 150 px, amplitude U[-3, 3] px/frame)",
}


def bench_config(name):
    """The workload as both arms print it (identical keys and values in both)."""
    w = WORKLOADS[name]
    out = {"workload": name, "frames": f"{w['W']}x{w['H']} uint8", "levels": w["levels"], "gamma": w["gamma"],
           "smoothIterations": w["smooth"], "maxflow": w["maxflow"], "l2": L2_NOTE}
    if "filter" in w:
        out["filter"] = w["filter"]
    return out


def level_shapes(w):
    h, wd = w["H"], w["W"]
    out = [(h, wd)]
    for _ in range(1, w["levels"]):
        h, wd = h // 2, wd // 2
        out.append((h, wd))
    return out


def frame_bytes(w):
    """Compulsory HBM bytes per frame: P0*1 + sum(delta) P_l*42 + P_top*24."""
    shapes = level_shapes(w)
    b = shapes[0][0] * shapes[0][1]
    for l, (h, wd) in enumerate(shapes):
        b += h * wd * (42 if l < len(shapes) - 1 else 24)
    return b


def level0_kernel_bytes(w):
    """Algorithmic bytes of one level-0 kernel launch: the uint8 frame (1 B/px) plus the
    delta level's state read and written and the coarse flow read (42 B/px)."""
    h, wd = w["H"], w["W"]
    return h * wd * (1 + (42 if w["levels"] > 1 else 24))


def kernels_per_frame(w, tuning: str) -> int:
    """Kernel launches of one frame: the pyramid (levels 1 and 2 in one launch, each deeper
    level one more), then per level one fused kernel (streaming or tile) or the per-stage
    kernels (model, 2N propagation passes, update, 2S smoothing passes)."""
    L = w["levels"]
    parts = [p.strip() for p in tuning.split(";")]
    # a two-level pyramid whose top level runs the tile kernel makes level 1 inside it
    if L == 2 and len(parts) > 1 and "tile" in parts[1]:
        n = 0
    else:
        n = L - 1 if L <= 2 else 1 + (L - 3)
    for l in range(L):
        m = w["maxflow"] / (2 ** min(l, L - 1))
        N = int(np.ceil(np.float32(m)))
        S = w["smooth"][l]
        fused = l < len(parts) and ("fused" in parts[l] or "tile" in parts[l])
        n += 1 if fused else 2 + 2 * N + 2 * S
    return n


def make_frames(w):
    from flowfilter_b200 import synthetic

    if w["seq"] == "constant":
        return synthetic.seq_constant(frames=w["ring"], height=w["H"], width=w["W"])
    if w["seq"] == "rotzoom":
        return synthetic.seq_rotzoom(frames=w["ring"], height=w["H"], width=w["W"])
    return synthetic.seq_bumps(frames=w["ring"], height=w["H"], width=w["W"])


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(name, key="dram_bytes_per_launch"):
    """A per-launch figure of the level-0 kernel from one ncu capture (profiles/)."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        d = json.load(f)
    v = d.get(name)
    return None if v is None or key not in v else float(v[key])


class ClockSampler:
    """SM clock and throttle reasons polled through NVML (read-only) every 2 ms while the
    timed region runs (no samples are reported when NVML is unavailable)."""

    # NVML clocks-event reason bits
    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown"}

    def __init__(self, gpu_uuid: str):
        self.uuid = gpu_uuid
        self.sm = []
        self.reasons = set()
        self.max_mhz = None
        self._stop = threading.Event()
        self._thread = None

    def __enter__(self):
        try:
            import pynvml

            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByUUID(self.uuid.encode() if isinstance(self.uuid, str) else self.uuid)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
            get_reasons = getattr(pynvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                pynvml.nvmlDeviceGetCurrentClocksThrottleReasons

            def poll():
                while not self._stop.is_set():
                    self.sm.append(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM))
                    bits = get_reasons(h)
                    for b, name in self.REASONS.items():
                        if bits & b:
                            self.reasons.add(name)
                    time.sleep(0.02)

            self._thread = threading.Thread(target=poll, daemon=True)
            self._thread.start()
        except Exception:
            self._thread = None
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._thread:
            self._thread.join(timeout=2)

    def summary(self):
        if not self.sm:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": [], "samples": 0, "source": "none"}
        return {"sm_mhz": statistics.median(self.sm), "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
                "samples": len(self.sm), "source": "nvml"}


def dist_backend() -> str:
    """NCCL between GPU ranks; gloo when there is no GPU (the CPU tests of the N>1 path)."""
    import torch

    return os.environ.get("FFB_DIST_BACKEND") or ("nccl" if torch.cuda.is_available() else "gloo")


def dist_setup():
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        backend = dist_backend()
        if backend == "nccl":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    elif torch.cuda.is_available():
        torch.cuda.set_device(local)
    return world, rank, local


def barrier(world):
    import torch

    if world > 1:
        import torch.distributed as dist

        dist.barrier()
    if torch.cuda.is_available():
        torch.cuda.synchronize()


def max_over_ranks(world, value: float) -> float:
    import torch

    if world == 1:
        return value
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(world: int, units_per_rank: int, max_ms: float) -> float:
    """Whole-job throughput: the units all ranks processed over the slowest rank's time."""
    return world * units_per_rank / (max_ms / 1000.0)


def gpu_uuid(local):
    import torch

    try:
        u = str(torch.cuda.get_device_properties(local).uuid)
        return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:
        return os.environ.get("CUDA_VISIBLE_DEVICES", str(local)).split(",")[local]


def make_filter(w):
    import flowfilter_b200 as ffb

    if w.get("filter") == "FlowFilter":
        f = ffb.FlowFilter(w["H"], w["W"])
        f.gamma = w["gamma"][0]
        f.smoothIterations = w["smooth"][0]
        f.maxflow = w["maxflow"]
        return f
    f = ffb.PyramidalFlowFilter(w["H"], w["W"], w["levels"])
    f.gamma = w["gamma"]
    f.smoothIterations = w["smooth"]
    f.maxflow = w["maxflow"]
    return f


TUNING_CACHE = os.path.join(os.path.expanduser("~"), ".cache", "flowfilter_b200", "tuning.json")


_LIB_DIGEST = None


def lib_digest():
    """sha256 prefix of the loaded libffb200.so: a tuning choice belongs to one build."""
    global _LIB_DIGEST
    if _LIB_DIGEST is None:
        import hashlib

        from flowfilter_b200 import _lib

        with open(_lib.LIB_PATH, "rb") as fh:
            _LIB_DIGEST = hashlib.sha256(fh.read()).hexdigest()[:16]
    return _LIB_DIGEST


def tuning_key(w):
    import torch

    return (f"{torch.cuda.get_device_name()}|{lib_digest()}|{w['H']}x{w['W']}|L{w['levels']}"
            f"|m{w['maxflow']}|s{w['smooth']}")


def load_tuning_cache():
    if os.path.exists(TUNING_CACHE):
        try:
            with open(TUNING_CACHE) as fh:
                return json.load(fh)
        except (OSError, ValueError):
            pass
    return {}


def store_tuning(key, state):
    cache = load_tuning_cache()
    cache[key] = state
    os.makedirs(os.path.dirname(TUNING_CACHE), exist_ok=True)
    with open(TUNING_CACHE, "w") as fh:
        json.dump(cache, fh, indent=1)


def tuned(f, w, key=None, flush=None):
    """Apply the cached autotuning result for this workload, GPU and library build, or
    autotune now (after the filter computed a frame) and cache it, so repeated runs of one
    build make the same choice."""
    key = key or tuning_key(w)
    cache = load_tuning_cache()
    if key in cache:
        f.setTuningState(cache[key])
        return
    f.autotune(5, flush)
    store_tuning(key, f.tuningState())


def pretune(w, dev_frames, flush, frames=9, rounds=3, timed_frames=60):
    """The kernel choice of workload w, made before any clock sampling and cached (the timed
    runs apply it through tuned()): `rounds` autotunes, each on a filter that computed
    `frames` frames, and of the choices they make the one whose frames run fastest in the
    bench's own timed loop (median of `timed_frames` frames, L2 flushed before each)."""
    import torch

    key = tuning_key(w)
    if key in load_tuning_cache():
        return
    ring = dev_frames.shape[0]
    best = None
    seen = []
    for _ in range(rounds):
        f = make_filter(w)
        for t in range(frames):
            f.loadImage(dev_frames[t % ring])
            f.computeAsync()
        torch.cuda.synchronize()
        f.autotune(5, flush)
        state = f.tuningState()
        if state in seen:
            continue
        seen.append(state)
        f.setGraphs(True)
        for t in range(5):
            f.loadImage(dev_frames[t % ring])
            f.computeAsync()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(timed_frames)]
        for k in range(timed_frames):
            flush.zero_()
            ev[k][0].record()
            f.loadImage(dev_frames[k % ring])
            f.computeAsync()
            ev[k][1].record()
        torch.cuda.synchronize()
        ms = sorted(a.elapsed_time(b) for a, b in ev)[timed_frames // 2]
        if best is None or ms < best[0]:
            best = (ms, state)
        del f
    store_tuning(key, best[1])


def device_run(w, dev_frames, steps, warmup, flush, graphs=True, profile=False, tune=True, label="timed"):
    """Device-timed frames; returns (summed step ms, per-level kernel ms or None, filter).

    The timed frames sit inside the NVTX range `label`, so a profiler can select them."""
    import torch

    f = make_filter(w)
    ring = dev_frames.shape[0]
    for t in range(warmup):
        f.loadImage(dev_frames[t % ring])
        f.computeAsync()
        if tune and t == 1:
            tuned(f, w, flush=flush)  # kernel choice per level on live data (results unchanged)
    f.setGraphs(graphs)
    torch.cuda.synchronize()
    if profile:
        f.setProfiling(steps)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    torch.cuda.nvtx.range_push(label)
    for k in range(steps):
        flush.zero_()
        ev[k][0].record()
        f.loadImage(dev_frames[(warmup + k) % ring])
        f.computeAsync()
        ev[k][1].record()
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    total = sum(a.elapsed_time(b) for a, b in ev)
    lv = None
    if profile:
        lv = [f.levelKernelTime(l) for l in range(w["levels"])]
    return total, lv, f


def e2e_run(w, frames, steps, warmup):
    """End to end through the public API with host buffers: every step uploads its frame from
    pinned host memory, computes, and downloads the smoothed flow into pinned host memory
    (PyramidalFlowFilter.processAsync: the three overlap across consecutive frames); the
    clock stops after synchronize() has delivered the last flow.  Wall-clock time."""
    import torch

    f = make_filter(w)
    ring = frames.shape[0]
    host = torch.from_numpy(frames).pin_memory()
    outs = [torch.empty((w["H"], w["W"], 2), dtype=torch.float32).pin_memory() for _ in range(4)]
    for t in range(warmup):
        f.processAsync(host[t % ring], outs[t % 4])
        if t == 1:
            f.synchronize()
            tuned(f, w)
    f.setGraphs(True)
    f.synchronize()
    t0 = time.perf_counter()
    for k in range(steps):
        f.processAsync(host[(warmup + k) % ring], outs[k % 4])
    f.synchronize()
    t1 = time.perf_counter()
    return (t1 - t0) * 1000.0


def oracle_filter(O, w):
    """The oracle's filter of a workload (the same kind and parameters as make_filter)."""
    if w.get("filter") == "FlowFilter":
        return O.Filter.flowfilter(w["H"], w["W"], smooth_iterations=w["smooth"][0], maxflow=w["maxflow"],
                                   gamma=w["gamma"][0])
    f = O.Filter.pyramidal(w["H"], w["W"], w["levels"])
    f.set_gammas(w["gamma"])
    f.set_smooths(w["smooth"])
    f.set_max_flow(w["maxflow"])
    return f


def cpu_port_fps(w, frames, seconds=10.0, max_frames=2000, threads=None):
    """The oracle (C++ restatement of the reference path) on the host cores."""
    import oracle as O

    threads = threads or os.cpu_count() or 1
    O.set_threads(threads)
    f = oracle_filter(O, w)
    ring = frames.shape[0]
    f.load(frames[0])
    f.compute()
    n = 0
    t0 = time.perf_counter()
    while n < max_frames and time.perf_counter() - t0 < seconds:
        f.load(frames[(n + 1) % ring])
        f.compute()
        n += 1
    dt = time.perf_counter() - t0
    O.set_threads(0)
    return n / dt, threads, n

BATCH_SIZES = [(240, 320), (480, 640), (720, 1280), (1080, 1920)]
BATCH_PER_SIZE = 16
BATCH_RING = 3


def batched_streams(seed=100):
    """64 streams, 16 at each size: levels in {1,2,3}, gamma log-uniform in [2, 100] per
    level, smoothing in {1..4} per level, maxflow 4 (seeded)."""
    rng = np.random.default_rng(seed)
    out = []
    for k, (h, w) in enumerate(BATCH_SIZES):
        for _ in range(BATCH_PER_SIZE):
            levels = int(rng.integers(1, 4))
            gamma = [float(np.exp(rng.uniform(np.log(2.0), np.log(100.0)))) for _ in range(levels)]
            smooth = [int(rng.integers(1, 5)) for _ in range(levels)]
            out.append(dict(H=h, W=w, levels=levels, gamma=gamma, smooth=smooth, maxflow=4.0, size=k))
    return out


def batched_sequences(streams, frames, ids=None):
    """Stream i's frames: the bump-flow sequence of its size from seed 100 + i (uint8
    [frames, H, W] each; ids: the streams' indices in the full mix), generated on a thread
    pool (numpy releases the GIL)."""
    from concurrent.futures import ThreadPoolExecutor

    from flowfilter_b200 import synthetic

    ids = list(range(len(streams))) if ids is None else list(ids)

    def one(k):
        s = streams[k]
        return synthetic.seq_bumps(frames=frames, height=s["H"], width=s["W"], seed=100 + ids[k])

    with ThreadPoolExecutor(min(8, os.cpu_count() or 1)) as ex:
        return list(ex.map(one, range(len(streams))))


def configure_stream(f, s):
    f.gamma = s["gamma"] if s["levels"] > 1 else s["gamma"][0]
    f.smoothIterations = s["smooth"] if s["levels"] > 1 else s["smooth"][0]
    f.maxflow = s["maxflow"]


def bench_batched(steps, warmup, world=1, rank=0):
    """The 64-stream mixed-size step: one BatchFlowFilter step against a loop that runs the
    64 streams one after another as single-stream filters (graph replay each), both over
    frames already in HBM.  The 64 streams' state (~1 GB) exceeds L2, so no flush.  With
    several ranks the 64 streams are split over them (BatchFlowFilter.shard, by compulsory
    bytes): each rank steps its own batch, and the rates are all streams over the slowest
    rank's time."""
    import torch
    from flowfilter_b200 import BatchFlowFilter, PyramidalFlowFilter, synthetic

    streams = batched_streams()
    total = len(streams)
    ids = list(range(total))
    if world > 1:
        ids = BatchFlowFilter.shard([(s["H"], s["W"], s["levels"]) for s in streams], world)[rank]
        streams = [streams[i] for i in ids]
    seqs = [torch.from_numpy(q).cuda() for q in batched_sequences(streams, BATCH_RING, ids)]
    batch = BatchFlowFilter([(s["H"], s["W"], s["levels"]) for s in streams])
    for i, s in enumerate(streams):
        configure_stream(batch.stream(i), s)
    packed = [batch.pack([seqs[i][r] for i in range(len(streams))]) for r in range(BATCH_RING)]

    def timed(run):
        for t in range(warmup):
            run(t)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for t in range(steps):
            run(warmup + t)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    b0_ms = timed(lambda t: batch.step(packed[t % BATCH_RING]))  # the default band rule
    t0 = time.perf_counter()
    bands = batch.autotune(packed[0], repetitions=5)  # per level size, on a scratch batch
    tune_s = time.perf_counter() - t0
    b_ms = timed(lambda t: batch.step(packed[t % BATCH_RING]))
    loop = []
    for s in streams:
        f = PyramidalFlowFilter(s["H"], s["W"], s["levels"])
        configure_stream(f, s)
        loop.append(f)

    def loop_step(t):
        for i, f in enumerate(loop):
            f.loadImage(seqs[i][t % BATCH_RING])
            f.computeAsync()
            if t == 0:
                f.setGraphs(True)

    l_ms = timed(loop_step)
    b0_ms, b_ms, l_ms = (max_over_ranks(world, v) for v in (b0_ms, b_ms, l_ms))
    px = sum(s["H"] * s["W"] for s in batched_streams())
    n = total
    return {
        "workload": f"{n} streams: {BATCH_PER_SIZE} each at " + ", ".join(f"{w}x{h}" for h, w in BATCH_SIZES)
                    + "; levels 1-3, gamma log-uniform [2,100], smoothing 1-4, maxflow 4 (seed 100)"
                    + (f"; split over {world} ranks by compulsory bytes ({len(streams)} streams here)"
                       if world > 1 else ""),
        "value": n * steps / (b_ms / 1e3), "unit": "stream-frames/s", "steps": steps,
        "ms_per_step": b_ms / steps, "mpix_per_s": px * steps / (b_ms / 1e3) / 1e6,
        "launches_per_step": batch.launches(),
        "autotune": {"bands": bands, "seconds": tune_s, "default_bands_ms_per_step": b0_ms / steps,
                     "method": "BatchFlowFilter.autotune: band rows per level size, largest first, each the "
                               "fastest of the default rule (0) and 8..128 rows by CUDA-event-timed "
                               "steps of a scratch batch"},
        "loop_value": n * steps / (l_ms / 1e3), "loop_ms_per_step": l_ms / steps,
        "speedup_vs_loop": l_ms / b_ms,
        "data": "synthetic: stream i is a seeded bump-flow sequence of its size from seed 100 + i",
    }


def graph_us(launch, n, per_graph=20):
    """Mean device microseconds of launch(stream) over replays of a CUDA graph holding
    per_graph back-to-back launches (host launch overhead not timed)."""
    import ctypes

    import torch

    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    st = ctypes.c_void_p(side.cuda_stream)
    with torch.cuda.stream(side):
        for _ in range(3):
            launch(st)  # first calls do any one-time set-up outside the capture
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=side):
        for _ in range(per_graph):
            launch(st)
    for _ in range(3):
        g.replay()
    reps = max(1, n // per_graph)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        g.replay()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) * 1e3 / (reps * per_graph)


def issue_roofline(warp_instructions, launch_ms, clocks):
    """The level-0 kernel against the instruction-issue ceiling that binds it: warp
    instructions per launch (ncu) / live launch time, over SMs x 4 schedulers x one
    instruction per clock at the median SM clock sampled during the timed region."""
    import torch

    if not warp_instructions or not clocks or not clocks.get("sm_mhz"):
        return None
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    peak = sms * 4 * clocks["sm_mhz"] * 1e6
    achieved = warp_instructions / (launch_ms * 1e-3)
    return {"warp_instructions": warp_instructions, "achieved": achieved, "peak": peak, "unit": "warp-inst/s",
            "frac": achieved / peak}


def bench_flow_to_color(filt, n):
    """Mean device microseconds of ff_flow_to_color per launch on the filter's current
    level-0 flow (a pitched device view), default wheel."""
    import ctypes

    import torch
    from flowfilter_b200 import lib

    flow = filt.getFlowDevice()
    h, w = flow.shape[:2]
    out = torch.empty((h, w, 4), dtype=torch.uint8, device="cuda")
    return graph_us(lambda st: lib().ff_flow_to_color(ctypes.c_void_p(flow.data_ptr()), flow.stride(0) * 4, h, w, 4.0,
                                                      None, ctypes.c_void_p(out.data_ptr()), out.stride(0), st), n)


def bench_rotational_predictor(n):
    """RotationalFlowImagePredictor on a 640x480 float image, 4 iterations: device
    microseconds per compute (one fused launch) and the bytes it must move."""
    import ctypes

    import torch
    from flowfilter_b200 import createPerspectiveCamera, lib

    h, w, it = 480, 640, 4
    img = torch.rand((h, w), dtype=torch.float32, device="cuda")
    flow = torch.empty((h, w, 2), dtype=torch.float32, device="cuda")
    out = torch.empty_like(img)
    cam = createPerspectiveCamera(0.004, h, w, 0.0036, 0.0048)
    vp = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    us = graph_us(lambda st: lib().ff_rotational_predict(ctypes.byref(cam.cam), 0.01, -0.02, 0.03, vp(img), w * 4, 1,
                                                         h, w, it, vp(flow), w * 8, vp(out), w * 4, None, 0, st), n)
    return {"workload": f"{w}x{h} float32 image, {it} iterations, rotational flow written", "launch_us": us,
            "launches": 1, "reference_launches": 1 + 2 * it,
            "bytes": h * w * 16, "achieved_GBps": h * w * 16 / (us * 1e-6) / 1e9}


def bench_differentiable(steps):
    """The differentiable filter on 16 sequences of 256x256 float frames, 32 frames each,
    2 levels (gamma [10, 50], smoothing [2, 4], maxflow 4): device time of the forward pass
    alone and of forward + backward of the mean endpoint error over frames 8-31 against the
    known flow, with the whole tape resident in HBM (no recompute) and with checkpoints every
    8 frames (each segment's forward recomputed in the backward pass)."""
    import torch
    from flowfilter_b200 import diff, synthetic

    B, T, H, W = 16, 32, 256, 256
    seqs = [synthetic.seq_bumps_float(frames=T, height=H, width=W, seed=200 + b, n_bumps=8, bump_sigma=40.0,
                                      amp=2.0) for b in range(B)]
    frames = torch.from_numpy(np.stack([q[0] for q in seqs])).cuda()
    truth = torch.from_numpy(np.stack([np.stack([q[1], q[2]], -1) for q in seqs])).cuda()[:, None]
    f = diff.DiffPyramidalFlowFilter(H, W, 2, [10.0, 50.0], [2, 4], maxflow=4.0, checkpoint_every=T)
    fc = diff.DiffPyramidalFlowFilter(H, W, 2, [10.0, 50.0], [2, 4], maxflow=4.0, checkpoint_every=8)

    def fwd():
        with torch.no_grad():
            return f(frames)

    def fwd_bwd(flt):
        def run():
            loss = diff.endpoint_error(flt(frames), truth.expand(B, T, H, W, 2), first=8)
            loss.backward()
            return loss
        return run

    def timed(fn, n):
        """Median over n calls, each bracketed by its own events (3 untimed calls first)."""
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        ms = []
        for _ in range(n):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        return statistics.median(ms)

    n = max(3, min(steps, 7))
    t_f = timed(fwd, n)
    t_fb = timed(fwd_bwd(f), n)
    t_fbc = timed(fwd_bwd(fc), n)
    tape = diff.lib().ff_diff_frame_tape_bytes(0, diff.ctypes.byref(diff._geom(f, B)))

    # the fit: Adam on per-level log gamma and smoothing weights, checkpoints every 8 frames
    ft = diff.DiffPyramidalFlowFilter(H, W, 2, [10.0, 50.0], [2, 4], maxflow=4.0, checkpoint_every=8)
    fit_steps = 200
    res = ft.fit(frames, truth.expand(B, T, H, W, 2), steps=fit_steps, lr=0.05, first=8, fit_weights=True)
    fit = {
        "steps": fit_steps,
        "optimizer": "Adam lr 0.05 on log gamma and on softmax logits of the 5-tap weights, checkpoint every 8",
        "epe_before": res["losses"][0], "epe_after": res["final"],
        "gamma": [float(x) for x in ft.gamma.detach().cpu()],
        "weights": [[float(x) for x in row] for row in ft.weights.detach().cpu()],
        "ms_per_step": res["ms"] / fit_steps,
        "loss_every_20": res["losses"][::20],
    }
    return {
        "workload": f"{B} sequences x {T} frames of {W}x{H} float32, 2 levels, gamma [10, 50], smoothing [2, 4], "
                    "maxflow 4, loss = mean endpoint error over frames 8-31",
        "fwd_ms": t_f, "fwd_note": "forward under torch.no_grad: no tape (ff_diff_frame_infer)",
        "fwd_bwd_ms": t_fb, "fwd_bwd_over_fwd": t_fb / t_f,
        "tape_bytes_per_frame": tape, "tape_note": "whole-sequence tape resident in HBM (no recompute)",
        "fwd_bwd_ckpt8_ms": t_fbc, "fwd_bwd_ckpt8_over_fwd": t_fbc / t_f,
        "fwd_frames_per_s": B * T / (t_f / 1e3), "fwd_bwd_frames_per_s": B * T / (t_fb / 1e3),
        "fit": fit,
        "dtype": "f32", "data": "synthetic: seeded bump flows (seed 200 + b), known flow",
    }


def workload_leg(world, name, steps, warmup, flush, hbm_peak):
    """Device-timed frames of one workload plus its level-0 kernel timed alone (L2 flushed
    before every frame and launch); returns (summary dict, tuned filter, frames on the host)."""
    import torch

    w = WORKLOADS[name]
    frames = make_frames(w)
    dev = torch.from_numpy(frames).cuda()
    barrier(world)
    ms, _, filt = device_run(w, dev, steps, warmup, flush, label="timed" if name == PRIMARY else "timed_" + name)
    barrier(world)
    ms = max_over_ranks(world, ms)
    fps = aggregate_rate(world, steps, ms)
    l0 = filt.timeLevel(0, min(steps, 1000), flush)
    l0_l2 = filt.timeLevel(0, min(steps, 1000), None)
    b0 = level0_kernel_bytes(w)
    N0 = int(np.ceil(np.float32(w["maxflow"])))
    kind = "delta level" if w["levels"] > 1 else "single level"
    out = {
        "workload": name, "value": fps, "unit": "frames/s", "steps": steps, "ms_per_step": ms / steps,
        "mpix_per_s": fps * w["H"] * w["W"] / 1e6, "kernels": filt.tuning(),
        "frame_bytes": frame_bytes(w), "frame_gbs": frame_bytes(w) * fps / world / 1e9,
        "frame_roofline_frac": frame_bytes(w) * fps / world / 1e9 / hbm_peak,
        "roofline": {"bound": "hbm", "kernel": f"level-0 step ({kind}, N={N0}, S={w['smooth'][0]}): "
                                               + filt.tuning().split(";")[0],
                     "achieved": b0 / (l0 / 1e3) / 1e9, "peak": hbm_peak, "unit": "GB/s",
                     "frac": b0 / (l0 / 1e3) / 1e9 / hbm_peak, "traffic": ncu_traffic(name),
                     "algorithmic_bytes": b0, "launch_ms": l0,
                     "l2_resident": {"launch_ms": l0_l2, "achieved": b0 / (l0_l2 / 1e3) / 1e9,
                                     "note": "same step without the L2 flush (state L2-resident)"}},
        "launches_per_frame": kernels_per_frame(w, filt.tuning()),
    }
    return out, filt, frames


def d2h_ceiling(nbytes, reps=20):
    """Frames/s that the device-to-host copy of one frame's flow alone allows (pinned host
    memory, one cudaMemcpyAsync per frame, back to back)."""
    import torch

    src = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    dst = torch.empty(nbytes, dtype=torch.uint8).pin_memory()
    for _ in range(3):
        dst.copy_(src, non_blocking=True)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        dst.copy_(src, non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    return {"fps": 1e3 / ms, "GBps": nbytes / (ms * 1e-3) / 1e9, "bytes": nbytes}


def bench_b200(args):
    import torch

    if args.config == 3:
        return bench_batched_line(args)
    if args.config == 4:
        return bench_differentiable_line(args)
    world, rank, local = dist_setup()
    hbm_peak, peak_kind = peaks()
    # --config 0 and 1 time that workload alone; the default run (config 2) adds the other legs
    name = CONFIGS[args.config] if args.config is not None else PRIMARY
    full = name == PRIMARY
    w = WORKLOADS[name]
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device="cuda")

    # kernel choice first, outside the clock sampling (its NVML polling must not disturb the
    # autotuner's per-frame timings)
    pretune(w, torch.from_numpy(make_frames(w)).cuda(), flush)
    # ---- timed region: device time of K frames, L2 flushed between frames
    barrier(world)
    with ClockSampler(gpu_uuid(local)) as clk:
        prim, filt, frames = workload_leg(world, name, args.steps, args.warmup, flush, hbm_peak)
    step_ms = prim["ms_per_step"] * args.steps
    value = prim["value"]

    # ---- elapsedTime() through the blocking drop-in calls (loadImage from host, compute),
    # the reference notebook's measure: mean over frames
    et = []
    for k in range(min(args.steps, 300)):
        filt.loadImage(frames[k % frames.shape[0]])
        filt.compute()
        et.append(filt.elapsedTime())
    elapsed_ms = float(np.mean(et))

    if full:
        # ---- FlowToColor of the level-0 flow (the step after the filter in the reference's
        # demos): device time per launch, back to back, the flow L2-resident as after a frame
        ftc_us = bench_flow_to_color(filt, min(args.steps, 1000))
        rot = bench_rotational_predictor(min(args.steps, 1000))

    # ---- end to end through the public API with host buffers
    e2e_steps = min(max(args.steps, 200), 2000)
    e2e_ms = max_over_ranks(world, e2e_run(w, frames, e2e_steps, args.warmup))
    e2e_fps = aggregate_rate(world, e2e_steps, e2e_ms)
    ceiling = d2h_ceiling(w["H"] * w["W"] * 8)

    if full:
        # ---- the reference's published configuration beside it
        extra, efilt, _ = workload_leg(world, EXTRA, min(args.steps * 4, 4000), args.warmup, flush, hbm_peak)
        extra["vs_published"] = extra["value"] / world / PUBLISHED_FPS[EXTRA]
        extra["published_fps"] = PUBLISHED_FPS[EXTRA]
        extra["sequence"] = SEQUENCE[WORKLOADS[EXTRA]["seq"]]

        # ---- the 64-stream batched step (each rank its own batch: replicas)
        barrier(world)
        batched = bench_batched(min(args.steps, 200), max(args.warmup, 3), world, rank)
        barrier(world)

        differentiable = bench_differentiable(args.steps)

    cpu = None
    if rank == 0 and world == 1:
        fps, cores, n = cpu_port_fps(w, frames)
        cpu = {"value": fps, "unit": "frames/s", "cores": cores, "kind": "port",
               "sample": f"{n} consecutive {w['W']}x{w['H']} frames, {w['levels']} levels, oracle/ C++ port, "
                         f"{cores} threads"}

    if rank == 0:
        roof = dict(prim["roofline"])
        roof["peak_kind"] = peak_kind
        instr = ncu_traffic(name, "warp_instructions_per_launch")
        if instr is not None:
            roof["issue"] = issue_roofline(instr, roof["launch_ms"], clk.summary())
        published = PUBLISHED_FPS.get(name)
        line = {
            "metric": metric_of(name), "value": value, "unit": "frames/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": value / world / published if published else None,
            "dtype": "f32", "data": "synthetic",
            "config": bench_config(name),
            "notes": {"sequence": SEQUENCE[w["seq"]], "step": "loadImage (device frame) + compute(), CUDA-graph replay",
                      "kernels": filt.tuning(), "parallelism": f"replicas x{world}",
                      "vs_baseline": (f"per GPU against the reference notebook's {published:.0f} frames/s "
                                      "(notebooks/GPU_example.ipynb:292)") if published else
                                     "null: the reference publishes no figure for this configuration"},
            "mpix_per_s": prim["mpix_per_s"],
            "frame_bytes": prim["frame_bytes"], "frame_gbs": prim["frame_gbs"],
            "frame_roofline_frac": prim["frame_roofline_frac"],
            "roofline": roof,
            "elapsed_time_ms": {"value": elapsed_ms, "frames": len(et),
                                "path": f"{w.get('filter', 'PyramidalFlowFilter')}.loadImage(host numpy) + compute(); "
                                        "mean elapsedTime(), as the reference notebook measures"},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_fps, "unit": "frames/s", "h2d_bytes_per_step": w["H"] * w["W"],
                    "d2h_bytes_per_step": w["H"] * w["W"] * 8, "steps": e2e_steps,
                    "d2h_ceiling": ceiling,
                    "path": f"flowfilter_b200.{w.get('filter', 'PyramidalFlowFilter')}.processAsync(pinned host frame "
                            "-> pinned host flow), synchronize() at the end; wall clock"},
            "gpu_launches": args.steps * prim["launches_per_frame"],
            "clocks": clk.summary(),
        }
        if full:
            line["flow_to_color"] = {"launch_us": ftc_us, "pixels": w["H"] * w["W"],
                                     "achieved_GBps": w["H"] * w["W"] * 12 / (ftc_us * 1e-6) / 1e9,
                                     "note": f"ff_flow_to_color on the {w['W']}x{w['H']} level-0 flow, default "
                                             "wheel; 12 B/px (float2 in, RGBA out)"}
            line["rotational_predictor"] = rot
            line["extra"] = extra
            line["batched"] = batched
            line["differentiable"] = differentiable
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def bench_batched_line(args):
    """--config 3: the 64-stream batched step as the line's metric (device-resident packed
    frames; the loop of single filters over the same streams beside it)."""
    world, rank, local = dist_setup()
    barrier(world)
    with ClockSampler(gpu_uuid(local)) as clk:
        b = bench_batched(args.steps, args.warmup, world, rank)
    if rank == 0:
        print(json.dumps({
            "metric": "stream-frames/s (BatchFlowFilter step over 64 mixed-size streams, each stream bit-exact with "
                      "its single filter)",
            "value": b["value"], "unit": "stream-frames/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": b["ms_per_step"], "higher_is_better": True,
            "scaling": "strong" if world > 1 else "weak", "vs_baseline": None, "dtype": "f32",
            "data": b["data"],
            "config": {"workload": "batched_64streams", "streams": b["workload"],
                       "l2": "no flush: the 64 streams' state (about 1 GB) exceeds L2"},
            "gpu_launches": args.steps * b["launches_per_step"],
            "e2e": None,
            "notes": {"e2e": "null: the batched step takes device-resident packed frames (BatchFlowFilter.pack); "
                             "no host-buffer entry point"},
            "clocks": clk.summary(), "batched": b,
        }), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def bench_differentiable_line(args):
    """--config 4: forward+backward of the differentiable filter as the line's metric."""
    world, rank, local = dist_setup()
    with ClockSampler(gpu_uuid(local)) as clk:
        d = bench_differentiable(args.steps)
    if rank == 0:
        print(json.dumps({
            "metric": "frames/s (differentiable PyramidalFlowFilter forward+backward, 16 x 32 frames of 256x256)",
            "value": d["fwd_bwd_frames_per_s"], "unit": "frames/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": d["fwd_bwd_ms"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": d["data"],
            "config": {"workload": "differentiable_16x32x256x256", "levels": 2, "gamma": [10.0, 50.0],
                       "smoothIterations": [2, 4], "maxflow": 4.0},
            "e2e": None,
            "gpu_launches": None,
            "notes": {"e2e": "null: frames and known flows are device-resident tensors; the fit's per-step time "
                             "(Adam, loss read back) is under differentiable.fit",
                      "gpu_launches": "not counted in this process; the launch list of one forward+backward is "
                                      "profiles/launches_differentiable_16x32x256x256.md"},
            "clocks": clk.summary(), "differentiable": d,
        }), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def bench_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if args.config in (3, 4):
        print(json.dumps({"impl": "reference", "unavailable": "the reference has no "
                          + ("batched step" if args.config == 3 else "gradient path")
                          + "; its per-stream filter is timed by --config 0-2"}), flush=True)
        return
    import oracle as O

    name = CONFIGS[args.config] if args.config is not None else PRIMARY
    w = WORKLOADS[name]
    frames = make_frames(w)
    threads = os.cpu_count() or 1
    O.set_threads(threads)
    f = oracle_filter(O, w)
    ring = frames.shape[0]
    for t in range(args.warmup):
        f.load(frames[t % ring])
        f.compute()
    t0 = time.perf_counter()
    for k in range(args.steps):
        f.load(frames[(args.warmup + k) % ring])
        f.compute()
    dt = time.perf_counter() - t0
    fps = args.steps / dt
    line = {
        "metric": metric_of(name), "value": fps, "unit": "frames/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dt * 1000.0 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
        "config": bench_config(name),
        "notes": {"sequence": SEQUENCE[w["seq"]],
                  "step": "one frame of the reference's CUDA path restated in C++ (oracle/), on the host cores"},
        "cpu_baseline": {"value": fps, "unit": "frames/s", "cores": threads, "kind": "port",
                         "sample": f"{args.steps} frames, reference CUDA path restated in C++ (oracle/), "
                                   f"{threads} host threads"},
        "e2e": {"value": fps, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def profile_next(args):
    """A profiler target for the kernels around the filter: --steps launches each of the
    flow-to-colour kernel (on a computed 640x480 flow, default wheel) and of the rotational
    predictor (640x480 float image, 4 iterations), inside the NVTX range "timed"."""
    import ctypes

    import torch
    from flowfilter_b200 import createPerspectiveCamera, lib

    w = dict(WORKLOADS["rotzoom_640x480_L2"])
    w["ring"] = 4
    dev = torch.from_numpy(make_frames(w)).cuda()
    f = make_filter(w)
    for t in range(args.warmup):
        f.loadImage(dev[t % 4])
        f.computeAsync()
    torch.cuda.synchronize()
    flow = f.getFlowDevice()
    h, wd = flow.shape[:2]
    rgba = torch.empty((h, wd, 4), dtype=torch.uint8, device="cuda")
    img = torch.rand((h, wd), dtype=torch.float32, device="cuda")
    rflow = torch.empty((h, wd, 2), dtype=torch.float32, device="cuda")
    pred = torch.empty_like(img)
    cam = createPerspectiveCamera(0.004, h, wd, 0.0036, 0.0048)
    vp = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for _ in range(3):  # set-up calls outside the range (default wheel upload, attributes)
        lib().ff_flow_to_color(vp(flow), flow.stride(0) * 4, h, wd, 4.0, None, vp(rgba), rgba.stride(0), st)
        lib().ff_rotational_predict(ctypes.byref(cam.cam), 0.01, -0.02, 0.03, vp(img), wd * 4, 1, h, wd, 4, vp(rflow),
                                    wd * 8, vp(pred), wd * 4, None, 0, st)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("timed")
    for _ in range(args.steps):
        lib().ff_flow_to_color(vp(flow), flow.stride(0) * 4, h, wd, 4.0, None, vp(rgba), rgba.stride(0), st)
        lib().ff_rotational_predict(ctypes.byref(cam.cam), 0.01, -0.02, 0.03, vp(img), wd * 4, 1, h, wd, 4, vp(rflow),
                                    wd * 8, vp(pred), wd * 4, None, 0, st)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    print(json.dumps({"profile": "next", "launches": 2 * args.steps}), flush=True)


def profile_batched(args):
    """A profiler target for the batched step: the 64-stream mix of the `batched` leg runs
    --warmup untimed steps, then --steps steps inside the NVTX range "timed"."""
    import torch
    from flowfilter_b200 import BatchFlowFilter, synthetic

    streams = batched_streams()
    seqs = [torch.from_numpy(q).cuda() for q in batched_sequences(streams, BATCH_RING)]
    batch = BatchFlowFilter([(s["H"], s["W"], s["levels"]) for s in streams])
    for i, s in enumerate(streams):
        configure_stream(batch.stream(i), s)
    packed = [batch.pack([seqs[i][r] for i in range(len(streams))]) for r in range(BATCH_RING)]
    for t in range(args.warmup):
        batch.step(packed[t % BATCH_RING])
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("timed")
    for t in range(args.steps):
        batch.step(packed[t % BATCH_RING])
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    print(json.dumps({"profile": "batched", "steps": args.steps, "launches_per_step": batch.launches()}), flush=True)


def profile_diff(args):
    """A profiler target for the differentiable filter: --warmup untimed passes, then --steps
    times one forward without a tape and one forward + backward with the whole tape, on the
    differentiable leg's batch (16 sequences x 32 frames of 256x256), in the NVTX range "timed"."""
    import torch
    from flowfilter_b200 import diff, synthetic

    B, T, H, W = 16, 32, 256, 256
    seqs = [synthetic.seq_bumps_float(frames=T, height=H, width=W, seed=200 + b, n_bumps=8, bump_sigma=40.0,
                                      amp=2.0) for b in range(B)]
    frames = torch.from_numpy(np.stack([q[0] for q in seqs])).cuda()
    truth = torch.from_numpy(np.stack([np.stack([q[1], q[2]], -1) for q in seqs])).cuda()[:, None]
    f = diff.DiffPyramidalFlowFilter(H, W, 2, [10.0, 50.0], [2, 4], maxflow=4.0, checkpoint_every=T)

    def once():
        with torch.no_grad():
            f(frames)
        diff.endpoint_error(f(frames), truth.expand(B, T, H, W, 2), first=8).backward()

    for _ in range(args.warmup):
        once()
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("timed")
    for _ in range(args.steps):
        once()
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    print(json.dumps({"profile": "diff", "steps": args.steps}), flush=True)


def profile_case(args):
    """A profiler target: the tuned filter of one workload runs --warmup untimed frames, then
    --steps frames inside the NVTX range "timed" (L2 flushed before each), and nothing else."""
    import torch

    w = dict(WORKLOADS[args.profile])
    w["ring"] = 4
    frames = make_frames(w)
    dev = torch.from_numpy(frames).cuda()
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    f = make_filter(w)
    for t in range(args.warmup):
        f.loadImage(dev[t % 4])
        f.computeAsync()
        if t == 1:
            tuned(f, w, flush=flush)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("timed")
    for t in range(args.steps):
        flush.zero_()
        f.loadImage(dev[t % 4])
        f.computeAsync()
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    print(json.dumps({"profile": args.profile, "frames": args.steps, "kernels": f.tuning()}), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--config", type=int, choices=sorted(CONFIGS), default=None,
                    help="one configuration alone: 0 320x240 FlowFilter, 1 640x480 2 levels, 2 2048x1088 3 levels "
                         "(the default run, with every other leg), 3 the 64-stream batched step, 4 the "
                         "differentiable filter")
    ap.add_argument("--profile-next", action="store_true",
                    help="profiler target: the flow-to-colour and rotational-predictor kernels (no JSON line)")
    ap.add_argument("--profile-batched", action="store_true",
                    help="profiler target: steps of the 64-stream batched step (no JSON line)")
    ap.add_argument("--profile-diff", action="store_true",
                    help="profiler target: the differentiable filter's forward and forward+backward (no JSON line)")
    ap.add_argument("--profile", choices=sorted(WORKLOADS), default=None,
                    help="profiler target: run --steps frames of one workload in the NVTX range 'timed' (no JSON line)")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.profile_next:
        profile_next(args)
    elif args.profile_diff:
        profile_diff(args)
    elif args.profile_batched:
        profile_batched(args)
    elif args.profile:
        profile_case(args)
    elif args.impl == "reference":
        bench_reference(args)
    else:
        bench_b200(args)


if __name__ == "__main__":
    main()
