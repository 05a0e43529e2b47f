"""Filters through the public API (C ABI) against the reference's own outputs and the oracle."""

from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from conftest import golden_case
from make_reference_fixtures import CASES, case_frames, sha, subsample_rows_cols

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ffb(cuda):
    import flowfilter_b200

    return flowfilter_b200


def make_gpu_filter(ffb, case, h, w):
    if case["levels"] == 0:
        return ffb.FlowFilter(h, w, case["smooth"][0], case["maxflow"], case["gamma"][0])
    f = ffb.PyramidalFlowFilter(h, w, case["levels"])
    f.gamma = case["gamma"]
    f.smoothIterations = case["smooth"]
    f.maxflow = case["maxflow"]
    return f


def run_gpu(f, frames, dump, fused=1):
    f.setFused(fused)
    out = []
    for t in range(frames.shape[0]):
        f.loadImage(frames[t])
        f.compute()
        if t in dump:
            out.append(f.getFlow())
    return np.stack(out)


@pytest.mark.parametrize("mode", [1, 3])
@pytest.mark.parametrize("name", list(CASES))
def test_reference_sequences_bit_exact(ffb, name, mode):
    """The GPU filter reproduces the reference library's flows bit for bit (sha256 per frame),
    with the streaming fused kernel (mode 1) and with the tile-fused kernel (mode 3)."""
    case = CASES[name]
    meta, arr = golden_case(name)
    frames = case_frames(case)
    assert sha(frames) == meta["frames_sha256"]
    f = make_gpu_filter(ffb, case, *frames.shape[1:])
    flows = run_gpu(f, frames, set(case["dump"]), mode)
    if meta["layout"] == "full":
        got = flows
    else:
        rows, cols = subsample_rows_cols(*frames.shape[1:])
        got = flows[:, rows][:, :, cols]
    assert np.max(np.abs(got - arr["flow"])) <= 1e-4  # the stated tolerance ...
    assert [sha(x) for x in flows] == meta["flow_sha256"]  # ... and in fact bit-exact


RANDOM_CASES = [
    # (h, w, levels, maxflow, gammas, smooths, border)
    (61, 77, 0, 2.5, [3.0], [2], 3),
    (40, 52, 0, 6.0, [20.0], [5], 0),
    (64, 96, 2, 5.0, [2.0, 25.0], [3, 1], 3),
    (98, 150, 3, 3.0, [4.0, 9.0, 30.0], [1, 3, 2], 5),
    (130, 130, 4, 8.0, [1.0, 2.0, 4.0, 8.0], [1, 1, 2, 3], 2),
    (9, 13, 2, 1.0, [1.0, 1.0], [1, 1], 3),
]


def oracle_filter(case):
    h, w, levels, maxflow, gammas, smooths, border = case
    if levels == 0:
        f = O.Filter.flowfilter(h, w, smooths[0], maxflow, gammas[0])
    else:
        f = O.Filter.pyramidal(h, w, levels)
        f.set_gammas(gammas)
        f.set_smooths(smooths)
        f.set_max_flow(maxflow)
    f.set_propagation_border(border)
    return f


def gpu_filter(ffb, case):
    h, w, levels, maxflow, gammas, smooths, border = case
    if levels == 0:
        f = ffb.FlowFilter(h, w, smooths[0], maxflow, gammas[0])
    else:
        f = ffb.PyramidalFlowFilter(h, w, levels)
        f.gamma = gammas
        f.smoothIterations = smooths
        f.maxflow = maxflow
    f.propagationBorder = border
    return f


@pytest.mark.parametrize("case", RANDOM_CASES)
@pytest.mark.parametrize("fused", [1, 0, 3])
def test_against_oracle(ffb, case, fused):
    h, w = case[:2]
    frames = case_frames(dict(seq="bumps", frames=12, kw=dict(height=h, width=w, sigma=1.0, seed=h * w,
                                                               n_bumps=2, bump_sigma=max(h, w) / 3, amp=2.0)))
    of = oracle_filter(case)
    gf = gpu_filter(ffb, case)
    gf.setFused(fused)
    for t in range(frames.shape[0]):
        of.load(frames[t])
        of.compute()
        gf.loadImage(frames[t])
        gf.compute()
        np.testing.assert_array_equal(gf.getFlow(), of.flow())
        np.testing.assert_array_equal(gf.getImage(), of.image())
    for lv in range(max(case[2], 1)):
        np.testing.assert_array_equal(gf.levelState(lv, 0), of.level_state(lv, 0))
        np.testing.assert_array_equal(gf.levelState(lv, 2), of.level_state(lv, 2))


def test_defaults_and_parameter_rules(ffb):
    f = ffb.FlowFilter(32, 48)
    assert f.height == 32 and f.width == 48
    assert f.gamma == pytest.approx(1.0 / (255.0 * 255.0))  # setGamma(1) scaled for uint8
    assert f.maxflow == 1.0 and f.propagationIterations == 1
    assert f.smoothIterations == 1 and f.propagationBorder == 3
    f.maxflow = 2.5
    assert f.propagationIterations == 3
    f.gamma = 10.0
    assert f.gamma == pytest.approx(10.0 / 65025.0)
    p = ffb.PyramidalFlowFilter(64, 64, 3)
    assert p.gamma == [1.0, 1.0, 1.0]  # configure() defaults are unscaled
    assert p.smoothIterations == [1, 1, 1]
    p.maxflow = 4.0
    assert [p.propagationIterationsAt(l) for l in range(3)] == [4, 2, 1]
    p.maxflow = 3.0
    assert [p.propagationIterationsAt(l) for l in range(3)] == [3, 2, 1]
    assert p.maxflow == 3.0
    with pytest.raises(RuntimeError):
        p.levels = 2
    with pytest.raises(RuntimeError):
        f.propagationIterations = 2


def test_argument_errors(ffb):
    f = ffb.FlowFilter(16, 16)
    with pytest.raises(ValueError):
        f.gamma = 0.0
    with pytest.raises(ValueError):
        f.gamma = -1.0
    with pytest.raises(ValueError):
        f.maxflow = 0.0
    with pytest.raises(ValueError):
        f.smoothIterations = 0
    with pytest.raises(ValueError):
        f.propagationBorder = -1
    with pytest.raises(ValueError):
        f.loadImage(np.zeros((16, 15), np.uint8))
    with pytest.raises(ValueError):
        f.loadImage(np.zeros((16, 16), np.float32))
    p = ffb.PyramidalFlowFilter(32, 32, 2)
    with pytest.raises(IndexError):
        p.setGamma(2, 1.0)
    with pytest.raises(IndexError):
        p.getSmoothIterations(-1)
    with pytest.raises(ValueError):
        ffb.PyramidalFlowFilter(4, 4, 4)  # level 3 would have zero size


def test_getflow_semantics(ffb):
    """Single level: getFlow() is the unsmoothed update output, downloadFlow the smoothed
    one (flowfilter.cu:238-240, 266-268); pyramids return the smoothed flow from both."""
    frames = case_frames(dict(seq="constant", frames=6, kw=dict(height=48, width=64, sigma=1.5, seed=3)))
    of = O.Filter.flowfilter(48, 64, 2, 3.0, 5.0)
    gf = ffb.FlowFilter(48, 64, 2, 3.0, 5.0)
    for t in range(6):
        of.load(frames[t]); of.compute()
        gf.loadImage(frames[t]); gf.compute()
    np.testing.assert_array_equal(gf.getFlowDevice().cpu().numpy(), of.get_flow())
    np.testing.assert_array_equal(gf.flowTensor().cpu().numpy(), of.flow())
    assert not np.array_equal(of.get_flow(), of.flow())
    p = ffb.PyramidalFlowFilter(48, 64, 2)
    p.loadImage(frames[0]); p.compute()
    np.testing.assert_array_equal(p.getFlowDevice().cpu().numpy(), p.getFlow())


def test_device_input_matches_host_input(ffb, cuda):
    frames = case_frames(dict(seq="constant", frames=5, kw=dict(height=40, width=56, sigma=1.5, seed=4)))
    a = ffb.PyramidalFlowFilter(40, 56, 2)
    b = ffb.PyramidalFlowFilter(40, 56, 2)
    for f in (a, b):
        f.maxflow = 3.0
    for t in range(5):
        a.loadImage(frames[t]); a.compute()
        b.loadImage(cuda.from_numpy(frames[t]).cuda()); b.compute()
        np.testing.assert_array_equal(a.getFlow(), b.getFlow())
    assert a.elapsedTime() > 0.0


def test_phase_api_matches_compute(ffb):
    frames = case_frames(dict(seq="constant", frames=5, kw=dict(height=33, width=45, sigma=1.5, seed=5)))
    a = ffb.FlowFilter(33, 45, 2, 2.0, 4.0)
    b = ffb.FlowFilter(33, 45, 2, 2.0, 4.0)
    for t in range(5):
        a.loadImage(frames[t]); a.compute()
        b.loadImage(frames[t]); b.computeImageModel(); b.computePropagation(); b.computeUpdate()
        np.testing.assert_array_equal(a.getFlow(), b.getFlow())


@pytest.mark.parametrize("dtype", ["uint8", "float32"])
def test_flowfilter_on_device_image(ffb, cuda, dtype):
    """FlowFilter(GPUImage): configure() defaults, float input uses gamma unscaled."""
    frames = case_frames(dict(seq="constant", frames=6, kw=dict(height=36, width=50, sigma=1.5, seed=6)))
    if dtype == "float32":
        frames = (frames.astype(np.float32) / 255.0).astype(np.float32)
    img = cuda.from_numpy(frames[0]).cuda()
    gf = ffb.FlowFilter.on_device(img)
    of = O.Filter.flowfilter_on(36, 50, 1 if dtype == "uint8" else 4)
    gf.gamma = 2.0
    of.set_gamma(0, 2.0)
    gf.maxflow = 2.0
    of.set_max_flow(2.0)
    for t in range(6):
        img.copy_(cuda.from_numpy(frames[t]))
        of.load(frames[t]); of.compute()
        gf.compute()
        np.testing.assert_array_equal(gf.getFlow(), of.flow())


def test_delta_filter_standalone(ffb, cuda):
    """DeltaFlowFilter(image, inputFlow) follows DeltaFlowFilter::compute (flowfilter.cu:429-457)."""
    rng = np.random.default_rng(9)
    h, w = 30, 44
    frames = case_frames(dict(seq="constant", frames=4, kw=dict(height=h, width=w, sigma=1.5, seed=9)))
    coarse = rng.normal(0, 0.5, (h // 2, w // 2, 2)).astype(np.float32)
    img = cuda.from_numpy(frames[0]).cuda()
    cf = cuda.from_numpy(coarse).cuda()
    gf = ffb.DeltaFlowFilter(img, cf)
    gf.gamma = 5.0
    gf.maxflow = 2.0
    gamma = np.float32(5.0) / np.float32(255.0 * 255.0)
    fs = np.zeros((h, w, 2), np.float32)
    iu = np.zeros((h, w), np.float32)
    du = np.zeros((h, w, 2), np.float32)
    for t in range(4):
        img.copy_(cuda.from_numpy(frames[t]))
        gf.compute()
        a0, g = O.image_model(frames[t])
        if t == 0:
            iu = a0.copy()
        _, ip, dp = O.propagate_payload(fs, iu, du, 2, 3)
        if t == 0:
            ip = a0.copy()
        fu, du, iu = O.delta_update(a0, g, ip, dp, coarse, gamma, 2.0)
        fs = O.smooth(fu, 1)
        np.testing.assert_array_equal(gf.getFlow(), fs)


@pytest.mark.parametrize("levels", [1, 2, 3, 4])
def test_graphs_side_streams_and_profiling(ffb, cuda, levels):
    """CUDA-graph replay (one graph per state parity), the side stream that runs levels
    0..L-3 concurrently, and the profiling events all leave results unchanged."""
    h, w = 96, 160
    frames = case_frames(dict(seq="bumps", frames=9, kw=dict(height=h, width=w, sigma=1.0, seed=21, n_bumps=2,
                                                              bump_sigma=40.0, amp=2.0)))
    ref = ffb.PyramidalFlowFilter(h, w, levels)
    g = ffb.PyramidalFlowFilter(h, w, levels)
    for f in (ref, g):
        f.maxflow = 4.0
        f.smoothIterations = [2] * levels if levels > 1 else 2
    g.setGraphs(True)
    dev = cuda.from_numpy(frames).cuda()
    for t in range(9):
        if t == 4:
            g.setProfiling(3)
        if t == 6:
            g.maxflow = 3.0  # parameter change re-captures the graphs
            ref.maxflow = 3.0
        ref.loadImage(frames[t]); ref.compute()
        g.loadImage(dev[t]); g.computeAsync()
        cuda.cuda.synchronize()
        np.testing.assert_array_equal(g.getFlow(), ref.getFlow())
    ms, n = g.levelKernelTime(0)
    assert n == 3 and ms > 0.0


def test_autotune_keeps_results(ffb, cuda):
    """Autotuning re-runs level steps on live data; the sequence is unchanged by it."""
    h, w = 272, 512
    frames = case_frames(dict(seq="bumps", frames=7, kw=dict(height=h, width=w, sigma=1.0, seed=31, n_bumps=3,
                                                              bump_sigma=60.0, amp=2.0)))
    ref = ffb.PyramidalFlowFilter(h, w, 3)
    tun = ffb.PyramidalFlowFilter(h, w, 3)
    for f in (ref, tun):
        f.gamma = [5.0, 20.0, 50.0]
        f.smoothIterations = [1, 2, 4]
        f.maxflow = 4.0
    ref.setFused(0)
    for t in range(7):
        ref.loadImage(frames[t]); ref.compute()
        tun.loadImage(frames[t]); tun.compute()
        if t == 2:
            with pytest.raises(ValueError):
                tun.autotune(0)
            choice = tun.autotune(2)
            assert choice.count("level") == 3 and "untuned" not in choice
            tun.setGraphs(True)
        np.testing.assert_array_equal(tun.getFlow(), ref.getFlow())
        np.testing.assert_array_equal(tun.getFlowDevice().cpu().numpy(), ref.getFlowDevice().cpu().numpy())
    fresh = ffb.PyramidalFlowFilter(h, w, 3)
    with pytest.raises(RuntimeError):
        fresh.autotune(1)  # needs one computed frame


def test_time_level_keeps_results(ffb, cuda):
    h, w = 96, 128
    frames = case_frames(dict(seq="bumps", frames=6, kw=dict(height=h, width=w, sigma=1.0, seed=41, n_bumps=2,
                                                              bump_sigma=30.0, amp=2.0)))
    ref = ffb.PyramidalFlowFilter(h, w, 3)
    tim = ffb.PyramidalFlowFilter(h, w, 3)
    for f in (ref, tim):
        f.maxflow = 4.0
    flush = cuda.empty(1 << 20, dtype=cuda.uint8, device="cuda")
    for t in range(6):
        ref.loadImage(frames[t]); ref.compute()
        tim.loadImage(frames[t]); tim.compute()
        if t >= 1:
            for lv in range(3):
                assert tim.timeLevel(lv, 3, flush if lv == 0 else None) > 0.0
        np.testing.assert_array_equal(tim.getFlow(), ref.getFlow())


TILE_CASES = [
    # (kind, h, w, item, maxflow, smooth, border)
    ("single", 37, 53, 1, 4.0, 2, 3),
    ("single", 120, 200, 4, 3.0, 4, 0),
    ("single", 5, 3, 1, 1.0, 1, 3),
    ("delta", 66, 90, 1, 4.0, 1, 3),
    ("delta", 97, 131, 4, 6.0, 3, 2),
    ("delta", 240, 320, 1, 2.0, 4, 3),
]


@pytest.mark.parametrize("case", TILE_CASES)
def test_tile_kernel_matches_per_stage(ffb, cuda, case):
    """The tile-fused kernel against the per-stage kernels, every tile shape, on FlowFilter
    and standalone DeltaFlowFilter over uint8 and float images."""
    kind, h, w, item, maxflow, smooth, border = case
    rng = np.random.default_rng(h * w + item)
    frames = case_frames(dict(seq="bumps", frames=5, kw=dict(height=h, width=w, sigma=1.0, seed=h + w, n_bumps=2,
                                                              bump_sigma=max(h, w) / 3, amp=2.0)))
    if item == 4:
        frames = (frames.astype(np.float32) / 255.0).astype(np.float32)
    coarse = cuda.from_numpy(rng.normal(0, 0.7, (max(h // 2, 1), max(w // 2, 1), 2)).astype(np.float32)).cuda()
    imgs = [cuda.from_numpy(frames[0]).cuda() for _ in range(2)]

    def make(img):
        f = ffb.DeltaFlowFilter(img, coarse) if kind == "delta" else ffb.FlowFilter.on_device(img)
        f.gamma = 10.0
        f.maxflow = maxflow
        f.smoothIterations = smooth
        f.propagationBorder = border
        return f

    ref = make(imgs[0])
    ref.setFused(0)
    tiles = []
    for c in range(64):  # every tile-shape index the library accepts
        f = make(imgs[1])
        try:
            f.setTuningState([(2, c)])
        except ValueError:
            break
        tiles.append((c, f))
    assert len(tiles) > 3
    for t in range(frames.shape[0]):
        for img in imgs:
            img.copy_(cuda.from_numpy(frames[t]))
        ref.compute()
        want = ref.getFlow()
        for c, f in tiles:
            f.compute()
            np.testing.assert_array_equal(f.getFlow(), want, err_msg=f"tile shape {c} frame {t} ({f.tuning()})")
            np.testing.assert_array_equal(f.getImage(), ref.getImage())


@pytest.mark.parametrize("levels", [0, 2, 3])
def test_pipelined_host_processing_matches_blocking_loop(ffb, cuda, levels):
    """processAsync (upload, compute and download overlapped on three streams) gives the
    blocking loadImage/compute/downloadFlow results, also with graphs and when the caller
    returns to the blocking calls afterwards."""
    h, w, t = 120, 160, 9
    frames = case_frames(dict(seq="bumps", frames=t, kw=dict(height=h, width=w, sigma=1.0, seed=51, n_bumps=2,
                                                              bump_sigma=40.0, amp=2.0)))

    def make():
        if levels == 0:
            return ffb.FlowFilter(h, w, 2, 4.0, 10.0)
        f = ffb.PyramidalFlowFilter(h, w, levels)
        f.maxflow = 4.0
        f.smoothIterations = [1, 2, 4][:levels]
        return f

    ref, pip = make(), make()
    want = []
    for k in range(t):
        ref.loadImage(frames[k])
        ref.compute()
        want.append(ref.flowTensor().cpu().numpy())
    hin = cuda.from_numpy(frames).pin_memory()
    outs = [cuda.empty((h, w, 2), dtype=cuda.float32).pin_memory() for _ in range(t)]
    for k in range(6):
        if k == 3:
            pip.setGraphs(True)
        pip.processAsync(hin[k], outs[k])
    pip.synchronize()
    for k in range(6):
        np.testing.assert_array_equal(outs[k].numpy(), want[k], err_msg=f"frame {k}")
    for k in range(6, t):  # back to the blocking path
        pip.loadImage(frames[k])
        pip.compute()
        np.testing.assert_array_equal(pip.flowTensor().cpu().numpy(), want[k], err_msg=f"frame {k}")
