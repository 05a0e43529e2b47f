"""Batched multi-stream step (BatchFlowFilter / ff_batch_*) against each stream filtered alone."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from make_reference_fixtures import case_frames

pytestmark = pytest.mark.gpu

# (height, width, levels, gamma per level, smooth per level, maxflow, border)
STREAMS = [
    (48, 64, 1, [7.0], [2], 3.0, 3),
    (61, 77, 2, [4.0, 30.0], [1, 3], 4.0, 3),
    (96, 128, 3, [5.0, 20.0, 50.0], [1, 2, 4], 4.0, 2),
    (120, 160, 2, [10.0, 50.0], [2, 4], 6.0, 3),
    (33, 45, 1, [2.0], [4], 1.0, 0),
    (130, 130, 4, [1.0, 2.0, 4.0, 8.0], [1, 1, 2, 3], 8.0, 3),
]


def configure(f, s):
    h, w, levels, gamma, smooth, maxflow, border = s
    f.gamma = gamma if levels > 1 else gamma[0]
    f.smoothIterations = smooth if levels > 1 else smooth[0]
    f.maxflow = maxflow
    f.propagationBorder = border


@pytest.fixture(scope="module")
def ffb(cuda):
    import flowfilter_b200

    return flowfilter_b200


def run_against_alone(ffb, cuda, streams, t_frames=8, tuning=None, retune=None, launches=None, level_bands=(),
                      prepare=None):
    """Steps a batch of `streams` and the same streams as single filters over seeded frames
    and asserts identical flow and image every frame.  tuning / retune: setTuning arguments
    before the first frame / from frame 3 on; level_bands: setLevelBand arguments from frame
    2 on; prepare(batch, step_buffer): called before the first frame."""
    seqs = [case_frames(dict(seq="bumps", frames=t_frames, kw=dict(height=s[0], width=s[1], sigma=1.0, seed=11 + i,
                                                                    n_bumps=2, bump_sigma=max(s[0], s[1]) / 3,
                                                                    amp=2.0)))
            for i, s in enumerate(streams)]
    alone = [ffb.PyramidalFlowFilter(s[0], s[1], s[2]) for s in streams]
    batch = ffb.BatchFlowFilter([s[:3] for s in streams])
    for f, b, s in zip(alone, [batch.stream(i) for i in range(len(streams))], streams):
        configure(f, s)
        configure(b, s)
    if tuning is not None:
        batch.setTuning(*tuning)
    if launches is not None:
        launches(batch.launches())
    dev = [cuda.from_numpy(q).cuda() for q in seqs]
    buf = cuda.empty(batch.frameBytes(), dtype=cuda.uint8, device="cuda")
    if prepare is not None:
        batch.pack([d[0] for d in dev], out=buf)
        prepare(batch, buf)
    for t in range(t_frames):
        if t == 2:
            for lb in level_bands:
                batch.setLevelBand(*lb)
        if t == 3 and retune is not None:
            batch.setTuning(*retune)
        if t == 5:  # a parameter change rebuilds the batch's job tables
            for f in (alone[2], batch.stream(2)):
                f.setGamma(1, 7.5)
            for f in (alone[4], batch.stream(4)):
                f.maxflow = 2.0
        batch.pack([d[t] for d in dev], out=buf)
        batch.step(buf)
        cuda.cuda.synchronize()
        for i, f in enumerate(alone):
            f.loadImage(seqs[i][t])
            f.compute()
            np.testing.assert_array_equal(batch.stream(i).getFlow(), f.getFlow(), err_msg=f"stream {i} frame {t}")
            np.testing.assert_array_equal(batch.stream(i).getImage(), f.getImage(), err_msg=f"stream {i} frame {t}")
    return batch


def test_batch_matches_streams_alone(ffb, cuda):
    def launches(n):
        # ingest with pyramid levels 1-2, pyramid depth 3, phase A's tile launch (its levels
        # are all below 200000 pixels), phase B's streaming launch and its tile launch (level 0
        # of the 2-level 120x160 stream has 6 propagation iterations, beyond the streaming
        # kernel's 4)
        assert n == 1 + 1 + 1 + 2

    run_against_alone(ffb, cuda, STREAMS, launches=launches)


def test_batch_streaming_launches_match_streams_alone(ffb, cuda):
    """Every level the streaming kernel can run goes to the batched streaming launches: bands
    chosen by the batch (one per level at these sizes), then bands of 8 rows from frame 3 on
    (band seams)."""
    seen = []
    run_against_alone(ffb, cuda, STREAMS, tuning=(0, 0), retune=(0, 8), launches=seen.append)
    assert seen[0] == 1 + 1 + 2 + 2  # both phases stream, and tile what has 6 or 8 iterations


def test_batch_level_bands_match_streams_alone(ffb, cuda):
    """Per-size band overrides (the autotuner's knob) from frame 2 on: 8-row bands at the
    96x128 and 130x130 level-0 sizes, 12 rows at 60x80, the default elsewhere."""
    run_against_alone(ffb, cuda, STREAMS, level_bands=[(96, 128, 8), (130, 130, 8), (60, 80, 12), (61, 77, 0)])


def test_batch_autotune_keeps_results_and_caches(ffb, cuda, tmp_path):
    """autotune() times a scratch batch (this batch is not stepped), applies one band per
    level size, stores the choice in the JSON cache and reapplies it from there; the batch
    still gives every stream's results alone."""
    cache = str(tmp_path / "bands.json")
    chosen = []

    def prepare(batch, buf):
        choice = batch.autotune(buf, repetitions=1, cache=cache, bands=(8, 16, 32))
        assert set(choice) == {f"{h}x{w}" for h, w in batch.levelSizes()}
        assert all(0 <= b <= int(k.split("x")[0]) for k, b in choice.items())
        again = batch.autotune(buf, repetitions=1, cache=cache)
        assert again == choice
        chosen.append(choice)

    run_against_alone(ffb, cuda, STREAMS[:4], t_frames=5, prepare=prepare)
    import json

    with open(cache) as fh:
        assert list(json.load(fh).values()) == chosen


def test_batch_mixed_kernels_match_streams_alone(ffb, cuda):
    """Levels of at least 3000 pixels stream and the rest tile: both kernels in both phases
    (top levels and levels L-3.. in phase A, levels L-2 in phase B), 16-row bands; back to
    the default selection from frame 3 on."""
    run_against_alone(ffb, cuda, STREAMS, tuning=(3000, 16), retune=(-1, 0))


def test_batch_default_selection_streams_large_levels(ffb, cuda):
    """By default phase-A levels of 200000 pixels or more and every phase-B level stream, the
    small phase-A levels tile: four launches."""
    streams = [
        (480, 640, 2, [10.0, 50.0], [2, 4], 4.0, 3),
        (544, 960, 1, [20.0], [3], 4.0, 3),
        (96, 128, 3, [5.0, 20.0, 50.0], [1, 2, 4], 4.0, 2),
        (480, 640, 3, [5.0, 10.0, 30.0], [1, 1, 2], 4.0, 3),
        (61, 77, 2, [4.0, 30.0], [1, 3], 2.0, 3),
    ]
    seen = []
    run_against_alone(ffb, cuda, streams, t_frames=6, launches=seen.append)
    assert seen[0] == 4  # ingest with pyramid, a streaming launch per phase, phase A's tiles


def test_batch_frame_layout_and_errors(ffb, cuda):
    from flowfilter_b200 import _lib

    batch = ffb.BatchFlowFilter([(10, 20, 1), (30, 17, 2)])
    offs = batch.frameOffsets()
    assert offs[0] == 0 and offs[1] == 256 and batch.frameBytes() == 256 + (30 * 17 + 255) // 256 * 256
    with pytest.raises(ValueError):
        batch.step(cuda.empty(batch.frameBytes() - 1, dtype=cuda.uint8, device="cuda"))
    st = _lib.lib().ff_filter_destroy(batch.stream(0)._h)
    assert st == _lib.FF_ERR_LOGIC  # streams belong to the batch
    h = ctypes.c_void_p()
    assert _lib.lib().ff_batch_stream(batch._h, 2, ctypes.byref(h)) == _lib.FF_ERR_OUT_OF_RANGE
    with pytest.raises(ValueError):
        ffb.BatchFlowFilter([])


def test_sixty_four_stream_mix_matches_streams_alone(ffb, cuda):
    """The benchmark's 64-stream mix (16 each at 320x240, 640x480, 1280x720, 1920x1080; levels,
    gamma and smoothing seeded per stream; stream i's frames from seed 100 + i) at the default
    kernel selection: every stream bit for bit equal to the same stream filtered alone, over
    four frames, in four launches: the large levels in the streaming launches at the batch's
    own bands, the small phase-A levels in the tile launch."""
    import bench

    streams = bench.batched_streams()
    assert len(streams) == 64
    seqs = bench.batched_sequences(streams, 4)
    alone = []
    batch = ffb.BatchFlowFilter([(s["H"], s["W"], s["levels"]) for s in streams])
    for i, s in enumerate(streams):
        f = ffb.PyramidalFlowFilter(s["H"], s["W"], s["levels"])
        bench.configure_stream(f, s)
        bench.configure_stream(batch.stream(i), s)
        alone.append(f)
    assert batch.launches() == 4  # ingest with pyramid, a streaming launch per phase, phase A's tiles
    dev = [cuda.from_numpy(q).cuda() for q in seqs]
    buf = cuda.empty(batch.frameBytes(), dtype=cuda.uint8, device="cuda")
    for t in range(4):
        batch.pack([d[t] for d in dev], out=buf)
        batch.step(buf)
        for f, d in zip(alone, dev):
            f.loadImage(d[t])
            f.computeAsync()
        cuda.cuda.synchronize()
        for i, f in enumerate(alone):
            np.testing.assert_array_equal(batch.stream(i).getFlow(), f.getFlow(), err_msg=f"stream {i} frame {t}")
