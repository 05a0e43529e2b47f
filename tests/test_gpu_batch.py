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


def run_against_alone(ffb, cuda, streams, t_frames=8, tuning=None, retune=None, launches=None):
    """Steps a batch of `streams` and the same streams as single filters over seeded frames
    and asserts identical flow and image every frame.  tuning / retune: setTuning arguments
    before the first frame / from frame 3 on."""
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
    for t in range(t_frames):
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
        assert n == 1 + (4 - 1) + 2  # ingest, 3 pyramid depths, the two tile launches

    run_against_alone(ffb, cuda, STREAMS, launches=launches)


def test_batch_streaming_launches_match_streams_alone(ffb, cuda):
    """Every level the streaming kernel can run goes to the batched streaming launches: bands
    chosen by the batch (one per level at these sizes), then bands of 8 rows from frame 3 on
    (band seams)."""
    seen = []
    run_against_alone(ffb, cuda, STREAMS, tuning=(0, 0), retune=(0, 8), launches=seen.append)
    assert seen[0] > 1 + (4 - 1) + 2


def test_batch_mixed_kernels_match_streams_alone(ffb, cuda):
    """Levels of at least 3000 pixels stream and the rest tile: both kernels in both phases
    (top levels and levels L-3.. in phase A, levels L-2 in phase B), 16-row bands; back to
    the default selection from frame 3 on."""
    run_against_alone(ffb, cuda, STREAMS, tuning=(3000, 16), retune=(-1, 0))


def test_batch_default_selection_streams_large_levels(ffb, cuda):
    """Levels as large as the ones a single filter streams take the streaming launches by
    default, beside small streams in the tile launches."""
    streams = [
        (480, 640, 2, [10.0, 50.0], [2, 4], 4.0, 3),
        (544, 960, 1, [20.0], [3], 4.0, 3),
        (96, 128, 3, [5.0, 20.0, 50.0], [1, 2, 4], 4.0, 2),
        (480, 640, 3, [5.0, 10.0, 30.0], [1, 1, 2], 4.0, 3),
        (61, 77, 2, [4.0, 30.0], [1, 3], 2.0, 3),
    ]
    seen = []
    run_against_alone(ffb, cuda, streams, t_frames=6, launches=seen.append)
    assert seen[0] > 1 + (3 - 1) + 2


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
    four frames.  Its large levels run the batched streaming kernel at the batch's own bands."""
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
    assert batch.launches() > 1 + 2 + 2  # streaming launches are in the step
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
