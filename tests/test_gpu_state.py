"""Checkpoint and resume (ff_filter_state_bytes / ff_filter_export_state /
ff_filter_import_state): a filter that imports another's state continues that stream
exactly; mismatched or corrupt state images are rejected."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from make_reference_fixtures import case_frames

pytestmark = pytest.mark.gpu

H, W = 96, 128


@pytest.fixture(scope="module")
def ffb(cuda):
    import flowfilter_b200

    return flowfilter_b200


def frames(t, seed=3):
    return case_frames(dict(seq="bumps", frames=t, kw=dict(height=H, width=W, sigma=1.0, seed=seed, n_bumps=2,
                                                          bump_sigma=W / 3, amp=2.0)))


def make(ffb, kind):
    if kind == "single":
        return ffb.FlowFilter(H, W, 2, 3.0, 10.0)
    f = ffb.PyramidalFlowFilter(H, W, 3)
    f.gamma = [5.0, 20.0, 50.0]
    f.smoothIterations = [1, 2, 4]
    f.maxflow = 4.0
    return f


@pytest.mark.parametrize("kind", ["single", "pyramidal"])
def test_resumed_filter_continues_the_stream(ffb, cuda, kind):
    seq = frames(8)
    a = make(ffb, kind)
    for t in range(4):
        a.loadImage(seq[t])
        a.compute()
    state = a.exportState()
    b = make(ffb, kind)
    if kind == "pyramidal":
        b.setGraphs(True)  # frames after the import replay graphs captured with the imported flags
    b.importState(state)
    np.testing.assert_array_equal(b.getFlow(), a.getFlow())
    np.testing.assert_array_equal(b.getImage(), a.getImage())
    for t in range(4, 8):
        for f in (a, b):
            f.loadImage(seq[t])
            f.compute()
        np.testing.assert_array_equal(b.getFlow(), a.getFlow(), err_msg=f"frame {t}")
        np.testing.assert_array_equal(b.getImage(), a.getImage(), err_msg=f"frame {t}")
    np.testing.assert_array_equal(b.exportState(), a.exportState())


def test_fresh_state_restarts_a_used_filter(ffb, cuda):
    seq = frames(6, seed=4)
    state0 = make(ffb, "pyramidal").exportState()
    used = make(ffb, "pyramidal")
    for t in range(3):
        used.loadImage(seq[5 - t])
        used.compute()
    used.importState(state0)
    new = make(ffb, "pyramidal")
    for t in range(3):
        for f in (used, new):
            f.loadImage(seq[t])
            f.compute()
        np.testing.assert_array_equal(used.getFlow(), new.getFlow(), err_msg=f"frame {t}")


def test_state_images_are_checked(ffb, cuda):
    from flowfilter_b200 import _lib

    a = make(ffb, "pyramidal")
    a.loadImage(frames(1)[0])
    a.compute()
    s = a.exportState()
    with pytest.raises(ValueError):
        ffb.PyramidalFlowFilter(H, W, 2).importState(s)  # level count
    with pytest.raises(ValueError):
        ffb.PyramidalFlowFilter(H, W + 2, 3).importState(s)  # level sizes
    with pytest.raises(ValueError):
        ffb.FlowFilter(H, W).importState(s)  # filter kind
    with pytest.raises(ValueError):
        a.importState(s[:-1])  # size
    bad = s.copy()
    bad[0] ^= 1
    with pytest.raises(ValueError):
        a.importState(bad)  # not a state image
    small = np.empty(s.size - 1, dtype=np.uint8)
    st = _lib.lib().ff_filter_export_state(a._h, small.ctypes.data_as(ctypes.c_void_p), small.size)
    assert st == _lib.FF_ERR_INVALID_ARGUMENT
    a.importState(s)  # the filter is unchanged by the rejected imports
    np.testing.assert_array_equal(a.exportState(), s)


def test_state_moves_between_frames_only(ffb, cuda):
    from flowfilter_b200._lib import FFLogicError

    f = make(ffb, "single")
    f.loadImage(frames(1)[0])
    f.computeImageModel()
    with pytest.raises(FFLogicError):
        f.exportState()
    f.computePropagation()
    f.computeUpdate()
    f.importState(f.exportState())


@pytest.mark.parametrize("kind", ["single", "pyramidal"])
def test_import_after_pipelined_frames_keeps_their_flows(ffb, cuda, kind):
    """importState right after processAsync (no synchronize in between) waits for the pipelined
    downloads: every output buffer holds the flow its frame computed, not the imported state."""
    import torch

    seq = frames(6, seed=5)
    want = make(ffb, kind)
    flows = []
    for t in range(4):
        want.loadImage(seq[t])
        want.compute()
        flows.append(want.getFlow())
    other = make(ffb, kind)
    for t in range(2):
        other.loadImage(seq[5 - t])
        other.compute()
    state = other.exportState()
    f = make(ffb, kind)
    host = torch.from_numpy(seq[:4].copy()).pin_memory()
    outs = [torch.full((H, W, 2), -7.0, dtype=torch.float32).pin_memory() for _ in range(4)]
    for t in range(4):
        f.processAsync(host[t], outs[t])
    f.importState(state)
    for t in range(4):
        np.testing.assert_array_equal(outs[t].numpy(), flows[t], err_msg=f"frame {t}")
    np.testing.assert_array_equal(f.exportState(), state)
    exported = f.exportState()
    g = make(ffb, kind)
    for t in range(2):
        g.processAsync(host[t], outs[t])
    e = g.exportState()  # export after pipelined frames sees their state
    np.testing.assert_array_equal(outs[1].numpy(), flows[1])
    h = make(ffb, kind)
    for t in range(2):
        h.loadImage(seq[t])
        h.compute()
    np.testing.assert_array_equal(e, h.exportState())
    assert exported.size == e.size
