"""Differentiable filter (ff_diff_* kernels, flowfilter_b200.diff): forward parity with the
oracle, adjoints against finite differences, FP64 gradients against the FP64 oracle."""

from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from oracle import diff_oracle as D

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dm(cuda):
    from flowfilter_b200 import diff

    return diff


def float_frames(B, T, H, W, seed):
    from flowfilter_b200 import synthetic

    seqs = [synthetic.seq_bumps_float(frames=T, height=H, width=W, seed=seed + b, n_bumps=2,
                                      bump_sigma=max(H, W) / 3, amp=1.5)[0] for b in range(B)]
    return np.stack(seqs).astype(np.float32)


def oracle_fp32_sequence(frames, gamma, smooth, maxflow, levels, border=3):
    """The float pyramidal filter composed from the FP32 oracle stages, as configure() wires
    ImagePyramid(float) + FlowFilter(GPUImage) + DeltaFlowFilter (flowfilter.cu:650-716)."""
    B, T, H, W = frames.shape
    mf = D.level_maxflow(maxflow, levels)
    iters = [int(np.ceil(m)) for m in mf]
    out = np.zeros((B, T, H, W, 2), np.float32)
    for b in range(B):
        shapes = [(H, W)]
        for _ in range(1, levels):
            shapes.append((shapes[-1][0] // 2, shapes[-1][1] // 2))
        st = [[np.zeros((h, w, 2), np.float32), np.zeros((h, w), np.float32), np.zeros((h, w, 2), np.float32)]
              for h, w in shapes]
        for t in range(T):
            first = t == 0
            imgs = [frames[b, t]]
            for _ in range(1, levels):
                imgs.append(O.pyramid_down(imgs[-1]))
            new = [None] * levels
            top = levels - 1
            a0, g = O.image_model(imgs[top])
            f = O.propagate(st[top][0], iters[top], border)
            fu, _ = O.update(a0, g, a0 if first else st[top][1], f, gamma[top], mf[top])
            new[top] = [O.smooth(fu, smooth[top]), a0, st[top][2]]
            for l in range(levels - 2, -1, -1):
                a0, g = O.image_model(imgs[l])
                f, s, v = O.propagate_payload(st[l][0], st[l][1], st[l][2], iters[l], border)
                coarse = fu if l == levels - 2 else st[l + 1][0]
                flow, d, _ = O.delta_update(a0, g, a0 if first else s, v, coarse, gamma[l], mf[l])
                new[l] = [O.smooth(flow, smooth[l]), a0, d]
            out[b, t] = new[0][0] if levels > 1 else fu
            st = new
    return out


@pytest.mark.parametrize("levels", [1, 2, 3])
def test_fp32_forward_equals_the_reference_float_path(dm, cuda, levels):
    B, T, H, W = 2, 5, 37, 53
    frames = float_frames(B, T, H, W, 3)
    gamma, smooth = [5.0, 20.0, 50.0][:levels], [2, 1, 3][:levels]
    f = dm.DiffPyramidalFlowFilter(H, W, levels, gamma, smooth, maxflow=4.0, checkpoint_every=2)
    with cuda.no_grad():
        got = f(cuda.from_numpy(frames).cuda()).cpu().numpy()
    want = oracle_fp32_sequence(frames, gamma, smooth, 4.0, levels)
    np.testing.assert_array_equal(got, want)


def test_fp32_forward_at_the_benchmark_size(dm, cuda):
    """The differentiable filter's float32 forward on the full benchmark batch (16 sequences of
    32 frames of 256x256, seeded bump flows from seed 200 + b, 2 levels, gamma [10, 50],
    smoothing [2, 4], maxflow 4) equals the reference float path composed from the oracle's
    stages, bit for bit."""
    from flowfilter_b200 import synthetic

    B, T, H, W = 16, 32, 256, 256
    frames = np.stack([synthetic.seq_bumps_float(frames=T, height=H, width=W, seed=200 + b, n_bumps=8,
                                                 bump_sigma=40.0, amp=2.0)[0] for b in range(B)])
    gamma, smooth = [10.0, 50.0], [2, 4]
    f = dm.DiffPyramidalFlowFilter(H, W, 2, gamma, smooth, maxflow=4.0, checkpoint_every=8)
    with cuda.no_grad():
        got = f(cuda.from_numpy(frames).cuda()).cpu().numpy()
    want = oracle_fp32_sequence(frames, gamma, smooth, 4.0, 2)
    assert np.max(np.abs(got - want)) <= 1e-4  # the stated tolerance ...
    np.testing.assert_array_equal(got, want)  # ... and in fact bit-exact


def test_fp64_forward_matches_fp64_oracle(dm, cuda):
    B, T, H, W = 2, 6, 24, 32
    frames = float_frames(B, T, H, W, 7).astype(np.float64)
    gamma, smooth = [3.0, 30.0], [1, 2]
    f = dm.DiffPyramidalFlowFilter(H, W, 2, gamma, smooth, maxflow=4.0, dtype=cuda.float64, checkpoint_every=3)
    w = np.full((2, 5), 0.2) + np.array([[0.01, -0.02, 0.03, 0.0, -0.01], [0.0, 0.01, -0.01, 0.02, 0.0]])
    with cuda.no_grad():
        f.weights.copy_(cuda.from_numpy(w))
        got = f(cuda.from_numpy(frames).cuda()).cpu().numpy()
    want = D.run(frames, gamma, w, 2, smooth, 4.0)
    assert np.max(np.abs(got - want)) <= 1e-12 * max(1.0, np.max(np.abs(want)))


def test_stage_adjoints_gradcheck(dm, cuda):
    """Every stage's adjoint kernel against numerical differentiation of its forward (FP64)."""
    F = dm.stages()
    gc = cuda.autograd.gradcheck
    rng = np.random.default_rng(0)
    dev = "cuda"

    def t(*shape, scale=1.0, offset=0.0):
        return cuda.tensor(rng.normal(offset, scale, shape), dtype=cuda.float64, device=dev, requires_grad=True)

    B, H, W = 2, 9, 11
    for ph, pw in [(9, 11), (20, 28), (35, 70)]:  # odd and even sizes; grids wider than one block
        assert gc(lambda x: F["Pyramid"].apply(x), (t(B, ph, pw),), eps=1e-6, atol=1e-8)
    assert gc(lambda x: F["Model"].apply(x), (t(B, H, W),), eps=1e-6, atol=1e-8)
    for axis in (0, 1):
        assert gc(lambda f: F["PropFlow"].apply(f, axis, 0.25, 2), (t(B, H, W, 2),), eps=1e-6, atol=1e-8)
        assert gc(lambda f: F["PropFlow"].apply(f, axis, 0.5, 0), (t(1, 12, 40, 2),), eps=1e-6, atol=1e-8)
        assert gc(lambda f, s, v: F["PropPayload"].apply(f, s, v, axis, 0.5, 1),
                  (t(B, H, W, 2), t(B, H, W), t(B, H, W, 2)), eps=1e-6, atol=1e-8)
        w5 = cuda.tensor([0.1, 0.25, 0.3, 0.2, 0.15], dtype=cuda.float64, device=dev, requires_grad=True)
        assert gc(lambda x, w: F["Smooth"].apply(x, w, axis), (t(B, H, W, 2), w5), eps=1e-6, atol=1e-8)
    gam = cuda.tensor([0.7], dtype=cuda.float64, device=dev, requires_grad=True)
    args = (t(B, H, W), t(B, H, W, 2, scale=0.3), t(B, H, W), t(B, H, W, 2, scale=0.5), gam)
    assert gc(lambda a0, g, old, fh, gm: F["Update"].apply(a0, g, old, fh, gm, 50.0), args, eps=1e-6, atol=1e-8)
    coarse = t(B, 4, 5, 2, scale=0.3)
    args = (t(B, H, W), t(B, H, W, 2, scale=0.3), t(B, H, W), t(B, H, W, 2, scale=0.5), coarse, gam)
    assert gc(lambda a0, g, old, dh, c, gm: F["DeltaUpdate"].apply(a0, g, old, dh, c, gm, 50.0), args, eps=1e-6,
              atol=1e-8)


def test_clamped_values_pass_no_gradient(dm, cuda):
    F = dm.stages()
    B, H, W = 1, 6, 7
    a0 = cuda.zeros((B, H, W), dtype=cuda.float64, device="cuda")
    g = cuda.full((B, H, W, 2), 0.1, dtype=cuda.float64, device="cuda")
    fh = cuda.full((B, H, W, 2), 5.0, dtype=cuda.float64, device="cuda", requires_grad=True)
    gam = cuda.tensor([1.0], dtype=cuda.float64, device="cuda", requires_grad=True)
    out = F["Update"].apply(a0, g, a0, fh, gam, 1.0)  # |solution| ~ 5 > maxflow 1: clamped everywhere
    out.sum().backward()
    assert float(fh.grad.abs().max()) == 0.0 and float(gam.grad.abs().max()) == 0.0


def sequence_loss(flows, proj):
    return (flows * proj).sum()


def test_sequence_gradients_match_fp64_oracle_finite_differences(dm, cuda):
    """Gradients of a whole sequence (2 levels, checkpointed) w.r.t. gamma, the smoothing
    weights and input pixels, FP64 GPU adjoints vs central differences of the FP64 oracle."""
    B, T, H, W = 2, 6, 20, 28
    frames = float_frames(B, T, H, W, 11).astype(np.float64)
    gamma, smooth = [2.0, 15.0], [1, 2]
    rng = np.random.default_rng(1)
    proj = rng.normal(0, 1, (B, T, H, W, 2))
    f = dm.DiffPyramidalFlowFilter(H, W, 2, gamma, smooth, maxflow=4.0, dtype=cuda.float64, checkpoint_every=2)
    x = cuda.from_numpy(frames).cuda().requires_grad_(True)
    loss = sequence_loss(f(x), cuda.from_numpy(proj).cuda())
    loss.backward()
    g_gamma = f.gamma.grad.cpu().numpy()
    g_w = f.weights.grad.cpu().numpy()
    g_x = x.grad.cpu().numpy()

    w0 = np.full((2, 5), 0.2)

    def L(gm=gamma, w=w0, fr=frames):
        return float((D.run(fr, gm, w, 2, smooth, 4.0) * proj).sum())

    def fd(fun, h):
        return (fun(+h) - fun(-h)) / (2 * h)

    def close(a, b, what):
        assert abs(a - b) <= 1e-6 * max(abs(b), 1e-4), (what, a, b)

    for l in range(2):
        h = 1e-6 * gamma[l]
        num = fd(lambda e: L(gm=[g + (e if i == l else 0.0) for i, g in enumerate(gamma)]), h)
        close(g_gamma[l], num, f"gamma[{l}]")
    for l, k in [(0, 0), (0, 2), (1, 1), (1, 4)]:
        def fw(e, l=l, k=k):
            w = w0.copy()
            w[l, k] += e
            return L(w=w)

        close(g_w[l, k], fd(fw, 1e-6), f"weights[{l},{k}]")
    for (b, t, yy, xx) in [(0, 0, 5, 7), (1, 3, 10, 14), (0, 5, 19, 0)]:
        def fx(e, b=b, t=t, yy=yy, xx=xx):
            fr = frames.copy()
            fr[b, t, yy, xx] += e
            return L(fr=fr)

        # h = 1e-5: rounding noise of the loss / h stays near 1e-11, truncation below that
        close(g_x[b, t, yy, xx], fd(fx, 1e-5), f"frame[{b},{t},{yy},{xx}]")


def test_fp32_gradients_follow_fp64(dm, cuda):
    B, T, H, W = 2, 5, 24, 32
    frames = float_frames(B, T, H, W, 13)
    proj = np.random.default_rng(2).normal(0, 1, (B, T, H, W, 2))
    grads = []
    for dtype in (cuda.float32, cuda.float64):
        f = dm.DiffPyramidalFlowFilter(H, W, 2, [4.0, 25.0], [2, 1], maxflow=4.0, dtype=dtype, checkpoint_every=3)
        flows = f(cuda.from_numpy(frames).cuda().to(dtype))
        sequence_loss(flows, cuda.from_numpy(proj).cuda().to(dtype)).backward()
        grads.append(np.concatenate([f.gamma.grad.double().cpu().numpy(), f.weights.grad.double().cpu().numpy().ravel()]))
    assert np.linalg.norm(grads[0] - grads[1]) <= 1e-3 * np.linalg.norm(grads[1])


def test_checkpointing_leaves_gradients_unchanged(dm, cuda):
    B, T, H, W = 1, 7, 16, 24
    frames = cuda.from_numpy(float_frames(B, T, H, W, 17).astype(np.float64)).cuda()
    proj = cuda.from_numpy(np.random.default_rng(3).normal(0, 1, (B, T, H, W, 2))).cuda()
    out = []
    for every in (2, 100):
        f = dm.DiffPyramidalFlowFilter(H, W, 2, [3.0, 9.0], [1, 1], maxflow=4.0, dtype=cuda.float64,
                                       checkpoint_every=every)
        sequence_loss(f(frames), proj).backward()
        out.append(np.concatenate([f.gamma.grad.cpu().numpy(), f.weights.grad.cpu().numpy().ravel()]))
    np.testing.assert_allclose(out[0], out[1], rtol=1e-12, atol=1e-14)


def test_fitting_gamma_lowers_endpoint_error(dm, cuda):
    """A few Adam steps (DiffPyramidalFlowFilter.fit) on log-gamma, then on log-gamma and the
    smoothing weights, against the known flow of a synthetic sequence."""
    from flowfilter_b200 import synthetic

    B, T, H, W = 2, 10, 48, 64
    seqs, truth = [], []
    for b in range(B):
        fr, u, v = synthetic.seq_bumps_float(frames=T, height=H, width=W, seed=40 + b, n_bumps=2, bump_sigma=20.0,
                                             amp=1.0)
        seqs.append(fr)
        truth.append(np.broadcast_to(np.stack([u, v], -1), (T, H, W, 2)))
    frames = cuda.from_numpy(np.stack(seqs)).cuda()
    truth = cuda.from_numpy(np.ascontiguousarray(np.stack(truth)).astype(np.float32)).cuda()
    f = dm.DiffPyramidalFlowFilter(H, W, 2, [200.0, 200.0], [1, 1], maxflow=4.0, checkpoint_every=5)
    res = f.fit(frames, truth, steps=12, lr=0.3, first=4, fit_weights=False)
    assert res["final"] < res["losses"][0]
    # gamma and the smoothing weights together: finite throughout, weights positive summing to 1
    g = dm.DiffPyramidalFlowFilter(H, W, 2, [200.0, 200.0], [1, 1], maxflow=4.0, checkpoint_every=5)
    res = g.fit(frames, truth, steps=12, lr=0.1, first=4, fit_weights=True)
    assert np.all(np.isfinite(res["losses"])) and res["final"] < res["losses"][0]
    w = g.weights.detach().cpu().numpy()
    assert (w > 0).all() and np.allclose(w.sum(1), 1.0, atol=1e-5)
    assert (g.gamma.detach().cpu().numpy() > 0).all()


@pytest.mark.parametrize("levels,smooth", [(1, [1]), (2, [1, 2]), (3, [1, 2, 1]), (2, [0, 1]), (3, [2, 0, 1])])
def test_frame_node_matches_per_stage_nodes(dm, cuda, levels, smooth):
    """The single autograd node per frame (ff_diff_frame_forward / _backward) gives the
    per-stage nodes' flows and gradients, zero smoothing iterations included."""
    B, T, H, W = 2, 5, 26, 34
    frames = cuda.from_numpy(float_frames(B, T, H, W, 23).astype(np.float64)).cuda()
    proj = cuda.from_numpy(np.random.default_rng(5).normal(0, 1, (B, T, H, W, 2))).cuda()
    res = []
    for per_stage in (False, True):
        f = dm.DiffPyramidalFlowFilter(H, W, levels, [3.0, 12.0, 40.0][:levels], smooth, maxflow=4.0,
                                       dtype=cuda.float64, checkpoint_every=2)
        f.per_stage = per_stage
        x = frames.clone().requires_grad_(True)
        flows = f(x)
        sequence_loss(flows, proj).backward()
        res.append((flows.detach().cpu().numpy(), f.gamma.grad.cpu().numpy(), f.weights.grad.cpu().numpy(),
                    x.grad.cpu().numpy()))
    np.testing.assert_array_equal(res[0][0], res[1][0])
    for a, b in zip(res[0][1:], res[1][1:]):
        np.testing.assert_allclose(a, b, rtol=1e-11, atol=1e-13)


def test_frame_node_rejects_bad_geometry(dm, cuda):
    """Level sizes that do not halve are refused by the library before any launch."""
    f = dm.DiffPyramidalFlowFilter(20, 28, 2, dtype=cuda.float32)
    g = dm._geom(f, 1)
    g.height[1] = 11
    assert dm.lib().ff_diff_frame_tape_bytes(0, dm.ctypes.byref(g)) == 0
    with pytest.raises(ValueError):
        dm._workspace("ff_diff_frame_tape_bytes", 0, g, cuda.zeros(1, device="cuda"))


@pytest.mark.parametrize("levels,dtype", [(1, "float32"), (2, "float32"), (3, "float64")])
def test_forward_without_tape_equals_forward_with_tape(dm, cuda, levels, dtype):
    """Under no_grad the frames run without a tape (ff_diff_frame_infer): the flows are the
    ones the taped forward gives, bit for bit."""
    B, T, H, W = 2, 6, 40, 56
    frames = cuda.from_numpy(float_frames(B, T, H, W, 11).astype(dtype)).cuda()
    gamma, smooth = [4.0, 15.0, 40.0][:levels], [1, 3, 0][:levels]
    f = dm.DiffPyramidalFlowFilter(H, W, levels, gamma, smooth, maxflow=3.0, checkpoint_every=T,
                                   dtype=getattr(cuda, dtype))
    with cuda.no_grad():
        free = f(frames)
    taped = f(frames.clone().requires_grad_(True)).detach()
    assert free.dtype == taped.dtype
    np.testing.assert_array_equal(free.cpu().numpy(), taped.cpu().numpy())


@pytest.mark.parametrize("first,eps,broadcast,dtype", [(0, 0.0, False, "float32"), (8, 1e-12, True, "float32"),
                                                       (3, 0.0, True, "float64"), (1, 0.5, False, "float64")])
def test_endpoint_error_kernels_match_the_formula(dm, cuda, first, eps, broadcast, dtype):
    """ff_diff_epe / ff_diff_epe_bwd (the loss on CUDA tensors) against the formula through
    torch autograd, with a broadcast truth frame and exact zeros in the difference."""
    torch = cuda
    dt = getattr(torch, dtype)
    rng = np.random.default_rng(first + 11)
    B, T, H, W = 3, 10, 17, 29
    flows = torch.from_numpy(rng.normal(0, 1, (B, T, H, W, 2))).to(dt).cuda()
    truth = torch.from_numpy(rng.normal(0, 1, (B, 1 if broadcast else T, H, W, 2))).to(dt).cuda()
    if broadcast:
        truth = truth.expand(B, T, H, W, 2)
    flows[0, -1, 0, :3] = truth[0, -1, 0, :3]  # |d| = 0 pixels
    res = []
    for fn in (dm.endpoint_error, lambda f, t, a, e: ((f[:, a:] - t[:, a:]) ** 2).sum(-1).add(e).sqrt().mean()):
        x = flows.clone().requires_grad_(True)
        loss = fn(x, truth, first, eps)
        (3.0 * loss).backward()
        res.append((loss.item(), x.grad.double().cpu().numpy()))
    tol = 1e-5 if dtype == "float32" else 1e-12
    assert res[0][0] == pytest.approx(res[1][0], rel=tol)
    g0, g1 = res[0][1], res[1][1]
    if eps == 0:  # the formula's gradient is NaN where |d| = 0; the kernel's is zero
        assert not g0[0, -1, 0, :3].any()
        g0[0, -1, 0, :3] = g1[0, -1, 0, :3] = 0
    np.testing.assert_allclose(g0, g1, rtol=tol, atol=tol * np.abs(g1).max())
    assert not g0[:, :first].any()
