"""The endpoint-error loss of the differentiable filter (flowfilter_b200.diff.endpoint_error):
its single autograd node gives the value and the flow gradient of the plain formula
sqrt(dx^2 + dy^2 + eps) averaged over frames first.. (torch on the CPU, float64)."""

from __future__ import annotations

import numpy as np
import pytest


def reference(flows, truth, first, eps):
    d = flows[:, first:] - truth[:, first:]
    return (d[..., 0] ** 2 + d[..., 1] ** 2 + eps).sqrt().mean()


@pytest.mark.parametrize("first,eps,broadcast", [(0, 0.0, False), (2, 0.0, True), (3, 1e-12, False), (1, 0.25, True)])
def test_endpoint_error_matches_the_formula(first, eps, broadcast):
    torch = pytest.importorskip("torch")
    from flowfilter_b200 import diff

    rng = np.random.default_rng(7 + first)
    B, T, H, W = 2, 5, 6, 7
    flows = torch.from_numpy(rng.normal(0, 1, (B, T, H, W, 2)))
    truth = torch.from_numpy(rng.normal(0, 1, (B, 1 if broadcast else T, H, W, 2)))
    if broadcast:
        truth = truth.expand(B, T, H, W, 2)
    grads = []
    for fn in (diff.endpoint_error, reference):
        x = flows.clone().requires_grad_(True)
        loss = fn(x, truth, first, eps)
        loss.backward()
        grads.append((loss.item(), x.grad.numpy()))
    assert grads[0][0] == pytest.approx(grads[1][0], rel=1e-12)
    np.testing.assert_allclose(grads[0][1], grads[1][1], rtol=1e-10, atol=1e-15)
    assert not grads[0][1][:, :first].any()


def test_endpoint_error_gradient_is_zero_where_the_flow_is_exact():
    torch = pytest.importorskip("torch")
    from flowfilter_b200 import diff

    flows = torch.zeros(1, 2, 3, 4, 2, dtype=torch.float64, requires_grad=True)
    truth = torch.zeros(1, 2, 3, 4, 2, dtype=torch.float64)
    truth[0, 1, 0, 0, 0] = 3.0
    truth[0, 1, 0, 0, 1] = 4.0
    loss = diff.endpoint_error(flows, truth)
    loss.backward()
    assert loss.item() == pytest.approx(5.0 / 24)
    g = flows.grad.numpy()
    np.testing.assert_allclose(g[0, 1, 0, 0], [-3.0 / 5 / 24, -4.0 / 5 / 24])
    g[0, 1, 0, 0] = 0
    assert not g.any() and np.isfinite(g).all()
