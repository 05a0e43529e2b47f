"""FP64 ORACLE of the differentiable (float-input) filter — TEST INFRASTRUCTURE ONLY.

A numpy float64 restatement of the pyramidal filter's per-frame recurrence on float images
(the reference's float path: pyramid_k.cu:81-145, imagemodel_k.cu:31-133,
propagation_k.cu:16-334, update_k.cu:15-173, flowsmoothing_k.cu:21-87, schedule
flowfilter.cu:685-716), with per-level 5-tap smoothing weights (0.2 each is the reference's
box).  tests/ use it to check the float64 GPU path's forward values and, by central finite
differences, its adjoint gradients.  The product never imports it.

Arrays: images (B, H, W), flows (B, H, W, 2).
"""

from __future__ import annotations

import math

import numpy as np

S5 = np.array([1 / 16, 1 / 4, 3 / 8, 1 / 4, 1 / 16])
D5 = np.array([-1 / 8, -1 / 4, 0.0, 1 / 4, 1 / 8])


def shift(a, axis: int, k: int):
    """a sampled at index + k along `axis`, clamped to the edge."""
    n = a.shape[axis]
    idx = np.clip(np.arange(n) + k, 0, n - 1)
    return np.take(a, idx, axis=axis)


def pyramid(img):
    """pyramid_k.cu:81-145 (float): X pass then Y pass of 0.5 c + 0.25 (m + p) at 2x."""
    B, H, W = img.shape
    h, w = H // 2, W // 2
    cx = lambda o: np.clip(2 * np.arange(w) + o, 0, W - 1)  # noqa: E731
    X = 0.5 * img[:, :, cx(0)] + 0.25 * (img[:, :, cx(-1)] + img[:, :, cx(1)])
    cy = lambda o: np.clip(2 * np.arange(h) + o, 0, H - 1)  # noqa: E731
    return 0.5 * X[:, cy(0), :] + 0.25 * (X[:, cy(-1), :] + X[:, cy(1), :])


def model(img):
    """imagemodel_k.cu:31-133: a0, (ax, ay)."""
    by = sum(S5[r] * shift(img, 1, r - 2) for r in range(5))
    bx = sum(S5[c] * shift(img, 2, c - 2) for c in range(5))
    a0 = sum(S5[c] * shift(by, 2, c - 2) for c in range(5))
    ax = sum(D5[c] * shift(by, 2, c - 2) for c in range(5))
    ay = sum(D5[r] * shift(bx, 1, r - 2) for r in range(5))
    return a0, np.stack([ax, ay], -1)


def inside(shape, border: int):
    B, H, W = shape[:3]
    y = np.arange(H)[:, None]
    x = np.arange(W)[None, :]
    return ((x >= border) & (x < W - border) & (y >= border) & (y < H - border))[None]


def propagate(f, s, v, axis: int, dt: float, border: int):
    """One upwind sub-step along axis 0 (X) or 1 (Y) (propagation_k.cu:16-334); s, v may be None."""
    ax = 2 if axis == 0 else 1
    fm, fp = shift(f, ax, -1), shift(f, ax, 1)
    vm, vp = fm[..., axis], fp[..., axis]
    dv = np.where(np.abs(vp) - np.abs(vm) > 0, vp, vm)
    t = dt * dv
    ins = inside(f.shape, border)

    def up(g):
        gm, gp = shift(g, ax, -1), shift(g, ax, 1)
        tt = t if g.ndim == 3 else t[..., None]
        dd = dv if g.ndim == 3 else dv[..., None]
        o = g - tt * np.where(dd >= 0, g - gm, gp - g)
        m = ins if g.ndim == 3 else ins[..., None]
        return np.where(m, o, g)

    return up(f), (up(s) if s is not None else None), (up(v) if v is not None else None)


def solve(gamma, grad, yt, fh):
    ax, ay = grad[..., 0], grad[..., 1]
    n00, n11, n01 = gamma + ay * ay, gamma + ax * ax, -ax * ay
    rdet = 1.0 / (gamma * (gamma + ax * ax + ay * ay))
    qx, qy = gamma * fh[..., 0] + ax * yt, gamma * fh[..., 1] + ay * yt
    return np.stack([(n00 * qx + n01 * qy) * rdet, (n01 * qx + n11 * qy) * rdet], -1)


def sanitize(a):
    return np.where(np.isfinite(a), a, 0.0)


def update(a0, grad, old, fh, gamma, maxflow):
    """flowUpdate_k (update_k.cu:15-79)."""
    return sanitize(np.clip(solve(gamma, grad, old - a0, fh), -maxflow, maxflow))


def upmap(n: int, nc: int):
    """Coarse index of each fine index: normalised coordinate truncated to 21 bits (texture)."""
    out = np.empty(n, dtype=np.int64)
    for i in range(n):
        u = np.float32(i) / np.float32(n - 1) if n > 1 else np.float32(np.nan)
        if not (u == u):
            out[i] = 0
            continue
        q = int(math.floor(float(np.float32(u * np.float32(2097152.0)))))
        out[i] = min(max((q * nc) >> 21, 0), nc - 1)
    return out


def delta_update(a0, grad, old, dh, coarse, gamma, maxflow):
    """deltaFlowUpdate_k (update_k.cu:82-173): returns (flow, delta)."""
    B, H, W = a0.shape
    hm = 0.5 * maxflow
    d = np.clip(sanitize(solve(gamma, grad, old - a0, dh)), -hm, hm)
    up = coarse[:, upmap(H, coarse.shape[1])][:, :, upmap(W, coarse.shape[2])]
    return np.clip(d + 2.0 * up, -maxflow, maxflow), d


def smooth(x, w, axis: int):
    ax = 2 if axis == 0 else 1
    return sum(w[k] * shift(x, ax, k - 2) for k in range(5))


def level_maxflow(maxflow: float, levels: int):
    out, m = [], np.float32(maxflow)
    for _ in range(levels - 1):
        out.append(float(m))
        m = np.float32(m / np.float32(2.0))
    out.append(float(m))
    return out if levels > 1 else [float(np.float32(maxflow))]


def run(frames, gamma, weights, levels: int, smooth_iters, maxflow: float, border: int = 3):
    """frames (B, T, H, W) float64 -> level-0 flow per frame (B, T, H, W, 2)."""
    frames = np.asarray(frames, np.float64)
    B, T, H, W = frames.shape
    L = levels
    mf = level_maxflow(maxflow, L)
    iters = [int(math.ceil(m)) for m in mf]
    shapes = [(H, W)]
    for _ in range(1, L):
        shapes.append((shapes[-1][0] // 2, shapes[-1][1] // 2))
    st = [[np.zeros((B, h, w, 2)), np.zeros((B, h, w)), np.zeros((B, h, w, 2))] for h, w in shapes]
    out = []
    for t in range(T):
        first = t == 0
        imgs = [frames[:, t]]
        for _ in range(1, L):
            imgs.append(pyramid(imgs[-1]))
        new = [None] * L
        top = L - 1
        a0, g = model(imgs[top])
        f = st[top][0]
        for _ in range(iters[top]):
            f = propagate(f, None, None, 0, 1.0 / iters[top], border)[0]
            f = propagate(f, None, None, 1, 1.0 / iters[top], border)[0]
        fu = update(a0, g, a0 if first else st[top][1], f, gamma[top], mf[top])
        fs = fu
        for _ in range(smooth_iters[top]):
            fs = smooth(smooth(fs, weights[top], 0), weights[top], 1)
        new[top] = [fs, a0, st[top][2]]
        for l in range(L - 2, -1, -1):
            a0, g = model(imgs[l])
            f, s, v = st[l]
            for _ in range(iters[l]):
                f, s, v = propagate(f, s, v, 0, 1.0 / iters[l], border)
                f, s, v = propagate(f, s, v, 1, 1.0 / iters[l], border)
            coarse = fu if l == L - 2 else st[l + 1][0]
            flow, d = delta_update(a0, g, a0 if first else s, v, coarse, gamma[l], mf[l])
            for _ in range(smooth_iters[l]):
                flow = smooth(smooth(flow, weights[l], 0), weights[l], 1)
            new[l] = [flow, a0, d]
        out.append(new[0][0] if L > 1 else fu)
        st = new
    return np.stack(out, 1)
