"""Differentiable flow filter: hand-written adjoint kernels behind torch.autograd.Function.

No counterpart in the reference.  The forward recurrence is the reference's pyramidal
filter on float32 images in [0, 1] (the float path of ImagePyramid, FlowFilter(GPUImage)
and DeltaFlowFilter, src/gpu/flowfilter.cu:621-716; gamma used unscaled for float input,
:279-284), run by the ff_diff_* kernels of libffb200.so in float32 or float64.  Every stage
has an autograd Function whose backward is the matching adjoint kernel (``stages()``); the
filter itself runs each frame as one autograd node (FrameStep) that calls the same forward
kernels and, in its backward, the adjoint kernels in reverse order.  The time recurrence
is chained by autograd and cut into checkpointed segments (recomputed in the backward pass)
of ``checkpoint_every`` frames.

Parameters with gradients: per-level gamma, per-level 5-tap smoothing weights (the reference
smooths with the 0.2 box, the default here, which reproduces it bit for bit in float32) and
the input frames.
"""

from __future__ import annotations

import ctypes
import math

from ._lib import call


def _torch():
    import torch

    return torch


def _dt(x) -> int:
    return 1 if x.dtype == _torch().float64 else 0


def _stream():
    return ctypes.c_void_p(_torch().cuda.current_stream().cuda_stream)


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _c(t):
    return t.contiguous() if t is not None else None


def _zeros_like(t):
    return _torch().zeros_like(t)


def _grad_or_zero(g, like):
    return _c(g) if g is not None else _zeros_like(like)


def _functions():
    torch = _torch()
    Function = torch.autograd.Function

    class Pyramid(Function):
        @staticmethod
        def forward(ctx, img):
            img = _c(img)
            B, H, W = img.shape
            out = img.new_empty((B, H // 2, W // 2))
            call("ff_diff_pyramid", _dt(img), B, H, W, _p(img), _p(out), _stream())
            ctx.shape = (B, H, W)
            return out

        @staticmethod
        def backward(ctx, g):
            B, H, W = ctx.shape
            g = _c(g)
            gin = g.new_zeros((B, H, W))
            call("ff_diff_pyramid_bwd", _dt(g), B, H, W, _p(g), _p(gin), _stream())
            return gin

    class Model(Function):
        @staticmethod
        def forward(ctx, img):
            img = _c(img)
            B, H, W = img.shape
            a0 = img.new_empty((B, H, W))
            grad = img.new_empty((B, H, W, 2))
            call("ff_diff_model", _dt(img), B, H, W, _p(img), _p(a0), _p(grad), _stream())
            ctx.shape = (B, H, W)
            return a0, grad

        @staticmethod
        def backward(ctx, ga0, ggrad):
            B, H, W = ctx.shape
            like = ga0 if ga0 is not None else ggrad
            dtype, dev = like.dtype, like.device
            ga0 = _c(ga0) if ga0 is not None else torch.zeros((B, H, W), dtype=dtype, device=dev)
            ggrad = _c(ggrad) if ggrad is not None else torch.zeros((B, H, W, 2), dtype=dtype, device=dev)
            gby = torch.empty((B, H, W), dtype=dtype, device=dev)
            gbx = torch.empty((B, H, W), dtype=dtype, device=dev)
            gimg = torch.zeros((B, H, W), dtype=dtype, device=dev)
            call("ff_diff_model_bwd", _dt(ga0), B, H, W, _p(ga0), _p(ggrad), _p(gby), _p(gbx), _p(gimg), _stream())
            return gimg

    class PropFlow(Function):
        @staticmethod
        def forward(ctx, f, axis, dt, border):
            f = _c(f)
            B, H, W, _ = f.shape
            fo = torch.empty_like(f)
            call("ff_diff_propagate", _dt(f), B, H, W, axis, 0, dt, border, _p(f), None, None, _p(fo), None, None,
                 _stream())
            ctx.save_for_backward(f)
            ctx.args = (axis, dt, border)
            return fo

        @staticmethod
        def backward(ctx, gfo):
            (f,) = ctx.saved_tensors
            axis, dt, border = ctx.args
            B, H, W, _ = f.shape
            gfo = _grad_or_zero(gfo, f)
            gf = torch.zeros_like(f)
            call("ff_diff_propagate_bwd", _dt(f), B, H, W, axis, 0, dt, border, _p(f), None, None, _p(gfo), None,
                 None, _p(gf), None, None, _stream())
            return gf, None, None, None

    class PropPayload(Function):
        @staticmethod
        def forward(ctx, f, s, v, axis, dt, border):
            f, s, v = _c(f), _c(s), _c(v)
            B, H, W, _ = f.shape
            fo, so, vo = torch.empty_like(f), torch.empty_like(s), torch.empty_like(v)
            call("ff_diff_propagate", _dt(f), B, H, W, axis, 1, dt, border, _p(f), _p(s), _p(v), _p(fo), _p(so),
                 _p(vo), _stream())
            ctx.save_for_backward(f, s, v)
            ctx.args = (axis, dt, border)
            return fo, so, vo

        @staticmethod
        def backward(ctx, gfo, gso, gvo):
            f, s, v = ctx.saved_tensors
            axis, dt, border = ctx.args
            B, H, W, _ = f.shape
            gfo, gso, gvo = _grad_or_zero(gfo, f), _grad_or_zero(gso, s), _grad_or_zero(gvo, v)
            gf, gs, gv = torch.zeros_like(f), torch.zeros_like(s), torch.zeros_like(v)
            call("ff_diff_propagate_bwd", _dt(f), B, H, W, axis, 1, dt, border, _p(f), _p(s), _p(v), _p(gfo),
                 _p(gso), _p(gvo), _p(gf), _p(gs), _p(gv), _stream())
            return gf, gs, gv, None, None, None

    class Update(Function):
        @staticmethod
        def forward(ctx, a0, grad, old, fhat, gamma, maxflow):
            a0, grad, old, fhat, gamma = _c(a0), _c(grad), _c(old), _c(fhat), _c(gamma)
            B, H, W = a0.shape
            out = torch.empty_like(fhat)
            call("ff_diff_update", _dt(a0), B, H, W, _p(a0), _p(grad), _p(old), _p(fhat), _p(gamma), maxflow, _p(out),
                 _stream())
            ctx.save_for_backward(a0, grad, old, fhat, gamma)
            ctx.maxflow = maxflow
            return out

        @staticmethod
        def backward(ctx, gout):
            a0, grad, old, fhat, gamma = ctx.saved_tensors
            B, H, W = a0.shape
            gout = _grad_or_zero(gout, fhat)
            ga0, ggrad, gold, gfhat = (torch.zeros_like(t) for t in (a0, grad, old, fhat))
            ggamma = torch.zeros_like(gamma)
            call("ff_diff_update_bwd", _dt(a0), B, H, W, _p(a0), _p(grad), _p(old), _p(fhat), _p(gamma), ctx.maxflow,
                 _p(gout), _p(ga0), _p(ggrad), _p(gold), _p(gfhat), _p(ggamma), _stream())
            return ga0, ggrad, gold, gfhat, ggamma, None

    class DeltaUpdate(Function):
        @staticmethod
        def forward(ctx, a0, grad, old, dhat, coarse, gamma, maxflow):
            a0, grad, old, dhat, coarse, gamma = (_c(t) for t in (a0, grad, old, dhat, coarse, gamma))
            B, H, W = a0.shape
            Hc, Wc = coarse.shape[1:3]
            flow, delta = torch.empty_like(dhat), torch.empty_like(dhat)
            call("ff_diff_delta_update", _dt(a0), B, H, W, Hc, Wc, _p(a0), _p(grad), _p(old), _p(dhat), _p(coarse),
                 _p(gamma), maxflow, _p(flow), _p(delta), _stream())
            ctx.save_for_backward(a0, grad, old, dhat, coarse, gamma)
            ctx.maxflow = maxflow
            return flow, delta

        @staticmethod
        def backward(ctx, gflow, gdelta):
            a0, grad, old, dhat, coarse, gamma = ctx.saved_tensors
            B, H, W = a0.shape
            Hc, Wc = coarse.shape[1:3]
            gflow, gdelta = _grad_or_zero(gflow, dhat), _grad_or_zero(gdelta, dhat)
            ga0, ggrad, gold, gdhat, gcoarse, ggamma = (torch.zeros_like(t) for t in (a0, grad, old, dhat, coarse,
                                                                                     gamma))
            call("ff_diff_delta_update_bwd", _dt(a0), B, H, W, Hc, Wc, _p(a0), _p(grad), _p(old), _p(dhat),
                 _p(coarse), _p(gamma), ctx.maxflow, _p(gflow), _p(gdelta), _p(ga0), _p(ggrad), _p(gold), _p(gdhat),
                 _p(gcoarse), _p(ggamma), _stream())
            return ga0, ggrad, gold, gdhat, gcoarse, ggamma, None

    class Smooth(Function):
        @staticmethod
        def forward(ctx, x, w5, axis):
            x, w5 = _c(x), _c(w5)
            B, H, W, _ = x.shape
            out = torch.empty_like(x)
            call("ff_diff_smooth", _dt(x), B, H, W, axis, _p(w5), _p(x), _p(out), _stream())
            ctx.save_for_backward(x, w5)
            ctx.axis = axis
            return out

        @staticmethod
        def backward(ctx, gout):
            x, w5 = ctx.saved_tensors
            B, H, W, _ = x.shape
            gout = _grad_or_zero(gout, x)
            gx, gw = torch.zeros_like(x), torch.zeros_like(w5)
            call("ff_diff_smooth_bwd", _dt(x), B, H, W, ctx.axis, _p(w5), _p(x), _p(gout), _p(gx), _p(gw), _stream())
            return gx, gw, None

    return dict(Pyramid=Pyramid, Model=Model, PropFlow=PropFlow, PropPayload=PropPayload, Update=Update,
                DeltaUpdate=DeltaUpdate, Smooth=Smooth)


_F = None


def stages():
    """The stage autograd Functions (built on first use so importing needs no torch)."""
    global _F
    if _F is None:
        _F = _functions()
    return _F


def level_maxflow(maxflow: float, levels: int) -> list[float]:
    """Per-level maxflow of a pyramid: halved per level, the top at maxflow / 2^(L-1)
    (flowfilter.cu:849-866), computed in float32 as the filter does."""
    import numpy as np

    out, m = [], np.float32(maxflow)
    for _ in range(levels - 1):
        out.append(float(m))
        m = np.float32(m / np.float32(2.0))
    out.append(float(m))
    return out if levels > 1 else [float(np.float32(maxflow))]


class DiffPyramidalFlowFilter:
    """The pyramidal filter as a differentiable function of its frames and parameters.

    ``f = DiffPyramidalFlowFilter(height, width, levels, gamma, smoothIterations, maxflow)``;
    ``flows = f(frames)`` with ``frames`` a (B, T, H, W) CUDA tensor (float32 or float64,
    values in [0, 1]) returns the level-0 smoothed flow of every frame, (B, T, H, W, 2).
    ``f.gamma`` (L,) and ``f.weights`` (L, 5) are leaf tensors with ``requires_grad``.
    """

    def __init__(self, height: int, width: int, levels: int = 2, gamma=None, smoothIterations=None,
                 maxflow: float = 4.0, border: int = 3, dtype=None, checkpoint_every: int = 8, device="cuda"):
        torch = _torch()
        dtype = dtype or torch.float32
        self.H, self.W, self.L = int(height), int(width), int(levels)
        self.shapes = [(self.H, self.W)]
        for _ in range(1, self.L):
            h, w = self.shapes[-1]
            self.shapes.append((h // 2, w // 2))
        gamma = gamma if gamma is not None else [1.0] * self.L
        smooth = smoothIterations if smoothIterations is not None else [1] * self.L
        if len(gamma) != self.L or len(smooth) != self.L:
            raise ValueError("gamma and smoothIterations need one entry per level")
        self.gamma = torch.tensor(gamma, dtype=dtype, device=device, requires_grad=True)
        self.weights = torch.full((self.L, 5), 0.2, dtype=dtype, device=device, requires_grad=True)
        self.smooth = [int(s) for s in smooth]
        self.maxflow = level_maxflow(maxflow, self.L)
        self.iters = [int(math.ceil(m)) for m in self.maxflow]
        self.border = int(border)
        self.dtype = dtype
        self.checkpoint_every = int(checkpoint_every)
        self.per_stage = False

    def parameters(self):
        return [self.gamma, self.weights]

    def _smooth(self, x, l):
        F = stages()
        w = self.weights[l]
        for _ in range(self.smooth[l]):
            x = F["Smooth"].apply(x, w, 0)
            x = F["Smooth"].apply(x, w, 1)
        return x

    def initial_state(self, B: int):
        torch = _torch()
        st = []
        for l, (h, w) in enumerate(self.shapes):
            z2 = torch.zeros((B, h, w, 2), dtype=self.dtype, device=self.gamma.device)
            z1 = torch.zeros((B, h, w), dtype=self.dtype, device=self.gamma.device)
            st.append((z2, z1, z2.clone()))  # smoothed flow, old image, delta flow
        return st

    def step(self, frame, state, first: bool):
        """One frame for every sequence of the batch; returns (level-0 flow, new state).
        The whole frame is one autograd node (frame_step) unless per_stage is set, in which
        case every stage is its own node (the same kernels, checked one by one)."""
        if not self.per_stage:
            return frame_step(self, frame.contiguous(), state, first)
        F = stages()
        imgs = [frame]
        for _ in range(1, self.L):
            imgs.append(F["Pyramid"].apply(imgs[-1]))
        new = [None] * self.L
        top = self.L - 1
        a0, g = F["Model"].apply(imgs[top])
        f = state[top][0]
        dt = 1.0 / self.iters[top]
        for _ in range(self.iters[top]):
            f = F["PropFlow"].apply(f, 0, dt, self.border)
            f = F["PropFlow"].apply(f, 1, dt, self.border)
        old = a0 if first else state[top][1]
        fu = F["Update"].apply(a0, g, old, f, self.gamma[top:top + 1], self.maxflow[top])
        fs = self._smooth(fu, top)
        new[top] = (fs, a0, state[top][2])
        out = fu if self.L == 1 else None
        for l in range(self.L - 2, -1, -1):
            a0, g = F["Model"].apply(imgs[l])
            f, s, v = state[l]
            dt = 1.0 / self.iters[l]
            for _ in range(self.iters[l]):
                f, s, v = F["PropPayload"].apply(f, s, v, 0, dt, self.border)
                f, s, v = F["PropPayload"].apply(f, s, v, 1, dt, self.border)
            old = a0 if first else s
            coarse = fu if l == self.L - 2 else state[l + 1][0]
            flow, delta = F["DeltaUpdate"].apply(a0, g, old, v, coarse, self.gamma[l:l + 1], self.maxflow[l])
            fs_l = self._smooth(flow, l)
            new[l] = (fs_l, a0, delta)
        level0 = new[0][0] if self.L > 1 else out
        return level0, new

    def __call__(self, frames):
        torch = _torch()
        from torch.utils.checkpoint import checkpoint

        if frames.dim() != 4 or tuple(frames.shape[2:]) != (self.H, self.W):
            raise ValueError(f"frames should be (B, T, {self.H}, {self.W})")
        frames = frames.to(self.dtype)
        B, T = frames.shape[:2]
        state = self.initial_state(B)
        flat = lambda st: [t for lvl in st for t in lvl]  # noqa: E731
        unflat = lambda ts: [tuple(ts[3 * l:3 * l + 3]) for l in range(self.L)]  # noqa: E731
        outs = []
        t0 = 0
        while t0 < T:
            t1 = min(T, t0 + self.checkpoint_every)
            first = t0 == 0

            def segment(fr, gamma, weights, *st, _t0=t0, _t1=t1, _first=first):
                stl = unflat(list(st))
                ys = []
                for t in range(_t1 - _t0):
                    y, stl = self.step(fr[:, t], stl, _first and t == 0)
                    ys.append(y)
                return (torch.stack(ys, 1), *flat(stl))

            seg_in = frames[:, t0:t1]
            if self.checkpoint_every < T and torch.is_grad_enabled():
                res = checkpoint(segment, seg_in, self.gamma, self.weights, *flat(state), use_reentrant=False)
            else:
                res = segment(seg_in, self.gamma, self.weights, *flat(state))
            outs.append(res[0])
            state = unflat(list(res[1:]))
            t0 = t1
        return torch.cat(outs, 1)


def endpoint_error(flows, truth, first: int = 0):
    """Mean endpoint error over frames first.. of flows (B, T, H, W, 2) against truth of the
    same shape (or broadcastable)."""
    d = flows[:, first:] - truth[:, first:]
    return (d[..., 0] ** 2 + d[..., 1] ** 2).sqrt().mean()


class _Kernels:
    """Direct calls of the ff_diff_* kernels for one dtype (no autograd bookkeeping)."""

    def __init__(self, dtype):
        torch = _torch()
        self.torch = torch
        self.d = 1 if dtype == torch.float64 else 0
        self.item = 8 if self.d else 4

    def at(self, t, i: int):
        """Device pointer of element i of a contiguous 1-D or 2-D parameter tensor."""
        return ctypes.c_void_p(t.data_ptr() + i * self.item)

    def pyr(self, x):
        B, H, W = x.shape
        out = x.new_empty((B, H // 2, W // 2))
        call("ff_diff_pyramid", self.d, B, H, W, _p(x), _p(out), _stream())
        return out

    def pyr_bwd(self, g, gin):
        B, H, W = gin.shape
        call("ff_diff_pyramid_bwd", self.d, B, H, W, _p(g), _p(gin), _stream())

    def model(self, img):
        B, H, W = img.shape
        a0, grad = img.new_empty((B, H, W)), img.new_empty((B, H, W, 2))
        call("ff_diff_model", self.d, B, H, W, _p(img), _p(a0), _p(grad), _stream())
        return a0, grad

    def model_bwd(self, ga0, ggrad, gimg):
        B, H, W = gimg.shape
        gby, gbx = gimg.new_empty((B, H, W)), gimg.new_empty((B, H, W))
        call("ff_diff_model_bwd", self.d, B, H, W, _p(ga0), _p(ggrad), _p(gby), _p(gbx), _p(gimg), _stream())

    def prop(self, f, s, v, axis, dt, border):
        B, H, W, _ = f.shape
        fo = self.torch.empty_like(f)
        so = self.torch.empty_like(s) if s is not None else None
        vo = self.torch.empty_like(v) if v is not None else None
        call("ff_diff_propagate", self.d, B, H, W, axis, 1 if s is not None else 0, dt, border, _p(f), _p(s), _p(v),
             _p(fo), _p(so), _p(vo), _stream())
        return fo, so, vo

    def prop_bwd(self, f, s, v, gfo, gso, gvo, gf, gs, gv, axis, dt, border):
        B, H, W, _ = f.shape
        call("ff_diff_propagate_bwd", self.d, B, H, W, axis, 1 if s is not None else 0, dt, border, _p(f), _p(s),
             _p(v), _p(gfo), _p(gso), _p(gvo), _p(gf), _p(gs), _p(gv), _stream())

    def update(self, a0, grad, old, fh, gamma, l, maxflow):
        B, H, W = a0.shape
        out = self.torch.empty_like(fh)
        call("ff_diff_update", self.d, B, H, W, _p(a0), _p(grad), _p(old), _p(fh), self.at(gamma, l), maxflow,
             _p(out), _stream())
        return out

    def update_bwd(self, a0, grad, old, fh, gamma, l, maxflow, gout, ga0, ggrad, gold, gfh, ggamma):
        B, H, W = a0.shape
        call("ff_diff_update_bwd", self.d, B, H, W, _p(a0), _p(grad), _p(old), _p(fh), self.at(gamma, l), maxflow,
             _p(gout), _p(ga0), _p(ggrad), _p(gold), _p(gfh), self.at(ggamma, l), _stream())

    def dupdate(self, a0, grad, old, dh, coarse, gamma, l, maxflow):
        B, H, W = a0.shape
        Hc, Wc = coarse.shape[1:3]
        flow, delta = self.torch.empty_like(dh), self.torch.empty_like(dh)
        call("ff_diff_delta_update", self.d, B, H, W, Hc, Wc, _p(a0), _p(grad), _p(old), _p(dh), _p(coarse),
             self.at(gamma, l), maxflow, _p(flow), _p(delta), _stream())
        return flow, delta

    def dupdate_bwd(self, a0, grad, old, dh, coarse, gamma, l, maxflow, gflow, gdelta, ga0, ggrad, gold, gdh, gcoarse,
                    ggamma):
        B, H, W = a0.shape
        Hc, Wc = coarse.shape[1:3]
        call("ff_diff_delta_update_bwd", self.d, B, H, W, Hc, Wc, _p(a0), _p(grad), _p(old), _p(dh), _p(coarse),
             self.at(gamma, l), maxflow, _p(gflow), _p(gdelta), _p(ga0), _p(ggrad), _p(gold), _p(gdh), _p(gcoarse),
             self.at(ggamma, l), _stream())

    def smooth(self, x, weights, l, axis):
        B, H, W, _ = x.shape
        out = self.torch.empty_like(x)
        call("ff_diff_smooth", self.d, B, H, W, axis, self.at(weights, 5 * l), _p(x), _p(out), _stream())
        return out

    def smooth_bwd(self, x, weights, l, axis, gout, gin, gweights):
        B, H, W, _ = x.shape
        call("ff_diff_smooth_bwd", self.d, B, H, W, axis, self.at(weights, 5 * l), _p(x), _p(gout), _p(gin),
             self.at(gweights, 5 * l), _stream())


def _frame_forward(k, flt, frame, gamma, weights, state, first: bool, keep: bool):
    """One frame of the pyramidal filter by direct kernel calls.  Returns (new state, fu of
    the top level, tape); the tape holds every intermediate the adjoint needs (if keep)."""
    L = flt.L
    tape = {"imgs": [frame]}
    for _ in range(1, L):
        tape["imgs"].append(k.pyr(tape["imgs"][-1]))
    new = [None] * L
    top = L - 1
    a0, g = k.model(tape["imgs"][top])
    dt, border = 1.0 / flt.iters[top], flt.border
    fs = [state[top][0]]
    for _ in range(flt.iters[top]):
        fs.append(k.prop(fs[-1], None, None, 0, dt, border)[0])
        fs.append(k.prop(fs[-1], None, None, 1, dt, border)[0])
    old = a0 if first else state[top][1]
    fu = k.update(a0, g, old, fs[-1], gamma, top, flt.maxflow[top])
    sm = [fu]
    for _ in range(flt.smooth[top]):
        sm.append(k.smooth(sm[-1], weights, top, 0))
        sm.append(k.smooth(sm[-1], weights, top, 1))
    new[top] = (sm[-1], a0, state[top][2])
    if keep:
        tape[top] = dict(a0=a0, g=g, prop=fs[:-1], fh=fs[-1], old=old, sm=sm[:-1])
    for l in range(L - 2, -1, -1):
        a0, g = k.model(tape["imgs"][l])
        dt = 1.0 / flt.iters[l]
        fsv = [tuple(state[l])]
        for _ in range(flt.iters[l]):
            fsv.append(k.prop(*fsv[-1], 0, dt, border))
            fsv.append(k.prop(*fsv[-1], 1, dt, border))
        f_h, s_h, v_h = fsv[-1]
        old = a0 if first else s_h
        coarse = fu if l == L - 2 else state[l + 1][0]
        flow, delta = k.dupdate(a0, g, old, v_h, coarse, gamma, l, flt.maxflow[l])
        sm = [flow]
        for _ in range(flt.smooth[l]):
            sm.append(k.smooth(sm[-1], weights, l, 0))
            sm.append(k.smooth(sm[-1], weights, l, 1))
        new[l] = (sm[-1], a0, delta)
        if keep:
            tape[l] = dict(a0=a0, g=g, prop=fsv[:-1], vh=v_h, old=old, coarse=coarse, sm=sm[:-1])
    return new, fu, tape


def _smooth_backward(k, sm, weights, l, g, gweights):
    """Adjoint of the 2S smoothing passes whose inputs are sm[0..2S-1]; g: output gradient."""
    torch = k.torch
    for j in range(len(sm) - 1, -1, -1):
        gin = torch.zeros_like(sm[j])
        k.smooth_bwd(sm[j], weights, l, j % 2, g, gin, gweights)
        g = gin
    return g


def _frame_backward(k, flt, tape, gamma, weights, state, first: bool, g_new, g_fu_out):
    """Reverse of _frame_forward.  g_new[l] = gradients of the new state (fs, io, d) (None =
    zero); g_fu_out = gradient of the top level's fu as an output (single level).  Returns
    (g_frame, g_gamma, g_weights, g_state)."""
    torch = k.torch
    L = flt.L
    top = L - 1
    z = lambda t: torch.zeros_like(t)  # noqa: E731
    g_gamma, g_weights = torch.zeros_like(gamma), torch.zeros_like(weights)
    g_state = [[z(state[l][0]), z(state[l][1]), z(state[l][2])] for l in range(L)]
    g_img = [z(im) for im in tape["imgs"]]
    g_fu = z(tape[top]["sm"][0])
    if g_fu_out is not None:
        g_fu += g_fu_out
    border = flt.border

    def gn(l, i, like):
        t = g_new[l][i]
        return t.contiguous() if t is not None else z(like)

    for l in range(0, L - 1):
        T = tape[l]
        g_flow = _smooth_backward(k, T["sm"], weights, l, gn(l, 0, T["sm"][0]), g_weights)
        ga0, gg, gold, gvh = z(T["a0"]), z(T["g"]), z(T["old"]), z(T["vh"])
        gcoarse = z(T["coarse"])
        k.dupdate_bwd(T["a0"], T["g"], T["old"], T["vh"], T["coarse"], gamma, l, flt.maxflow[l], g_flow,
                      gn(l, 2, T["vh"]), ga0, gg, gold, gvh, gcoarse, g_gamma)
        ga0 += gn(l, 1, T["a0"])
        if l == L - 2:
            g_fu += gcoarse
        else:
            g_state[l + 1][0] += gcoarse
        if first:
            ga0 += gold
            gs = z(T["old"])
        else:
            gs = gold
        gf, gv = z(T["prop"][0][0]), gvh
        dt = 1.0 / flt.iters[l]
        for j in range(len(T["prop"]) - 1, -1, -1):
            f, s, v = T["prop"][j]
            nf, ns, nv = z(f), z(s), z(v)
            k.prop_bwd(f, s, v, gf, gs, gv, nf, ns, nv, j % 2, dt, border)
            gf, gs, gv = nf, ns, nv
        g_state[l][0] += gf
        g_state[l][1] += gs
        g_state[l][2] += gv
        k.model_bwd(ga0, gg, g_img[l])

    T = tape[top]
    g_fu += _smooth_backward(k, T["sm"], weights, top, gn(top, 0, T["sm"][0]), g_weights)
    ga0, gg, gold, gfh = z(T["a0"]), z(T["g"]), z(T["old"]), z(T["fh"])
    k.update_bwd(T["a0"], T["g"], T["old"], T["fh"], gamma, top, flt.maxflow[top], g_fu, ga0, gg, gold, gfh, g_gamma)
    ga0 += gn(top, 1, T["a0"])
    if first:
        ga0 += gold
    else:
        g_state[top][1] += gold
    g_state[top][2] += gn(top, 2, state[top][2])
    gf = gfh
    dt = 1.0 / flt.iters[top]
    for j in range(len(T["prop"]) - 1, -1, -1):
        nf = z(T["prop"][j])
        k.prop_bwd(T["prop"][j], None, None, gf, None, None, nf, None, None, j % 2, dt, border)
        gf = nf
    g_state[top][0] += gf
    k.model_bwd(ga0, gg, g_img[top])
    for l in range(L - 1, 0, -1):
        k.pyr_bwd(g_img[l], g_img[l - 1])
    return g_img[0], g_gamma, g_weights, g_state


def _pack(obj, out: list):
    """obj with every tensor replaced by its index in out (tensors appended to out)."""
    torch = _torch()
    if isinstance(obj, torch.Tensor):
        out.append(obj)
        return ("#", len(out) - 1)
    if isinstance(obj, dict):
        return {k: _pack(v, out) for k, v in obj.items()}
    if isinstance(obj, (list, tuple)):
        return type(obj)(_pack(v, out) for v in obj)
    return obj


def _unpack(obj, ts):
    if isinstance(obj, tuple) and len(obj) == 2 and obj[0] == "#":
        return ts[obj[1]]
    if isinstance(obj, dict):
        return {k: _unpack(v, ts) for k, v in obj.items()}
    if isinstance(obj, (list, tuple)):
        return type(obj)(_unpack(v, ts) for v in obj)
    return obj


def _frame_function():
    torch = _torch()

    class FrameStep(torch.autograd.Function):
        """One frame of the pyramidal filter as a single autograd node: the forward runs the
        stage kernels, the backward their adjoints in reverse order over the saved tape."""

        @staticmethod
        def forward(ctx, flt, first, frame, gamma, weights, *state_flat):
            k = _Kernels(frame.dtype)
            L = flt.L
            state = [tuple(t.contiguous() for t in state_flat[3 * l:3 * l + 3]) for l in range(L)]
            frame, gamma, weights = frame.contiguous(), gamma.contiguous(), weights.contiguous()
            keep = torch.is_grad_enabled() or any(ctx.needs_input_grad)
            new, fu, tape = _frame_forward(k, flt, frame, gamma, weights, state, first, keep)
            ctx.flt, ctx.first = flt, first
            if keep:
                # everything the adjoint reads goes through save_for_backward, so an enclosing
                # checkpoint can drop it and recompute the frame in the backward pass
                flat = []
                ctx.skeleton = _pack({"tape": tape, "state": state, "params": (gamma, weights)}, flat)
                ctx.save_for_backward(*flat)
            outs = [t for lvl in new for t in lvl]
            # the top level's delta slot passes its input through: return a copy so every
            # output is a distinct tensor
            outs[3 * (L - 1) + 2] = outs[3 * (L - 1) + 2].clone()
            return (*outs, fu.clone() if L == 1 else fu.new_zeros(0))

        @staticmethod
        def backward(ctx, *grads):
            flt = ctx.flt
            saved = _unpack(ctx.skeleton, ctx.saved_tensors)
            gamma, weights = saved["params"]
            k = _Kernels(gamma.dtype)
            L = flt.L
            g_new = [tuple(grads[3 * l:3 * l + 3]) for l in range(L)]
            g_fu = grads[3 * L] if L == 1 and grads[3 * L] is not None and grads[3 * L].numel() else None
            g_frame, g_gamma, g_weights, g_state = _frame_backward(k, flt, saved["tape"], gamma, weights,
                                                                   saved["state"], ctx.first, g_new, g_fu)
            return (None, None, g_frame, g_gamma, g_weights, *[t for lvl in g_state for t in lvl])

    return FrameStep


_FrameStep = None


def frame_step(flt, frame, state, first: bool):
    """One frame through the single-node FrameStep; returns (level-0 flow, new state)."""
    global _FrameStep
    if _FrameStep is None:
        _FrameStep = _frame_function()
    L = flt.L
    out = _FrameStep.apply(flt, first, frame, flt.gamma, flt.weights, *[t for lvl in state for t in lvl])
    new = [tuple(out[3 * l:3 * l + 3]) for l in range(L)]
    y = out[3 * L] if L == 1 else new[0][0]
    return y, new
