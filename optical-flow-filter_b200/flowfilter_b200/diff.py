"""Differentiable flow filter: hand-written adjoint kernels behind torch.autograd.Function.

No counterpart in the reference.  The forward recurrence is the reference's pyramidal
filter on float32 images in [0, 1] (the float path of ImagePyramid, FlowFilter(GPUImage)
and DeltaFlowFilter, src/gpu/flowfilter.cu:621-716; gamma used unscaled for float input,
:279-284), run by the ff_diff_* kernels of libffb200.so in float32 or float64.  Every stage
has an autograd Function whose backward is the matching adjoint kernel (``stages()``); the
filter itself runs each frame as one autograd node (FrameStep) whose forward is one
ff_diff_frame_forward call (the same forward kernels, launched by the library) and whose
backward is one ff_diff_frame_backward call (the adjoint kernels in reverse order).  The time recurrence
is chained by autograd and cut into checkpointed segments (recomputed in the backward pass)
of ``checkpoint_every`` frames.

Parameters with gradients: per-level gamma, per-level 5-tap smoothing weights (the reference
smooths with the 0.2 box, the default here, which reproduces it bit for bit in float32) and
the input frames.
"""

from __future__ import annotations

import ctypes
import math

from ._lib import call, lib


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

    def fit(self, frames, truth, steps: int = 200, lr: float = 0.05, first: int = 8, fit_weights: bool = True,
            group=None):
        """Fits the per-level gamma and, with fit_weights, the per-level 5-tap smoothing
        weights by Adam on the mean endpoint error of the flows against ``truth``
        (B, T, H, W, 2) over frames first.. .  gamma is fitted through its logarithm (it stays
        positive), the weights through a softmax of five logits per level (they stay positive
        and sum to 1, as the reference's 0.2 box does, which is the softmax of equal logits).
        Checkpointing follows ``checkpoint_every``.  Returns the loss of every step, the final
        loss and the device milliseconds of the steps; the fitted values are left in gamma /
        weights.

        Data parallel: when torch.distributed is initialised with more than one rank (or
        ``group`` is given), each rank passes its own share of the sequences (equal batch
        sizes) and every step averages the parameter gradients and the loss over the ranks
        (one all-reduce each), so all ranks take the same Adam steps."""
        torch = _torch()
        log_g = torch.log(self.gamma.detach().clone()).requires_grad_(True)
        w0 = self.weights.detach().clone()
        logits = torch.log(w0 / w0.sum(1, keepdim=True)).requires_grad_(fit_weights)
        opt = torch.optim.Adam([log_g, logits] if fit_weights else [log_g], lr=lr)
        losses = []
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(int(steps)):
            self.gamma = log_g.exp()
            self.weights = torch.softmax(logits, 1) if fit_weights else w0
            loss = endpoint_error(self(frames), truth, first=first, eps=1e-12)
            opt.zero_grad()
            loss.backward()
            params = [log_g, logits] if fit_weights else [log_g]
            average_over_ranks([p.grad for p in params], group)
            lv = loss.detach().reshape(1).clone()
            average_over_ranks([lv], group)
            opt.step()
            losses.append(lv[0])
        e1.record()
        torch.cuda.synchronize()
        self.gamma = log_g.detach().exp().requires_grad_(True)
        self.weights = (torch.softmax(logits.detach(), 1) if fit_weights else w0).clone().requires_grad_(True)
        with torch.no_grad():
            fl = endpoint_error(self(frames), truth, first=first).reshape(1).clone()
            average_over_ranks([fl], group)
            final = float(fl[0])
        return {"losses": [float(x) for x in losses], "final": final, "ms": e0.elapsed_time(e1)}

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


def average_over_ranks(tensors, group=None) -> int:
    """Replaces every tensor with its mean over the ranks of ``group`` (the default process
    group when torch.distributed is initialised; nothing happens with one rank): one
    all-reduce of their flattened concatenation.  Returns the number of ranks."""
    torch = _torch()
    dist = torch.distributed
    if group is None and not (dist.is_available() and dist.is_initialized()):
        return 1
    world = dist.get_world_size(group)
    if world == 1 or not tensors:
        return world
    flat = torch.cat([t.reshape(-1) for t in tensors])
    dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=group)
    flat /= world
    at = 0
    for t in tensors:
        t.copy_(flat[at:at + t.numel()].view_as(t))
        at += t.numel()
    return world


def endpoint_error(flows, truth, first: int = 0, eps: float = 0.0):
    """Mean endpoint error over frames first.. of flows (B, T, H, W, 2) against truth of the
    same shape (or broadcastable).  eps > 0 is added under the square root, which keeps the
    gradient finite where a flow equals the truth exactly (used by fit()); with eps = 0 the
    gradient there is zero.  One autograd node: the backward writes the flow gradient in one
    pass (zero for the frames before ``first``)."""
    torch = _torch()
    if isinstance(truth, torch.Tensor) and truth.requires_grad:
        d = flows[:, first:] - truth[:, first:]
        return (d[..., 0] ** 2 + d[..., 1] ** 2 + eps).sqrt().mean()
    global _EPE
    if _EPE is None:
        _EPE = _epe_function()
    return _EPE.apply(flows, truth, int(first), float(eps))


_EPE = None


def _epe_function():
    torch = _torch()

    def on_device(flows, first):
        return (flows.is_cuda and flows.dtype in (torch.float32, torch.float64) and flows.dim() == 5
                and flows.shape[-1] == 2 and 0 <= first < flows.shape[1])

    class EndpointError(torch.autograd.Function):
        """CUDA float tensors: ff_diff_epe / ff_diff_epe_bwd (one pass each way); otherwise
        the same arithmetic from torch operations."""

        @staticmethod
        def forward(ctx, flows, truth, first, eps):
            ctx.first, ctx.eps, ctx.shape = first, eps, flows.shape
            if on_device(flows, first):
                f = flows.contiguous()
                tr = torch.as_tensor(truth, dtype=f.dtype, device=f.device).expand(f.shape)
                if tr.stride()[2:] != f.stride()[2:]:
                    tr = tr.contiguous()
                B, T, H, W = f.shape[:4]
                d = _dt(f)
                loss = f.new_empty(())
                scratch = f.new_empty(lib().ff_diff_epe_scratch_bytes(d) // f.element_size())
                call("ff_diff_epe", d, B, T, H, W, first, eps, _p(f), _p(tr), tr.stride(0), tr.stride(1), _p(loss),
                     _p(scratch), _stream())
                ctx.device = True
                ctx.save_for_backward(f, tr)
                return loss
            d = flows[:, first:] - truth[:, first:]
            n = torch.linalg.vector_norm(d, dim=-1)
            if eps > 0:
                n = n.square_().add_(eps).sqrt_()
            ctx.device = False
            ctx.save_for_backward(d, n)
            return n.mean()

        @staticmethod
        def backward(ctx, g):
            if ctx.device:
                f, tr = ctx.saved_tensors
                B, T, H, W = f.shape[:4]
                out = torch.empty_like(f)
                call("ff_diff_epe_bwd", _dt(f), B, T, H, W, ctx.first, ctx.eps, _p(f), _p(tr), tr.stride(0),
                     tr.stride(1), _p(g.contiguous()), _p(out), _stream())
                return out, None, None, None
            d, n = ctx.saved_tensors
            # d |d|^-1 g / count; where |d| = 0 (eps = 0) so is d, and the gradient is zero
            scale = torch.div(g / n.numel(), n.clamp_min(1e-30))
            out = d.new_empty(ctx.shape)
            out[:, :ctx.first].zero_()
            torch.mul(d, scale.unsqueeze(-1), out=out[:, ctx.first:])
            return out, None, None, None

    return EndpointError


MAX_LEVELS = 8  # FF_DIFF_MAX_LEVELS


class _Geom(ctypes.Structure):
    """ff_diff_geom of include/ffb200.h."""

    _fields_ = [("batch", ctypes.c_int), ("levels", ctypes.c_int), ("border", ctypes.c_int),
                ("height", ctypes.c_int * MAX_LEVELS), ("width", ctypes.c_int * MAX_LEVELS),
                ("iterations", ctypes.c_int * MAX_LEVELS), ("smooth", ctypes.c_int * MAX_LEVELS),
                ("maxflow", ctypes.c_double * MAX_LEVELS)]


def _geom(flt, B: int) -> _Geom:
    if flt.L > MAX_LEVELS:
        raise ValueError(f"at most {MAX_LEVELS} levels")
    g = _Geom()
    g.batch, g.levels, g.border = int(B), flt.L, flt.border
    for l, (h, w) in enumerate(flt.shapes):
        g.height[l], g.width[l] = h, w
        g.iterations[l], g.smooth[l] = flt.iters[l], flt.smooth[l]
        g.maxflow[l] = flt.maxflow[l]
    return g


def _workspace(name: str, d: int, g: _Geom, like):
    """A device buffer of the size ff_diff_frame_{tape,scratch}_bytes gives."""
    n = getattr(lib(), name)(d, ctypes.byref(g))
    if n == 0:
        raise ValueError("bad differentiable-filter geometry")
    return _torch().empty(n // (8 if d else 4), dtype=like.dtype, device=like.device)


def _ptrs(ts):
    return (ctypes.c_void_p * len(ts))(*[t.data_ptr() if t is not None else None for t in ts])


def _frame_forward(flt, frame, gamma, weights, state_flat, first: bool):
    """One frame through ff_diff_frame_forward (one host call launches the whole frame).
    Returns (new state, flat; the top level's unsmoothed flow for one level, else None; the
    tape the adjoint reads; for several levels a copy of level 0's smoothed flow, the frame's
    output, else None)."""
    d = _dt(frame)
    B = frame.shape[0]
    g = _geom(flt, B)
    tape = _workspace("ff_diff_frame_tape_bytes", d, g, frame)
    new = []
    for h, w in flt.shapes:
        new += [frame.new_empty((B, h, w, 2)), frame.new_empty((B, h, w)), frame.new_empty((B, h, w, 2))]
    fu = frame.new_empty((B,) + tuple(flt.shapes[0]) + (2,)) if flt.L == 1 else None
    y = frame.new_empty((B,) + tuple(flt.shapes[0]) + (2,)) if flt.L > 1 else None
    call("ff_diff_frame_forward", d, ctypes.byref(g), 1 if first else 0, _p(frame), _p(gamma), _p(weights),
         _ptrs(state_flat), _ptrs(new), _p(fu), _p(y), _p(tape), _stream())
    return new, fu, tape, y


def _frame_backward(flt, first: bool, frame, gamma, weights, state_flat, new_flat, tape, g_new, g_fu, g_y=None):
    """Adjoint of one frame through ff_diff_frame_backward: gradients of the new state (None
    = zero), of the top level's unsmoothed flow and of the frame's output y -> gradients of
    the frame, gamma, weights and the input state."""
    torch = _torch()
    d = _dt(frame)
    g = _geom(flt, frame.shape[0])
    scratch = _workspace("ff_diff_frame_scratch_bytes", d, g, frame)
    # the gradients the adjoint adds into, carved from one zeroed buffer (one fill per frame);
    # every piece starts at an even element, so two-element pairs stay aligned
    like = [frame, gamma, weights] + list(state_flat)
    sizes = [(t.numel() + 1) & ~1 for t in like]
    flat = torch.zeros(sum(sizes), dtype=frame.dtype, device=frame.device)
    views, at = [], 0
    for t, n in zip(like, sizes):
        views.append(flat[at:at + t.numel()].view(t.shape))
        at += n
    g_frame, g_gamma, g_weights, g_state = views[0], views[1], views[2], views[3:]
    g_new = [_c(t) for t in g_new]
    # y's gradient is often one frame of a (B, T, H, W, 2) gradient: read in place when its
    # images are dense (any image stride)
    if g_y is not None and (g_y.dim() != 4 or g_y.stride()[1:] != (2 * g_y.shape[2], 2, 1) or g_y.stride(0) % 2):
        g_y = g_y.contiguous()
    call("ff_diff_frame_backward", d, ctypes.byref(g), 1 if first else 0, _p(frame), _p(gamma), _p(weights),
         _ptrs(state_flat), _ptrs(new_flat), _p(tape), _ptrs(g_new), _p(_c(g_fu)), _p(g_y),
         g_y.stride(0) if g_y is not None else 0, _p(g_frame), _p(g_gamma), _p(g_weights), _ptrs(g_state),
         _p(scratch), _stream())
    return g_frame, g_gamma, g_weights, g_state


def _frame_function():
    torch = _torch()

    class FrameStep(torch.autograd.Function):
        """One frame of the pyramidal filter as a single autograd node: the forward is one
        ff_diff_frame_forward call (every stage kernel, intermediates kept in a tape), the
        backward one ff_diff_frame_backward call (the adjoint kernels in reverse order)."""

        @staticmethod
        def forward(ctx, flt, first, frame, gamma, weights, *state_flat):
            state_flat = [t.contiguous() for t in state_flat]
            frame, gamma, weights = frame.contiguous(), gamma.contiguous(), weights.contiguous()
            new, fu, tape, y = _frame_forward(flt, frame, gamma, weights, state_flat, first)
            ctx.flt, ctx.first = flt, first
            ctx.set_materialize_grads(False)  # outputs nobody differentiates: None, not zeros
            if torch.is_grad_enabled() or any(ctx.needs_input_grad):
                # the tape and the outputs the adjoint reads go through save_for_backward, so an
                # enclosing checkpoint can drop them and recompute the frame in the backward pass
                ctx.save_for_backward(frame, gamma, weights, tape, *state_flat, *new)
            empty = frame.new_zeros(0)
            # outputs: the new state, the top level's unsmoothed flow (one level), the frame's
            # output (several levels: a copy of level 0's smoothed flow, so that its gradient
            # and the next frame's state gradient reach the adjoint separately)
            return (*new, fu if fu is not None else empty, y if y is not None else empty)

        @staticmethod
        def backward(ctx, *grads):
            flt = ctx.flt
            L = flt.L
            saved = ctx.saved_tensors
            frame, gamma, weights, tape = saved[:4]
            state_flat, new_flat = list(saved[4:4 + 3 * L]), list(saved[4 + 3 * L:])
            g_fu = grads[3 * L] if L == 1 and grads[3 * L] is not None and grads[3 * L].numel() else None
            g_y = grads[3 * L + 1] if L > 1 and grads[3 * L + 1] is not None and grads[3 * L + 1].numel() else None
            g_frame, g_gamma, g_weights, g_state = _frame_backward(flt, ctx.first, frame, gamma, weights, state_flat,
                                                                   new_flat, tape, list(grads[:3 * L]), g_fu, g_y)
            return (None, None, g_frame, g_gamma, g_weights, *g_state)

    return FrameStep


_FrameStep = None


def _frame_infer(flt, frame, gamma, weights, state_flat, first: bool):
    """One frame without a tape (ff_diff_frame_infer): the same outputs as _frame_forward, the
    intermediates in a scratch buffer kept on the filter and reused every frame."""
    d = _dt(frame)
    B = frame.shape[0]
    g = _geom(flt, B)
    key = (d, B, frame.device)
    cache = flt.__dict__.setdefault("_infer_scratch", {})
    if key not in cache:
        cache.clear()
        cache[key] = _workspace("ff_diff_frame_infer_bytes", d, g, frame)
    scratch = cache[key]
    new = []
    for h, w in flt.shapes:
        new += [frame.new_empty((B, h, w, 2)), frame.new_empty((B, h, w)), frame.new_empty((B, h, w, 2))]
    fu = frame.new_empty((B,) + tuple(flt.shapes[0]) + (2,)) if flt.L == 1 else None
    call("ff_diff_frame_infer", d, ctypes.byref(g), 1 if first else 0, _p(frame), _p(gamma), _p(weights),
         _ptrs(state_flat), _ptrs(new), _p(fu), _p(scratch), _stream())
    return new, fu


def frame_step(flt, frame, state, first: bool):
    """One frame through the single-node FrameStep; returns (level-0 flow, new state).  With
    gradients off (torch.no_grad or inference mode) the frame runs without a tape."""
    global _FrameStep
    if _FrameStep is None:
        _FrameStep = _frame_function()
    L = flt.L
    torch = _torch()
    if not torch.is_grad_enabled():
        state_flat = [t.contiguous() for lvl in state for t in lvl]
        new, fu = _frame_infer(flt, frame.contiguous(), flt.gamma.detach().contiguous(),
                               flt.weights.detach().contiguous(), state_flat, first)
        out = (*new, fu if fu is not None else frame.new_zeros(0))
        newst = [tuple(out[3 * l:3 * l + 3]) for l in range(L)]
        return (out[3 * L] if L == 1 else newst[0][0]), newst
    out = _FrameStep.apply(flt, first, frame, flt.gamma, flt.weights, *[t for lvl in state for t in lvl])
    new = [tuple(out[3 * l:3 * l + 3]) for l in range(L)]
    y = out[3 * L] if L == 1 else out[3 * L + 1]
    return y, new
