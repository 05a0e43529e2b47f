"""Stage-level operations on CUDA tensors (the reference's stage classes).

Each function wraps one ``ff_stage_*`` entry point of the C ABI and runs on the current
torch CUDA stream.  Images are (H, W) uint8 or float32, flows (H, W, 2) float32.
Mirrors ImagePyramid, ImageModel, FlowPropagator, FlowPropagatorPayload, FlowUpdate,
DeltaFlowUpdate and FlowSmoother (src/gpu/{pyramid,imagemodel,propagation,update,
flowsmoothing}.cu).
"""

from __future__ import annotations

import ctypes

from ._lib import call, lib

__all__ = ["pyramid_down", "image_model", "propagate", "propagate_payload", "update", "delta_update", "smooth"]


def _torch():
    import torch

    return torch


def _stream():
    return ctypes.c_void_p(_torch().cuda.current_stream().cuda_stream)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _rowpitch(t) -> int:
    return t.stride(0) * t.element_size()


def _check(t, dims, dtype=None, channels=None, name="tensor"):
    torch = _torch()
    if not (isinstance(t, torch.Tensor) and t.is_cuda):
        raise ValueError(f"{name} should be a CUDA tensor")
    if t.dim() != dims:
        raise ValueError(f"{name} should have {dims} dimensions, got shape {tuple(t.shape)}")
    if dtype is not None and t.dtype != dtype:
        raise ValueError(f"{name} dtype should be {dtype}, got {t.dtype}")
    if channels is not None and t.shape[2] != channels:
        raise ValueError(f"{name} should have {channels} channels")
    inner = t.stride(-1) == 1 and (dims == 2 or t.stride(1) == t.shape[2])
    if not inner:
        raise ValueError(f"{name} rows must be contiguous")


def _flow(h, w):
    return _torch().empty((h, w, 2), device="cuda", dtype=_torch().float32)


def _img(h, w):
    return _torch().empty((h, w), device="cuda", dtype=_torch().float32)


def pyramid_down(img):
    """One pyramid step: X then Y [1/4, 1/2, 1/4] at stride 2 (pyramid_k.cu:14-145)."""
    torch = _torch()
    _check(img, 2, name="image")
    if img.dtype not in (torch.uint8, torch.float32):
        raise ValueError("image dtype should be uint8 or float32")
    h, w = img.shape
    out = torch.empty((h // 2, w // 2), device="cuda", dtype=img.dtype)
    if out.numel():
        call("ff_stage_pyramid_down", _ptr(img), _rowpitch(img), img.element_size(), h, w, _ptr(out), _rowpitch(out),
             _stream())
    return out


def image_model(img):
    """Image model (a0, gradient) of a uint8 or float32 image (imagemodel_k.cu:31-133)."""
    torch = _torch()
    _check(img, 2, name="image")
    if img.dtype not in (torch.uint8, torch.float32):
        raise ValueError("image dtype should be uint8 or float32")
    h, w = img.shape
    a0, grad = _img(h, w), _flow(h, w)
    call("ff_stage_image_model", _ptr(img), _rowpitch(img), img.element_size(), h, w, _ptr(a0), _rowpitch(a0),
         _ptr(grad), _rowpitch(grad), _stream())
    return a0, grad


def propagate(flow, iterations: int, border: int = 3):
    """FlowPropagator: ``iterations`` upwind sub-steps with dt = 1/iterations."""
    torch = _torch()
    _check(flow, 3, torch.float32, 2, "flow")
    h, w, _ = flow.shape
    out = _flow(h, w)
    ws = torch.empty(lib().ff_stage_propagate_workspace_size(h, w), device="cuda", dtype=torch.uint8)
    call("ff_stage_propagate", _ptr(flow), _rowpitch(flow), h, w, int(iterations), int(border), _ptr(out),
         _rowpitch(out), _ptr(ws), _stream())
    return out


def propagate_payload(flow, scalar, vector, iterations: int, border: int = 3):
    """FlowPropagatorPayload: flow, scalar and vector payload advected together."""
    torch = _torch()
    _check(flow, 3, torch.float32, 2, "flow")
    _check(scalar, 2, torch.float32, name="scalar")
    _check(vector, 3, torch.float32, 2, "vector")
    h, w, _ = flow.shape
    of, osc, ove = _flow(h, w), _img(h, w), _flow(h, w)
    ws = torch.empty(lib().ff_stage_propagate_payload_workspace_size(h, w), device="cuda", dtype=torch.uint8)
    call("ff_stage_propagate_payload", _ptr(flow), _rowpitch(flow), _ptr(scalar), _rowpitch(scalar), _ptr(vector),
         _rowpitch(vector), h, w, int(iterations), int(border), _ptr(of), _rowpitch(of), _ptr(osc), _rowpitch(osc),
         _ptr(ove), _rowpitch(ove), _ptr(ws), _stream())
    return of, osc, ove


def update(a0, grad, a0_old, flow, gamma: float, maxflow: float):
    """FlowUpdate: returns (flow, image); ``gamma`` is used as given (no 1/255^2 scaling)."""
    torch = _torch()
    for t, d, c, n in ((a0, 2, None, "a0"), (grad, 3, 2, "grad"), (a0_old, 2, None, "a0_old"), (flow, 3, 2, "flow")):
        _check(t, d, torch.float32, c, n)
    h, w = a0.shape
    of, oi = _flow(h, w), _img(h, w)
    call("ff_stage_update", _ptr(a0), _rowpitch(a0), _ptr(grad), _rowpitch(grad), _ptr(a0_old), _rowpitch(a0_old),
         _ptr(flow), _rowpitch(flow), h, w, float(gamma), float(maxflow), _ptr(of), _rowpitch(of), _ptr(oi),
         _rowpitch(oi), _stream())
    return of, oi


def delta_update(a0, grad, a0_old, delta, coarse, gamma: float, maxflow: float):
    """DeltaFlowUpdate: returns (flow, delta, image)."""
    torch = _torch()
    for t, d, c, n in ((a0, 2, None, "a0"), (grad, 3, 2, "grad"), (a0_old, 2, None, "a0_old"),
                       (delta, 3, 2, "delta"), (coarse, 3, 2, "coarse")):
        _check(t, d, torch.float32, c, n)
    h, w = a0.shape
    hc, wc, _ = coarse.shape
    of, od, oi = _flow(h, w), _flow(h, w), _img(h, w)
    call("ff_stage_delta_update", _ptr(a0), _rowpitch(a0), _ptr(grad), _rowpitch(grad), _ptr(a0_old),
         _rowpitch(a0_old), _ptr(delta), _rowpitch(delta), _ptr(coarse), _rowpitch(coarse), hc, wc, h, w,
         float(gamma), float(maxflow), _ptr(of), _rowpitch(of), _ptr(od), _rowpitch(od), _ptr(oi), _rowpitch(oi),
         _stream())
    return of, od, oi


def smooth(flow, iterations: int):
    """FlowSmoother: ``iterations`` x (5-tap box X, then Y)."""
    torch = _torch()
    _check(flow, 3, torch.float32, 2, "flow")
    h, w, _ = flow.shape
    out = _flow(h, w)
    ws = torch.empty(lib().ff_stage_smooth_workspace_size(h, w), device="cuda", dtype=torch.uint8)
    call("ff_stage_smooth", _ptr(flow), _rowpitch(flow), h, w, int(iterations), _ptr(out), _rowpitch(out), _ptr(ws),
         _stream())
    return out
