"""Flow colour encoding: the reference's ``flowfilter.gpu.display.FlowToColor``
(python/flowfilter/gpu/display.pyx:18-72, src/gpu/display.cu:20-142) over
``ff_flow_to_color``.

``FlowToColor(inputFlow, maxflow)`` takes a (H, W, 2) float32 CUDA tensor (for example a
filter's ``getFlowDevice()``), and ``compute()`` writes a (H, W, 4) uint8 RGBA image that
``getColorFlow()`` returns as a CUDA tensor and ``download()`` as a numpy array.  The
colour wheel is the library's default (the reference's own 256x256 RGBA table, byte for
byte) unless ``setColorWheel`` gives another one.
"""

from __future__ import annotations

import ctypes

import numpy as np

from ._lib import FF_ERR_LOGIC, FFLogicError, call

WHEEL_SIZE = 256


def _torch():
    import torch

    return torch


def color_wheel() -> np.ndarray:
    """The library's default colour wheel, (256, 256, 4) uint8 (row = y, column = x)."""
    w = np.empty((WHEEL_SIZE, WHEEL_SIZE, 4), np.uint8)
    call("ff_color_wheel_default", w.ctypes.data_as(ctypes.c_void_p))
    return w


def _check_flow(flow):
    torch = _torch()
    if not isinstance(flow, torch.Tensor) or not flow.is_cuda or flow.dtype != torch.float32:
        raise ValueError("input flow should be a float32 CUDA tensor of shape (H, W, 2)")
    if flow.dim() != 3 or flow.shape[2] != 2:
        raise ValueError(f"input flow should have depth 2: {tuple(flow.shape)}")
    if flow.stride(2) != 1 or flow.stride(1) != 2:
        raise ValueError("input flow rows should hold interleaved (x, y) pairs contiguously")
    return flow


class FlowToColor:
    """Colour encoding of an optical flow field through a colour wheel (FlowToColor stage)."""

    def __init__(self, inputFlow=None, maxflow: float = 1.0):
        self._flow = None
        self._color = None
        self._wheel = None
        self._maxflow = 1.0
        self._ms = 0.0
        self._configured = False
        if inputFlow is None:
            return
        self.setInputFlow(inputFlow)
        self.maxflow = maxflow
        self.configure()

    def configure(self) -> None:
        """Allocate the colour output for the input flow (display.cu:52-84)."""
        if self._flow is None:
            raise FFLogicError(FF_ERR_LOGIC, "FlowToColor::configure(): input flow not set")
        h, w = self._flow.shape[:2]
        self._color = _torch().empty((h, w, 4), dtype=_torch().uint8, device=self._flow.device)
        self._configured = True

    def compute(self) -> None:
        """Colour-encode the input flow into getColorFlow() (display.cu:87-110)."""
        if not self._configured:
            raise FFLogicError(FF_ERR_LOGIC, "FlowToColor::compute(): Stage not configured")
        torch = _torch()
        f, c = self._flow, self._color
        stream = torch.cuda.current_stream(f.device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        call("ff_flow_to_color", ctypes.c_void_p(f.data_ptr()), f.stride(0) * 4, f.shape[0], f.shape[1],
             self._maxflow, ctypes.c_void_p(self._wheel.data_ptr()) if self._wheel is not None else None,
             ctypes.c_void_p(c.data_ptr()), c.stride(0), ctypes.c_void_p(stream.cuda_stream))
        e1.record(stream)
        e1.synchronize()
        self._ms = e0.elapsed_time(e1)

    def elapsedTime(self) -> float:
        """Milliseconds of the last compute()."""
        return self._ms

    def setInputFlow(self, inputFlow) -> None:
        """Set the (H, W, 2) float32 CUDA flow to encode (display.cu:113-121)."""
        self._flow = _check_flow(inputFlow)
        if self._color is not None and self._color.shape[:2] != inputFlow.shape[:2]:
            self._configured = False

    def getColorFlow(self):
        """The (H, W, 4) uint8 RGBA output on the device."""
        if self._color is None:
            raise FFLogicError(FF_ERR_LOGIC, "FlowToColor: not configured")
        return self._color

    def download(self) -> np.ndarray:
        """Host copy of the colour output, (H, W, 4) uint8."""
        return self.getColorFlow().cpu().numpy()

    def setColorWheel(self, wheel=None) -> None:
        """Use another (256, 256, 4) uint8 RGBA wheel (numpy or tensor); None: the default."""
        if wheel is None:
            self._wheel = None
            return
        torch = _torch()
        t = torch.as_tensor(np.asarray(wheel) if not isinstance(wheel, torch.Tensor) else wheel)
        if t.dtype != torch.uint8 or tuple(t.shape) != (WHEEL_SIZE, WHEEL_SIZE, 4):
            raise ValueError("the colour wheel should be a (256, 256, 4) uint8 RGBA table")
        dev = self._flow.device if self._flow is not None else torch.device("cuda")
        self._wheel = t.to(dev).contiguous()

    @property
    def maxflow(self) -> float:
        return self._maxflow

    @maxflow.setter
    def maxflow(self, value: float) -> None:
        if not float(value) > 0.0:
            raise ValueError(f"FlowToColor::setMaxFlow(): maxflow should be greater than 0.0: {value}")
        self._maxflow = float(value)
