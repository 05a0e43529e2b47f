"""Camera model, Lax-Wendroff image propagation and the rotational image predictor: the
reference's ``flowfilter.gpu.camera`` (python/flowfilter/gpu/camera.pyx:12-75),
``flowfilter.gpu.propagation.LaxWendroffPropagator`` (python/flowfilter/gpu/propagation.pyx:
254-330) and ``flowfilter.gpu.rotation.RotationalFlowImagePredictor``
(python/flowfilter/gpu/rotation.pyx:16-97), over ``ff_camera_perspective``,
``ff_lax_wendroff`` and ``ff_rotational_predict``.

Images are float32 CUDA tensors of shape (H, W) or (H, W, 4); flows (H, W, 2).  Outputs are
CUDA tensors owned by the object and rewritten by every ``compute()``.
"""

from __future__ import annotations

import ctypes

import numpy as np

from ._lib import FF_ERR_LOGIC, FFLogicError, call, lib


def _torch():
    import torch

    return torch


class _Camera(ctypes.Structure):
    """ff_camera of include/ffb200.h."""

    _fields_ = [("alphaX", ctypes.c_float), ("alphaY", ctypes.c_float), ("centerX", ctypes.c_float),
                ("centerY", ctypes.c_float)]


class PerspectiveCamera:
    """Pinhole camera intrinsics (alphaX, alphaY, centerX, centerY), read-only as in the
    reference."""

    def __init__(self):
        self.cam = _Camera()

    def getIntrinsicsMatrix(self) -> np.ndarray:
        K = np.zeros((3, 3), dtype=np.float32)
        K[0, 0], K[0, 2] = self.alphaX, self.centerX
        K[1, 1], K[1, 2] = self.alphaY, self.centerY
        K[2, 2] = 1.0
        return K

    def _ro(name):  # noqa: N805
        def get(self):
            return getattr(self.cam, name)

        def put(self, value):
            raise RuntimeError(f"{name} cannot be set")

        return property(get, put)

    alphaX = _ro("alphaX")
    alphaY = _ro("alphaY")
    centerX = _ro("centerX")
    centerY = _ro("centerY")
    del _ro


def createPerspectiveCamera(focalLength: float, height: int, width: int, sensorHeight: float,
                            sensorWidth: float) -> PerspectiveCamera:
    """Camera of a sensor of the given physical size imaged on height x width pixels
    (createPerspectiveCamera, src/gpu/camera.cu:15-31)."""
    cam = PerspectiveCamera()
    call("ff_camera_perspective", focalLength, int(height), int(width), sensorHeight, sensorWidth,
         ctypes.byref(cam.cam))
    return cam


def _image(t, what: str):
    torch = _torch()
    if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype != torch.float32:
        raise ValueError(f"{what} should be a float32 CUDA tensor")
    depth = 1 if t.dim() == 2 else (t.shape[2] if t.dim() == 3 else 0)
    if depth not in (1, 4):
        raise ValueError(f"{what} should have depth 1 or 4, got shape {tuple(t.shape)}")
    if t.stride(-1) != 1 or (depth == 4 and t.stride(1) != 4):
        raise ValueError(f"{what} rows should be contiguous")
    return t, depth


def _flow(t):
    torch = _torch()
    if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype != torch.float32:
        raise ValueError("input flow should be a float32 CUDA tensor of shape (H, W, 2)")
    if t.dim() != 3 or t.shape[2] != 2:
        raise ValueError(f"input flow should have depth 2: {tuple(t.shape)}")
    if t.stride(2) != 1 or t.stride(1) != 2:
        raise ValueError("input flow rows should hold interleaved (x, y) pairs contiguously")
    return t


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


class _Timed:
    def _run(self, fn):
        torch = _torch()
        stream = torch.cuda.current_stream()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn(ctypes.c_void_p(stream.cuda_stream))
        e1.record(stream)
        e1.synchronize()
        self._ms = e0.elapsed_time(e1)

    def elapsedTime(self) -> float:
        """Milliseconds of the last compute()."""
        return self._ms

    def _workspace(self, like):
        """A second image for runs of more than ff_lax_wendroff_max_fused() iterations."""
        if max(self._iterations, 1) <= lib().ff_lax_wendroff_max_fused():
            return None
        if self._ws is None or self._ws.shape != like.shape:
            self._ws = _torch().empty_like(like)
        return self._ws


class LaxWendroffPropagator(_Timed):
    """Lax-Wendroff propagation of an image (depth 1 or 4) by a flow field."""

    def __init__(self, inputFlow=None, inputImage=None):
        self._flow = self._img = self._out = self._ws = None
        self._depth = 1
        self._iterations = 0
        self._ms = 0.0
        self._configured = False
        if inputFlow is None or inputImage is None:
            return
        self.setInputFlow(inputFlow)
        self.setInputImage(inputImage)
        self.configure()

    def configure(self) -> None:
        if self._flow is None:
            raise FFLogicError(FF_ERR_LOGIC, "LaxWendroffPropagator::configure(): input flow has not been set")
        if self._img is None:
            raise FFLogicError(FF_ERR_LOGIC, "LaxWendroffPropagator::configure(): input image has not been set")
        self._out = _torch().empty_like(self._img, memory_format=_torch().contiguous_format)
        self._configured = True

    def compute(self) -> None:
        if not self._configured:
            raise FFLogicError(FF_ERR_LOGIC, "LaxWendroffPropagator::compute(): stage not configured")
        f, i, o = self._flow, self._img, self._out
        ws = self._workspace(o)
        h, w = i.shape[:2]
        self._run(lambda s: call("ff_lax_wendroff", _p(f), f.stride(0) * 4, _p(i), i.stride(0) * 4, self._depth, h, w,
                                 self._iterations, _p(o), o.stride(0) * 4, _p(ws),
                                 ws.stride(0) * 4 if ws is not None else 0, s))

    def setInputFlow(self, inputFlow) -> None:
        self._flow = _flow(inputFlow)

    def setInputImage(self, img) -> None:
        t, d = _image(img, "input image")
        if self._flow is not None and tuple(t.shape[:2]) != tuple(self._flow.shape[:2]):
            raise ValueError("LaxWendroffPropagator::setInputImage(): image shape does not match with input flow")
        self._img, self._depth = t, d

    def getFlow(self):
        return self._flow

    def getPropagatedImage(self):
        return self._out

    def getDt(self) -> float:
        return float(np.float32(1.0) / np.float32(self._iterations)) if self._iterations > 0 else 0.0

    @property
    def iterations(self) -> int:
        return self._iterations

    @iterations.setter
    def iterations(self, n: int) -> None:
        if int(n) <= 0:
            raise ValueError(f"LaxWendroffPropagator::setIterations(): iterations less than zero: {n}")
        self._iterations = int(n)


class RotationalFlowImagePredictor(_Timed):
    """The image a camera rotating at a given angular velocity sees next: the rotational flow
    field of the camera model and the input image propagated along it (Lax-Wendroff).

    As in the reference, configure() starts a new propagator, so the iterations go back to
    0 (one pass pair with dt = 0, the image unchanged) until they are set again."""

    def __init__(self, cam: PerspectiveCamera | None = None, inputImage=None):
        self._cam = None
        self._w = (0.0, 0.0, 0.0)
        self._img = self._flow = self._out = self._ws = None
        self._depth = 1
        self._iterations = 0
        self._ms = 0.0
        self._configured = False
        if cam is None or inputImage is None:
            return
        self.setCamera(cam)
        self.setInputImage(inputImage)
        self.configure()

    def configure(self) -> None:
        if self._img is None:
            raise FFLogicError(FF_ERR_LOGIC, "RotationalFlowImagePredictor::configure(): input image not set")
        torch = _torch()
        h, w = self._img.shape[:2]
        self._flow = torch.empty((h, w, 2), dtype=torch.float32, device=self._img.device)
        self._out = torch.empty_like(self._img, memory_format=torch.contiguous_format)
        self._iterations = 0
        self._configured = True

    def compute(self) -> None:
        if not self._configured:
            raise FFLogicError(FF_ERR_LOGIC, "RotationalFlowImagePredictor::compute(): stage not configured")
        if self._cam is None:
            raise FFLogicError(FF_ERR_LOGIC, "RotationalFlowImagePredictor::compute(): camera not set")
        i, f, o = self._img, self._flow, self._out
        ws = self._workspace(o)
        h, w = i.shape[:2]
        self._run(lambda s: call("ff_rotational_predict", ctypes.byref(self._cam.cam), *self._w, _p(i),
                                 i.stride(0) * 4, self._depth, h, w, self._iterations, _p(f), f.stride(0) * 4, _p(o),
                                 o.stride(0) * 4, _p(ws), ws.stride(0) * 4 if ws is not None else 0, s))

    def setInputImage(self, inputImage) -> None:
        self._img, self._depth = _image(inputImage, "input image")

    def getPredictedImage(self):
        return self._out

    def getOpticalFlow(self):
        return self._flow

    def setCamera(self, cam: PerspectiveCamera) -> None:
        self._cam = cam

    def setAngularVelocity(self, wx: float, wy: float, wz: float) -> None:
        self._w = (float(wx), float(wy), float(wz))

    @property
    def iterations(self) -> int:
        return self._iterations

    @iterations.setter
    def iterations(self, n: int) -> None:
        if int(n) <= 0:
            raise ValueError(f"LaxWendroffPropagator::setIterations(): iterations less than zero: {n}")
        self._iterations = int(n)
