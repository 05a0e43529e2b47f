"""The reference's stage classes on CUDA tensors: GPUImage, ImageModel, ImagePyramid,
FlowPropagator, FlowPropagatorPayload, FlowUpdate, DeltaFlowUpdate and FlowSmoother.

They keep the reference's life cycle and names (python/flowfilter/gpu/{image,imagemodel,
pyramid,propagation,update}.pyx; FlowSmoother from include/flowfilter/gpu/flowsmoothing.h:22):
a stage is built on its input images, ``configure()`` allocates its outputs once, and every
``compute()`` overwrites those outputs in place.  Images are shared handles, as the
reference's GPUImage is (include/flowfilter/gpu/image.h:47-123): the ``GPUImage`` a getter
returns is the stage's output buffer itself, so stages wired to each other's outputs see every
new result without copies, and pipelines such as FlowFilter's (update -> smoother ->
propagator -> update, src/gpu/flowfilter.cu:84-122) can be rebuilt stage by stage.

Every compute() is one ``ff_stage_*`` call of the C ABI on torch's current CUDA stream; the
arithmetic is the library's (bit-identical with the reference).  Differences from the
reference: GPUImage buffers start cleared (the reference leaves a new buffer undefined), and
argument errors raise ValueError (invalid values) or RuntimeError (unconfigured stages) where
the reference throws std::exception or exits.
"""

from __future__ import annotations

import ctypes

import numpy as np

from ._lib import call, lib

__all__ = ["GPUImage", "ImageModel", "ImagePyramid", "FlowPropagator", "FlowPropagatorPayload", "FlowUpdate",
           "DeltaFlowUpdate", "FlowSmoother"]


def _torch():
    import torch

    return torch


def _stream():
    return ctypes.c_void_p(_torch().cuda.current_stream().cuda_stream)


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _pitch(t) -> int:
    return t.stride(0) * t.element_size()


class GPUImage:
    """A device image of height x width x depth items of itemSize bytes (1: uint8, 4: float32)
    held as a CUDA tensor; copies of the handle alias one buffer (image.pyx:16)."""

    def __init__(self, shape=None, itemSize: int = 4, *, tensor=None):
        torch = _torch()
        if tensor is not None:
            if not (isinstance(tensor, torch.Tensor) and tensor.is_cuda) or tensor.dim() not in (2, 3):
                raise ValueError("tensor should be a 2- or 3-dimensional CUDA tensor")
            if tensor.dtype not in (torch.uint8, torch.float32) or tensor.stride(-1) != 1:
                raise ValueError("tensor should be uint8 or float32 with contiguous rows")
            self.tensor = tensor
            return
        if shape is None:
            self.tensor = None
            return
        if len(shape) not in (2, 3):
            raise ValueError(f"number of dimensions must be 2 or 3, got: {len(shape)}")
        if itemSize not in (1, 4):
            raise ValueError("itemSize should be 1 (uint8) or 4 (float32)")
        dims = tuple(int(s) for s in shape)
        if len(dims) == 3 and dims[2] == 1:
            dims = dims[:2]
        self.tensor = torch.zeros(dims, dtype=torch.uint8 if itemSize == 1 else torch.float32, device="cuda")

    # ---- the reference's accessors
    def _t(self):
        if self.tensor is None:
            raise RuntimeError("GPUImage has no buffer")
        return self.tensor

    @property
    def shape(self):
        return tuple(self._t().shape)

    @property
    def height(self) -> int:
        return self._t().shape[0]

    @property
    def width(self) -> int:
        return self._t().shape[1]

    @property
    def depth(self) -> int:
        t = self._t()
        return 1 if t.dim() == 2 else t.shape[2]

    @property
    def itemSize(self) -> int:
        return self._t().element_size()

    @property
    def pitch(self) -> int:
        return _pitch(self._t())

    def upload(self, img) -> None:
        """Copy a host array of this image's shape and item type into the buffer."""
        t = self._t()
        a = np.ascontiguousarray(img)
        if a.shape != tuple(t.shape) and not (a.ndim == 3 and a.shape[2] == 1 and a.shape[:2] == tuple(t.shape)):
            raise ValueError(f"image shape {a.shape} does not match {tuple(t.shape)}")
        if a.itemsize != t.element_size():
            raise ValueError(f"item size {a.itemsize} does not match {t.element_size()}")
        t.copy_(_torch().from_numpy(a.reshape(t.shape)))

    def download(self, dtype=None, output=None) -> np.ndarray:
        """The buffer as a host array (image.pyx:43-62)."""
        t = self._t()
        host = t.cpu().numpy()
        if dtype is not None:
            host = host.view(np.dtype(dtype)) if np.dtype(dtype).itemsize == host.itemsize else host.astype(dtype)
        if output is None:
            return host
        np.copyto(output.reshape(host.shape), host)
        return output

    def copyFrom(self, other: "GPUImage") -> None:
        """Copy another image of the same shape and item size into this buffer (image.cu:139-166)."""
        src = other._t()
        t = self._t()
        if src.shape != t.shape or src.dtype != t.dtype:
            raise ValueError("copyFrom: images differ in shape or item size")
        t.copy_(src)

    def clear(self) -> None:
        self._t().zero_()

    def __repr__(self):
        return f"GPUImage(shape={self.shape if self.tensor is not None else None}, itemSize=" \
               f"{self.itemSize if self.tensor is not None else None})"


def _as_image(img, what: str) -> GPUImage:
    torch = _torch()
    if isinstance(img, GPUImage):
        img._t()
        return img
    if isinstance(img, torch.Tensor):
        return GPUImage(tensor=img)
    raise ValueError(f"{what} should be a GPUImage or a CUDA tensor")


def _need(img: GPUImage, depth: int, what: str, item_sizes=(4,)) -> None:
    if img.depth != depth or img.itemSize not in item_sizes:
        raise ValueError(f"{what} should have depth {depth} and item size in {item_sizes}, got depth {img.depth}, "
                         f"item size {img.itemSize}")


class _Stage:
    """configure/compute life cycle and elapsedTime() of a stage (src/gpu/pipeline.cu:63-88)."""

    def __init__(self):
        self._configured = False
        self._ev = None

    def _run(self, fn) -> None:
        if not self._configured:
            raise RuntimeError(f"{type(self).__name__}.compute(): stage not configured")
        torch = _torch()
        if self._ev is None:
            self._ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
        self._ev[0].record()
        fn()
        self._ev[1].record()

    def elapsedTime(self) -> float:
        """Milliseconds the last compute() took on the device."""
        if self._ev is None:
            return 0.0
        self._ev[1].synchronize()
        return self._ev[0].elapsed_time(self._ev[1])


class ImageModel(_Stage):
    """Image constant a0 and gradient (ax, ay) of a uint8 or float32 image
    (imagemodel.pyx:14, src/gpu/imagemodel.cu:93-113)."""

    def __init__(self, inputImage=None):
        super().__init__()
        self._in = None
        if inputImage is not None:
            self.setInputImage(inputImage)
            self.configure()

    def setInputImage(self, inputImage) -> None:
        img = _as_image(inputImage, "inputImage")
        _need(img, 1, "input image", (1, 4))
        self._in = img

    def configure(self) -> None:
        if self._in is None:
            raise RuntimeError("ImageModel.configure(): input image not set")
        h, w = self._in.height, self._in.width
        self._a0 = GPUImage((h, w), 4)
        self._grad = GPUImage((h, w, 2), 4)
        self._configured = True

    def compute(self) -> None:
        def run():
            i, a0, g = self._in.tensor, self._a0.tensor, self._grad.tensor
            call("ff_stage_image_model", _p(i), _pitch(i), i.element_size(), i.shape[0], i.shape[1], _p(a0),
                 _pitch(a0), _p(g), _pitch(g), _stream())
        self._run(run)

    def getImageConstant(self) -> GPUImage:
        return self._a0

    def getImageGradient(self) -> GPUImage:
        return self._grad


class ImagePyramid(_Stage):
    """Levels of an image by repeated [1/4, 1/2, 1/4] X then Y passes at stride 2
    (pyramid.pyx:13, src/gpu/pyramid.cu:49-219); level 0 is the input image itself."""

    def __init__(self, inputImage=None, levels: int = 1):
        super().__init__()
        self._in = None
        self._levels = 1
        self.levels = levels
        if inputImage is not None:
            self.setInputImage(inputImage)
            self.configure()

    def setInputImage(self, inputImage) -> None:
        img = _as_image(inputImage, "inputImage")
        _need(img, 1, "input image", (1, 4))
        self._in = img

    @property
    def levels(self) -> int:
        return self._levels

    @levels.setter
    def levels(self, levels: int) -> None:
        if int(levels) <= 0:
            raise ValueError(f"levels should be greater than zero: {levels}")
        self._levels = int(levels)
        if self._configured:
            self.configure()

    def configure(self) -> None:
        if self._in is None:
            raise RuntimeError("ImagePyramid.configure(): input image not set")
        h, w = self._in.height, self._in.width
        self._imgs = [self._in]
        for _ in range(1, self._levels):
            h, w = h // 2, w // 2
            if h < 1 or w < 1:
                raise ValueError("ImagePyramid: too many levels for the image size")
            self._imgs.append(GPUImage((h, w), self._in.itemSize))
        self._configured = True

    def compute(self) -> None:
        def run():
            for l in range(1, self._levels):
                a, b = self._imgs[l - 1].tensor, self._imgs[l].tensor
                call("ff_stage_pyramid_down", _p(a), _pitch(a), a.element_size(), a.shape[0], a.shape[1], _p(b),
                     _pitch(b), _stream())
        self._run(run)

    def getImage(self, level: int) -> GPUImage:
        if not 0 <= level < self._levels:
            raise IndexError(f"level index out of bounds: {level}")
        if not self._configured:
            raise RuntimeError("ImagePyramid.getImage(): stage not configured")
        return self._imgs[level]


class _PropBase(_Stage):
    def __init__(self, iterations: int):
        super().__init__()
        self._border = 3
        self._iterations = 1
        self.iterations = iterations

    @property
    def iterations(self) -> int:
        return self._iterations

    @iterations.setter
    def iterations(self, n: int) -> None:
        # the reference rejects negative counts (propagation.cu:137-148); a compute() runs at
        # least one sub-step pair, so 0 is refused here as well
        if int(n) <= 0:
            raise ValueError(f"iterations should be greater than zero: {n}")
        self._iterations = int(n)

    @property
    def dt(self) -> float:
        return float(np.float32(1.0) / np.float32(self._iterations))

    @property
    def border(self) -> int:
        return self._border

    @border.setter
    def border(self, b: int) -> None:
        if int(b) < 0:
            raise ValueError(f"border should be >= 0: {b}")
        self._border = int(b)

    def setIterations(self, n: int) -> None:
        self.iterations = n

    def getIterations(self) -> int:
        return self._iterations

    def setBorder(self, b: int) -> None:
        self.border = b

    def getBorder(self) -> int:
        return self._border

    def getDt(self) -> float:
        return self.dt


class FlowPropagator(_PropBase):
    """Upwind propagation of a flow field by itself over ``iterations`` X/Y sub-step pairs,
    dt = 1/iterations, border frozen (propagation.pyx:15, src/gpu/propagation.cu:80-210)."""

    def __init__(self, inputFlow=None, iterations: int = 1):
        super().__init__(iterations)
        self._in = None
        self._invert = False
        if inputFlow is not None:
            self.setInputFlow(inputFlow)
            self.configure()

    def setInputFlow(self, inputFlow) -> None:
        img = _as_image(inputFlow, "inputFlow")
        _need(img, 2, "input flow")
        self._in = img

    @property
    def invertInputFlow(self) -> bool:
        return self._invert

    @invertInputFlow.setter
    def invertInputFlow(self, invert: bool) -> None:
        self._invert = bool(invert)

    def setInvertInputFlow(self, invert: bool) -> None:
        self.invertInputFlow = invert

    def getInvertInputFlow(self) -> bool:
        return self._invert

    def configure(self) -> None:
        if self._in is None:
            raise RuntimeError("FlowPropagator.configure(): input flow not set")
        h, w = self._in.height, self._in.width
        torch = _torch()
        self._out = GPUImage((h, w, 2), 4)
        self._neg = GPUImage((h, w, 2), 4)
        self._ws = torch.empty(lib().ff_stage_propagate_workspace_size(h, w), dtype=torch.uint8, device="cuda")
        self._configured = True

    def compute(self) -> None:
        def run():
            src = self._in.tensor
            if self._invert:  # scalarProductF2_k with -1 (propagation.cu:92-96): an exact negation
                _torch().neg(src, out=self._neg.tensor)
                src = self._neg.tensor
            o = self._out.tensor
            call("ff_stage_propagate", _p(src), _pitch(src), src.shape[0], src.shape[1], self._iterations,
                 self._border, _p(o), _pitch(o), _p(self._ws), _stream())
        self._run(run)

    def getPropagatedFlow(self) -> GPUImage:
        return self._out


class FlowPropagatorPayload(_PropBase):
    """Propagation of a flow field with a scalar and a 2-vector payload advected by the same
    velocities (propagation.pyx:118, src/gpu/propagation.cu:262-412)."""

    def __init__(self, inputFlow=None, inputScalar=None, inputVector=None, iterations: int = 1):
        super().__init__(iterations)
        self._in = self._sc = self._vec = None
        if inputFlow is not None and inputScalar is not None and inputVector is not None:
            self.setInputFlow(inputFlow)
            self.setScalarPayload(inputScalar)
            self.setVectorPayload(inputVector)
            self.configure()

    def setInputFlow(self, inputFlow) -> None:
        img = _as_image(inputFlow, "inputFlow")
        _need(img, 2, "input flow")
        self._in = img

    def setScalarPayload(self, scalarField) -> None:
        img = _as_image(scalarField, "scalarField")
        _need(img, 1, "scalar payload")
        self._sc = img

    def setVectorPayload(self, vectorField) -> None:
        img = _as_image(vectorField, "vectorField")
        _need(img, 2, "vector payload")
        self._vec = img

    def configure(self) -> None:
        if self._in is None or self._sc is None or self._vec is None:
            raise RuntimeError("FlowPropagatorPayload.configure(): inputs not set")
        h, w = self._in.height, self._in.width
        if (self._sc.height, self._sc.width) != (h, w) or (self._vec.height, self._vec.width) != (h, w):
            raise ValueError("FlowPropagatorPayload: payload shapes differ from the flow's")
        torch = _torch()
        self._of = GPUImage((h, w, 2), 4)
        self._os = GPUImage((h, w), 4)
        self._ov = GPUImage((h, w, 2), 4)
        self._ws = torch.empty(lib().ff_stage_propagate_payload_workspace_size(h, w), dtype=torch.uint8,
                               device="cuda")
        self._configured = True

    def compute(self) -> None:
        def run():
            f, s, v = self._in.tensor, self._sc.tensor, self._vec.tensor
            of, os_, ov = self._of.tensor, self._os.tensor, self._ov.tensor
            call("ff_stage_propagate_payload", _p(f), _pitch(f), _p(s), _pitch(s), _p(v), _pitch(v), f.shape[0],
                 f.shape[1], self._iterations, self._border, _p(of), _pitch(of), _p(os_), _pitch(os_), _p(ov),
                 _pitch(ov), _p(self._ws), _stream())
        self._run(run)

    def getPropagatedFlow(self) -> GPUImage:
        return self._of

    def getPropagatedScalar(self) -> GPUImage:
        return self._os

    def getPropagatedVector(self) -> GPUImage:
        return self._ov


class _UpdateBase(_Stage):
    def __init__(self, gamma: float, maxflow: float):
        super().__init__()
        self._gamma = 1.0
        self._maxflow = 1.0
        self.gamma = gamma
        self.maxflow = maxflow

    @property
    def gamma(self) -> float:
        return self._gamma

    @gamma.setter
    def gamma(self, g: float) -> None:
        g = float(np.float32(g))
        if not g > 0:  # update.cu:123-131
            raise ValueError(f"gamma should be greater than zero: {g}")
        self._gamma = g

    @property
    def maxflow(self) -> float:
        return self._maxflow

    @maxflow.setter
    def maxflow(self, m: float) -> None:
        self._maxflow = float(np.float32(m))

    def setGamma(self, g: float) -> None:
        self.gamma = g

    def getGamma(self) -> float:
        return self._gamma

    def setMaxFlow(self, m: float) -> None:
        self.maxflow = m

    def getMaxFlow(self) -> float:
        return self._maxflow


class FlowUpdate(_UpdateBase):
    """The regularised 2x2 update of the top level (update.pyx:13, src/gpu/update.cu:30-116).
    The old image is the stage's own updated-image buffer, read and then overwritten with the
    new image constant by every compute()."""

    def __init__(self, inputFlow=None, inputImage=None, inputImageGradient=None, gamma: float = 1.0,
                 maxflow: float = 1.0):
        super().__init__(gamma, maxflow)
        self._flow = self._img = self._grad = None
        if inputFlow is not None and inputImage is not None and inputImageGradient is not None:
            self.setInputFlow(inputFlow)
            self.setInputImage(inputImage)
            self.setInputImageGradient(inputImageGradient)
            self.configure()

    def setInputFlow(self, inputFlow) -> None:
        img = _as_image(inputFlow, "inputFlow")
        _need(img, 2, "input flow")
        self._flow = img

    def setInputImage(self, image) -> None:
        img = _as_image(image, "image")
        _need(img, 1, "input image")
        self._img = img

    def setInputImageGradient(self, imageGradient) -> None:
        img = _as_image(imageGradient, "imageGradient")
        _need(img, 2, "input image gradient")
        self._grad = img

    def configure(self) -> None:
        if self._flow is None or self._img is None or self._grad is None:
            raise RuntimeError("FlowUpdate.configure(): inputs not set")
        h, w = self._flow.height, self._flow.width
        if (self._img.height, self._img.width) != (h, w) or (self._grad.height, self._grad.width) != (h, w):
            raise ValueError("FlowUpdate.configure(): input buffers do not match height and width")
        self._oflow = GPUImage((h, w, 2), 4)
        self._oimg = GPUImage((h, w), 4)
        self._configured = True

    def compute(self) -> None:
        def run():
            a0, g, f = self._img.tensor, self._grad.tensor, self._flow.tensor
            of, oi = self._oflow.tensor, self._oimg.tensor
            call("ff_stage_update", _p(a0), _pitch(a0), _p(g), _pitch(g), _p(oi), _pitch(oi), _p(f), _pitch(f),
                 a0.shape[0], a0.shape[1], self._gamma, self._maxflow, _p(of), _pitch(of), _p(oi), _pitch(oi),
                 _stream())
        self._run(run)

    def getUpdatedFlow(self) -> GPUImage:
        return self._oflow

    def getUpdatedImage(self) -> GPUImage:
        return self._oimg


class DeltaFlowUpdate(_UpdateBase):
    """The update of a finer pyramid level: the 2x2 solve on the propagated delta flow, then
    the coarse flow (``inputFlow``, half the size) upsampled by point sampling and added twice
    (update.pyx:100, src/gpu/update.cu:219-349)."""

    def __init__(self, inputFlow=None, inputDeltaFlow=None, inputImageOld=None, inputImage=None,
                 inputImageGradient=None, gamma: float = 1.0, maxflow: float = 1.0):
        super().__init__(gamma, maxflow)
        self._flow = self._delta = self._old = self._img = self._grad = None
        if all(x is not None for x in (inputFlow, inputDeltaFlow, inputImageOld, inputImage, inputImageGradient)):
            self.setInputFlow(inputFlow)
            self.setInputDeltaFlow(inputDeltaFlow)
            self.setInputImageOld(inputImageOld)
            self.setInputImage(inputImage)
            self.setInputImageGradient(inputImageGradient)
            self.configure()

    def setInputFlow(self, inputFlow) -> None:
        img = _as_image(inputFlow, "inputFlow")
        _need(img, 2, "input (coarse) flow")
        self._flow = img

    def setInputDeltaFlow(self, inputDeltaFlow) -> None:
        img = _as_image(inputDeltaFlow, "inputDeltaFlow")
        _need(img, 2, "input delta flow")
        self._delta = img

    def setInputImageOld(self, inputImageOld) -> None:
        img = _as_image(inputImageOld, "inputImageOld")
        _need(img, 1, "input old image")
        self._old = img

    def setInputImage(self, image) -> None:
        img = _as_image(image, "image")
        _need(img, 1, "input image")
        self._img = img

    def setInputImageGradient(self, imageGradient) -> None:
        img = _as_image(imageGradient, "imageGradient")
        _need(img, 2, "input image gradient")
        self._grad = img

    def configure(self) -> None:
        if any(x is None for x in (self._flow, self._delta, self._old, self._img, self._grad)):
            raise RuntimeError("DeltaFlowUpdate.configure(): inputs not set")
        h, w = self._delta.height, self._delta.width
        for x in (self._old, self._img, self._grad):
            if (x.height, x.width) != (h, w):
                raise ValueError("DeltaFlowUpdate.configure(): input buffers do not match height and width")
        self._oflow = GPUImage((h, w, 2), 4)
        self._odelta = GPUImage((h, w, 2), 4)
        self._oimg = GPUImage((h, w), 4)
        self._configured = True

    def compute(self) -> None:
        def run():
            a0, g, old, d, c = self._img.tensor, self._grad.tensor, self._old.tensor, self._delta.tensor, \
                self._flow.tensor
            of, od, oi = self._oflow.tensor, self._odelta.tensor, self._oimg.tensor
            call("ff_stage_delta_update", _p(a0), _pitch(a0), _p(g), _pitch(g), _p(old), _pitch(old), _p(d),
                 _pitch(d), _p(c), _pitch(c), c.shape[0], c.shape[1], a0.shape[0], a0.shape[1], self._gamma,
                 self._maxflow, _p(of), _pitch(of), _p(od), _pitch(od), _p(oi), _pitch(oi), _stream())
        self._run(run)

    def getUpdatedFlow(self) -> GPUImage:
        return self._oflow

    def getUpdatedDeltaFlow(self) -> GPUImage:
        return self._odelta

    def getUpdatedImage(self) -> GPUImage:
        return self._oimg


class FlowSmoother(_Stage):
    """``iterations`` passes of the 5-tap box filter along X then Y (include/flowfilter/gpu/
    flowsmoothing.h:22, src/gpu/flowsmoothing.cu:74-127)."""

    def __init__(self, inputFlow=None, iterations: int = 1):
        super().__init__()
        self._in = None
        self._iterations = 1
        self.iterations = iterations
        if inputFlow is not None:
            self.setInputFlow(inputFlow)
            self.configure()

    @property
    def iterations(self) -> int:
        return self._iterations

    @iterations.setter
    def iterations(self, n: int) -> None:
        if int(n) <= 0:  # flowsmoothing.cu:117-127
            raise ValueError(f"iterations should be greater than zero: {n}")
        self._iterations = int(n)

    def setIterations(self, n: int) -> None:
        self.iterations = n

    def getIterations(self) -> int:
        return self._iterations

    def setInputFlow(self, inputFlow) -> None:
        img = _as_image(inputFlow, "inputFlow")
        _need(img, 2, "input flow")
        self._in = img

    def configure(self) -> None:
        if self._in is None:
            raise RuntimeError("FlowSmoother.configure(): input flow not set")
        h, w = self._in.height, self._in.width
        torch = _torch()
        self._out = GPUImage((h, w, 2), 4)
        self._ws = torch.empty(lib().ff_stage_smooth_workspace_size(h, w), dtype=torch.uint8, device="cuda")
        self._configured = True

    def compute(self) -> None:
        def run():
            f, o = self._in.tensor, self._out.tensor
            call("ff_stage_smooth", _p(f), _pitch(f), f.shape[0], f.shape[1], self._iterations, _p(o), _pitch(o),
                 _p(self._ws), _stream())
        self._run(run)

    def getSmoothedFlow(self) -> GPUImage:
        return self._out
