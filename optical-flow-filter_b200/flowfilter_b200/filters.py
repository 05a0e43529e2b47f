"""Python filter classes mirroring the reference's Cython API.

``FlowFilter`` and ``PyramidalFlowFilter`` keep the names, arguments, properties and
error behaviour of python/flowfilter/gpu/flowfilters.pyx:15-455 (loadImage / compute /
getFlow / getImage / elapsedTime; gamma, maxflow, smoothIterations,
propagationIterations, propagationBorder).  Inputs may be numpy arrays (synchronous
host upload, as in the reference) or torch tensors (CPU or CUDA).  Everything runs
through the C ABI of libffb200.so; there is no host-side fallback.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import FFImage, call, lib

__all__ = ["FlowFilter", "PyramidalFlowFilter", "DeltaFlowFilter", "BatchFlowFilter", "device_view"]


def _torch():
    import torch  # imported lazily: numpy-only use does not need it

    return torch


class _CudaArray:
    """__cuda_array_interface__ wrapper for a pitched device buffer owned by a filter."""

    def __init__(self, ptr: int, shape, strides, typestr: str, owner):
        self.__cuda_array_interface__ = {
            "shape": tuple(shape),
            "strides": tuple(strides),
            "typestr": typestr,
            "data": (ptr, False),
            "version": 3,
        }
        self._owner = owner


def device_view(ptr: int, pitch: int, height: int, width: int, channels: int, owner=None):
    """torch.float32 view (H, W[, C]) of a pitched device buffer (no copy)."""
    torch = _torch()
    if channels == 1:
        shape, strides = (height, width), (pitch, 4)
    else:
        shape, strides = (height, width, channels), (pitch, 4 * channels, 4)
    return torch.as_tensor(_CudaArray(ptr, shape, strides, "<f4", owner), device="cuda")


def _host_image(arr: np.ndarray, depth: int) -> tuple[FFImage, np.ndarray]:
    arr = np.ascontiguousarray(arr)
    img = FFImage()
    img.height = arr.shape[0]
    img.width = arr.shape[1]
    img.depth = depth
    img.itemSize = arr.dtype.itemsize
    img.pitch = arr.strides[0]
    img.data = arr.ctypes.data_as(ctypes.c_void_p)
    return img, arr


def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


def _torch_cuda() -> bool:
    try:
        return _torch().cuda.is_available()
    except ImportError:
        return False


def _host_array(x, dtype, shape) -> np.ndarray:
    """A C-contiguous numpy view of a host buffer (numpy array or CPU tensor), no copy."""
    arr = x.numpy() if _is_torch(x) else x
    if not isinstance(arr, np.ndarray) or arr.dtype != dtype or arr.shape != shape or not arr.flags["C_CONTIGUOUS"]:
        raise ValueError(f"expected a contiguous host {np.dtype(dtype).name} buffer of shape {shape}")
    return arr


class _FilterBase:
    _h = None

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h and _lib._lib is not None:
            lib().ff_filter_destroy(h)

    # ------------------------------------------------------------ helpers
    def _shape(self):
        h, w, l = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        call("ff_filter_shape", self._h, ctypes.byref(h), ctypes.byref(w), ctypes.byref(l))
        return h.value, w.value, l.value

    def _item(self) -> int:
        return 1

    def loadImage(self, img) -> None:
        """Load the next frame: numpy (H, W) uint8 uploads synchronously (flowfilter.cu:218-220);
        a CUDA tensor is copied device-to-device on the current torch stream."""
        dtype = np.uint8 if self._item() == 1 else np.float32
        if _is_torch(img) and img.is_cuda:
            torch = _torch()
            want = torch.uint8 if dtype == np.uint8 else torch.float32
            if img.dtype != want or tuple(img.shape) != (self.height, self.width):
                raise ValueError(f"expected a {want} tensor of shape {(self.height, self.width)}, "
                                 f"got {img.dtype} {tuple(img.shape)}")
            if img.stride(1) != 1:
                img = img.contiguous()
            stream = torch.cuda.current_stream().cuda_stream
            call("ff_filter_load_image_device_async", self._h, ctypes.c_void_p(img.data_ptr()),
                 img.stride(0) * img.element_size(), ctypes.c_void_p(stream))
            self._keep_input = img
            return
        if _is_torch(img):
            img = img.numpy()
        img = np.asarray(img)
        if img.ndim != 2:
            raise ValueError(f"image should be 2-D (height, width), got shape {img.shape}")
        if img.dtype != dtype:
            raise ValueError(f"image dtype should be {np.dtype(dtype)}, got {img.dtype}")
        fimg, keep = _host_image(img, 1)
        call("ff_filter_load_image_host", self._h, ctypes.byref(fimg))

    def compute(self) -> None:
        """One frame; blocks until done (flowfilter.cu:125-153, 685-716)."""
        call("ff_filter_compute", self._h)

    def computeAsync(self, stream=None) -> None:
        """Enqueue one frame on ``stream`` (default: the current torch stream)."""
        if stream is None:
            stream = _torch().cuda.current_stream().cuda_stream
        elif hasattr(stream, "cuda_stream"):
            stream = stream.cuda_stream
        call("ff_filter_compute_async", self._h, ctypes.c_void_p(stream))

    def processAsync(self, frame, flow, stream=None) -> None:
        """Pipelined loadImage + compute + downloadFlow for host buffers: ``frame`` (H, W) and
        ``flow`` (H, W, 2) float32 are numpy arrays or CPU tensors (pinned for overlap); the
        call returns at once and ``flow`` is filled once ``synchronize()`` returns.  Keep
        both buffers untouched until then."""
        dtype = np.uint8 if self._item() == 1 else np.float32
        fin = _host_array(frame, dtype, (self.height, self.width))
        fout = _host_array(flow, np.float32, (self.height, self.width, 2))
        img_in, _ = _host_image(fin, 1)
        img_out, _ = _host_image(fout, 2)
        if stream is None:
            stream = _torch().cuda.current_stream().cuda_stream if _torch_cuda() else 0
        elif hasattr(stream, "cuda_stream"):
            stream = stream.cuda_stream
        call("ff_filter_process_host_async", self._h, ctypes.byref(img_in), ctypes.byref(img_out),
             ctypes.c_void_p(stream))

    def synchronize(self) -> None:
        """Wait for everything queued on the filter, pipelined copies included."""
        call("ff_filter_synchronize", self._h)

    def elapsedTime(self) -> float:
        ms = ctypes.c_float()
        call("ff_filter_elapsed_ms", self._h, ctypes.byref(ms))
        return ms.value

    def exportState(self) -> np.ndarray:
        """The filter's state after its latest frame as a uint8 array (checkpoint): per level
        the smoothed flow, old image, delta or unsmoothed flow and the first-frame flag.
        Parameters are not part of it."""
        n = ctypes.c_size_t()
        call("ff_filter_state_bytes", self._h, ctypes.byref(n))
        out = np.empty(n.value, dtype=np.uint8)
        call("ff_filter_export_state", self._h, out.ctypes.data_as(ctypes.c_void_p), n.value)
        return out

    def importState(self, state) -> None:
        """Resume from exportState() of a filter of the same kind and level sizes."""
        a = np.ascontiguousarray(np.asarray(state, dtype=np.uint8).reshape(-1))
        call("ff_filter_import_state", self._h, a.ctypes.data_as(ctypes.c_void_p), a.size)

    def getFlow(self, flow: np.ndarray | None = None) -> np.ndarray:
        """Smoothed level-0 flow as (H, W, 2) float32 (downloadFlow, flowfilter.cu:238-240)."""
        if flow is None:
            flow = np.zeros((self.height, self.width, 2), dtype=np.float32)
        if flow.dtype != np.float32 or flow.shape != (self.height, self.width, 2) or not flow.flags["C_CONTIGUOUS"]:
            raise ValueError("flow buffer should be a contiguous float32 array of shape (H, W, 2)")
        fimg, _ = _host_image(flow, 2)
        call("ff_filter_download_flow_host", self._h, ctypes.byref(fimg))
        return flow

    def getImage(self, image: np.ndarray | None = None) -> np.ndarray:
        """Level-0 updated image (current a0), (H, W) float32 (downloadImage)."""
        if image is None:
            image = np.zeros((self.height, self.width), dtype=np.float32)
        if image.dtype != np.float32 or image.shape != (self.height, self.width) or not image.flags["C_CONTIGUOUS"]:
            raise ValueError("image buffer should be a contiguous float32 array of shape (H, W)")
        fimg, _ = _host_image(image, 1)
        call("ff_filter_download_image_host", self._h, ctypes.byref(fimg))
        return image

    def _device_result(self, which: int, channels: int):
        p, pitch = ctypes.c_void_p(), ctypes.c_size_t()
        call("ff_filter_device_result", self._h, which, ctypes.byref(p), ctypes.byref(pitch))
        return device_view(p.value, pitch.value, self.height, self.width, channels, owner=self)

    def getFlowDevice(self):
        """torch view of getFlow() on the device (valid until the next compute)."""
        return self._device_result(1, 2)

    def flowTensor(self):
        """torch view of the smoothed level-0 flow on the device (valid until the next compute)."""
        return self._device_result(0, 2)

    def imageTensor(self):
        """torch view of the level-0 updated image on the device."""
        return self._device_result(2, 1)

    def levelState(self, level: int, which: int) -> np.ndarray:
        """Host copy of a level's state: 0 smoothed flow, 1 unsmoothed flow (top level),
        2 old image, 3 delta flow (delta levels)."""
        h, w = ctypes.c_int(), ctypes.c_int()
        call("ff_filter_level_shape", self._h, level, ctypes.byref(h), ctypes.byref(w))
        ch = 1 if which == 2 else 2
        out = np.zeros((h.value, w.value, ch) if ch == 2 else (h.value, w.value), np.float32)
        call("ff_filter_level_state_host", self._h, level, which, out.ctypes.data_as(ctypes.c_void_p),
             out.strides[0])
        return out

    def setFused(self, mode) -> None:
        """Kernel selection: False/0 per-stage kernels, True/1 streaming fused per-level kernels,
        2 automatic (the default: the autotuned choice, else the streaming kernel for levels
        of at least 200,000 pixels and the tile-fused kernel below), 3 tile-fused kernels.
        Results are identical."""
        call("ff_filter_set_fused", self._h, int(mode))

    def setGraphs(self, enabled: bool) -> None:
        """Replay the frame step from captured CUDA graphs (one per state parity)."""
        call("ff_filter_set_graphs", self._h, 1 if enabled else 0)

    def autotune(self, repetitions: int = 5, flush=None) -> str:
        """Time each level's kernel choices on the current inputs, then (pyramids) whole frames
        over combinations of the best ones, and keep the fastest; returns the choice per level.
        ``flush`` (a CUDA tensor) is overwritten before every timed whole frame.  Needs one
        computed frame; results are unchanged."""
        if flush is None:
            call("ff_filter_autotune", self._h, int(repetitions))
        else:
            call("ff_filter_autotune_flush", self._h, int(repetitions), ctypes.c_void_p(flush.data_ptr()),
                 flush.numel() * flush.element_size())
        return self.tuning()

    def tuningState(self) -> list:
        """[(path, band)] per level: path -1 untuned, 0 per-stage, 1 streaming fused (band =
        rows per band, 0 automatic), 2 tile-fused (band = tile-shape index, 0 automatic)."""
        out = []
        for l in range(self._shape()[2]):
            p, b = ctypes.c_int(), ctypes.c_int()
            call("ff_filter_get_level_tuning", self._h, l, ctypes.byref(p), ctypes.byref(b))
            out.append((p.value, b.value))
        return out

    def setTuningState(self, state) -> None:
        for l, (p, b) in enumerate(state):
            call("ff_filter_set_level_tuning", self._h, l, int(p), int(b))

    def tuning(self) -> str:
        buf = ctypes.create_string_buffer(512)
        call("ff_filter_tuning", self._h, buf, 512)
        return buf.value.decode()

    def timeLevel(self, level: int, reps: int = 100, flush=None) -> float:
        """Mean device milliseconds of one level step in its current configuration, replayed
        as a captured graph; ``flush`` (a CUDA tensor) is overwritten before every launch."""
        ms = ctypes.c_float()
        fp = ctypes.c_void_p(flush.data_ptr()) if flush is not None else None
        nb = flush.numel() * flush.element_size() if flush is not None else 0
        call("ff_filter_time_level", self._h, int(level), int(reps), fp, nb, ctypes.byref(ms))
        return ms.value / reps

    def setBand(self, rows: int) -> None:
        """Rows per warp band of the fused kernels (0 = automatic)."""
        call("ff_filter_set_band", self._h, int(rows))

    def setProfiling(self, max_frames: int) -> None:
        """Record per-level kernel events for the next ``max_frames`` computes."""
        call("ff_filter_set_profiling", self._h, int(max_frames))

    def levelKernelTime(self, level: int) -> tuple[float, int]:
        """(summed milliseconds, frames) of the level's kernels since setProfiling."""
        ms, n = ctypes.c_float(), ctypes.c_int()
        call("ff_filter_level_kernel_ms", self._h, int(level), ctypes.byref(ms), ctypes.byref(n))
        return ms.value, n.value

    def setStream(self, stream) -> None:
        if hasattr(stream, "cuda_stream"):
            stream = stream.cuda_stream
        call("ff_filter_set_stream", self._h, ctypes.c_void_p(stream))

    # ------------------------------------------------------------ properties
    @property
    def height(self) -> int:
        return self._shape()[0]

    @height.setter
    def height(self, value):
        raise RuntimeError("Filter height cannot be set after instantiation")

    @property
    def width(self) -> int:
        return self._shape()[1]

    @width.setter
    def width(self, value):
        raise RuntimeError("Filter width cannot be set after instantiation")

    @property
    def maxflow(self) -> float:
        v = ctypes.c_float()
        call("ff_filter_get_max_flow", self._h, ctypes.byref(v))
        return v.value

    @maxflow.setter
    def maxflow(self, value: float) -> None:
        call("ff_filter_set_max_flow", self._h, float(value))

    @property
    def propagationBorder(self) -> int:
        v = ctypes.c_int()
        call("ff_filter_get_propagation_border", self._h, ctypes.byref(v))
        return v.value

    @propagationBorder.setter
    def propagationBorder(self, value: int) -> None:
        call("ff_filter_set_propagation_border", self._h, int(value))

    def _get_gamma(self, level: int) -> float:
        v = ctypes.c_float()
        call("ff_filter_get_gamma", self._h, level, ctypes.byref(v))
        return v.value

    def _get_smooth(self, level: int) -> int:
        v = ctypes.c_int()
        call("ff_filter_get_smooth_iterations", self._h, level, ctypes.byref(v))
        return v.value

    def _get_iters(self, level: int) -> int:
        v = ctypes.c_int()
        call("ff_filter_get_propagation_iterations", self._h, level, ctypes.byref(v))
        return v.value


class FlowFilter(_FilterBase):
    """Single-level filter, flowfilters.pyx:15-200 / flowfilter.cu:45-76.

    ``FlowFilter(height, width, smoothIterations=1, maxflow=1.0, gamma=1.0)`` owns a
    uint8 input image.  ``FlowFilter.on_device(tensor)`` is FlowFilter(GPUImage): it
    reads a caller-owned uint8 or float32 CUDA image on every compute.
    """

    def __init__(self, height: int, width: int, smoothIterations: int = 1, maxflow: float = 1.0,
                 gamma: float = 1.0):
        h = ctypes.c_void_p()
        call("ff_filter_create", int(height), int(width), int(smoothIterations), float(maxflow), float(gamma),
             ctypes.byref(h))
        self._h = h
        self._itemsize = 1

    @classmethod
    def on_device(cls, image) -> "FlowFilter":
        """FlowFilter(GPUImage): configure() defaults (gamma 1 unscaled, maxflow 1, 1 smoothing)."""
        torch = _torch()
        if not (_is_torch(image) and image.is_cuda and image.dim() == 2):
            raise ValueError("expected a 2-D CUDA tensor")
        if image.dtype not in (torch.uint8, torch.float32):
            raise ValueError("image dtype should be uint8 or float32")
        if image.stride(1) != 1:
            raise ValueError("image rows must be contiguous")
        self = cls.__new__(cls)
        h = ctypes.c_void_p()
        item = image.element_size()
        call("ff_filter_create_on_device_image", ctypes.c_void_p(image.data_ptr()), image.stride(0) * item, item,
             image.shape[0], image.shape[1], ctypes.byref(h))
        self._h = h
        self._itemsize = item
        self._keep_input = image
        return self

    def _item(self) -> int:
        return self._itemsize

    def configure(self) -> None:
        """Kept for API compatibility; the filter is configured at construction."""

    def computeImageModel(self) -> None:
        call("ff_filter_compute_image_model", self._h)

    def computePropagation(self) -> None:
        call("ff_filter_compute_propagation", self._h)

    def computeUpdate(self) -> None:
        call("ff_filter_compute_update", self._h)

    @property
    def gamma(self) -> float:
        return self._get_gamma(0)

    @gamma.setter
    def gamma(self, value: float) -> None:
        call("ff_filter_set_gamma", self._h, 0, float(value))

    @property
    def smoothIterations(self) -> int:
        return self._get_smooth(0)

    @smoothIterations.setter
    def smoothIterations(self, value: int) -> None:
        call("ff_filter_set_smooth_iterations", self._h, 0, int(value))

    @property
    def propagationIterations(self) -> int:
        return self._get_iters(0)

    @propagationIterations.setter
    def propagationIterations(self, value):
        raise RuntimeError("propagation iterations cannot be set, use maxflow instead")


class DeltaFlowFilter(_FilterBase):
    """DeltaFlowFilter(GPUImage image, GPUImage inputFlow), flowfilter.cu:349-426, over CUDA
    tensors: ``image`` (H, W) uint8/float32 and ``coarse_flow`` (Hc, Wc, 2) float32."""

    def __init__(self, image, coarse_flow):
        torch = _torch()
        if not (_is_torch(image) and image.is_cuda and image.dim() == 2 and image.stride(1) == 1):
            raise ValueError("image should be a 2-D CUDA tensor with contiguous rows")
        if image.dtype not in (torch.uint8, torch.float32):
            raise ValueError("image dtype should be uint8 or float32")
        if not (_is_torch(coarse_flow) and coarse_flow.is_cuda and coarse_flow.dim() == 3
                and coarse_flow.shape[2] == 2 and coarse_flow.dtype == torch.float32
                and coarse_flow.stride(2) == 1 and coarse_flow.stride(1) == 2):
            raise ValueError("coarse flow should be a (Hc, Wc, 2) float32 CUDA tensor with contiguous rows")
        h = ctypes.c_void_p()
        item = image.element_size()
        call("ff_delta_filter_create", ctypes.c_void_p(image.data_ptr()), image.stride(0) * item, item,
             image.shape[0], image.shape[1], ctypes.c_void_p(coarse_flow.data_ptr()), coarse_flow.stride(0) * 4,
             coarse_flow.shape[0], coarse_flow.shape[1], ctypes.byref(h))
        self._h = h
        self._itemsize = item
        self._keep = (image, coarse_flow)

    def _item(self) -> int:
        return self._itemsize

    def computeImageModel(self) -> None:
        call("ff_filter_compute_image_model", self._h)

    def computePropagation(self) -> None:
        call("ff_filter_compute_propagation", self._h)

    def computeUpdate(self) -> None:
        call("ff_filter_compute_update", self._h)

    @property
    def gamma(self) -> float:
        return self._get_gamma(0)

    @gamma.setter
    def gamma(self, value: float) -> None:
        call("ff_filter_set_gamma", self._h, 0, float(value))

    @property
    def smoothIterations(self) -> int:
        return self._get_smooth(0)

    @smoothIterations.setter
    def smoothIterations(self, value: int) -> None:
        call("ff_filter_set_smooth_iterations", self._h, 0, int(value))

    @property
    def propagationIterations(self) -> int:
        return self._get_iters(0)


class PyramidalFlowFilter(_FilterBase):
    """Pyramidal filter, flowfilters.pyx:204-455 / flowfilter.cu:621-897."""

    def __init__(self, height: int, width: int, levels: int):
        h = ctypes.c_void_p()
        call("ff_pyramidal_create", int(height), int(width), int(levels), ctypes.byref(h))
        self._h = h

    def configure(self) -> None:
        """Kept for API compatibility; the filter is configured at construction."""

    @property
    def levels(self) -> int:
        return self._shape()[2]

    @levels.setter
    def levels(self, value):
        raise RuntimeError("Filter levels cannot be set after instantiation")

    @property
    def gamma(self):
        if self.levels == 1:
            return self._get_gamma(0)
        return [self._get_gamma(h) for h in range(self.levels)]

    @gamma.setter
    def gamma(self, g) -> None:
        if self.levels == 1:
            call("ff_filter_set_gamma", self._h, 0, float(g))
        else:
            for h in range(self.levels):
                call("ff_filter_set_gamma", self._h, h, float(g[h]))

    def setGamma(self, level: int, gamma: float) -> None:
        call("ff_filter_set_gamma", self._h, int(level), float(gamma))

    def getGamma(self, level: int) -> float:
        return self._get_gamma(int(level))

    @property
    def smoothIterations(self):
        if self.levels == 1:
            return self._get_smooth(0)
        return [self._get_smooth(h) for h in range(self.levels)]

    @smoothIterations.setter
    def smoothIterations(self, n) -> None:
        if self.levels == 1:
            call("ff_filter_set_smooth_iterations", self._h, 0, int(n))
        else:
            for h in range(self.levels):
                call("ff_filter_set_smooth_iterations", self._h, h, int(n[h]))

    def setSmoothIterations(self, level: int, n: int) -> None:
        call("ff_filter_set_smooth_iterations", self._h, int(level), int(n))

    def getSmoothIterations(self, level: int) -> int:
        return self._get_smooth(int(level))

    def propagationIterationsAt(self, level: int) -> int:
        return self._get_iters(int(level))


class _BatchStream(PyramidalFlowFilter):
    """One stream of a BatchFlowFilter: a PyramidalFlowFilter owned by the batch."""

    def __init__(self, handle, batch):
        self._h = handle
        self._batch = batch  # keeps the batch (and so this stream) alive

    def __del__(self):
        self._h = None  # the batch destroys its streams


class BatchFlowFilter:
    """Many independent pyramidal streams advanced together (no reference counterpart).

    ``BatchFlowFilter([(height, width, levels), ...])``.  ``stream(i)`` is stream i as a
    PyramidalFlowFilter (set gamma / smoothIterations / maxflow / propagationBorder, read
    getFlow() / getFlowDevice()); ``step(frames)`` advances every stream by one frame, where
    ``frames`` is one uint8 CUDA tensor of ``frameBytes()`` bytes holding stream i's frame
    at ``frameOffsets()[i]`` (``pack()`` builds it from a list of (H, W) tensors).  A step
    runs ``launches()`` kernels, a number that does not grow with the number of streams;
    every stream's results equal those of the same stream filtered alone.
    """

    def __init__(self, shapes):
        shapes = [tuple(int(v) for v in s) for s in shapes]
        n = len(shapes)
        if n == 0:
            raise ValueError("a batch needs at least one stream")
        arr = (ctypes.c_int * n)
        hs, ws, ls = arr(*[s[0] for s in shapes]), arr(*[s[1] for s in shapes]), arr(*[s[2] for s in shapes])
        h = ctypes.c_void_p()
        call("ff_batch_create", n, hs, ws, ls, ctypes.byref(h))
        self._h = h
        self.shapes = shapes
        offs = (ctypes.c_size_t * n)()
        total = ctypes.c_size_t()
        call("ff_batch_frame_layout", self._h, offs, ctypes.byref(total))
        self._offsets = list(offs)
        self._total = total.value
        self._streams = []
        for i in range(n):
            fh = ctypes.c_void_p()
            call("ff_batch_stream", self._h, i, ctypes.byref(fh))
            self._streams.append(_BatchStream(fh, self))

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h and _lib._lib is not None:
            lib().ff_batch_destroy(h)

    def __len__(self) -> int:
        return len(self.shapes)

    def stream(self, i: int) -> PyramidalFlowFilter:
        return self._streams[i]

    def frameOffsets(self) -> list:
        return list(self._offsets)

    def frameBytes(self) -> int:
        return self._total

    def launches(self) -> int:
        n = ctypes.c_int()
        call("ff_batch_launches", self._h, ctypes.byref(n))
        return n.value

    def setTuning(self, minPixels: int = -1, band: int = 0) -> None:
        """Top levels and levels reading the previous frame's coarse flow (phase A) below
        ``minPixels`` pixels run the tile kernel (-1: 200000), every other level the streaming
        kernel covers runs it in bands of ``band`` rows (0: the default rule).  Results are
        unchanged."""
        call("ff_batch_set_tuning", self._h, int(minPixels), int(band))

    @staticmethod
    def streamBytes(height: int, width: int, levels: int) -> int:
        """Compulsory HBM bytes of one frame of a stream: the uint8 frame, 40 B of state read
        and written plus 2 B of coarse flow per pixel of every delta level, 24 B per pixel of
        the top level."""
        total, h, w = height * width, height, width
        for l in range(levels):
            total += h * w * (24 if l == levels - 1 else 42)
            h, w = h // 2, w // 2
        return total

    @staticmethod
    def shard(shapes, ranks: int) -> list:
        """Streams split over ``ranks`` GPUs (one batch each): the stream indices of every
        rank, assigned greedily, largest compulsory bytes first, each to the rank with the
        least so far."""
        order = sorted(range(len(shapes)), key=lambda i: (-BatchFlowFilter.streamBytes(*shapes[i]), i))
        load = [0] * ranks
        out = [[] for _ in range(ranks)]
        for i in order:
            r = min(range(ranks), key=lambda k: (load[k], k))
            out[r].append(i)
            load[r] += BatchFlowFilter.streamBytes(*shapes[i])
        return [sorted(v) for v in out]

    def setLevelBand(self, height: int, width: int, band: int) -> None:
        """Levels of ``height`` x ``width`` pixels run in bands of ``band`` rows (0: no
        override).  Results are unchanged."""
        call("ff_batch_set_level_band", self._h, int(height), int(width), int(band))

    def levelSizes(self) -> list:
        """Distinct (height, width) of the streams' pyramid levels, largest first."""
        sizes = set()
        for hh, ww, L in self.shapes:
            for l in range(L):
                sizes.add((hh >> l, ww >> l))
        return sorted(sizes, key=lambda s: (-s[0] * s[1], s))

    def _signature(self) -> str:
        import hashlib
        import json

        streams = [[list(sh), st.gamma, st.smoothIterations, st.maxflow, st.propagationBorder]
                   for sh, st in zip(self.shapes, self._streams)]
        return hashlib.sha256(json.dumps(streams).encode()).hexdigest()

    def autotune(self, frames, repetitions: int = 3, cache: str | None = None,
                 bands=(8, 12, 16, 24, 32, 48, 64, 96, 128)) -> dict:
        """Picks the streaming kernel's band rows per level size by timing: a scratch batch
        with this batch's streams and parameters steps on ``frames`` (a packed step buffer,
        see pack()); level sizes are tuned one at a time, largest first, each keeping the band
        whose step is fastest (median of ``repetitions`` CUDA-event-timed steps) with the
        sizes before it fixed (0: the batch's default rule stays).  The choice is applied
        here (setLevelBand) and returned as {"HxW": band}.  With ``cache`` (a JSON file), a choice stored for the same streams and
        parameters is applied without timing, and a new one is stored.  This batch's streams
        are not stepped, and results do not depend on the choice."""
        import json
        import os

        torch = _torch()
        key = self._signature()
        store = {}
        if cache and os.path.exists(cache):
            with open(cache) as fh:
                store = json.load(fh)
            if key in store:
                choice = store[key]
                for name, b in choice.items():
                    hh, ww = (int(v) for v in name.split("x"))
                    self.setLevelBand(hh, ww, b)
                return choice
        scratch = BatchFlowFilter(self.shapes)
        for st, mine in zip(scratch._streams, self._streams):
            st.gamma = mine.gamma
            st.smoothIterations = mine.smoothIterations
            st.maxflow = mine.maxflow
            st.propagationBorder = mine.propagationBorder
        scratch.step(frames)  # the first frame runs each stream on its own

        def step_ms():
            scratch.step(frames)  # rebuilds the step graph after a band change
            ms = []
            for _ in range(max(1, int(repetitions))):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                scratch.step(frames)
                e1.record()
                e1.synchronize()
                ms.append(e0.elapsed_time(e1))
            return sorted(ms)[len(ms) // 2]

        choice = {}
        for hh, ww in self.levelSizes():
            best = None
            # 0: the batch's own band rule (no override), kept unless a band beats it
            for b in [0] + sorted({min(int(v), hh) for v in bands if v > 0}):
                scratch.setLevelBand(hh, ww, b)
                t = step_ms()
                if best is None or t < best[0]:
                    best = (t, b)
            scratch.setLevelBand(hh, ww, best[1])
            choice[f"{hh}x{ww}"] = best[1]
        del scratch
        for name, b in choice.items():
            hh, ww = (int(v) for v in name.split("x"))
            self.setLevelBand(hh, ww, b)
        if cache:
            store[key] = choice
            with open(cache, "w") as fh:
                json.dump(store, fh, indent=1, sort_keys=True)
        return choice

    def pack(self, frames, out=None):
        """Pack one (H, W) uint8 CUDA tensor per stream into a step buffer (device copies)."""
        torch = _torch()
        if out is None:
            out = torch.empty(self._total, dtype=torch.uint8, device="cuda")
        for (hh, ww, _), off, f in zip(self.shapes, self._offsets, frames):
            if tuple(f.shape) != (hh, ww) or f.dtype != torch.uint8:
                raise ValueError(f"stream frame should be a uint8 tensor of shape {(hh, ww)}")
            out[off:off + hh * ww].view(hh, ww).copy_(f)
        return out

    def step(self, frames, stream=None) -> None:
        """Advance every stream by one frame (enqueued on ``stream``, default the current one)."""
        torch = _torch()
        if not (_is_torch(frames) and frames.is_cuda and frames.dtype == torch.uint8 and frames.is_contiguous()
                and frames.numel() >= self._total):
            raise ValueError(f"frames should be a contiguous uint8 CUDA tensor of {self._total} bytes")
        if stream is None:
            stream = torch.cuda.current_stream().cuda_stream
        elif hasattr(stream, "cuda_stream"):
            stream = stream.cuda_stream
        call("ff_batch_step", self._h, ctypes.c_void_p(frames.data_ptr()), ctypes.c_void_p(stream))
