"""flowfilter_b200 — the Adarve–Mahony optical flow filter's per-frame hot path on B200.

Python face of libffb200.so (include/ffb200.h).  ``FlowFilter``,
``PyramidalFlowFilter`` and ``DeltaFlowFilter`` mirror the reference's classes;
``BatchFlowFilter`` advances many independent streams together; the
``stages`` module exposes the individual stages on CUDA tensors as functions and
``stage_classes`` as the reference's stage classes (``GPUImage``, ``ImageModel``,
``ImagePyramid``, ``FlowPropagator``, ``FlowPropagatorPayload``, ``FlowUpdate``,
``DeltaFlowUpdate``, ``FlowSmoother``); ``FlowToColor`` colour-
encodes a flow field; ``RotationalFlowImagePredictor`` and ``LaxWendroffPropagator``
predict an image under camera rotation.
"""

from ._lib import FFError, FFIndexError, FFLogicError, FFValueError, lib, set_log_callback  # noqa: F401
from .display import FlowToColor, color_wheel  # noqa: F401
from .rotation import (LaxWendroffPropagator, PerspectiveCamera, RotationalFlowImagePredictor,  # noqa: F401
                       createPerspectiveCamera)
from .filters import BatchFlowFilter, DeltaFlowFilter, FlowFilter, PyramidalFlowFilter, device_view  # noqa: F401
from .stage_classes import (DeltaFlowUpdate, FlowPropagator, FlowPropagatorPayload, FlowSmoother,  # noqa: F401
                            FlowUpdate, GPUImage, ImageModel, ImagePyramid)

__all__ = [
    "FlowFilter",
    "PyramidalFlowFilter",
    "DeltaFlowFilter",
    "BatchFlowFilter",
    "FlowToColor",
    "color_wheel",
    "PerspectiveCamera",
    "createPerspectiveCamera",
    "LaxWendroffPropagator",
    "RotationalFlowImagePredictor",
    "GPUImage",
    "ImageModel",
    "ImagePyramid",
    "FlowPropagator",
    "FlowPropagatorPayload",
    "FlowUpdate",
    "DeltaFlowUpdate",
    "FlowSmoother",
    "FFError",
    "FFValueError",
    "FFIndexError",
    "FFLogicError",
    "device_view",
    "lib",
    "set_log_callback",
]
