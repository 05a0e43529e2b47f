"""ctypes binding of the C ABI in include/ffb200.h (libffb200.so, built in place).

The library is loaded from this package directory; importing a filter when the
library is missing raises immediately — there is no fallback implementation.
"""

from __future__ import annotations

import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libffb200.so")

FF_OK = 0
FF_ERR_INVALID_ARGUMENT = 1
FF_ERR_LOGIC = 2
FF_ERR_OUT_OF_RANGE = 3
FF_ERR_SHAPE = 4
FF_ERR_CUDA = 5
FF_ERR_OUT_OF_MEMORY = 6
FF_ERR_UNSUPPORTED = 7


class FFError(RuntimeError):
    """Raised for CUDA failures and unsupported requests."""

    def __init__(self, status: int, msg: str):
        super().__init__(msg)
        self.status = status


class FFValueError(FFError, ValueError):
    """Invalid argument / shape mismatch (the reference's std::invalid_argument)."""


class FFIndexError(FFError, IndexError):
    """Level index out of range."""


class FFLogicError(FFError):
    """Operation on an object in the wrong state (the reference's std::logic_error)."""


class FFImage(ctypes.Structure):
    # flowfilter::image_t (include/flowfilter/image.h:30-49)
    _fields_ = [
        ("height", ctypes.c_int),
        ("width", ctypes.c_int),
        ("depth", ctypes.c_int),
        ("pitch", ctypes.c_size_t),
        ("itemSize", ctypes.c_size_t),
        ("data", ctypes.c_void_p),
    ]


_i = ctypes.c_int
_f = ctypes.c_float
_sz = ctypes.c_size_t
_vp = ctypes.c_void_p
_ip = ctypes.POINTER(ctypes.c_int)
_fp = ctypes.POINTER(ctypes.c_float)
_szp = ctypes.POINTER(ctypes.c_size_t)
_vpp = ctypes.POINTER(ctypes.c_void_p)
_st = ctypes.c_int
LOG_FN = ctypes.CFUNCTYPE(None, ctypes.c_int, ctypes.c_char_p, ctypes.c_void_p)
FF_LOG_ERROR = 0
FF_LOG_INFO = 1

SIGNATURES = {
    "ff_last_error": (ctypes.c_char_p, []),
    "ff_set_log_callback": (_st, [LOG_FN, _vp]),
    "ff_status_string": (ctypes.c_char_p, [_st]),
    "ff_version": (_i, []),
    "ff_set_device": (_st, [_i]),
    "ff_malloc_pitch": (_st, [_vpp, _szp, _sz, _sz]),
    "ff_free": (_st, [_vp]),
    "ff_memcpy2d": (_st, [_vp, _sz, _vp, _sz, _sz, _sz, _i]),
    "ff_memset2d": (_st, [_vp, _sz, _i, _sz, _sz]),
    "ff_filter_create": (_st, [_i, _i, _i, _f, _f, _vpp]),
    "ff_filter_create_on_device_image": (_st, [_vp, _sz, _i, _i, _i, _vpp]),
    "ff_delta_filter_create": (_st, [_vp, _sz, _i, _i, _i, _vp, _sz, _i, _i, _vpp]),
    "ff_pyramidal_create": (_st, [_i, _i, _i, _vpp]),
    "ff_filter_destroy": (_st, [_vp]),
    "ff_filter_shape": (_st, [_vp, _ip, _ip, _ip]),
    "ff_filter_kind": (_st, [_vp, _ip]),
    "ff_filter_level_shape": (_st, [_vp, _i, _ip, _ip]),
    "ff_filter_set_gamma": (_st, [_vp, _i, _f]),
    "ff_filter_get_gamma": (_st, [_vp, _i, _fp]),
    "ff_filter_set_max_flow": (_st, [_vp, _f]),
    "ff_filter_get_max_flow": (_st, [_vp, _fp]),
    "ff_filter_set_smooth_iterations": (_st, [_vp, _i, _i]),
    "ff_filter_get_smooth_iterations": (_st, [_vp, _i, _ip]),
    "ff_filter_set_propagation_border": (_st, [_vp, _i]),
    "ff_filter_get_propagation_border": (_st, [_vp, _ip]),
    "ff_filter_get_propagation_iterations": (_st, [_vp, _i, _ip]),
    "ff_filter_set_fused": (_st, [_vp, _i]),
    "ff_filter_set_graphs": (_st, [_vp, _i]),
    "ff_filter_set_band": (_st, [_vp, _i]),
    "ff_filter_autotune": (_st, [_vp, _i]),
    "ff_filter_autotune_flush": (_st, [_vp, _i, _vp, _sz]),
    "ff_filter_tuning": (_st, [_vp, ctypes.c_char_p, _sz]),
    "ff_filter_get_level_tuning": (_st, [_vp, _i, _ip, _ip]),
    "ff_filter_set_level_tuning": (_st, [_vp, _i, _i, _i]),
    "ff_filter_set_profiling": (_st, [_vp, _i]),
    "ff_filter_level_kernel_ms": (_st, [_vp, _i, _fp, _ip]),
    "ff_filter_time_level": (_st, [_vp, _i, _i, _vp, _sz, _fp]),
    "ff_filter_set_stream": (_st, [_vp, _vp]),
    "ff_filter_load_image_host": (_st, [_vp, ctypes.POINTER(FFImage)]),
    "ff_filter_load_image_device_async": (_st, [_vp, _vp, _sz, _vp]),
    "ff_filter_bind_image_device": (_st, [_vp, _vp, _sz]),
    "ff_filter_compute": (_st, [_vp]),
    "ff_filter_compute_async": (_st, [_vp, _vp]),
    "ff_filter_process_host_async": (_st, [_vp, ctypes.POINTER(FFImage), ctypes.POINTER(FFImage), _vp]),
    "ff_filter_synchronize": (_st, [_vp]),
    "ff_filter_compute_image_model": (_st, [_vp]),
    "ff_filter_compute_propagation": (_st, [_vp]),
    "ff_filter_compute_update": (_st, [_vp]),
    "ff_filter_elapsed_ms": (_st, [_vp, _fp]),
    "ff_filter_state_bytes": (_st, [_vp, _szp]),
    "ff_filter_export_state": (_st, [_vp, _vp, _sz]),
    "ff_filter_import_state": (_st, [_vp, _vp, _sz]),
    "ff_filter_download_flow_host": (_st, [_vp, ctypes.POINTER(FFImage)]),
    "ff_filter_download_image_host": (_st, [_vp, ctypes.POINTER(FFImage)]),
    "ff_filter_device_result": (_st, [_vp, _i, _vpp, _szp]),
    "ff_filter_level_state_host": (_st, [_vp, _i, _i, _vp, _sz]),
    "ff_stage_pyramid_down": (_st, [_vp, _sz, _i, _i, _i, _vp, _sz, _vp]),
    "ff_stage_image_model": (_st, [_vp, _sz, _i, _i, _i, _vp, _sz, _vp, _sz, _vp]),
    "ff_stage_propagate_workspace_size": (_sz, [_i, _i]),
    "ff_stage_propagate": (_st, [_vp, _sz, _i, _i, _i, _i, _vp, _sz, _vp, _vp]),
    "ff_stage_propagate_payload_workspace_size": (_sz, [_i, _i]),
    "ff_stage_propagate_payload": (_st, [_vp, _sz, _vp, _sz, _vp, _sz, _i, _i, _i, _i, _vp, _sz, _vp, _sz, _vp, _sz,
                                         _vp, _vp]),
    "ff_stage_update": (_st, [_vp, _sz, _vp, _sz, _vp, _sz, _vp, _sz, _i, _i, _f, _f, _vp, _sz, _vp, _sz, _vp]),
    "ff_stage_delta_update": (_st, [_vp, _sz, _vp, _sz, _vp, _sz, _vp, _sz, _vp, _sz, _i, _i, _i, _i, _f, _f, _vp, _sz,
                                    _vp, _sz, _vp, _sz, _vp]),
    "ff_stage_smooth_workspace_size": (_sz, [_i, _i]),
    "ff_stage_smooth": (_st, [_vp, _sz, _i, _i, _i, _vp, _sz, _vp, _vp]),
    "ff_stage_scale_flow": (_st, [_vp, _sz, _i, _i, ctypes.c_float, _vp, _sz, _vp]),
    "ff_stage_smooth_noalloc": (_st, [_vp, _sz, _i, _i, _i, _vp, _sz, _vp]),
    "ff_batch_create": (_st, [_i, _ip, _ip, _ip, _vpp]),
    "ff_batch_destroy": (_st, [_vp]),
    "ff_batch_size": (_st, [_vp, _ip]),
    "ff_batch_stream": (_st, [_vp, _i, _vpp]),
    "ff_batch_frame_layout": (_st, [_vp, _szp, _szp]),
    "ff_batch_launches": (_st, [_vp, _ip]),
    "ff_batch_step": (_st, [_vp, _vp, _vp]),
    "ff_debug_fail_allocation_after": (_st, [ctypes.c_longlong]),
    "ff_batch_set_tuning": (_st, [_vp, ctypes.c_longlong, _i]),
    "ff_batch_set_level_band": (_st, [_vp, _i, _i, _i]),
    "ff_diff_pyramid": (_st, [_i, _i, _i, _i, _vp, _vp, _vp]),
    "ff_diff_pyramid_bwd": (_st, [_i, _i, _i, _i, _vp, _vp, _vp]),
    "ff_diff_model": (_st, [_i, _i, _i, _i, _vp, _vp, _vp, _vp]),
    "ff_diff_model_bwd": (_st, [_i, _i, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp]),
    "ff_diff_propagate": (_st, [_i, _i, _i, _i, _i, _i, ctypes.c_double, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "ff_diff_propagate_bwd": (_st, [_i, _i, _i, _i, _i, _i, ctypes.c_double, _i] + [_vp] * 10),
    "ff_diff_update": (_st, [_i, _i, _i, _i, _vp, _vp, _vp, _vp, _vp, ctypes.c_double, _vp, _vp]),
    "ff_diff_update_bwd": (_st, [_i, _i, _i, _i, _vp, _vp, _vp, _vp, _vp, ctypes.c_double] + [_vp] * 7),
    "ff_diff_delta_update": (_st, [_i, _i, _i, _i, _i, _i] + [_vp] * 6 + [ctypes.c_double, _vp, _vp, _vp]),
    "ff_diff_delta_update_bwd": (_st, [_i, _i, _i, _i, _i, _i] + [_vp] * 6 + [ctypes.c_double] + [_vp] * 9),
    "ff_diff_smooth": (_st, [_i, _i, _i, _i, _i, _vp, _vp, _vp, _vp]),
    "ff_diff_smooth_bwd": (_st, [_i, _i, _i, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp]),
    "ff_flow_to_color": (_st, [_vp, ctypes.c_size_t, _i, _i, ctypes.c_float, _vp, _vp, ctypes.c_size_t, _vp]),
    "ff_color_wheel_default": (_st, [_vp]),
    "ff_camera_perspective": (_st, [ctypes.c_float, _i, _i, ctypes.c_float, ctypes.c_float, _vp]),
    "ff_rotational_flow": (_st, [_vp, ctypes.c_float, ctypes.c_float, ctypes.c_float, _vp, ctypes.c_size_t, _i, _i,
                                 _vp]),
    "ff_lax_wendroff_max_fused": (_i, []),
    "ff_lax_wendroff": (_st, [_vp, ctypes.c_size_t, _vp, ctypes.c_size_t, _i, _i, _i, _i, _vp, ctypes.c_size_t, _vp,
                              ctypes.c_size_t, _vp]),
    "ff_rotational_predict": (_st, [_vp, ctypes.c_float, ctypes.c_float, ctypes.c_float, _vp, ctypes.c_size_t, _i, _i,
                                    _i, _i, _vp, ctypes.c_size_t, _vp, ctypes.c_size_t, _vp, ctypes.c_size_t, _vp]),
    "ff_diff_frame_tape_bytes": (ctypes.c_size_t, [_i, _vp]),
    "ff_diff_frame_scratch_bytes": (ctypes.c_size_t, [_i, _vp]),
    "ff_diff_frame_forward": (_st, [_i, _vp, _i] + [_vp] * 9),
    "ff_diff_frame_infer_bytes": (ctypes.c_size_t, [_i, _vp]),
    "ff_diff_frame_infer": (_st, [_i, _vp, _i] + [_vp] * 8),
    "ff_diff_epe_scratch_bytes": (ctypes.c_size_t, [_i]),
    "ff_diff_epe": (_st, [_i] * 6 + [ctypes.c_double, _vp, _vp, ctypes.c_longlong, ctypes.c_longlong, _vp, _vp, _vp]),
    "ff_diff_epe_bwd": (_st, [_i] * 6 + [ctypes.c_double, _vp, _vp, ctypes.c_longlong, ctypes.c_longlong, _vp, _vp,
                                         _vp]),
    "ff_diff_frame_backward": (_st, [_i, _vp, _i] + [_vp] * 9 + [ctypes.c_longlong] + [_vp] * 6),
}

_lib = None
_lock = threading.Lock()


def lib() -> ctypes.CDLL:
    """Load libffb200.so from the package directory (raises if it was not built)."""
    global _lib
    if _lib is None:
        with _lock:
            if _lib is None:
                if not os.path.exists(LIB_PATH):
                    raise ImportError(
                        f"{LIB_PATH} is missing: build it with `make -C optical-flow-filter_b200` "
                        "(or __graft_entry__.build()); there is no fallback implementation")
                L = ctypes.CDLL(LIB_PATH)
                for name, (res, args) in SIGNATURES.items():
                    fn = getattr(L, name)
                    fn.restype = res
                    fn.argtypes = args
                _lib = L
    return _lib


def check(status: int) -> None:
    """Raise the Python exception matching an ff_status."""
    if status == FF_OK:
        return
    msg = lib().ff_last_error().decode(errors="replace")
    if status in (FF_ERR_INVALID_ARGUMENT, FF_ERR_SHAPE):
        raise FFValueError(status, msg)
    if status == FF_ERR_OUT_OF_RANGE:
        raise FFIndexError(status, msg)
    if status == FF_ERR_LOGIC:
        raise FFLogicError(status, msg)
    raise FFError(status, msg)


def call(name: str, *args) -> None:
    check(getattr(lib(), name)(*args))


_log_callback = None  # the ctypes thunk the library holds, kept alive here


def set_log_callback(fn) -> None:
    """Send the library's log to ``fn(level, message)`` (level FF_LOG_ERROR or FF_LOG_INFO;
    message a str); ``None`` switches it off.  The library is silent by default."""
    global _log_callback
    if fn is None:
        call("ff_set_log_callback", LOG_FN(), None)
        _log_callback = None
        return
    thunk = LOG_FN(lambda level, msg, user: fn(int(level), msg.decode(errors="replace")))
    call("ff_set_log_callback", thunk, None)
    _log_callback = thunk
