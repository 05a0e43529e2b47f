"""The C ABI library: it loads, exports every entry point include/ffb200.h declares,
and rejects invalid arguments before touching the GPU (runs without a GPU)."""

from __future__ import annotations

import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT

import flowfilter_b200 as ffb
from flowfilter_b200 import _lib


def declared_entry_points():
    text = open(os.path.join(ROOT, "include", "ffb200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ff_[a-z0-9_]+)\s*\(", text)))


def test_library_loads_and_exports_every_declared_symbol():
    L = _lib.lib()
    names = declared_entry_points()
    assert len(names) >= 45
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    # every binding the Python layer uses is declared in the header
    assert set(_lib.SIGNATURES) <= set(names)
    assert set(names) <= set(_lib.SIGNATURES), set(names) - set(_lib.SIGNATURES)


def test_bindings_pass_as_many_arguments_as_the_header_declares():
    """Every ctypes binding has one argument type per parameter of its declaration (a binding
    out of step with its declaration would pass arguments in the wrong places)."""
    text = open(os.path.join(ROOT, "include", "ffb200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    wrong = {}
    for name, params in re.findall(r"\b(ff_[a-z0-9_]+)\s*\(([^;{]*?)\)\s*;", text, flags=re.S):
        params = params.strip()
        n = 0 if params in ("", "void") else params.count(",") + 1
        if name in _lib.SIGNATURES and len(_lib.SIGNATURES[name][1]) != n:
            wrong[name] = (n, len(_lib.SIGNATURES[name][1]))
    assert not wrong, wrong


def test_allocation_failure_injection_switches_on_and_off():
    L = _lib.lib()
    assert L.ff_debug_fail_allocation_after(3) == _lib.FF_OK
    assert L.ff_debug_fail_allocation_after(-1) == _lib.FF_OK
    assert L.ff_debug_fail_allocation_after(-5) == _lib.FF_OK


def test_state_calls_reject_null_handles():
    L = _lib.lib()
    n = ctypes.c_size_t()
    buf = (ctypes.c_uint8 * 16)()
    assert L.ff_filter_state_bytes(None, ctypes.byref(n)) == _lib.FF_ERR_INVALID_ARGUMENT
    assert L.ff_filter_export_state(None, buf, 16) == _lib.FF_ERR_INVALID_ARGUMENT
    assert L.ff_filter_import_state(None, buf, 16) == _lib.FF_ERR_INVALID_ARGUMENT


def test_log_callback_receives_errors_until_switched_off():
    seen = []
    ffb.set_log_callback(lambda level, msg: seen.append((level, msg)))
    try:
        assert _lib.lib().ff_filter_compute(None) == _lib.FF_ERR_INVALID_ARGUMENT
        assert seen == [(_lib.FF_LOG_ERROR, "invalid argument: null filter")]
        assert _lib.lib().ff_last_error().decode() == "null filter"
    finally:
        ffb.set_log_callback(None)
    assert _lib.lib().ff_filter_compute(None) == _lib.FF_ERR_INVALID_ARGUMENT
    assert len(seen) == 1  # silent again


def test_version_and_status_strings():
    L = _lib.lib()
    assert L.ff_version() >= 10000
    assert L.ff_status_string(_lib.FF_ERR_SHAPE) == b"shape mismatch"
    assert L.ff_status_string(99) == b"unknown status"


@pytest.mark.parametrize("h,w", [(0, 10), (10, 0), (-3, 5)])
def test_flowfilter_rejects_bad_shape(h, w):
    with pytest.raises(ValueError):
        ffb.FlowFilter(h, w)


@pytest.mark.parametrize("levels", [0, -1])
def test_pyramid_rejects_bad_levels(levels):
    with pytest.raises(ValueError):
        ffb.PyramidalFlowFilter(64, 64, levels)


def test_null_output_handle_is_invalid_argument():
    L = _lib.lib()
    assert L.ff_filter_create(10, 10, 1, 1.0, 1.0, None) == _lib.FF_ERR_INVALID_ARGUMENT
    assert b"null" in L.ff_last_error()
    assert L.ff_pyramidal_create(10, 10, 2, None) == _lib.FF_ERR_INVALID_ARGUMENT


def test_null_filter_handle():
    L = _lib.lib()
    g = ctypes.c_float()
    assert L.ff_filter_get_gamma(None, 0, ctypes.byref(g)) == _lib.FF_ERR_INVALID_ARGUMENT
    assert L.ff_filter_compute(None) == _lib.FF_ERR_INVALID_ARGUMENT
    assert L.ff_filter_destroy(None) == _lib.FF_OK


def test_stage_argument_checks():
    L = _lib.lib()
    assert L.ff_stage_propagate(None, 0, 4, 4, 1, 3, None, 0, None, None) == _lib.FF_ERR_INVALID_ARGUMENT
    assert L.ff_stage_image_model(None, 0, 1, 4, 4, None, 0, None, 0, None) == _lib.FF_ERR_INVALID_ARGUMENT
    fake = ctypes.c_void_p(16)  # never dereferenced: rejected by the shape/parameter checks first
    assert L.ff_stage_propagate(fake, 64, 4, 4, 0, 3, fake, 64, fake, None) == _lib.FF_ERR_INVALID_ARGUMENT
    assert L.ff_stage_propagate(fake, 64, 4, 4, 2, -1, fake, 64, fake, None) == _lib.FF_ERR_INVALID_ARGUMENT
    assert L.ff_stage_smooth(fake, 64, 4, 4, 0, fake, 64, fake, None) == _lib.FF_ERR_INVALID_ARGUMENT
    assert L.ff_stage_image_model(fake, 64, 2, 4, 4, fake, 64, fake, 64, None) == _lib.FF_ERR_INVALID_ARGUMENT
    assert L.ff_stage_update(fake, 64, fake, 64, fake, 64, fake, 64, 4, 4, 0.0, 1.0, fake, 64, fake, 64,
                             None) == _lib.FF_ERR_INVALID_ARGUMENT
    assert L.ff_stage_pyramid_down(fake, 64, 1, 0, 4, fake, 64, None) == _lib.FF_ERR_INVALID_ARGUMENT


def test_workspace_sizes():
    L = _lib.lib()
    assert L.ff_stage_propagate_workspace_size(0, 5) == 0
    assert L.ff_stage_propagate_workspace_size(3, 5) >= 3 * 5 * 8
    assert L.ff_stage_propagate_payload_workspace_size(3, 5) >= 3 * 5 * 20
    assert L.ff_stage_smooth_workspace_size(7, 9) >= 7 * 9 * 8


def test_memcpy_kind_checked():
    L = _lib.lib()
    a = np.zeros(4, np.uint8)
    p = a.ctypes.data_as(ctypes.c_void_p)
    assert L.ff_memcpy2d(p, 4, p, 4, 4, 1, 7) == _lib.FF_ERR_INVALID_ARGUMENT


def test_cpp_dropin_library_exports_the_reference_classes():
    """libflowfilter_gpu.so carries the flowfilter::gpu classes the reference's callers link."""
    import subprocess

    lib = os.path.join(ROOT, "optical-flow-filter_b200", "flowfilter_b200", "libflowfilter_gpu.so")
    assert os.path.exists(lib)
    syms = subprocess.run(["nm", "-DC", "--defined-only", lib], capture_output=True, text=True, check=True).stdout
    for name in ["flowfilter::gpu::GPUImage::upload(", "flowfilter::gpu::GPUImage::download(",
                 "flowfilter::gpu::ImageModel::getImageGradient()", "flowfilter::gpu::FlowFilter::FlowFilter(int, int)",
                 "flowfilter::gpu::FlowFilter::FlowFilter(flowfilter::gpu::GPUImage)",
                 "flowfilter::gpu::FlowFilter::getFlow()", "flowfilter::gpu::FlowFilter::computeUpdate()",
                 "flowfilter::gpu::DeltaFlowFilter::DeltaFlowFilter(flowfilter::gpu::GPUImage, flowfilter::gpu::GPUImage)",
                 "flowfilter::gpu::PyramidalFlowFilter::PyramidalFlowFilter(int, int, int)",
                 "flowfilter::gpu::PyramidalFlowFilter::setGamma(std::vector<float, std::allocator<float> > const&)",
                 "flowfilter::gpu::PyramidalFlowFilter::setSmoothIterations(int, int)",
                 "flowfilter::gpu::Stage::elapsedTime() const"]:
        assert name in syms, name


def test_cpp_dropin_headers_compile(tmp_path):
    import subprocess

    src = tmp_path / "use.cpp"
    src.write_text('#include "flowfilter/gpu/flowfilter.h"\n#include "flowfilter/gpu/imagemodel.h"\n'
                   "int main() { flowfilter::image_t t{}; (void)t; return 0; }\n")
    subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-I", os.path.join(ROOT, "include"), str(src)], check=True)


def test_log_callback_receives_errors_of_every_module():
    """Failing calls of the differentiable, colour and Lax-Wendroff entry points (rejected
    before any GPU work) reach the log callback like the filter's."""
    seen = []
    ffb.set_log_callback(lambda level, msg: seen.append((level, msg)))
    try:
        L = _lib.lib()
        assert L.ff_diff_smooth(0, 0, 4, 4, 0, None, None, None, None) == _lib.FF_ERR_INVALID_ARGUMENT
        assert L.ff_diff_smooth(0, 1, 4, 4, 2, None, None, None, None) == _lib.FF_ERR_INVALID_ARGUMENT
        assert L.ff_flow_to_color(None, 8, 1, 1, 0.0, None, None, 4, None) == _lib.FF_ERR_INVALID_ARGUMENT
        assert L.ff_color_wheel_default(None) == _lib.FF_ERR_INVALID_ARGUMENT
        assert seen == [(_lib.FF_LOG_ERROR, "invalid argument: batch, height and width must be positive"),
                        (_lib.FF_LOG_ERROR, "invalid argument: axis must be 0 or 1"),
                        (_lib.FF_LOG_ERROR, "invalid argument: flow_to_color: maxflow should be greater than 0.0"),
                        (_lib.FF_LOG_ERROR, "invalid argument: rgba must not be NULL")]
        assert L.ff_last_error().decode() == "rgba must not be NULL"
    finally:
        ffb.set_log_callback(None)
