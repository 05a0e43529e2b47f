"""ff_stage_smooth_noalloc (static device scratch) against ff_stage_smooth (caller workspace).

Both calls go through the C ABI. This file is collected last so the static-scratch entry
point also runs after every other GPU test has used the library on the same device.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FF_OK = 0
FF_ERR_INVALID_ARGUMENT = 1
STATIC_SCRATCH_BYTES = 32 << 20


@pytest.fixture(scope="module")
def lib(cuda):
    from flowfilter_b200 import _lib

    return _lib.lib()


def flows(cuda, h, w, seed, n):
    rng = np.random.default_rng(seed)
    return [cuda.from_numpy(rng.normal(0, 1.5, (h, w, 2)).astype(np.float32)).cuda() for _ in range(n)]


def smooth_ws(cuda, lib, x, s):
    h, w = x.shape[:2]
    out = cuda.empty_like(x)
    ws = cuda.empty(lib.ff_stage_smooth_workspace_size(h, w), dtype=cuda.uint8, device="cuda")
    st = lib.ff_stage_smooth(x.data_ptr(), w * 8, h, w, s, out.data_ptr(), w * 8, ws.data_ptr(),
                             ctypes.c_void_p(cuda.cuda.current_stream().cuda_stream))
    assert st == FF_OK, lib.ff_last_error()
    return out


def smooth_static(cuda, lib, x, s, out):
    h, w = x.shape[:2]
    return lib.ff_stage_smooth_noalloc(x.data_ptr(), w * 8, h, w, s, out.data_ptr(), w * 8,
                                       ctypes.c_void_p(cuda.cuda.current_stream().cuda_stream))


@pytest.mark.parametrize("h,w,s", [(53, 70, 1), (480, 640, 2), (1088, 2048, 4), (2048, 2048, 1)])
def test_two_calls_in_a_row_match_workspace_entry_point(cuda, lib, h, w, s):
    a, b = flows(cuda, h, w, 11 + s, 2)
    want_a, want_b = smooth_ws(cuda, lib, a, s), smooth_ws(cuda, lib, b, s)
    got_a, got_b = cuda.empty_like(a), cuda.empty_like(b)
    # queued back to back on one stream: the second call reuses the scratch the first wrote
    assert smooth_static(cuda, lib, a, s, got_a) == FF_OK, lib.ff_last_error()
    assert smooth_static(cuda, lib, b, s, got_b) == FF_OK, lib.ff_last_error()
    cuda.cuda.synchronize()
    assert cuda.equal(got_a, want_a)
    assert cuda.equal(got_b, want_b)


def test_sizes_alternate_on_one_stream(cuda, lib):
    big = flows(cuda, 1088, 2048, 5, 1)[0]
    small = flows(cuda, 61, 77, 6, 1)[0]
    outs = []
    for x in (big, small, big):
        o = cuda.empty_like(x)
        assert smooth_static(cuda, lib, x, 2, o) == FF_OK, lib.ff_last_error()
        outs.append(o)
    cuda.cuda.synchronize()
    for x, o in zip((big, small, big), outs):
        assert cuda.equal(o, smooth_ws(cuda, lib, x, 2))


def test_in_place_matches(cuda, lib):
    x = flows(cuda, 240, 320, 7, 1)[0]
    want = smooth_ws(cuda, lib, x, 3)
    assert smooth_static(cuda, lib, x, 3, x) == FF_OK, lib.ff_last_error()
    cuda.cuda.synchronize()
    assert cuda.equal(x, want)


@pytest.mark.parametrize("h,w", [(2049, 2048), (2048, 2049), (1, (1 << 22) + 1)])
def test_rejects_flows_above_the_static_scratch(cuda, lib, h, w):
    assert ((w * 8 + 511) // 512 * 512) * h > STATIC_SCRATCH_BYTES
    x = cuda.zeros((1, 1, 2), device="cuda")  # never read: the size check comes first
    st = lib.ff_stage_smooth_noalloc(x.data_ptr(), w * 8, h, w, 1, x.data_ptr(), w * 8, None)
    assert st == FF_ERR_INVALID_ARGUMENT
    msg = lib.ff_last_error().decode()
    assert "static" in msg and str(STATIC_SCRATCH_BYTES) in msg


def test_rejects_bad_arguments(cuda, lib):
    x = cuda.zeros((4, 4, 2), device="cuda")
    assert lib.ff_stage_smooth_noalloc(None, 32, 4, 4, 1, x.data_ptr(), 32, None) == FF_ERR_INVALID_ARGUMENT
    assert lib.ff_stage_smooth_noalloc(x.data_ptr(), 32, 4, 4, 0, x.data_ptr(), 32, None) == FF_ERR_INVALID_ARGUMENT
    assert lib.ff_stage_smooth_noalloc(x.data_ptr(), 32, 0, 4, 1, x.data_ptr(), 32, None) == FF_ERR_INVALID_ARGUMENT
