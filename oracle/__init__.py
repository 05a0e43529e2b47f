"""ctypes view of the CPU oracle (oracle/oracle.cpp) — TEST INFRASTRUCTURE ONLY.

Imported by tests/, by ``__graft_entry__.smoke()`` (as the checker) and by the
CPU-baseline leg of bench.py.  The product never imports this package.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
REF_DRIVER = os.path.join(HERE, "_ref", "ref_driver")

# variant keys (oracle.h)
V_MODEL_FMA, V_PROP_FMA, V_UPD_NFMA, V_UPD_Q, V_UPD_OX, V_UPD_OY, V_SMOOTH_FMA, V_UPMAP = range(8)

_lib = None
_f32p = ctypes.POINTER(ctypes.c_float)
_u8p = ctypes.POINTER(ctypes.c_uint8)


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        i = ctypes.c_int
        f = ctypes.c_float
        sigs = {
            "or_set_variant": (None, [i, i]),
            "or_get_variant": (i, [i]),
            "or_set_norm_table": (None, [_f32p]),
            "or_get_norm_table": (None, [_f32p]),
            "or_set_threads": (None, [i]),
            "or_pyramid_down_u8": (None, [_u8p, i, i, _u8p]),
            "or_pyramid_down_f32": (None, [_f32p, i, i, _f32p]),
            "or_image_model": (None, [vp, i, i, i, _f32p, _f32p]),
            "or_propagate": (None, [_f32p, i, i, i, i, _f32p]),
            "or_propagate_payload": (None, [_f32p, _f32p, _f32p, i, i, i, i, _f32p, _f32p, _f32p]),
            "or_update": (None, [_f32p, _f32p, _f32p, _f32p, i, i, f, f, _f32p, _f32p]),
            "or_delta_update": (None, [_f32p, _f32p, _f32p, _f32p, _f32p, i, i, i, i, f, f, _f32p, _f32p, _f32p]),
            "or_smooth": (None, [_f32p, i, i, i, _f32p]),
            "or_upmap_index": (i, [i, i, i]),
            "or_camera_perspective": (None, [f, i, i, f, f, _f32p]),
            "or_rotational_flow": (None, [_f32p, f, f, f, i, i, _f32p]),
            "or_lax_wendroff": (None, [_f32p, _f32p, i, i, i, i, _f32p]),
            "or_flowfilter_create": (vp, [i, i, i, f, f]),
            "or_flowfilter_create_on": (vp, [i, i, i]),
            "or_pyramidal_create": (vp, [i, i, i]),
            "or_filter_destroy": (None, [vp]),
            "or_filter_levels": (i, [vp]),
            "or_filter_set_gamma": (i, [vp, i, f]),
            "or_filter_get_gamma": (f, [vp, i]),
            "or_filter_set_max_flow": (i, [vp, f]),
            "or_filter_get_max_flow": (f, [vp]),
            "or_filter_set_smooth_iterations": (i, [vp, i, i]),
            "or_filter_get_smooth_iterations": (i, [vp, i]),
            "or_filter_set_propagation_border": (i, [vp, i]),
            "or_filter_get_propagation_iterations": (i, [vp, i]),
            "or_filter_load": (None, [vp, vp]),
            "or_filter_compute": (None, [vp]),
            "or_filter_download_flow": (None, [vp, _f32p]),
            "or_filter_get_flow": (None, [vp, _f32p]),
            "or_filter_download_image": (None, [vp, _f32p]),
            "or_filter_level_state": (ctypes.c_size_t, [vp, i, i, _f32p]),
            "or_filter_level_shape": (None, [vp, i, ctypes.POINTER(i), ctypes.POINTER(i)]),
        }
        for name, (res, args) in sigs.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _p(a: np.ndarray, t=_f32p):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(t)


def set_variant(key: int, value: int) -> None:
    lib().or_set_variant(key, value)


def get_variant(key: int) -> int:
    return lib().or_get_variant(key)


def set_threads(n: int) -> None:
    lib().or_set_threads(n)


def set_norm_table(t: np.ndarray) -> None:
    t = np.ascontiguousarray(t, dtype=np.float32)
    lib().or_set_norm_table(_p(t))


def norm_table() -> np.ndarray:
    t = np.empty(256, np.float32)
    lib().or_get_norm_table(_p(t))
    return t


def pyramid_down(img: np.ndarray) -> np.ndarray:
    h, w = img.shape
    img = np.ascontiguousarray(img)
    if img.dtype == np.uint8:
        out = np.empty((h // 2, w // 2), np.uint8)
        lib().or_pyramid_down_u8(_p(img, _u8p), h, w, _p(out, _u8p))
    else:
        img = img.astype(np.float32)
        out = np.empty((h // 2, w // 2), np.float32)
        lib().or_pyramid_down_f32(_p(img), h, w, _p(out))
    return out


def image_model(img: np.ndarray):
    h, w = img.shape
    img = np.ascontiguousarray(img)
    item = 1 if img.dtype == np.uint8 else 4
    if item == 4:
        img = img.astype(np.float32)
    a0 = np.empty((h, w), np.float32)
    grad = np.empty((h, w, 2), np.float32)
    lib().or_image_model(img.ctypes.data_as(ctypes.c_void_p), item, h, w, _p(a0), _p(grad))
    return a0, grad


def propagate(flow: np.ndarray, n: int, border: int = 3) -> np.ndarray:
    h, w, _ = flow.shape
    flow = np.ascontiguousarray(flow, np.float32)
    out = np.empty_like(flow)
    lib().or_propagate(_p(flow), h, w, n, border, _p(out))
    return out


def propagate_payload(flow, scalar, vector, n: int, border: int = 3):
    h, w, _ = flow.shape
    flow = np.ascontiguousarray(flow, np.float32)
    scalar = np.ascontiguousarray(scalar, np.float32)
    vector = np.ascontiguousarray(vector, np.float32)
    of, os_, ov = np.empty_like(flow), np.empty_like(scalar), np.empty_like(vector)
    lib().or_propagate_payload(_p(flow), _p(scalar), _p(vector), h, w, n, border, _p(of), _p(os_), _p(ov))
    return of, os_, ov


def update(a0, grad, a0old, flow, gamma: float, maxflow: float):
    h, w = a0.shape
    args = [np.ascontiguousarray(x, np.float32) for x in (a0, grad, a0old, flow)]
    of = np.empty((h, w, 2), np.float32)
    oi = np.empty((h, w), np.float32)
    lib().or_update(*[_p(x) for x in args], h, w, gamma, maxflow, _p(of), _p(oi))
    return of, oi


def delta_update(a0, grad, a0old, delta, coarse, gamma: float, maxflow: float):
    h, w = a0.shape
    hc, wc, _ = coarse.shape
    args = [np.ascontiguousarray(x, np.float32) for x in (a0, grad, a0old, delta, coarse)]
    of = np.empty((h, w, 2), np.float32)
    od = np.empty((h, w, 2), np.float32)
    oi = np.empty((h, w), np.float32)
    lib().or_delta_update(*[_p(x) for x in args], hc, wc, h, w, gamma, maxflow, _p(of), _p(od), _p(oi))
    return of, od, oi


def smooth(flow: np.ndarray, s: int) -> np.ndarray:
    h, w, _ = flow.shape
    flow = np.ascontiguousarray(flow, np.float32)
    out = np.empty_like(flow)
    lib().or_smooth(_p(flow), h, w, s, _p(out))
    return out


def camera_perspective(focal: float, h: int, w: int, sensor_h: float, sensor_w: float) -> np.ndarray:
    """[alphaX, alphaY, centerX, centerY] (createPerspectiveCamera, camera.cu:15-31)."""
    cam = np.zeros(4, np.float32)
    lib().or_camera_perspective(focal, h, w, sensor_h, sensor_w, _p(cam))
    return cam


def rotational_flow(cam: np.ndarray, wx: float, wy: float, wz: float, h: int, w: int) -> np.ndarray:
    cam = np.ascontiguousarray(cam, np.float32)
    out = np.zeros((h, w, 2), np.float32)
    lib().or_rotational_flow(_p(cam), wx, wy, wz, h, w, _p(out))
    return out


def lax_wendroff(flow: np.ndarray, image: np.ndarray, iterations: int) -> np.ndarray:
    """image (H, W) or (H, W, 4) float32 propagated by flow (H, W, 2)."""
    flow = np.ascontiguousarray(flow, np.float32)
    image = np.ascontiguousarray(image, np.float32)
    h, w = image.shape[:2]
    d = 1 if image.ndim == 2 else image.shape[2]
    out = np.zeros_like(image)
    lib().or_lax_wendroff(_p(flow), _p(image), d, h, w, iterations, _p(out))
    return out


def upmap_index(x: int, w: int, wc: int) -> int:
    return lib().or_upmap_index(x, w, wc)


class Filter:
    """Oracle filter mirroring FlowFilter / PyramidalFlowFilter of the reference."""

    def __init__(self, handle, height: int, width: int, item: int = 1):
        if not handle:
            raise ValueError("oracle filter creation failed")
        self._h = handle
        self.height = height
        self.width = width
        self.item = item

    @classmethod
    def flowfilter(cls, height, width, smooth_iterations=1, maxflow=1.0, gamma=1.0):
        return cls(lib().or_flowfilter_create(height, width, smooth_iterations, maxflow, gamma), height, width)

    @classmethod
    def flowfilter_on(cls, height, width, item_size):
        return cls(lib().or_flowfilter_create_on(height, width, item_size), height, width, item_size)

    @classmethod
    def pyramidal(cls, height, width, levels):
        return cls(lib().or_pyramidal_create(height, width, levels), height, width)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().or_filter_destroy(self._h)
            self._h = None

    @property
    def levels(self) -> int:
        return lib().or_filter_levels(self._h)

    def set_gamma(self, level: int, g: float) -> None:
        if lib().or_filter_set_gamma(self._h, level, g) != 0:
            raise ValueError("bad gamma/level")

    def set_gammas(self, gs) -> None:
        for lv, g in enumerate(gs):
            self.set_gamma(lv, g)

    def set_max_flow(self, m: float) -> None:
        lib().or_filter_set_max_flow(self._h, m)

    def set_smooth_iterations(self, level: int, n: int) -> None:
        if lib().or_filter_set_smooth_iterations(self._h, level, n) != 0:
            raise ValueError("bad smooth iterations/level")

    def set_smooths(self, ss) -> None:
        for lv, s in enumerate(ss):
            self.set_smooth_iterations(lv, s)

    def set_propagation_border(self, b: int) -> None:
        lib().or_filter_set_propagation_border(self._h, b)

    def propagation_iterations(self, level: int) -> int:
        return lib().or_filter_get_propagation_iterations(self._h, level)

    def gamma(self, level: int) -> float:
        return lib().or_filter_get_gamma(self._h, level)

    def load(self, img: np.ndarray) -> None:
        img = np.ascontiguousarray(img)
        assert img.shape == (self.height, self.width)
        want = np.uint8 if self.item == 1 else np.float32
        img = img.astype(want, copy=False)
        self._keep = img
        lib().or_filter_load(self._h, img.ctypes.data_as(ctypes.c_void_p))

    def compute(self) -> None:
        lib().or_filter_compute(self._h)

    def flow(self) -> np.ndarray:
        out = np.empty((self.height, self.width, 2), np.float32)
        lib().or_filter_download_flow(self._h, _p(out))
        return out

    def get_flow(self) -> np.ndarray:
        out = np.empty((self.height, self.width, 2), np.float32)
        lib().or_filter_get_flow(self._h, _p(out))
        return out

    def image(self) -> np.ndarray:
        out = np.empty((self.height, self.width), np.float32)
        lib().or_filter_download_image(self._h, _p(out))
        return out

    def level_shape(self, level: int):
        h, w = ctypes.c_int(), ctypes.c_int()
        lib().or_filter_level_shape(self._h, level, ctypes.byref(h), ctypes.byref(w))
        return h.value, w.value

    def level_state(self, level: int, which: int) -> np.ndarray | None:
        n = lib().or_filter_level_state(self._h, level, which, None)
        if n == 0:
            return None
        out = np.empty(n, np.float32)
        lib().or_filter_level_state(self._h, level, which, _p(out))
        h, w = self.level_shape(level)
        return out.reshape(h, w, -1) if n == 2 * h * w else out.reshape(h, w)


def run_case(case: dict, frames: np.ndarray, dump=None):
    """Run a parity case (dict as in make_reference_fixtures.CASES) over ``frames``;
    returns the smoothed level-0 flow at the dumped frame indices."""
    t, h, w = frames.shape
    if case["levels"] == 0:
        f = Filter.flowfilter(h, w, case["smooth"][0], case["maxflow"], case["gamma"][0])
    else:
        f = Filter.pyramidal(h, w, case["levels"])
        f.set_gammas(case["gamma"])
        f.set_smooths(case["smooth"])
        f.set_max_flow(case["maxflow"])
    dump = case["dump"] if dump is None else dump
    out = []
    for i in range(t):
        f.load(frames[i])
        f.compute()
        if i in dump:
            out.append(f.flow())
    return np.stack(out) if out else np.zeros((0, h, w, 2), np.float32)
