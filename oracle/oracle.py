"""ORACLE -- test infrastructure only (tests/, the smoke check and bench.py's
CPU-baseline leg). ctypes binding of liboracle.so, the CPU restatement of
VISAR's imgproc path in visar_oracle.cpp. Same call shapes as the product
binding (visar_b200) so parity tests compare like with like.

`build()` compiles liboracle.so with oracle/Makefile if it is missing.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

_DEPTH = {np.uint8: 0, np.int8: 1, np.uint16: 2, np.int16: 3, np.int32: 4, np.float32: 5, np.float64: 6, np.float16: 7}


def build():
    src = os.path.join(HERE, "visar_oracle.cpp")
    if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


class Image(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_uint32),
        ("height", ctypes.c_uint32),
        ("channels", ctypes.c_uint32),
        ("depth", ctypes.c_uint32),
        ("stride", ctypes.c_size_t),
        ("data", ctypes.c_void_p),
    ]


build()
lib = ctypes.CDLL(LIB_PATH)
lib.oracle_last_error.restype = ctypes.c_char_p
lib.oracle_border_map.restype = ctypes.c_longlong
lib.oracle_border_map.argtypes = [ctypes.c_longlong, ctypes.c_longlong, ctypes.c_int]
lib.oracle_cv_exp.restype = ctypes.c_double
lib.oracle_cv_exp.argtypes = [ctypes.c_double]
for _n in ("oracle_sat_u8_f32", "oracle_sat_i16_f32", "oracle_satv_u8_f32", "oracle_satv_i16_f32"):
    getattr(lib, _n).argtypes = [ctypes.c_float]


class OracleError(RuntimeError):
    def __init__(self, status, name):
        super().__init__(f"{status}: {name}")
        self.status = status
        self.name = name


def _check(rc):
    if rc != 0:
        raise OracleError(rc, lib.oracle_last_error().decode())


def desc(a):
    if a.ndim == 2:
        h, w = a.shape
        c = 1
    else:
        h, w, c = a.shape
    if a.strides[-1] != a.itemsize or (a.ndim == 3 and a.strides[1] != a.itemsize * c):
        raise ValueError("pixels must be packed")
    return Image(w, h, c, _DEPTH[a.dtype.type], a.strides[0], a.ctypes.data)


def _shape(a, w=None, h=None, c=None):
    H, W = a.shape[:2]
    C = a.shape[2] if a.ndim == 3 else 1
    w = W if w is None else w
    h = H if h is None else h
    c = C if c is None else c
    return (h, w) if c == 1 else (h, w, c)


def set_num_threads(n):
    lib.oracle_set_num_threads(int(n))


def get_num_threads():
    return int(lib.oracle_get_num_threads())


_COLOR_CN = {
    0: (3, 4), 1: (4, 3), 2: (3, 4), 3: (4, 3), 4: (3, 3), 5: (4, 4), 6: (3, 1), 7: (3, 1),
    8: (1, 3), 9: (1, 4), 10: (4, 1), 11: (4, 1), 36: (3, 3), 37: (3, 3), 38: (3, 3), 39: (3, 3),
    40: (3, 3), 41: (3, 3), 54: (3, 3), 55: (3, 3),
}


def cvt_color(a, code, dst=None):
    dst = np.empty(_shape(a, c=_COLOR_CN.get(code, (0, 1))[1]), a.dtype) if dst is None else dst
    _check(lib.oracle_cvt_color(ctypes.byref(desc(a)), ctypes.byref(desc(dst)), code))
    return dst


def resize(a, size, interpolation=1, dst=None):
    dst = np.empty(_shape(a, w=size[0], h=size[1]), a.dtype) if dst is None else dst
    _check(lib.oracle_resize(ctypes.byref(desc(a)), ctypes.byref(desc(dst)), interpolation))
    return dst


def gaussian_blur(a, ksize, sigma_x, sigma_y=0, border=4, dst=None):
    dst = np.empty_like(a) if dst is None else dst
    _check(lib.oracle_gaussian_blur(ctypes.byref(desc(a)), ctypes.byref(desc(dst)), ksize[0], ksize[1],
                                    ctypes.c_double(sigma_x), ctypes.c_double(sigma_y), border))
    return dst


def box_filter(a, ksize, normalize=True, border=4, dst=None):
    dst = np.empty_like(a) if dst is None else dst
    _check(lib.oracle_box_filter(ctypes.byref(desc(a)), ctypes.byref(desc(dst)), ksize[0], ksize[1], int(normalize), border))
    return dst


def sobel(a, ddepth, dx, dy, ksize=3, scale=1.0, border=4, dst=None):
    dst = np.empty(a.shape, dtype=ddepth) if dst is None else dst
    _check(lib.oracle_sobel(ctypes.byref(desc(a)), ctypes.byref(desc(dst)), dx, dy, ksize, ctypes.c_double(scale), border))
    return dst


def sep_filter_2d(a, ddepth, kx, ky, border=4, dst=None):
    kxa = np.ascontiguousarray(kx, np.float32).ravel()
    kya = np.ascontiguousarray(ky, np.float32).ravel()
    dst = np.empty(a.shape, dtype=ddepth) if dst is None else dst
    fp = ctypes.POINTER(ctypes.c_float)
    _check(lib.oracle_sep_filter_2d(ctypes.byref(desc(a)), ctypes.byref(desc(dst)), kxa.ctypes.data_as(fp), len(kxa),
                                    kya.ctypes.data_as(fp), len(kya), border))
    return dst


def threshold(a, thresh, maxval, kind, dst=None):
    dst = np.empty_like(a) if dst is None else dst
    used = ctypes.c_double(0)
    _check(lib.oracle_threshold(ctypes.byref(desc(a)), ctypes.byref(desc(dst)), ctypes.c_double(thresh),
                                ctypes.c_double(maxval), kind, ctypes.byref(used)))
    return used.value, dst


def resize_generic_u8(a, size, interpolation=1):
    """VISAR's generic u8 kernels (linear: resize.zig:284-423; area:
    areaGeneric), which its resize tests hold the dispatched fast paths to."""
    w, h = size
    dst = np.empty(_shape(a, w, h), np.uint8)
    _check(lib.oracle_resize_generic_u8(ctypes.byref(desc(a)), ctypes.byref(desc(dst)), interpolation))
    return dst


def gray_downsample(a, k, dst=None):
    """grayDownsample (frame.zig:169-335): BGR/BGRA u8 -> (w // k) x (h // k) gray."""
    if dst is None:
        dst = np.empty((a.shape[0] // k if k > 0 else 0, a.shape[1] // k if k > 0 else 0), np.uint8)
    _check(lib.oracle_gray_downsample(ctypes.byref(desc(a)), ctypes.byref(desc(dst)), int(k)))
    return dst


def pyr_down(a, border=4, dst=None):
    if dst is None:
        dst = np.empty(_shape(a, (a.shape[1] + 1) // 2, (a.shape[0] + 1) // 2), a.dtype)
    _check(lib.oracle_pyr_down(ctypes.byref(desc(a)), ctypes.byref(desc(dst)), int(border)))
    return dst


def pyr_up(a, border=4, dst=None):
    if dst is None:
        dst = np.empty(_shape(a, 2 * a.shape[1], 2 * a.shape[0]), a.dtype)
    _check(lib.oracle_pyr_up(ctypes.byref(desc(a)), ctypes.byref(desc(dst)), int(border)))
    return dst


_DP = ctypes.POINTER(ctypes.c_double)
lib.oracle_undistort.argtypes = [ctypes.c_void_p, ctypes.c_void_p, _DP, _DP, ctypes.c_size_t, _DP]
lib.oracle_init_undistort_rectify_map.argtypes = [_DP, _DP, ctypes.c_size_t, _DP, _DP, ctypes.c_void_p, ctypes.c_void_p]
lib.oracle_remap.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double]


def _dv(v, n=None):
    if v is None:
        return None, 0
    a = np.ascontiguousarray(np.asarray(v, np.float64).ravel())
    if n is not None and a.size != n:
        raise ValueError(f"expected {n} values")
    return a, a.size


def _pp(a):
    return None if a is None else a.ctypes.data_as(_DP)


def undistort(a, k, dist=None, new_k=None, dst=None):
    dst = np.empty_like(a) if dst is None else dst
    km, _ = _dv(k, 9)
    dv, nd = _dv(dist)
    nk, _ = _dv(new_k, 9)
    _check(lib.oracle_undistort(ctypes.byref(desc(a)), ctypes.byref(desc(dst)), _pp(km), _pp(dv), nd, _pp(nk)))
    return dst


def init_undistort_rectify_map(k, dist, r, new_k, size):
    w, h = size
    mx = np.empty((h, w), np.float32)
    my = np.empty((h, w), np.float32)
    km, _ = _dv(k, 9)
    dv, nd = _dv(dist)
    rm, _ = _dv(r, 9)
    nk, _ = _dv(new_k, 9)
    _check(lib.oracle_init_undistort_rectify_map(_pp(km), _pp(dv), nd, _pp(rm), _pp(nk), ctypes.byref(desc(mx)),
                                                 ctypes.byref(desc(my))))
    return mx, my


def remap(a, mapx, mapy, value=0.0, dst=None):
    dst = np.empty(_shape(a, mapx.shape[1], mapx.shape[0]), np.uint8) if dst is None else dst
    _check(lib.oracle_remap(ctypes.byref(desc(a)), ctypes.byref(desc(dst)), ctypes.byref(desc(mapx)), ctypes.byref(desc(mapy)),
                            ctypes.c_double(value)))
    return dst


def equalize_hist(a, dst=None):
    dst = np.empty_like(a) if dst is None else dst
    _check(lib.oracle_equalize_hist(ctypes.byref(desc(a)), ctypes.byref(desc(dst))))
    return dst


lib.oracle_adaptive_threshold.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_double]


def adaptive_threshold(a, maxval, method, kind, block, delta, dst=None):
    dst = np.empty_like(a) if dst is None else dst
    _check(lib.oracle_adaptive_threshold(ctypes.byref(desc(a)), ctypes.byref(desc(dst)), maxval, method, kind, block, delta))
    return dst


class Background:
    """The running-average background model (track.zig:17-82) on the host."""

    def __init__(self, w, h, shift):
        self.model = np.zeros((h, w), np.uint16)
        self.primed = ctypes.c_int(0)
        self.shift = shift

    def apply(self, frame, threshold, mask=None):
        mask = np.empty_like(frame) if mask is None else mask
        _check(lib.oracle_background_apply(self.model.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)),
                                           ctypes.byref(self.primed), self.shift, ctypes.byref(desc(frame)),
                                           ctypes.byref(desc(mask)), int(threshold)))
        return mask


lib.oracle_connected_components.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                            ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_double),
                                            ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]


def connected_components(a, connectivity=8, max_stats=None):
    """(count, labels int32, stats (count x 5), centroids (count x 2))."""
    labels = np.empty(a.shape[:2], np.int32)
    cap = max_stats if max_stats is not None else a.shape[0] * a.shape[1] + 1
    stats = np.zeros((cap, 5), np.int32)
    cents = np.zeros((cap, 2), np.float64)
    n = ctypes.c_size_t(0)
    _check(lib.oracle_connected_components(ctypes.byref(desc(a)), ctypes.byref(desc(labels)), int(connectivity),
                                           stats.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                           cents.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), cap, ctypes.byref(n)))
    k = min(n.value, cap)
    return n.value, labels, stats[:k], cents[:k]


def morphology(a, op, shape, ksize, iterations=1, dst=None):
    dst = np.empty_like(a) if dst is None else dst
    _check(lib.oracle_morphology(ctypes.byref(desc(a)), ctypes.byref(desc(dst)), op, shape, ksize[0], ksize[1], iterations))
    return dst


def warp_affine(a, m, size, interpolation=1, border=0, value=0.0, dst=None):
    dst = np.empty(_shape(a, w=size[0], h=size[1]), a.dtype) if dst is None else dst
    arr = (ctypes.c_double * 6)(*np.asarray(m, dtype=np.float64).ravel())
    _check(lib.oracle_warp_affine(ctypes.byref(desc(a)), ctypes.byref(desc(dst)), arr, interpolation, border, ctypes.c_double(value)))
    return dst


def warp_perspective(a, m, size, interpolation=1, border=0, value=0.0, dst=None):
    dst = np.empty(_shape(a, w=size[0], h=size[1]), a.dtype) if dst is None else dst
    arr = (ctypes.c_double * 9)(*np.asarray(m, dtype=np.float64).ravel())
    _check(lib.oracle_warp_perspective(ctypes.byref(desc(a)), ctypes.byref(desc(dst)), arr, interpolation, border,
                                       ctypes.c_double(value)))
    return dst


# ---------------------------------------------------------- known answers

def gaussian_kernel(n, sigma):
    out = np.zeros(n, np.float64)
    lib.oracle_gaussian_kernel(out.ctypes.data_as(ctypes.c_void_p), n, ctypes.c_double(sigma))
    return out


def gaussian_kernel_fixed(n, sigma, bits):
    if bits == 8:
        out = np.zeros(n, np.uint16)
        lib.oracle_gaussian_kernel_fixed_u16(out.ctypes.data_as(ctypes.c_void_p), n, ctypes.c_double(sigma))
    else:
        out = np.zeros(n, np.uint32)
        lib.oracle_gaussian_kernel_fixed_u32(out.ctypes.data_as(ctypes.c_void_p), n, ctypes.c_double(sigma))
    return out


def deriv_kernel(n, order, ksize):
    out = np.zeros(n, np.int32)
    rc = lib.oracle_deriv_kernel(out.ctypes.data_as(ctypes.c_void_p), n, order, ksize)
    return out if rc == 0 else None


def border_map(p, n, border):
    r = lib.oracle_border_map(p, n, border)
    return None if r < 0 else int(r)


def sat_u8(x):
    return lib.oracle_sat_u8_f32(ctypes.c_float(x))


def sat_i16(x):
    return lib.oracle_sat_i16_f32(ctypes.c_float(x))


def satv_u8(x):
    return lib.oracle_satv_u8_f32(ctypes.c_float(x))


def satv_i16(x):
    return lib.oracle_satv_i16_f32(ctypes.c_float(x))


def cv_exp(x):
    return lib.oracle_cv_exp(x)


def structuring_element(shape, w, h):
    out = np.zeros((h, w), np.uint8)
    lib.oracle_structuring_element(shape, w, h, out.ctypes.data_as(ctypes.c_void_p))
    return out
