"""visar-b200: VISAR's imgproc stencil-and-warp path on NVIDIA B200.

Python binding of the C ABI in include/visar.h (libvisar_b200.so, built
in-tree by visar_b200.build). The functions mirror VISAR's ctypes test
binding (tests/py/visar_ctypes.py in VISAR): same names, argument order and
OpenCV constant numbering, NumPy arrays in OpenCV layout (H x W or
H x W x C). CUDA torch tensors of the same layout are accepted too and are
processed in place on the device (zero copy).

There is no CPU fallback: importing this module fails if the CUDA library
is missing, and calls fail (VisarError) when no CUDA device is present.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("VISAR_B200_LIB", os.path.join(_HERE, "libvisar_b200.so"))

_DEPTH = {np.uint8: 0, np.int8: 1, np.uint16: 2, np.int16: 3, np.int32: 4, np.float32: 5, np.float64: 6, np.float16: 7}
_DTYPE = {v: k for k, v in _DEPTH.items()}

# OpenCV constants used by the path.
INTER_NEAREST, INTER_LINEAR, INTER_CUBIC, INTER_AREA, INTER_LANCZOS4 = 0, 1, 2, 3, 4
BORDER_CONSTANT, BORDER_REPLICATE, BORDER_REFLECT, BORDER_WRAP, BORDER_REFLECT_101 = 0, 1, 2, 3, 4
THRESH_BINARY, THRESH_BINARY_INV, THRESH_TRUNC, THRESH_TOZERO, THRESH_TOZERO_INV = 0, 1, 2, 3, 4
THRESH_OTSU, THRESH_TRIANGLE = 8, 16
MORPH_ERODE, MORPH_DILATE, MORPH_OPEN, MORPH_CLOSE, MORPH_GRADIENT, MORPH_TOPHAT, MORPH_BLACKHAT = range(7)
MORPH_RECT, MORPH_CROSS, MORPH_ELLIPSE = 0, 1, 2
COLOR_BGR2GRAY, COLOR_RGB2GRAY, COLOR_BGRA2GRAY = 6, 7, 10


class Image(ctypes.Structure):
    """visar_image (include/visar.h): stride in bytes."""
    _fields_ = [
        ("width", ctypes.c_uint32),
        ("height", ctypes.c_uint32),
        ("channels", ctypes.c_uint32),
        ("depth", ctypes.c_uint32),
        ("stride", ctypes.c_size_t),
        ("data", ctypes.c_void_p),
    ]


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"visar_b200: CUDA library not built ({LIB_PATH}); run `python visar_b200/build.py`")
    lib = ctypes.CDLL(LIB_PATH)
    lib.visar_version.restype = ctypes.c_char_p
    lib.visar_build_info.restype = ctypes.c_char_p
    lib.visar_last_error.restype = ctypes.c_char_p
    lib.visar_cuda_launch_count.restype = ctypes.c_uint64
    lib.visar_cuda_set_stream.argtypes = [ctypes.c_void_p]
    dp = ctypes.POINTER(ctypes.c_double)
    lib.visar_undistort.argtypes = [ctypes.c_void_p, ctypes.c_void_p, dp, dp, ctypes.c_size_t, dp]
    lib.visar_init_undistort_rectify_map.argtypes = [dp, dp, ctypes.c_size_t, dp, dp, ctypes.c_void_p, ctypes.c_void_p]
    lib.visar_remap.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double]
    lib.visar_connected_components.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int32),
                                               ctypes.POINTER(ctypes.c_double), ctypes.c_size_t,
                                               ctypes.POINTER(ctypes.c_size_t)]
    lib.visar_background_create.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
    lib.visar_background_apply.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
    lib.visar_background_free.argtypes = [ctypes.c_void_p]
    lib.visar_background_free.restype = None
    return lib


lib = _load()


class VisarError(RuntimeError):
    def __init__(self, status, name):
        super().__init__(f"{status}: {name}")
        self.status = status
        self.name = name


def _check(rc):
    if rc != 0:
        raise VisarError(rc, lib.visar_last_error().decode())


def _is_torch(a):
    return type(a).__module__.startswith("torch")


_TORCH_DEPTH = None


def _torch_depth(t):
    global _TORCH_DEPTH
    if _TORCH_DEPTH is None:
        import torch
        _TORCH_DEPTH = {torch.uint8: 0, torch.int8: 1, torch.uint16: 2, torch.int16: 3, torch.int32: 4,
                        torch.float32: 5, torch.float64: 6, torch.float16: 7}
    return _TORCH_DEPTH[t.dtype]


def desc(a):
    """visar_image describing a NumPy array or CUDA tensor (rows may be strided; pixels packed)."""
    if a.ndim == 2:
        h, w = a.shape
        c = 1
    elif a.ndim == 3:
        h, w, c = a.shape
    else:
        raise ValueError("expected 2-D or 3-D array")
    if _is_torch(a):
        es = a.element_size()
        st = a.stride()
        if st[1] != c or (a.ndim == 3 and st[2] != 1):
            raise ValueError("pixels must be packed")
        return Image(w, h, c, _torch_depth(a), st[0] * es, a.data_ptr())
    t = a.dtype.type
    if t not in _DEPTH:
        raise ValueError(f"unsupported dtype {a.dtype}")
    if a.strides[-1] != a.itemsize or (a.ndim == 3 and a.strides[1] != a.itemsize * c):
        raise ValueError("pixels must be packed")
    return Image(w, h, c, _DEPTH[t], a.strides[0], a.ctypes.data)


def _shape(a, w=None, h=None, c=None):
    H, W = a.shape[:2]
    C = a.shape[2] if a.ndim == 3 else 1
    w = W if w is None else w
    h = H if h is None else h
    c = C if c is None else c
    return (h, w) if c == 1 else (h, w, c)


def _out(like, shape, dtype=None):
    if _is_torch(like):
        import torch
        return torch.empty(shape, dtype=like.dtype if dtype is None else dtype, device=like.device)
    return np.empty(shape, dtype=like.dtype if dtype is None else dtype)


def version():
    return lib.visar_version().decode()


def build_info():
    return lib.visar_build_info().decode()


def set_num_threads(n):
    lib.visar_set_num_threads(n)


def launch_count():
    """CUDA kernels launched by the library since it was loaded."""
    return int(lib.visar_cuda_launch_count())


def set_stream(stream):
    """Run this thread's calls on `stream` (a torch.cuda.Stream, a raw handle, or None)."""
    h = getattr(stream, "cuda_stream", stream)
    _check(lib.visar_cuda_set_stream(ctypes.c_void_p(h or 0)))


def set_async(flag):
    _check(lib.visar_cuda_set_async(int(bool(flag))))


_COLOR_CN = {
    0: (3, 4), 1: (4, 3), 2: (3, 4), 3: (4, 3), 4: (3, 3), 5: (4, 4), 6: (3, 1), 7: (3, 1),
    8: (1, 3), 9: (1, 4), 10: (4, 1), 11: (4, 1), 36: (3, 3), 37: (3, 3), 38: (3, 3), 39: (3, 3),
    40: (3, 3), 41: (3, 3), 54: (3, 3), 55: (3, 3),
}


def cvt_color(a, code, dst=None):
    dst = _out(a, _shape(a, c=_COLOR_CN.get(code, (0, 1))[1])) if dst is None else dst
    _check(lib.visar_cvt_color(ctypes.byref(desc(a)), ctypes.byref(desc(dst)), code))
    return dst


def resize(a, size, interpolation=1, dst=None):
    dst = _out(a, _shape(a, w=size[0], h=size[1])) if dst is None else dst
    _check(lib.visar_resize(ctypes.byref(desc(a)), ctypes.byref(desc(dst)), interpolation))
    return dst


def resize_linear_u8_noalloc(a, dst):
    """INTER_LINEAR resize of a uint8 CUDA tensor into `dst` (a CUDA tensor
    the caller owns) through visar_resize_linear_u8_noalloc: no device memory
    is allocated by the call; destination sides up to 16384."""
    _check(lib.visar_resize_linear_u8_noalloc(ctypes.byref(desc(a)), ctypes.byref(desc(dst))))
    return dst


def gray_downsample(a, k, dst=None):
    """visar_gray_downsample: BT.601 gray of a BGR / BGRA u8 image shrunk by the
    integer factor k (1-16) with box averaging, in one pass."""
    if dst is None:
        dst = _out(a, (a.shape[0] // k if k > 0 else 0, a.shape[1] // k if k > 0 else 0))
    _check(lib.visar_gray_downsample(ctypes.byref(desc(a)), ctypes.byref(desc(dst)), int(k)))
    return dst


def pyr_down(a, border=4, dst=None):
    """visar_pyr_down: 5x5 Gaussian, then every other row and column; dst is ((w+1)//2, (h+1)//2)."""
    if dst is None:
        dst = _out(a, _shape(a, (a.shape[1] + 1) // 2, (a.shape[0] + 1) // 2))
    _check(lib.visar_pyr_down(ctypes.byref(desc(a)), ctypes.byref(desc(dst)), int(border)))
    return dst


def pyr_up(a, border=4, dst=None):
    """visar_pyr_up: upsample by 2 and blur with the 5x5 Gaussian times 4; dst is (2w, 2h)."""
    if dst is None:
        dst = _out(a, _shape(a, 2 * a.shape[1], 2 * a.shape[0]))
    _check(lib.visar_pyr_up(ctypes.byref(desc(a)), ctypes.byref(desc(dst)), int(border)))
    return dst


def _dptr(v, n=None):
    """(pointer, length) of a float64 vector, or (None, 0)."""
    if v is None:
        return None, 0
    a = np.ascontiguousarray(np.asarray(v, np.float64).ravel())
    if n is not None and a.size != n:
        raise ValueError(f"expected {n} values")
    return a, a.size


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def undistort(a, k, dist=None, new_k=None, dst=None):
    """visar_undistort: 8U images of 1-4 channels; k and new_k 3x3, dist 0/4/5/8 coefficients."""
    dst = _out(a, tuple(a.shape)) if dst is None else dst
    km, _ = _dptr(k, 9)
    dv, nd = _dptr(dist)
    nk, _ = _dptr(new_k, 9)
    _check(lib.visar_undistort(ctypes.byref(desc(a)), ctypes.byref(desc(dst)), _p(km), _p(dv), ctypes.c_size_t(nd), _p(nk)))
    return dst


def init_undistort_rectify_map(k, dist, r, new_k, size, mapx=None, mapy=None, like=None):
    """visar_init_undistort_rectify_map: f32 maps of size (w, h); `like` picks host (NumPy, default) or a CUDA tensor."""
    w, h = size

    def alloc():
        if like is not None and _is_torch(like):
            import torch
            return torch.empty((h, w), dtype=torch.float32, device=like.device)
        return np.empty((h, w), np.float32)

    mapx = alloc() if mapx is None else mapx
    mapy = alloc() if mapy is None else mapy
    km, _ = _dptr(k, 9)
    dv, nd = _dptr(dist)
    rm, _ = _dptr(r, 9)
    nk, _ = _dptr(new_k, 9)
    _check(lib.visar_init_undistort_rectify_map(_p(km), _p(dv), ctypes.c_size_t(nd), _p(rm), _p(nk),
                                                ctypes.byref(desc(mapx)), ctypes.byref(desc(mapy))))
    return mapx, mapy


def remap(a, mapx, mapy, value=0.0, dst=None):
    """visar_remap: 8U 1-4 channels through f32 maps (INTER_LINEAR, constant border `value`)."""
    if dst is None:
        dst = _out(a, _shape(a, mapx.shape[1], mapx.shape[0]))
    _check(lib.visar_remap(ctypes.byref(desc(a)), ctypes.byref(desc(dst)), ctypes.byref(desc(mapx)),
                           ctypes.byref(desc(mapy)), ctypes.c_double(value)))
    return dst


def equalize_hist(a, dst=None):
    """visar_equalize_hist: 8U one channel."""
    dst = _out(a, tuple(a.shape)) if dst is None else dst
    _check(lib.visar_equalize_hist(ctypes.byref(desc(a)), ctypes.byref(desc(dst))))
    return dst


def adaptive_threshold(a, maxval, method, kind, block, delta, dst=None):
    """visar_adaptive_threshold: method 0 MEAN_C / 1 GAUSSIAN_C, kind 0 BINARY / 1 BINARY_INV."""
    dst = _out(a, tuple(a.shape)) if dst is None else dst
    _check(lib.visar_adaptive_threshold(ctypes.byref(desc(a)), ctypes.byref(desc(dst)), ctypes.c_double(maxval),
                                        int(method), int(kind), int(block), ctypes.c_double(delta)))
    return dst


def connected_components(a, connectivity=8, labels=None, max_stats=None):
    """visar_connected_components: (count, labels int32, stats (n x 5 int32), centroids (n x 2 f64))."""
    if labels is None:
        if _is_torch(a):
            import torch
            labels = torch.empty(tuple(a.shape[:2]), dtype=torch.int32, device=a.device)
        else:
            labels = np.empty(tuple(a.shape[:2]), np.int32)
    cap = max_stats if max_stats is not None else int(a.shape[0]) * int(a.shape[1]) + 1
    stats = np.zeros((max(cap, 1), 5), np.int32)
    cents = np.zeros((max(cap, 1), 2), np.float64)
    n = ctypes.c_size_t(0)
    _check(lib.visar_connected_components(ctypes.byref(desc(a)), ctypes.byref(desc(labels)), int(connectivity),
                                          stats.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                          cents.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), cap, ctypes.byref(n)))
    k = min(n.value, cap)
    return n.value, labels, stats[:k], cents[:k]


class Background:
    """visar_background_*: the running-average background model (its state on the device)."""

    def __init__(self, width, height, shift=4):
        h = ctypes.c_void_p()
        _check(lib.visar_background_create(ctypes.c_uint32(width), ctypes.c_uint32(height), int(shift), ctypes.byref(h)))
        self._h = h

    def apply(self, frame, threshold, mask=None):
        mask = _out(frame, tuple(frame.shape)) if mask is None else mask
        _check(lib.visar_background_apply(self._h, ctypes.byref(desc(frame)), ctypes.byref(desc(mask)), int(threshold)))
        return mask

    def close(self):
        if getattr(self, "_h", None) and lib is not None:
            lib.visar_background_free(self._h)
            self._h = None

    def __del__(self):
        self.close()


def gaussian_blur(a, ksize, sigma_x, sigma_y=0, border=4, dst=None):
    dst = _out(a, tuple(a.shape)) if dst is None else dst
    _check(lib.visar_gaussian_blur(ctypes.byref(desc(a)), ctypes.byref(desc(dst)), ksize[0], ksize[1],
                                   ctypes.c_double(sigma_x), ctypes.c_double(sigma_y), border))
    return dst


def box_filter(a, ksize, normalize=True, border=4, dst=None):
    dst = _out(a, tuple(a.shape)) if dst is None else dst
    _check(lib.visar_box_filter(ctypes.byref(desc(a)), ctypes.byref(desc(dst)), ksize[0], ksize[1], int(normalize), border))
    return dst


def sobel(a, ddepth, dx, dy, ksize=3, scale=1.0, border=4, dst=None):
    if dst is None:
        if _is_torch(a):
            import torch
            td = {np.int16: torch.int16, np.float32: torch.float32}[np.dtype(ddepth).type]
            dst = torch.empty(tuple(a.shape), dtype=td, device=a.device)
        else:
            dst = np.empty(a.shape, dtype=ddepth)
    _check(lib.visar_sobel(ctypes.byref(desc(a)), ctypes.byref(desc(dst)), dx, dy, ksize, ctypes.c_double(scale), border))
    return dst


def sep_filter_2d(a, ddepth, kx, ky, border=4, dst=None):
    """sepFilter2D (VISAR's Zig API; an added C entry point here)."""
    kxa = np.ascontiguousarray(kx, np.float32).ravel()
    kya = np.ascontiguousarray(ky, np.float32).ravel()
    if dst is None:
        if _is_torch(a):
            import torch
            td = {np.uint8: torch.uint8, np.uint16: torch.uint16, np.int16: torch.int16,
                  np.float32: torch.float32}[np.dtype(ddepth).type]
            dst = torch.empty(tuple(a.shape), dtype=td, device=a.device)
        else:
            dst = np.empty(a.shape, dtype=ddepth)
    fp = ctypes.POINTER(ctypes.c_float)
    _check(lib.visar_sep_filter_2d(ctypes.byref(desc(a)), ctypes.byref(desc(dst)), kxa.ctypes.data_as(fp), len(kxa),
                                   kya.ctypes.data_as(fp), len(kya), border))
    return dst


def threshold(a, thresh, maxval, kind, dst=None):
    dst = _out(a, tuple(a.shape)) if dst is None else dst
    used = ctypes.c_double(0)
    _check(lib.visar_threshold(ctypes.byref(desc(a)), ctypes.byref(desc(dst)), ctypes.c_double(thresh),
                               ctypes.c_double(maxval), kind, ctypes.byref(used)))
    return used.value, dst


def morphology(a, op, shape, ksize, iterations=1, dst=None):
    dst = _out(a, tuple(a.shape)) if dst is None else dst
    _check(lib.visar_morphology(ctypes.byref(desc(a)), ctypes.byref(desc(dst)), op, shape, ksize[0], ksize[1], iterations))
    return dst


def warp_affine(a, m, size, interpolation=1, border=0, value=0.0, dst=None):
    dst = _out(a, _shape(a, w=size[0], h=size[1])) if dst is None else dst
    arr = (ctypes.c_double * 6)(*np.asarray(m, dtype=np.float64).ravel())
    _check(lib.visar_warp_affine(ctypes.byref(desc(a)), ctypes.byref(desc(dst)), arr, interpolation, border, ctypes.c_double(value)))
    return dst


def warp_perspective(a, m, size, interpolation=1, border=0, value=0.0, dst=None):
    """warpPerspective (VISAR's Zig API; an added C entry point here)."""
    dst = _out(a, _shape(a, w=size[0], h=size[1])) if dst is None else dst
    arr = (ctypes.c_double * 9)(*np.asarray(m, dtype=np.float64).ravel())
    _check(lib.visar_warp_perspective(ctypes.byref(desc(a)), ctypes.byref(desc(dst)), arr, interpolation, border,
                                      ctypes.c_double(value)))
    return dst
