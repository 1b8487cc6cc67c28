"""Python binding of the batched form (include/visar_batch.h).

    plan = Batch(images, [gray(), gaussian((5, 5)), morphology(MORPH_OPEN, MORPH_ELLIPSE, (5, 5)),
                          resize(0.5, 0.5)])
    plan.run()                    # or plan.run_graph()
    out = plan.output(i)          # torch tensor view of image i's result (device)

`images` are CUDA torch tensors (H x W or H x W x C; rows may be padded) or
(height, width, channels, dtype) tuples for plan-owned inputs, which
`plan.input(i)` exposes for filling. Views returned by input() / output()
alias plan memory and stay valid while the plan lives.
"""
import ctypes

import numpy as np

from . import Image, VisarError, _DEPTH, _DTYPE, _check, desc, lib

STAGE_GRAY, STAGE_GAUSSIAN, STAGE_MORPHOLOGY, STAGE_RESIZE, STAGE_THRESHOLD = 1, 2, 3, 4, 5
STAGE_WARP_AFFINE, STAGE_WARP_PERSPECTIVE = 6, 7


class Stage(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int),
        ("i", ctypes.c_int * 5),
        ("d", ctypes.c_double * 10),
        ("per_image", ctypes.POINTER(ctypes.c_double)),
    ]


class BatchInfo(ctypes.Structure):
    _fields_ = [(k, ctypes.c_size_t) for k in
                ("images", "stages", "launches", "fallback_calls", "pool_bytes", "bytes_moved", "pixels_in")]


lib.visar_batch_create.argtypes = [ctypes.POINTER(Image), ctypes.c_size_t, ctypes.POINTER(Stage), ctypes.c_size_t,
                                   ctypes.POINTER(ctypes.c_void_p)]
for _fn in ("visar_batch_input", "visar_batch_output"):
    getattr(lib, _fn).argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(Image)]
lib.visar_batch_stage_output.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_size_t, ctypes.POINTER(Image)]
lib.visar_batch_run.argtypes = [ctypes.c_void_p]
lib.visar_batch_run_graph.argtypes = [ctypes.c_void_p]
lib.visar_batch_get_info.argtypes = [ctypes.c_void_p, ctypes.POINTER(BatchInfo)]
lib.visar_batch_destroy.argtypes = [ctypes.c_void_p]
lib.visar_batch_destroy.restype = None
lib.visar_batch_set_input.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(Image)]
lib.visar_batch_upload.argtypes = [ctypes.c_void_p, ctypes.POINTER(Image), ctypes.c_size_t]
lib.visar_batch_download.argtypes = [ctypes.c_void_p, ctypes.POINTER(Image), ctypes.c_size_t]
lib.visar_batch_profile.argtypes = [ctypes.c_void_p, ctypes.c_int]


class LaunchStat(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 48), ("stage", ctypes.c_int), ("images", ctypes.c_size_t),
                ("tiles", ctypes.c_size_t), ("bytes", ctypes.c_size_t), ("grid", ctypes.c_int), ("ms", ctypes.c_float)]


lib.visar_batch_launch_stat_get.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(LaunchStat)]
lib.visar_tune_load.argtypes = [ctypes.c_char_p]
lib.visar_tune_set.argtypes = [ctypes.c_char_p, ctypes.c_int]
lib.visar_tune_get.argtypes = [ctypes.c_char_p, ctypes.c_int]


def _stage(kind, i=(), d=(), per_image=None):
    s = Stage()
    s.kind = kind
    for k, v in enumerate(i):
        s.i[k] = int(v)
    for k, v in enumerate(d):
        s.d[k] = float(v)
    keep = None
    if per_image is not None:
        keep = np.ascontiguousarray(per_image, dtype=np.float64)
        s.per_image = keep.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    return s, keep


def gray():
    return _stage(STAGE_GRAY)


def gaussian(ksize, sigma_x=0.0, sigma_y=0.0, border=4):
    return _stage(STAGE_GAUSSIAN, (ksize[0], ksize[1], border), (sigma_x, sigma_y))


def morphology(op, shape, ksize, iterations=1):
    return _stage(STAGE_MORPHOLOGY, (op, shape, ksize[0], ksize[1], iterations))


def resize(fx, fy, interpolation=1):
    return _stage(STAGE_RESIZE, (interpolation,), (fx, fy))


def threshold(thresh, maxval, type_):
    return _stage(STAGE_THRESHOLD, (type_,), (thresh, maxval))


def warp_affine(m=None, interpolation=1, border=0, value=0.0, per_image=None):
    d = list(np.asarray(m, dtype=np.float64).reshape(6)) if m is not None else [0.0] * 6
    return _stage(STAGE_WARP_AFFINE, (interpolation, border), d + [value], per_image)


def warp_perspective(m=None, interpolation=1, border=0, value=0.0, per_image=None):
    d = list(np.asarray(m, dtype=np.float64).reshape(9)) if m is not None else [0.0] * 9
    return _stage(STAGE_WARP_PERSPECTIVE, (interpolation, border), d + [value], per_image)


_TYPESTR = {0: "|u1", 2: "<u2", 3: "<i2", 5: "<f4"}


class _DevView:
    """__cuda_array_interface__ over a visar_image in device memory."""

    def __init__(self, img, owner):
        es = np.dtype(_DTYPE[img.depth]).itemsize
        c = img.channels
        shape = (img.height, img.width) if c == 1 else (img.height, img.width, c)
        strides = (img.stride, es) if c == 1 else (img.stride, es * c, es)
        self.owner = owner
        self.__cuda_array_interface__ = {"shape": shape, "typestr": _TYPESTR[img.depth], "strides": strides,
                                         "data": (img.data, False), "version": 3}


def _as_tensor(img, owner):
    import torch
    return torch.as_tensor(_DevView(img, owner), device="cuda")


class Batch:
    """A plan over images and stages (visar_batch_create)."""

    def __init__(self, images, stages):
        descs = []
        self._keep = []
        for im in images:
            if isinstance(im, tuple):
                h, w, c, dt = im
                descs.append(Image(w, h, c, _DEPTH[np.dtype(dt).type], 0, None))
            else:
                descs.append(desc(im))
                self._keep.append(im)
        arr = (Image * max(1, len(descs)))(*descs)
        sts = []
        for s in stages:
            st, keep = s
            sts.append(st)
            self._keep.append(keep)
        sarr = (Stage * max(1, len(sts)))(*sts)
        h = ctypes.c_void_p()
        _check(lib.visar_batch_create(arr, len(descs), sarr, len(sts), ctypes.byref(h)))
        self._h = h
        self.n = len(descs)
        self.nstages = len(sts)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and lib is not None:  # (module globals are gone at interpreter exit)
            lib.visar_batch_destroy(h)
            self._h = None

    def run(self):
        _check(lib.visar_batch_run(self._h))

    def run_graph(self):
        _check(lib.visar_batch_run_graph(self._h))

    def info(self):
        inf = BatchInfo()
        _check(lib.visar_batch_get_info(self._h, ctypes.byref(inf)))
        return {k: getattr(inf, k) for k, _ in BatchInfo._fields_}

    def input(self, i):
        img = Image()
        _check(lib.visar_batch_input(self._h, i, ctypes.byref(img)))
        return _as_tensor(img, self)

    def output(self, i):
        img = Image()
        _check(lib.visar_batch_output(self._h, i, ctypes.byref(img)))
        return _as_tensor(img, self)

    def set_input(self, i, x):
        """Rebinds input i to device tensor x (same shape, dtype, row stride and alignment)."""
        self._keep.append(x)
        _check(lib.visar_batch_set_input(self._h, i, ctypes.byref(desc(x))))

    def upload(self, hosts):
        """Host -> device copy of every input from NumPy arrays (pinned for asynchrony)."""
        arr = (Image * len(hosts))(*[desc(h) for h in hosts])
        _check(lib.visar_batch_upload(self._h, arr, len(hosts)))

    def download(self, hosts):
        """Device -> host copy of every final output into NumPy arrays."""
        arr = (Image * len(hosts))(*[desc(h) for h in hosts])
        _check(lib.visar_batch_download(self._h, arr, len(hosts)))

    def profile(self, enable=True):
        _check(lib.visar_batch_profile(self._h, int(bool(enable))))

    def launch_stats(self):
        out = []
        for i in range(self.info()["launches"]):
            st = LaunchStat()
            _check(lib.visar_batch_launch_stat_get(self._h, i, ctypes.byref(st)))
            out.append({"name": st.name.decode(), "stage": st.stage, "images": st.images, "tiles": st.tiles,
                        "bytes": st.bytes, "grid": st.grid, "ms": st.ms})
        return out

    def stage_output(self, stage, i):
        img = Image()
        _check(lib.visar_batch_stage_output(self._h, stage, i, ctypes.byref(img)))
        return _as_tensor(img, self)


def tune_load(path=None):
    _check(lib.visar_tune_load(None if path is None else str(path).encode()))


def tune_set(key, value):
    _check(lib.visar_tune_set(key.encode(), int(value)))


def tune_get(key, fallback=-1):
    return int(lib.visar_tune_get(key.encode(), int(fallback)))


__all__ = ["Batch", "VisarError", "gray", "gaussian", "morphology", "resize", "threshold", "warp_affine",
           "warp_perspective", "tune_load", "tune_set", "tune_get"]
