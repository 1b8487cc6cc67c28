import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests through the C ABI")


def natural(h, w, c=3, dtype=np.uint8, seed=1234):
    """A photo-like test image: gradients, sines, N(0, 8) noise, a bright
    rectangle and a dark disc (the shape of VISAR's difftest generator,
    tests/py/test_core_vs_opencv.py:25-44, with its own seed)."""
    rng = np.random.default_rng(seed + 7919 * h + 104729 * w + c)
    y, x = np.mgrid[0:h, 0:w].astype(np.float32)
    base = 127 + 60 * np.sin(x / 37.0) * np.cos(y / 23.0) + 40 * (x / max(w, 1) - 0.5)
    planes = [base + 30 * np.sin((x + y * (k + 1)) / 11.0) + rng.normal(0, 8, (h, w)) for k in range(c)]
    img = np.stack(planes, axis=-1) if c > 1 else planes[0]
    img = np.clip(img, 0, 255).astype(np.uint8)
    y0, y1, x0, x1 = h // 5, h // 2, w // 5, w // 2
    img[y0:y1 + 1, x0:x1 + 1] = 255
    cy, cx, r = 2 * h // 3, 2 * w // 3, max(1, min(h, w) // 6)
    yy, xx = np.mgrid[0:h, 0:w]
    img[(yy - cy) ** 2 + (xx - cx) ** 2 <= r * r] = 0
    if dtype == np.uint16:
        return img.astype(np.uint16) * 257
    if dtype == np.float32:
        return img.astype(np.float32) / 255.0
    if dtype == np.int16:
        return img.astype(np.int16) - 128
    return img


def assert_same(ours, ref, dtype_tol=None, what=""):
    """Bit-exact for integer samples; |a-b| <= tol*max(1,|b|) for f32 (tol default 1e-5)."""
    ours = np.asarray(ours)
    ref = np.asarray(ref)
    assert ours.shape == ref.shape, f"{what}: shape {ours.shape} vs {ref.shape}"
    assert ours.dtype == ref.dtype, f"{what}: dtype {ours.dtype} vs {ref.dtype}"
    if ours.dtype.kind == "f":
        tol = 1e-5 if dtype_tol is None else dtype_tol
        a = ours.astype(np.float64)
        b = ref.astype(np.float64)
        both_nan = np.isnan(a) & np.isnan(b)
        err = np.where(both_nan, 0, np.abs(a - b) / np.maximum(1.0, np.abs(b)))
        mx = float(np.nanmax(err)) if err.size else 0.0
        assert mx <= tol, f"{what}: max rel err {mx} > {tol}"
    else:
        diff = np.nonzero(ours != ref)
        n = len(diff[0])
        assert n == 0, f"{what}: {n} samples differ, first at {tuple(d[0] for d in diff)}: {ours[tuple(d[0] for d in diff)]} vs {ref[tuple(d[0] for d in diff)]}"
