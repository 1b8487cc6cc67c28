"""Cross-checks the CPU oracle against OpenCV (cv2 4.13 with the IPP HAL, which
VISAR's difftest reports as matching exactly on x86). VISAR's own
differential suite (tests/py/test_core_vs_opencv.py) pins VISAR to OpenCV 5.0
with the tolerances used below; cases where OpenCV 4 and 5 differ in
arithmetic (warpAffine: INTER_BITS tables in 4.x, float kernel in 5.x) are
checked with a loose bound only. CPU only."""
import numpy as np
import pytest

from conftest import natural
from oracle import oracle as O

cv2 = pytest.importorskip("cv2")

SIZES = [(480, 640), (37, 53), (1, 1), (7, 1), (1, 9)]


def close(ours, ref, tol=0.0, pct=100.0):
    d = np.abs(ours.astype(np.float64) - np.asarray(ref).astype(np.float64))
    mx = float(d.max()) if d.size else 0.0
    frac = 100.0 * float((d > (1e-5 if ours.dtype.kind == "f" else 0)).mean()) if d.size else 0.0
    return mx <= tol and frac <= pct, (mx, frac)


@pytest.mark.parametrize("h,w", SIZES)
def test_color(h, w):
    bgr = natural(h, w, 3)
    bgra = np.dstack([bgr, natural(h, w, 1)])
    gray = natural(h, w, 1)
    for code, src in [(6, bgr), (7, bgr), (10, bgra), (4, bgr), (0, bgr), (1, bgra), (2, bgr), (8, gray), (9, gray),
                      (40, bgr), (41, bgr), (36, bgr), (38, bgr)]:
        ok, info = close(O.cvt_color(src, code), cv2.cvtColor(src, code))
        assert ok, (code, info)
    f = natural(h, w, 3, np.float32)
    assert close(O.cvt_color(f, 6), cv2.cvtColor(f, 6), 1e-5)[0]
    assert close(O.cvt_color(f, 40), cv2.cvtColor(f, 40), 1e-3)[0]
    u16 = natural(h, w, 3, np.uint16)
    assert close(O.cvt_color(u16, 6), cv2.cvtColor(u16, 6))[0]


@pytest.mark.parametrize("h,w", SIZES)
def test_resize(h, w):
    bgr = natural(h, w, 3)
    f = natural(h, w, 3, np.float32)
    for dw, dh in [(max(1, w // 2), max(1, h // 2)), (w * 2, h * 2), (max(1, w * 3 // 4), max(1, h * 2 // 3)), (113, 71)]:
        for interp, tol in [(0, 0), (1, 1), (3, 0), (2, 1)]:
            ok, info = close(O.resize(bgr, (dw, dh), interp), cv2.resize(bgr, (dw, dh), interpolation=interp), tol)
            assert ok, (interp, dw, dh, info)
        assert close(O.resize(f, (dw, dh), 1), cv2.resize(f, (dw, dh), interpolation=1), 1e-4)[0]


def test_resize_area_exact():
    for (sw, sh), (dw, dh) in [((640, 480), (416, 312)), ((1920, 1080), (640, 360)), ((1920, 1080), (1280, 720)),
                               ((1280, 720), (320, 180)), ((97, 61), (53, 37)), ((640, 480), (60, 45)),
                               ((640, 480), (7, 5)), ((640, 480), (640, 300)), ((640, 480), (320, 480)),
                               ((640, 480), (639, 479)), ((97, 61), (130, 80)), ((97, 61), (50, 80))]:
        for cn in (1, 3, 4):
            a = natural(sh, sw, cn)
            ok, info = close(O.resize(a, (dw, dh), 3), cv2.resize(a, (dw, dh), interpolation=cv2.INTER_AREA))
            assert ok, (sw, sh, dw, dh, cn, info)


@pytest.mark.parametrize("h,w", SIZES)
def test_filters(h, w):
    bgr = natural(h, w, 3)
    gray = natural(h, w, 1)
    f = natural(h, w, 3, np.float32)
    for k, s in [(3, 0), (5, 0), (7, 0), (0, 1.5), (9, 2.0), (0, 3.0)]:
        assert close(O.gaussian_blur(bgr, (k, k), s), cv2.GaussianBlur(bgr, (k, k), s))[0], (k, s)
        assert close(O.gaussian_blur(f, (k, k), s), cv2.GaussianBlur(f, (k, k), s), 1e-5)[0], (k, s)
    for border in (1, 2, 0):
        assert close(O.gaussian_blur(gray, (5, 5), 0, border=border), cv2.GaussianBlur(gray, (5, 5), 0, borderType=border))[0]
    for k in [(3, 3), (5, 5), (7, 3), (15, 15)]:
        assert close(O.box_filter(bgr, k), cv2.blur(bgr, k), 1)[0], k
    for dx, dy, ks in [(1, 0, 3), (0, 1, 3), (1, 1, 3), (1, 0, 5), (2, 0, 5), (1, 0, -1)]:
        assert close(O.sobel(gray, np.int16, dx, dy, ks), cv2.Sobel(gray, cv2.CV_16S, dx, dy, ksize=ks))[0]
        assert close(O.sobel(gray, np.float32, dx, dy, ks), cv2.Sobel(gray, cv2.CV_32F, dx, dy, ksize=ks), 1e-3)[0]


def test_gaussian_sweep_u8_u16():
    # tests/py/test_core_vs_opencv.py:164-181 (a subset of the sigmas).
    for dt in (np.uint8, np.uint16):
        a = natural(120, 160, 1, dt)
        for k in range(1, 32, 2):
            for s in (0, 1.3, 4.1):
                assert close(O.gaussian_blur(a, (k, k), s), cv2.GaussianBlur(a, (k, k), s))[0], (dt, k, s)
        for s in (0.3, 1.0, 2.2, 5.0, 7.5):
            assert close(O.gaussian_blur(a, (0, 0), s), cv2.GaussianBlur(a, (0, 0), s))[0], (dt, s)


def test_gaussian_shapes_borders():
    for cn in (1, 3, 4):
        for h, w in [(37, 53), (1, 1), (7, 1), (1, 9), (2, 40), (31, 3)]:
            a = natural(h, w, cn)
            for (kw, kh), sx, sy in [((3, 15), 0, 0), ((21, 5), 0, 0), ((1, 9), 0, 0), ((13, 1), 0, 0),
                                     ((11, 7), 1.4, 3.2), ((0, 0), 1.2, 2.9), ((0, 17), 2.1, 0), ((25, 0), 0, 1.8)]:
                for border in (0, 1, 2, 4):
                    ours = O.gaussian_blur(a, (kw, kh), sx, sy, border=border)
                    ref = cv2.GaussianBlur(a, (kw, kh), sx, sigmaY=sy, borderType=border)
                    assert close(ours, ref)[0], (cn, h, w, kw, kh, sx, sy, border)


@pytest.mark.parametrize("h,w", SIZES)
def test_threshold_and_morphology(h, w):
    bgr = natural(h, w, 3)
    gray = natural(h, w, 1)
    f = natural(h, w, 3, np.float32)
    for kind in range(5):
        assert close(O.threshold(bgr, 127.5, 200, kind)[1], cv2.threshold(bgr, 127.5, 200, kind)[1])[0]
        assert close(O.threshold(f, 0.5, 1.0, kind)[1], cv2.threshold(f, 0.5, 1.0, kind)[1])[0]
    for auto in (8, 16):
        assert O.threshold(gray, 0, 255, auto)[0] == cv2.threshold(gray, 0, 255, auto)[0]
    for op in range(7):
        for shape in range(3):
            for ks in [(3, 3), (5, 7)]:
                el = cv2.getStructuringElement(shape, ks)
                assert close(O.morphology(bgr, op, shape, ks), cv2.morphologyEx(bgr, op, el))[0], (op, shape, ks)
    el = cv2.getStructuringElement(0, (3, 3))
    assert close(O.morphology(gray, 0, 0, (3, 3), 3), cv2.erode(gray, el, iterations=3))[0]


def test_warp_affine_loose():
    # OpenCV 4 blends with INTER_BITS fixed-point tables; VISAR (and OpenCV 5)
    # with f32 fmas. They agree to within one level on nearly every sample.
    bgr = natural(480, 640, 3)
    m = cv2.getRotationMatrix2D((320, 240), 30, 0.9)
    ok, info = close(O.warp_affine(bgr, m, (640, 480), 1), cv2.warpAffine(bgr, m, (640, 480), flags=cv2.INTER_LINEAR), 4, 10)
    assert ok, info
