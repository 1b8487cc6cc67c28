"""The CUDA library on the pinning cases of tests/test_oracle_pins.py: VISAR's
own resize property tests (resize.zig:642-743), the NumPy restatements of the
generic linear and cubic kernels, the analytic warp known answers and
sepFilter2D against cv2. Each result is compared with the same expected
array the oracle is held to."""
import numpy as np
import pytest

import pins_resize as PR
import pins_warp
from conftest import natural
from oracle import oracle as O

vb = pytest.importorskip("visar_b200")
torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def both(a):
    """The same image as host memory and as a CUDA tensor."""
    return [a, torch.from_numpy(np.ascontiguousarray(a)).cuda()]


def host(x):
    return x.cpu().numpy() if hasattr(x, "cpu") else np.asarray(x)


@pytest.mark.parametrize("cn", [1, 2, 3, 4])
def test_u8_linear_equals_generic_kernel(cn):
    src = PR.lcg_image(150, 64, cn, 12345)
    for w, h in PR.LINEAR_SIZES:
        want = O.resize_generic_u8(src, (w, h), 1)
        for s in both(src):
            assert np.array_equal(host(vb.resize(s, (w, h), 1)), want), (cn, w, h)


def test_constant_stays_constant():
    src = np.full((10, 10, 3), 100, np.uint8)
    for interp in (0, 1, 3, 2):
        assert (host(vb.resize(src, (7, 13), interp)) == 100).all(), interp


@pytest.mark.parametrize("cn", [1, 2, 3, 4])
def test_nearest_equals_naive_mapping(cn):
    src = PR.hash_image(37, 11, cn)
    for w, h in PR.NEAREST_SIZES:
        assert np.array_equal(host(vb.resize(src, (w, h), 0)), PR.nearest_naive(src, w, h)), (cn, w, h)


@pytest.mark.parametrize("cn", [1, 2, 3, 4])
def test_area_equals_generic_and_integer_rounding(cn):
    src = PR.lcg_image(97, 61, cn, 777)
    for w, h in PR.AREA_SIZES:
        assert np.array_equal(host(vb.resize(src, (w, h), 3)), O.resize_generic_u8(src, (w, h), 3)), (cn, w, h)
    s2 = np.ascontiguousarray(src[:60, :96])
    for fx, fy in [(4, 3), (4, 4)]:
        assert np.array_equal(host(vb.resize(s2, (96 // fx, 60 // fy), 3)), PR.area_int_naive(s2, fx, fy)), (cn, fx, fy)


SHAPES = [(480, 640), (37, 53), (64, 150), (1, 9), (7, 1), (61, 97)]


def _dsizes(h, w):
    out = [(max(1, w * 3 // 4), max(1, h * 2 // 3)), (113, 71), (w * 2, h * 2), (75, 32), (max(1, w // 2), max(1, h // 2))]
    return [d for d in out if d != (w, h)]


@pytest.mark.parametrize("h,w", SHAPES)
def test_generic_linear_f32_u16(h, w):
    for cn in (1, 2, 3, 4):
        for dt in (np.float32, np.uint16):
            a = natural(h, w, cn, dt)
            for dw, dh in _dsizes(h, w):
                assert np.array_equal(host(vb.resize(a, (dw, dh), 1)), PR.linear_generic(a, dw, dh)), (cn, dt, dw, dh)


@pytest.mark.parametrize("h,w", SHAPES)
def test_u8_linear_and_cubic(h, w):
    import cv2
    for cn in (1, 2, 3, 4):
        a = natural(h, w, cn)
        for dw, dh in _dsizes(h, w):
            ours = host(vb.resize(a, (dw, dh), 2))
            assert np.array_equal(ours, PR.cubic_u8(a, dw, dh, "visar")), ("cubic", cn, dw, dh)
            if cn == 2 and (dw * 2, dh * 2) == (w, h):
                continue
            ours = host(vb.resize(a, (dw, dh), 1))
            assert np.array_equal(ours, cv2.resize(a, (dw, dh), interpolation=1).reshape(ours.shape)), ("linear", cn, dw, dh)


def test_warp_known_answers():
    bad = pins_warp.check_all(vb)
    assert not bad, bad[:10]


def test_warp_known_answers_device_images():
    class Dev:
        """The CUDA binding on device copies of every input."""

        @staticmethod
        def warp_affine(src, m, dsize, interp, border, value):
            return host(vb.warp_affine(torch.from_numpy(np.ascontiguousarray(src)).cuda(), m, dsize, interp, border, value))

        @staticmethod
        def warp_perspective(src, m, dsize, interp, border, value):
            return host(vb.warp_perspective(torch.from_numpy(np.ascontiguousarray(src)).cuda(), m, dsize, interp, border,
                                            value))

    bad = pins_warp.check_all(Dev)
    assert not bad, bad[:10]


@pytest.mark.parametrize("h,w", [(37, 53), (1, 9), (7, 1), (64, 150)])
def test_sep_filter_2d_against_cv2(h, w):
    import cv2
    ints = [([1, -2, 1], [1, 2, 1]), ([1, 4, 6, 4, 1], [-1, 0, 1]), ([3], [1, 1, 1, 1, 1, 1, 1]), ([2, -1, 0, 5, 1], [1, 3, -2])]
    floats = [([0.1, 0.25, 0.3, 0.25, 0.1], [0.2, 0.6, 0.2]), ([-0.5, 0.0, 1.5], [0.7]),
              ([1.0 / 3] * 3, [0.05, 0.9, 0.05, 0.3, -0.1])]
    for cn in (1, 3):
        u8 = natural(h, w, cn)
        f = natural(h, w, cn, np.float32)
        for border in (0, 1, 2, 4):
            for kx, ky in ints:
                ours = host(vb.sep_filter_2d(u8, np.uint8, kx, ky, border))
                ref = cv2.sepFilter2D(u8, -1, np.float32(kx), np.float32(ky), borderType=border).reshape(ours.shape)
                assert np.array_equal(ours, ref), (cn, border, kx, ky)
                assert np.array_equal(ours, O.sep_filter_2d(u8, np.uint8, kx, ky, border))
            for kx, ky in ints + floats:
                ours = host(vb.sep_filter_2d(f, np.float32, kx, ky, border))
                ref = cv2.sepFilter2D(f, -1, np.float32(kx), np.float32(ky), borderType=border).reshape(ours.shape)
                err = np.abs(ours.astype(np.float64) - ref) / np.maximum(1.0, np.abs(ref))
                assert err.max() <= 1e-5, (cn, border, kx, ky, err.max())
                assert np.array_equal(ours, O.sep_filter_2d(f, np.float32, kx, ky, border))
