"""Pins the CPU oracle to VISAR's own known answers (the inline Zig unit tests
cited beside each check) and to its property tests. CPU only."""
import struct

import numpy as np
import pytest

from conftest import natural
from oracle import oracle as O


def _bits(v):
    return struct.unpack("<Q", struct.pack("<d", v))[0]


def test_gaussian_kernel_bit_patterns():
    # src/imgproc/filter.zig:930-935: cv2.getGaussianKernel(3, 0.9, CV_64F) bit for bit.
    k = O.gaussian_kernel(3, 0.9)
    assert _bits(k[0]) == 0x3FD09B4B1DC450D8
    assert _bits(k[1]) == 0x3FDEC969C4775E50
    assert k[2] == k[0]


def test_gaussian_fixed_taps():
    # src/imgproc/filter.zig:936-946: error-diffused fixed point sums to 2^bits.
    assert O.gaussian_kernel_fixed(13, 0, 8).tolist() == [1, 5, 10, 19, 30, 41, 44, 41, 30, 19, 10, 5, 1]
    assert O.gaussian_kernel_fixed(13, 0, 16).tolist() == [380, 1075, 2516, 4877, 7823, 10388, 11418, 10388, 7823, 4877,
                                                           2516, 1075, 380]
    assert O.gaussian_kernel_fixed(9, 0, 8).tolist() == [4, 13, 30, 51, 60, 51, 30, 13, 4]
    for n in range(1, 128, 2):
        for s in (0, 0.7, 2.5):
            assert int(O.gaussian_kernel_fixed(n, s, 8).astype(np.int64).sum()) == 256
            assert int(O.gaussian_kernel_fixed(n, s, 16).astype(np.int64).sum()) == 65536


def test_gaussian_3x3_hand_values():
    # src/imgproc/filter.zig:916-928
    src = np.zeros((5, 5), np.uint8)
    src[2, 2] = 255
    d = O.gaussian_blur(src, (3, 3), 0)
    assert (d[2, 2], d[2, 1], d[1, 1]) == (64, 32, 16)


def test_deriv_kernels():
    # src/imgproc/filter.zig:949-958
    assert O.deriv_kernel(3, 1, 3).tolist() == [-1, 0, 1]
    assert O.deriv_kernel(3, 0, 3).tolist() == [1, 2, 1]
    assert O.deriv_kernel(5, 1, 5).tolist() == [-1, -2, 0, 2, 1]
    assert O.deriv_kernel(3, 1, -1).tolist() == [-1, 0, 1]
    assert O.deriv_kernel(3, 0, -1).tolist() == [3, 10, 3]
    assert O.deriv_kernel(3, 3, 3) is None


def test_border_map_known_answers():
    # src/imgproc/border.zig:41-49
    assert O.border_map(-1, 5, 4) == 1
    assert O.border_map(-1, 5, 2) == 0
    assert O.border_map(5, 5, 4) == 3
    assert O.border_map(5, 5, 2) == 4
    assert O.border_map(5, 5, 3) == 0
    assert O.border_map(9, 5, 1) == 4
    assert O.border_map(-1, 5, 0) is None


def _closed_form(p, n, b):
    # The periodic form the CUDA library uses (visar_b200/csrc/vb_common.cuh border_map).
    if 0 <= p < n:
        return p
    if b == 0:
        return None
    if b == 1:
        return 0 if p < 0 else n - 1
    if b == 3:
        return p % n
    if n == 1:
        return 0
    if b == 2:
        q = p % (2 * n)
        return q if q < n else 2 * n - 1 - q
    q = p % (2 * n - 2)
    return q if q < n else 2 * n - 2 - q


def test_border_map_closed_form_equals_reflection_loop():
    for n in range(1, 12):
        for p in range(-60, 60):
            for b in range(5):
                assert _closed_form(p, n, b) == O.border_map(p, n, b), (p, n, b)


def test_saturate_known_answers():
    # src/core/saturate.zig:56-63 and src/core/simd.zig:217-223
    assert O.sat_u8(2.5) == 2 and O.sat_u8(3.5) == 4
    assert O.sat_i16(-1e9) == -32768
    v = [-1, 0.5, 1.5, 2.5, 254.5, 255.5, 300, float("nan")]
    assert [O.sat_u8(x) for x in v] == [0, 0, 2, 2, 254, 255, 255, 0]
    assert [O.sat_i16(x * -200) for x in v] == [200, -100, -300, -500, -32768, -32768, -32768, 0]


def test_threshold_known_answer():
    # src/imgproc/threshold.zig:288-299
    src = np.array([[10, 20, 30, 200, 210, 220, 15, 205]], np.uint8)
    _, dst = O.threshold(src, 100, 255, 0)
    assert dst.tolist() == [[0, 0, 0, 255, 255, 255, 0, 255]]
    t, _ = O.threshold(src, 0, 255, 8)
    assert 30 <= t < 200


def test_box_equals_naive_sum():
    # src/imgproc/filter.zig:960-986: every window against a naive sum, reflect101.
    for cn in (1, 2, 3, 4):
        rng = np.random.default_rng(99 + cn)
        src = rng.integers(0, 256, (23, 67, cn), dtype=np.uint8)
        src = src[..., 0] if cn == 1 else src
        for kw, kh in [(3, 3), (5, 5), (7, 3), (9, 1), (15, 15), (31, 31), (1, 9)]:
            dst = O.box_filter(src, (kw, kh))
            scale = np.float32(1.0 / (kw * kh))
            s3 = src.reshape(23, 67, cn).astype(np.int64)
            ys = np.array([[O.border_map(y + j - kh // 2, 23, 4) for j in range(kh)] for y in range(23)])
            xs = np.array([[O.border_map(x + i - kw // 2, 67, 4) for i in range(kw)] for x in range(67)])
            tot = s3[ys][:, :, xs].sum(axis=(1, 3))
            want = np.clip(np.rint((tot.astype(np.float32) * scale).astype(np.float64)), 0, 255).astype(np.uint8)
            assert np.array_equal(dst.reshape(23, 67, cn), want), (cn, kw, kh)


def test_morphology_equals_naive_min_max():
    # src/imgproc/morph.zig:672-698: 3x3 rect against a naive min/max ignoring outside pixels.
    for cn in (1, 2, 3, 4):
        for h, w in [(1, 1), (3, 2), (1, 37), (9, 1), (37, 53), (2, 70)]:
            src = (np.arange(h * w * cn, dtype=np.uint64) * 2654435761 >> 9).astype(np.uint8).reshape(h, w, cn)
            s = src[..., 0] if cn == 1 else src
            for op, fn, init in [(0, np.minimum, 255), (1, np.maximum, 0)]:
                d = O.morphology(s, op, 0, (3, 3)).reshape(h, w, cn)
                pad = np.pad(src, ((1, 1), (1, 1), (0, 0)), constant_values=init)
                want = pad[1:-1, 1:-1].copy()
                for dy in range(3):
                    for dx in range(3):
                        want = fn(want, pad[dy:dy + h, dx:dx + w])
                assert np.array_equal(d, want), (cn, h, w, op)


def test_structuring_elements():
    import cv2
    for shape in (0, 1, 2):
        for w, h in [(3, 3), (5, 5), (5, 7), (7, 7), (9, 3), (1, 1), (21, 13), (2, 4)]:
            assert np.array_equal(O.structuring_element(shape, w, h), cv2.getStructuringElement(shape, (w, h))), (shape, w, h)


def test_cv_exp_known_points():
    assert O.cv_exp(0.0) == 1.0
    assert O.cv_exp(float("-inf")) == 0.0
    for x in np.linspace(-30, 0, 301):
        assert abs(O.cv_exp(x) - np.exp(x)) <= 1e-14 * np.exp(x)


def test_hsv_tables_route_equals_scalar_formula():
    # color.zig:596-626: BGR->HSV on a 1-in-7 lattice equals rgb2hsvU8.
    vals = list(range(0, 256, 7)) + [255]
    b, g, r = np.meshgrid(vals, vals, vals, indexing="ij")
    img = np.stack([b.ravel(), g.ravel(), r.ravel()], -1).astype(np.uint8).reshape(1, -1, 3)
    out = O.cvt_color(img, 40)
    import cv2
    assert np.array_equal(out, cv2.cvtColor(img, cv2.COLOR_BGR2HSV))


@pytest.mark.parametrize("threads", [1, 3, 4, 8])
def test_threads_do_not_change_results(threads):
    a = natural(97, 131, 3)
    O.set_num_threads(1)
    ref = [O.gaussian_blur(a, (7, 7), 0), O.resize(a, (53, 37), 3), O.morphology(a, 2, 2, (5, 5))]
    O.set_num_threads(threads)
    got = [O.gaussian_blur(a, (7, 7), 0), O.resize(a, (53, 37), 3), O.morphology(a, 2, 2, (5, 5))]
    O.set_num_threads(0)
    for x, y in zip(ref, got):
        assert np.array_equal(x, y)
