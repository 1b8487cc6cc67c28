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


# ------------------------------------------------------------ resize property tests
# VISAR's own resize tests (resize.zig:642-743), on the oracle; the same cases
# run through the CUDA library in test_pins_gpu.py.

import pins_resize as PR  # noqa: E402


@pytest.mark.parametrize("cn", [1, 2, 3, 4])
def test_u8_linear_dispatch_equals_generic_kernel(cn):
    # resize.zig:654-682: the dispatched u8 INTER_LINEAR (exact half, exact 2x,
    # fast paths) equals the generic fixed-point `linear` kernel.
    src = PR.lcg_image(150, 64, cn, 12345)
    for w, h in PR.LINEAR_SIZES:
        assert np.array_equal(O.resize(src, (w, h), 1), O.resize_generic_u8(src, (w, h), 1)), (cn, w, h)


def test_resize_constant_stays_constant():
    # resize.zig:642-652: 10x10x3 of 100 -> 7x13 under every interpolation.
    src = np.full((10, 10, 3), 100, np.uint8)
    for interp in (0, 1, 3, 2):
        assert (O.resize(src, (7, 13), interp) == 100).all(), interp


@pytest.mark.parametrize("cn", [1, 2, 3, 4])
def test_nearest_equals_naive_mapping(cn):
    # resize.zig:684-700
    src = PR.hash_image(37, 11, cn)
    for w, h in PR.NEAREST_SIZES:
        assert np.array_equal(O.resize(src, (w, h), 0), PR.nearest_naive(src, w, h)), (cn, w, h)


@pytest.mark.parametrize("cn", [1, 2, 3, 4])
def test_area_dispatch_equals_generic_and_integer_rounding(cn):
    # resize.zig:702-743: the dispatched u8 INTER_AREA equals areaGeneric, and
    # 4x3 / 4x4 integer factors equal the f32 block-sum rounding.
    src = PR.lcg_image(97, 61, cn, 777)
    for w, h in PR.AREA_SIZES:
        assert np.array_equal(O.resize(src, (w, h), 3), O.resize_generic_u8(src, (w, h), 3)), (cn, w, h)
    s2 = np.ascontiguousarray(src[:60, :96])
    for fx, fy in [(4, 3), (4, 4)]:
        assert np.array_equal(O.resize(s2, (96 // fx, 60 // fy), 3), PR.area_int_naive(s2, fx, fy)), (cn, fx, fy)


# ---------------------------------------------------- linear / cubic against cv2 4.13

SHAPES = [(480, 640), (37, 53), (64, 150), (1, 9), (7, 1), (61, 97)]


def _dsizes(h, w):
    out = [(max(1, w * 3 // 4), max(1, h * 2 // 3)), (113, 71), (w * 2, h * 2), (75, 32)]
    return [d for d in out if d != (w, h)]


@pytest.mark.parametrize("h,w", SHAPES)
def test_generic_linear_f32_u16_pinned(h, w):
    # The NumPy restatement of the generic kernel (resize.zig:284-423) equals
    # the oracle bit for bit; given OpenCV 4's f32 source coordinates instead
    # of VISAR's f64 ones it equals cv2 4.13's portable build bit for bit, so
    # VISAR and OpenCV 4 differ only in that step. (Exact halvings are left out
    # of the cv2 side: OpenCV 4 runs them through INTER_AREA.)
    import cv2
    opt = cv2.useOptimized()
    cv2.setUseOptimized(False)
    try:
        for cn in (1, 2, 3, 4):
            for dt in (np.float32, np.uint16):
                a = natural(h, w, cn, dt)
                for dw, dh in _dsizes(h, w) + [(max(1, w // 2), max(1, h // 2))]:
                    ours = O.resize(a, (dw, dh), 1)
                    assert np.array_equal(ours, PR.linear_generic(a, dw, dh)), (cn, dt, dw, dh)
                    if (dw * 2, dh * 2) != (w, h):
                        ref = cv2.resize(a, (dw, dh), interpolation=cv2.INTER_LINEAR).reshape(ours.shape)
                        assert np.array_equal(PR.linear_generic(a, dw, dh, opencv4=True), ref), (cn, dt, dw, dh)
    finally:
        cv2.setUseOptimized(opt)


@pytest.mark.parametrize("h,w", SHAPES)
def test_u8_linear_equals_cv2(h, w):
    # u8 INTER_LINEAR (linearU8 / half / up2Linear) equals cv2 4.13 exactly,
    # except 2-channel exact halvings, which OpenCV 4 sends through its area path.
    import cv2
    for cn in (1, 2, 3, 4):
        a = natural(h, w, cn)
        for dw, dh in _dsizes(h, w) + [(max(1, w // 2), max(1, h // 2))]:
            if cn == 2 and (dw * 2, dh * 2) == (w, h):
                continue
            ours = O.resize(a, (dw, dh), 1)
            assert np.array_equal(ours, cv2.resize(a, (dw, dh), interpolation=1).reshape(ours.shape)), (cn, dw, dh)


@pytest.mark.parametrize("h,w", SHAPES)
def test_cubic_u8_pinned(h, w):
    # cubicU8 / up2Cubic: the NumPy restatement (taps, integer horizontal
    # pass, vcubic's fused f32 chain) equals the oracle bit for bit; with
    # OpenCV's unfused chain and integer row tail it equals cv2 4.13's portable
    # build bit for bit. Taps, offsets and horizontal sums are therefore
    # OpenCV's; only the fusing of the vertical chain differs.
    import cv2
    opt = cv2.useOptimized()
    cv2.setUseOptimized(False)
    try:
        for cn in (1, 2, 3, 4):
            a = natural(h, w, cn)
            for dw, dh in _dsizes(h, w) + [(max(1, w // 2), max(1, h // 2))]:
                ours = O.resize(a, (dw, dh), 2)
                assert np.array_equal(ours, PR.cubic_u8(a, dw, dh, "visar")), (cn, dw, dh)
                ref = cv2.resize(a, (dw, dh), interpolation=cv2.INTER_CUBIC).reshape(ours.shape)
                assert np.array_equal(PR.cubic_u8(a, dw, dh, "opencv4"), ref), (cn, dw, dh)
    finally:
        cv2.setUseOptimized(opt)


# ------------------------------------------------------------------ warp known answers

def test_warp_known_answers():
    import pins_warp
    bad = pins_warp.check_all(O)
    assert not bad, bad[:10]


# ----------------------------------------------------------------- sepFilter2D vs cv2

def _sep_cases():
    ints = [([1, -2, 1], [1, 2, 1]), ([1, 4, 6, 4, 1], [-1, 0, 1]), ([3], [1, 1, 1, 1, 1, 1, 1]), ([2, -1, 0, 5, 1], [1, 3, -2])]
    floats = [([0.1, 0.25, 0.3, 0.25, 0.1], [0.2, 0.6, 0.2]), ([-0.5, 0.0, 1.5], [0.7]), ([1.0 / 3] * 3, [0.05, 0.9, 0.05, 0.3, -0.1])]
    return ints, floats


@pytest.mark.parametrize("h,w", [(37, 53), (1, 9), (7, 1), (64, 150)])
def test_sep_filter_2d_against_cv2(h, w):
    # filter.zig:909-914 has no VISAR test. Integer taps on u8: every f32 sum
    # is an exact integer, so VISAR's vertical-first and OpenCV's
    # horizontal-first orders must agree exactly (saturated); f32 images agree
    # within the 1e-5 contract.
    import cv2
    ints, floats = _sep_cases()
    for cn in (1, 3):
        u8 = natural(h, w, cn)
        f = natural(h, w, cn, np.float32)
        for border in (0, 1, 2, 4):
            for kx, ky in ints:
                ours = O.sep_filter_2d(u8, np.uint8, kx, ky, border)
                ref = cv2.sepFilter2D(u8, -1, np.float32(kx), np.float32(ky), borderType=border).reshape(ours.shape)
                assert np.array_equal(ours, ref), (cn, border, kx, ky)
            for kx, ky in ints + floats:
                ours = O.sep_filter_2d(f, np.float32, kx, ky, border).astype(np.float64)
                assert ours.shape[:2] == (h, w)
                ref = cv2.sepFilter2D(f, -1, np.float32(kx), np.float32(ky), borderType=border).reshape(ours.shape)
                err = np.abs(ours - ref) / np.maximum(1.0, np.abs(ref))
                assert err.max() <= 1e-5, (cn, border, kx, ky, err.max())


def test_sep_filter_2d_even_kernels_refused():
    # filter.zig:122: kernels of even length are InvalidKernel.
    a = natural(9, 11, 1)
    for kx, ky in [([1, 1], [1]), ([1], [1, 2, 1, 0])]:
        with pytest.raises(O.OracleError) as e:
            O.sep_filter_2d(a, np.uint8, kx, ky, 4)
        assert e.value.status == -1 and "InvalidKernel" in e.value.name


# ------------------------------------------------------------ gray + integer shrink

def _luma_mean(src, k):
    h, w = src.shape[0] // k * k, src.shape[1] // k * k
    s = src[:h, :w].astype(np.float64)
    lum = (s[..., 0] * 1868 + s[..., 1] * 9617 + s[..., 2] * 4899) / 16384.0
    return lum.reshape(h // k, k, w // k, k).mean(axis=(1, 3))


@pytest.mark.parametrize("cn", [4, 3])
def test_gray_downsample_matches_gray_then_area(cn):
    # frame.zig:384-416: within 0.51 of the f64 mean of per-pixel lumas; at
    # k = 1 within 1 of cvtColor's gray.
    for k in (1, 2, 3, 4, 6, 8):
        rng = np.random.default_rng(k)
        src = rng.integers(0, 256, (9 * k, 70 * k + 1, cn), dtype=np.uint8)
        d = O.gray_downsample(src, k)
        assert d.shape == (9, 70 + (k == 1))
        assert np.abs(d - _luma_mean(src, k)).max() <= 0.51, (cn, k)
        if k == 1:
            g = O.cvt_color(src, 10 if cn == 4 else 6)
            assert np.abs(d.astype(int) - g.astype(int)).max() <= 1


def test_gray_downsample_refusals():
    src = np.zeros((40, 50, 3), np.uint8)
    for k, shape, want in [(0, (40, 50), (-1, "InvalidArgument")), (17, (2, 2), (-2, "SizeMismatch")),
                           (2, (20, 24), (-2, "SizeMismatch")), (2, (20, 25, 3), (-2, "SizeMismatch"))]:
        with pytest.raises(O.OracleError) as e:
            O.gray_downsample(src, k, dst=np.zeros(shape, np.uint8))
        assert (e.value.status, e.value.name) == want, (k, shape)
    with pytest.raises(O.OracleError) as e:
        O.gray_downsample(np.zeros((40, 50), np.uint8), 2)
    assert e.value.status == -2


# ------------------------------------------------------------------------ pyramids

import pins_pyr as PP  # noqa: E402

PYR_TYPES = [np.uint8, np.uint16, np.int16, np.float32]
PYR_SIZES = [(1, 1), (2, 3), (5, 4), (37, 19), (70, 9), (129, 7)]  # (w, h), pyramid.zig:626


@pytest.mark.parametrize("dtype", PYR_TYPES)
def test_pyr_down_up_equal_direct_sums(dtype):
    # pyramid.zig:624-644 (channel counts 1-5, every border but constant).
    for w, h in PYR_SIZES:
        for cn in (1, 2, 3, 4, 5):
            src = PP.fill_random(dtype, w, h, cn, w * 31 + cn)
            for b in (4, 2, 1, 3):
                got = O.pyr_down(src, b).reshape((h + 1) // 2, (w + 1) // 2, cn)
                want = PP.ref_down(src, b)
                if dtype == np.float32:
                    assert np.abs(got - want).max() <= 1e-5, (w, h, cn, b)
                else:
                    assert np.array_equal(got.astype(np.int64), want.astype(np.int64)), (w, h, cn, b)
            got = O.pyr_up(src, 4).reshape(2 * h, 2 * w, cn)
            want = PP.ref_up(src)
            if dtype == np.float32:
                assert np.abs(got - want).max() <= 1e-5, (w, h, cn)
            else:
                assert np.array_equal(got.astype(np.int64), want.astype(np.int64)), (w, h, cn)


def test_pyr_down_f32_scalar_order():
    # pyramid.zig:646-672: f32 3/4 channels equal the scalar formula exactly.
    for w, h in [(131, 12), (64, 9), (70, 7), (9, 5)]:
        for cn in (3, 4):
            src = PP.fill_random(np.float32, w, h, cn, w * 7 + cn)
            for b in (4, 1):
                got = O.pyr_down(src, b).reshape((h + 1) // 2, (w + 1) // 2, cn)
                assert np.array_equal(got, PP.down_f32_scalar(src, b)), (w, h, cn, b)


def test_pyramid_sizes_and_refusals():
    # pyramid.zig:674-688: levels of 101x50 are 51x25 ... 7x4; a constant image stays constant.
    lv = np.full((50, 101), 7, np.uint8)
    sizes = []
    for _ in range(4):
        lv = O.pyr_down(lv, 4)
        sizes.append(lv.shape)
    assert sizes == [(25, 51), (13, 26), (7, 13), (4, 7)] and (lv == 7).all()
    src = np.zeros((50, 101), np.uint8)
    for fn, dst, border, want in [(O.pyr_down, np.zeros((13, 26), np.uint8), 4, -2),
                                  (O.pyr_down, np.zeros((25, 51), np.uint8), 0, -3),
                                  (O.pyr_up, np.zeros((100, 202), np.uint8), 1, -3),
                                  (O.pyr_up, np.zeros((100, 201), np.uint8), 4, -2),
                                  (O.pyr_down, np.zeros((25, 51), np.uint8), 5, -3)]:
        with pytest.raises(O.OracleError) as e:
            fn(src, border, dst=dst)
        assert e.value.status == want, (fn.__name__, dst.shape, border)


# --------------------------------------------------------------- undistort / remap

import pins_calib as PC  # noqa: E402


def test_undistort_zero_distortion_is_identity():
    # undistort.zig:396-408: all but the last row and column come back unchanged.
    src = (np.arange(23 * 37 * 3) * 7 % 256).astype(np.uint8).reshape(23, 37, 3)
    d = O.undistort(src, [40, 0, 18, 0, 40, 11, 0, 0, 1], [])
    assert np.array_equal(d[:22, :36], src[:22, :36])


@pytest.mark.parametrize("cn", [1, 2, 3, 4])
def test_undistort_and_maps_equal_cv2(cn):
    import cv2
    rng = np.random.default_rng(cn)
    for w, h in [(640, 480), (97, 61), (1500, 1000), (4100, 9)]:
        img = rng.integers(0, 256, (h, w, cn), dtype=np.uint8)
        img = img[..., 0] if cn == 1 else img
        for K0, dist, nk in PC.CAMERAS:
            K = PC.scaled_camera(K0, w, h)
            d = np.array(dist) if dist else None
            ours = O.undistort(img, K, dist, nk)
            ref = cv2.undistort(img, K, d, newCameraMatrix=nk)
            # Equal but where a source coordinate lies within 1e-6 of a 1/64
            # pixel boundary (OpenCV's own map arithmetic may round it the
            # other way; undistort.zig:7-11).
            for y, x in {(int(a), int(b)) for a, b in np.argwhere((ours != ref).reshape(h, w, -1).any(axis=2))}:
                u, v = PC.undistort_coord(K, dist, nk, w, h, x, y)
                assert PC.near_tie(u) or PC.near_tie(v), (cn, w, h, dist, x, y, u, v)
            if cn == 1:
                R = np.array([[0.999, -0.01, 0.02], [0.011, 0.9995, -0.005], [-0.02, 0.006, 0.9992]])
                for r in (None, R):
                    mx, my = O.init_undistort_rectify_map(K, dist, r, nk, (w, h))
                    cx, cy = cv2.initUndistortRectifyMap(K, d, r, nk if nk is not None else K, (w, h), cv2.CV_32FC1)
                    if dist:
                        # Equal but at f64 values within 1e-9 of an f32 rounding tie.
                        for axis, (a, b) in enumerate(((mx, cx), (my, cy))):
                            for y, x in np.argwhere(a != b):
                                c = PC.undistort_coord(K, dist, nk, w, h, int(x), int(y), R=r, stripes=False)[axis]
                                assert PC.f32_tie(c, a[y, x], b[y, x]), (w, h, dist, r is None, x, y, c, a[y, x], b[y, x])
                    else:  # OpenCV inverts an identity-distortion camera by a route that can leave 1e-16 residues
                        for a, b in ((mx, cx), (my, cy)):
                            assert np.abs(a - b).max() <= 1e-6 * max(1.0, float(np.abs(b).max())), (w, h, r is None)


def test_remap_known_answers():
    bad = [name for name, src, mx, my, v, exp in PC.remap_cases() if not np.array_equal(O.remap(src, mx, my, v), exp)]
    assert not bad, bad[:10]


def test_undistort_remap_refusals():
    img = np.zeros((20, 30, 3), np.uint8)
    K = [40, 0, 15, 0, 40, 10, 0, 0, 1]
    with pytest.raises(O.OracleError) as e:
        O.undistort(img, K, [0.1, 0.2])
    assert e.value.status == -1
    with pytest.raises(O.OracleError) as e:
        O.undistort(img, K, [], dst=np.zeros((20, 31, 3), np.uint8))
    assert e.value.status == -2
    with pytest.raises(O.OracleError) as e:
        O.init_undistort_rectify_map([0] * 9, [], None, None, (30, 20))
    assert e.value.status == -1
    mx = np.zeros((20, 30), np.float32)
    with pytest.raises(O.OracleError) as e:
        O.remap(img, mx, np.zeros((20, 29), np.float32))
    assert e.value.status == -2
    with pytest.raises(O.OracleError) as e:
        O.remap(img, mx, mx, dst=np.zeros((20, 30), np.uint8))
    assert e.value.status == -3


# --------------------------------------------------------------- tracker tail

import pins_tail as PT  # noqa: E402


def test_equalize_known_answer_and_cv2():
    # hist.zig:67-75
    assert O.equalize_hist(np.array([[10, 10, 20, 30]], np.uint8)).tolist() == [[0, 0, 128, 255]]
    import cv2
    rng = np.random.default_rng(3)
    for img in (natural(120, 160, 1), rng.integers(40, 90, (37, 53), dtype=np.uint8), np.full((5, 7), 9, np.uint8)):
        assert np.array_equal(O.equalize_hist(img), cv2.equalizeHist(img))


@pytest.mark.parametrize("conn", [4, 8])
def test_connected_components_reference_patterns_and_cv2(conn):
    # components.zig:545-650 (patterns, sizes) against cv2 4.13's
    # connectedComponentsWithStats: labels, stats and centroids exactly.
    import cv2
    rng = np.random.default_rng(42)
    for w, h in PT.CC_SIZES:
        for pat in PT.PATTERNS:
            img = PT.cc_pattern(w, h, pat, rng)
            n, lab, st, ce = O.connected_components(img, conn)
            n2, lab2, st2, ce2 = cv2.connectedComponentsWithStats(img, connectivity=conn, ltype=cv2.CV_32S)
            assert n == n2 and np.array_equal(lab, lab2) and np.array_equal(st, st2), (w, h, pat)
            assert np.array_equal(np.isnan(ce), np.isnan(ce2)) and np.allclose(ce, ce2, rtol=0, atol=0, equal_nan=True)


def test_connected_components_two_components():
    # components.zig:545-559: a U shape that merges late and a separate dot.
    img = np.zeros((4, 6), np.uint8)
    for x, y in [(0, 0), (0, 1), (0, 2), (1, 2), (2, 2), (2, 1), (2, 0), (5, 3)]:
        img[y, x] = 255
    n, lab, st, _ = O.connected_components(img, 8)
    assert n == 3 and lab[0, 2] == 1 and lab[3, 5] == 2 and st[1, 4] == 7 and st[1, 2] == 3


def test_adaptive_threshold_against_cv2():
    # Mean: equal to cv2. Gaussian: equal but where the f32 blurred mean is
    # within 1e-3 of a rounding tie (OpenCV 4 sums the f32 taps in another order).
    import cv2
    g = natural(240, 320, 1)
    f = g.astype(np.float32)
    for kind in (0, 1):
        for block, delta in [(3, 0.0), (11, 2.5), (31, -3.2), (5, 7.0)]:
            assert np.array_equal(O.adaptive_threshold(g, 255, 0, kind, block, delta),
                                  cv2.adaptiveThreshold(g, 255, 0, kind, block, delta)), (kind, block, delta)
            ours = O.adaptive_threshold(g, 200.4, 1, kind, block, delta)
            ref = cv2.adaptiveThreshold(g, 200.4, 1, kind, block, delta)
            bad = np.argwhere(ours != ref)
            if len(bad):
                m = O.gaussian_blur(f, (block, block), 0, 0, 1)
                for y, x in bad:
                    assert abs(abs(m[y, x] - np.floor(m[y, x])) - 0.5) < 1e-3, (kind, block, delta, y, x, m[y, x])


def test_adaptive_threshold_refusals():
    g = natural(20, 30, 1)
    for args, want in [((255, 2, 0, 3, 0), -1), ((255, 0, 2, 3, 0), -1), ((255, 0, 0, 1, 0), -1), ((255, 0, 0, 4, 0), -1)]:
        with pytest.raises(O.OracleError) as e:
            O.adaptive_threshold(g, *args)
        assert e.value.status == want, args
    with pytest.raises(O.OracleError) as e:
        O.adaptive_threshold(natural(20, 30, 3), 255, 0, 0, 3, 0)
    assert e.value.status == -3


def test_background_model_sequence():
    rng = np.random.default_rng(5)
    frames = [np.clip(natural(60, 80, 1).astype(int) + rng.integers(-40, 40, (60, 80)), 0, 255).astype(np.uint8)
              for _ in range(6)]
    for shift, t in [(4, 28), (0, 5), (15, 0)]:
        bg = O.Background(80, 60, shift)
        want = PT.background_ref(frames, shift, t)
        for f, w_ in zip(frames, want):
            assert np.array_equal(bg.apply(f, t), w_)
        assert np.array_equal(bg.model, PT.background_model(frames, shift, t))
