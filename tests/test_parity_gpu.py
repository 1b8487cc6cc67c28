"""Parity: the CUDA library (through the C ABI) against the CPU oracle on the
same seeded inputs. Integer outputs must be bit-exact; f32 outputs within
1e-5 relative (|a-b| <= 1e-5 * max(1, |b|)); f32 paths that reproduce VISAR's
operation order are additionally checked bit-exact where stated.

Cases follow VISAR's differential suite (tests/py/test_core_vs_opencv.py:47,
164-297): sizes 640x480, 53x37, 1x1, 1x7, 9x1, strided views, every border.
"""
import numpy as np
import pytest

from conftest import assert_same, natural

pytestmark = pytest.mark.gpu

vb = pytest.importorskip("visar_b200")
from oracle import oracle as O  # noqa: E402

SIZES = [(480, 640), (37, 53), (1, 1), (7, 1), (1, 9)]
DTYPES = [np.uint8, np.uint16, np.int16, np.float32]


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    yield


def _both(fn_vb, fn_or, *args, tol=None, exact_f32=False, what="", **kw):
    ours = fn_vb(*args, **kw)
    ref = fn_or(*args, **kw)
    if isinstance(ours, tuple):
        assert ours[0] == ref[0], f"{what}: threshold {ours[0]} vs {ref[0]}"
        ours, ref = ours[1], ref[1]
    if exact_f32 and np.asarray(ref).dtype.kind == "f":
        assert_same(ours, ref, 0.0, what)
    else:
        assert_same(ours, ref, tol, what)


# ----------------------------------------------------------------- color

COLOR_CASES = [(6, 3), (7, 3), (10, 4), (11, 4), (4, 3), (0, 3), (1, 4), (2, 3), (3, 4), (5, 4), (8, 1), (9, 1),
               (40, 3), (41, 3), (36, 3), (37, 3), (38, 3), (39, 3), (54, 3), (55, 3)]


@pytest.mark.parametrize("h,w", SIZES)
@pytest.mark.parametrize("code,scn", COLOR_CASES)
def test_cvt_color_u8(h, w, code, scn):
    a = natural(h, w, scn)
    if code in (54, 55):
        a = a.copy()
        a[..., 0] = a[..., 0] % 180
    _both(vb.cvt_color, O.cvt_color, a, code, what=f"cvt {code}")


@pytest.mark.parametrize("dt", [np.uint16, np.float32])
@pytest.mark.parametrize("code,scn", [(6, 3), (7, 3), (10, 4), (4, 3), (0, 3), (8, 1)])
def test_cvt_color_other_depths(dt, code, scn):
    a = natural(37, 53, scn, dt)
    _both(vb.cvt_color, O.cvt_color, a, code, exact_f32=True, what=f"cvt {code} {dt}")


@pytest.mark.parametrize("code", [40, 41, 36, 37, 38, 39, 54, 55])
def test_cvt_color_f32_hsv_ycrcb(code):
    a = natural(37, 53, 3, np.float32)
    if code in (54, 55):
        a = a.copy()
        a[..., 0] *= 360.0
    _both(vb.cvt_color, O.cvt_color, a, code, exact_f32=True, what=f"cvt f32 {code}")


def test_cvt_color_exhaustive_u8_lattice():
    # Every 5th value in each channel (52^3 colours), as color.zig:628-681 does.
    v = np.minimum(np.arange(52) * 5, 255).astype(np.uint8)
    b, g, r = np.meshgrid(v, v, v, indexing="ij")
    img = np.stack([b.ravel(), g.ravel(), r.ravel()], -1).reshape(52 * 52, 52, 3)
    for code in (6, 7, 36, 37, 40, 41):
        _both(vb.cvt_color, O.cvt_color, np.ascontiguousarray(img), code, what=f"lattice {code}")


# -------------------------------------------------------------- Gaussian

@pytest.mark.parametrize("dt", DTYPES)
@pytest.mark.parametrize("k,s", [(1, 0), (3, 0), (5, 0), (7, 0), (9, 0), (11, 0), (15, 0.6), (31, 0), (0, 1.5),
                                 (9, 2.0), (0, 3.0), (13, 4.1), (21, 2.5)])
def test_gaussian_sweep(dt, k, s):
    a = natural(97, 131, 1, dt)
    _both(vb.gaussian_blur, O.gaussian_blur, a, (k, k), s, exact_f32=True, what=f"gauss k{k} s{s} {dt}")


@pytest.mark.parametrize("cn", [1, 3, 4])
@pytest.mark.parametrize("h,w", [(37, 53), (1, 1), (7, 1), (1, 9), (2, 40), (31, 3)])
@pytest.mark.parametrize("border", [0, 1, 2, 4])
def test_gaussian_shapes_borders(cn, h, w, border):
    for dt in DTYPES:
        a = natural(h, w, cn, dt)
        for (kw, kh), sx, sy in [((3, 15), 0, 0), ((21, 5), 0, 0), ((1, 9), 0, 0), ((13, 1), 0, 0), ((5, 5), 0, 0),
                                 ((11, 7), 1.4, 3.2), ((0, 0), 1.2, 2.9), ((0, 17), 2.1, 0), ((25, 0), 0, 1.8)]:
            _both(vb.gaussian_blur, O.gaussian_blur, a, (kw, kh), sx, sy, border=border, exact_f32=True,
                  what=f"gauss ({kw},{kh}) s{sx}/{sy} b{border} c{cn} {dt} {w}x{h}")


def test_gaussian_wrap_border():
    a = natural(37, 53, 3)
    _both(vb.gaussian_blur, O.gaussian_blur, a, (5, 5), 0, border=3, what="gauss wrap")


@pytest.mark.parametrize("cn", [1, 3])
def test_gaussian_strided_views(cn):
    big = natural(120, 160, cn)
    for y0, x0, h, w in [(3, 5, 37, 53), (1, 1, 97, 131), (10, 7, 9, 150)]:
        v = big[y0:y0 + h, x0:x0 + w]
        for k, s in [(3, 0), (7, 0), (13, 0), (19, 2.3), (31, 0)]:
            _both(vb.gaussian_blur, O.gaussian_blur, v, (k, k), s, what=f"view k{k}")


def test_gaussian_f32_workload_bit_exact():
    from visar_b200 import synth
    a = synth.normal_f32(1080, 1920, seed=3)
    _both(vb.gaussian_blur, O.gaussian_blur, a, (7, 7), 1.5, exact_f32=True, what="f32 7x7 s1.5 1920x1080")


# --------------------------------------------------------- box / Sobel

@pytest.mark.parametrize("dt", DTYPES)
@pytest.mark.parametrize("k", [(3, 3), (5, 5), (7, 3), (15, 15), (1, 9), (31, 31)])
@pytest.mark.parametrize("border", [0, 1, 4])
def test_box(dt, k, border):
    a = natural(37, 53, 3, dt)
    if dt == np.int16:
        a = np.abs(a).astype(np.int16)  # VISAR's i16 box accumulates in u32 (negative samples are undefined there)
    _both(vb.box_filter, O.box_filter, a, k, True, border, exact_f32=True, what=f"box {k} {dt} b{border}")
    _both(vb.box_filter, O.box_filter, a, k, False, border, exact_f32=True, what=f"box unnorm {k} {dt}")


@pytest.mark.parametrize("h,w", SIZES)
@pytest.mark.parametrize("dx,dy,ks", [(1, 0, 3), (0, 1, 3), (1, 1, 3), (1, 0, 5), (2, 0, 5), (1, 0, -1), (0, 1, -1),
                                      (1, 0, 1), (0, 1, 1), (2, 1, 7), (1, 2, 31)])
def test_sobel(h, w, dx, dy, ks):
    g = natural(h, w, 1)
    _both(vb.sobel, O.sobel, g, np.int16, dx, dy, ks, what=f"sobel i16 {dx}{dy}{ks}")
    _both(vb.sobel, O.sobel, g, np.float32, dx, dy, ks, exact_f32=True, what=f"sobel f32 {dx}{dy}{ks}")
    _both(vb.sobel, O.sobel, g, np.int16, dx, dy, ks, 0.5, what=f"sobel i16 scaled {dx}{dy}{ks}")


@pytest.mark.parametrize("dt", [np.uint16, np.int16, np.float32])
def test_sobel_other_sources(dt):
    a = natural(37, 53, 3, dt)
    _both(vb.sobel, O.sobel, a, np.float32, 1, 1, 3, 0.25, exact_f32=True, what=f"sobel {dt}")


@pytest.mark.parametrize("sdt", DTYPES)
@pytest.mark.parametrize("ddt", DTYPES)
def test_sep_filter_2d(sdt, ddt):
    a = natural(37, 53, 3, sdt)
    kx = np.array([0.1, -0.3, 0.55, 0.2, 0.15], np.float32)
    ky = np.array([0.25, 0.5, 0.25], np.float32)
    for border in (0, 1, 2, 4):
        _both(vb.sep_filter_2d, O.sep_filter_2d, a, ddt, kx, ky, border, exact_f32=True, what=f"sep2d {sdt}->{ddt}")
    _both(vb.sep_filter_2d, O.sep_filter_2d, a, ddt, [-1, 0, 1], [1, 2, 1], 4, exact_f32=True, what="sep2d odd")


# --------------------------------------------------------------- resize

@pytest.mark.parametrize("h,w", SIZES)
@pytest.mark.parametrize("interp", [0, 1, 2, 3])
def test_resize_u8(h, w, interp):
    bgr = natural(h, w, 3)
    for dw, dh in [(max(1, w // 2), max(1, h // 2)), (w * 2, h * 2), (max(1, w * 3 // 4), max(1, h * 2 // 3)), (113, 71)]:
        _both(vb.resize, O.resize, bgr, (dw, dh), interp, what=f"resize {interp} {w}x{h}->{dw}x{dh}")


@pytest.mark.parametrize("cn", [1, 3, 4])
def test_resize_area_u8(cn):
    for (sw, sh), (dw, dh) in [((640, 480), (416, 312)), ((1920, 1080), (640, 360)), ((1920, 1080), (1280, 720)),
                               ((1280, 720), (320, 180)), ((97, 61), (53, 37)), ((640, 480), (60, 45)),
                               ((640, 480), (7, 5)), ((640, 480), (640, 300)), ((640, 480), (320, 480)),
                               ((640, 480), (639, 479)), ((97, 61), (130, 80)), ((97, 61), (50, 80)),
                               ((96, 60), (24, 20)), ((96, 60), (24, 15))]:
        a = natural(sh, sw, cn)
        _both(vb.resize, O.resize, a, (dw, dh), 3, what=f"area c{cn} {sw}x{sh}->{dw}x{dh}")


@pytest.mark.parametrize("dt", [np.uint16, np.int16, np.float32])
@pytest.mark.parametrize("interp", [0, 1, 2, 3])
def test_resize_other_depths(dt, interp):
    a = natural(61, 97, 3, dt)
    for dw, dh in [(48, 30), (194, 122), (53, 37), (97, 61), (130, 80), (32, 61)]:
        _both(vb.resize, O.resize, a, (dw, dh), interp, exact_f32=True, what=f"resize {interp} {dt} ->{dw}x{dh}")


def test_resize_many_channels_u8():
    a = natural(31, 47, 6)
    for interp in (0, 1, 2, 3):
        for dw, dh in [(23, 15), (94, 62), (30, 20), (47, 31)]:
            _both(vb.resize, O.resize, a, (dw, dh), interp, what=f"resize c6 {interp} {dw}x{dh}")


# ---------------------------------------------------------------- warps

@pytest.mark.parametrize("h,w", SIZES)
@pytest.mark.parametrize("interp", [0, 1])
@pytest.mark.parametrize("border", [0, 1, 2, 3, 4])
def test_warp_affine(h, w, interp, border):
    from visar_b200 import synth
    bgr = natural(h, w, 3)
    m = synth.rotation_matrix_2d(w / 2, h / 2, 30, 0.9)
    _both(vb.warp_affine, O.warp_affine, bgr, m, (w, h), interp, border, 17.0, what=f"affine {interp} b{border}")


@pytest.mark.parametrize("dt", DTYPES)
def test_warp_affine_depths(dt):
    from visar_b200 import synth
    a = natural(61, 97, 3, dt)
    for seed in range(4):
        m = synth.affine_params(97, 61, seed)
        for interp in (0, 1):
            _both(vb.warp_affine, O.warp_affine, a, m, (97, 61), interp, 0, 3.0, exact_f32=True, what=f"affine {dt}")


@pytest.mark.parametrize("dt", DTYPES)
@pytest.mark.parametrize("border", [0, 1, 4])
def test_warp_perspective(dt, border):
    from visar_b200 import synth
    a = natural(61, 97, 3, dt)
    for seed in range(4):
        m = synth.perspective_params(97, 61, seed, jitter=20)
        for interp in (0, 1):
            _both(vb.warp_perspective, O.warp_perspective, a, m, (97, 61), interp, border, 9.0, exact_f32=True,
                  what=f"persp {dt} b{border}")


def test_warp_workload_full_size():
    from visar_b200 import synth
    img = synth.base_image(1080, 1920, 3, nrect=32, seed=1)
    m = synth.affine_params(1920, 1080, 11)
    _both(vb.warp_affine, O.warp_affine, img, m, (1920, 1080), 1, 0, 0.0, what="affine 1080p")
    hm = synth.perspective_params(1920, 1080, 12)
    _both(vb.warp_perspective, O.warp_perspective, img, hm, (1920, 1080), 1, 0, 0.0, what="persp 1080p")


# ------------------------------------------------------------ threshold

@pytest.mark.parametrize("h,w", SIZES)
@pytest.mark.parametrize("kind", [0, 1, 2, 3, 4])
def test_threshold(h, w, kind):
    bgr = natural(h, w, 3)
    for t in (127.5, 0, -3, 254.9, 255, 300):
        _both(vb.threshold, O.threshold, bgr, t, 200, kind, what=f"thr u8 {kind} {t}")
    f = natural(h, w, 3, np.float32)
    _both(vb.threshold, O.threshold, f, 0.5, 1.0, kind, exact_f32=True, what=f"thr f32 {kind}")
    for dt, ts in [(np.uint16, (30000.7, -5, 70000)), (np.int16, (10.2, -40000, 40000, -128))]:
        a = natural(h, w, 3, dt)
        for t in ts:
            _both(vb.threshold, O.threshold, a, t, 1000, kind, what=f"thr {dt} {kind} {t}")


@pytest.mark.parametrize("h,w", SIZES)
@pytest.mark.parametrize("auto", [8, 16])
def test_threshold_auto(h, w, auto):
    g = natural(h, w, 1)
    for kind in (0, 1, 2, 3, 4):
        _both(vb.threshold, O.threshold, g, 0, 255, kind | auto, what=f"auto {auto} {kind}")


def test_threshold_known_answer():
    src = np.array([[10, 20, 30, 200, 210, 220, 15, 205]], np.uint8)  # threshold.zig:288-299
    _, dst = vb.threshold(src, 100, 255, 0)
    assert dst.tolist() == [[0, 0, 0, 255, 255, 255, 0, 255]]
    t, _ = vb.threshold(src, 0, 255, 8)
    assert 30 <= t < 200


# ----------------------------------------------------------- morphology

@pytest.mark.parametrize("h,w", SIZES)
@pytest.mark.parametrize("op", range(7))
def test_morphology(h, w, op):
    bgr = natural(h, w, 3)
    for shape in (0, 1, 2):
        for ks in [(3, 3), (5, 7), (1, 1), (7, 1)]:
            _both(vb.morphology, O.morphology, bgr, op, shape, ks, what=f"morph op{op} sh{shape} {ks}")


@pytest.mark.parametrize("dt", DTYPES)
def test_morphology_depths_iterations(dt):
    a = natural(37, 53, 3, dt)
    for op in range(7):
        for shape, ks, it in [(0, (3, 3), 3), (2, (5, 5), 2), (1, (9, 3), 1), (2, (21, 13), 1), (0, (7, 7), 0)]:
            _both(vb.morphology, O.morphology, a, op, shape, ks, it, what=f"morph {dt} op{op} {ks} it{it}")


def test_morphology_large_element():
    g = natural(61, 97, 1)
    _both(vb.morphology, O.morphology, g, 0, 2, (61, 41), 1, what="morph big ellipse")
    _both(vb.morphology, O.morphology, g, 1, 0, (255, 3), 1, what="morph 255 wide")


# ------------------------------------------------------- device tensors

def test_device_tensors_match_host_path():
    import torch
    from visar_b200 import synth
    img = synth.base_image(480, 640, 3, seed=0)
    t = torch.from_numpy(img).cuda()
    g_dev = vb.cvt_color(t, 6)
    b_dev = vb.gaussian_blur(g_dev, (5, 5), 0)
    _, th_dev = vb.threshold(b_dev, 127, 255, 0)
    e_dev = vb.morphology(th_dev, 0, 0, (3, 3))
    d_dev = vb.morphology(e_dev, 1, 0, (3, 3))
    g = O.cvt_color(img, 6)
    b = O.gaussian_blur(g, (5, 5), 0)
    _, th = O.threshold(b, 127, 255, 0)
    e = O.morphology(th, 0, 0, (3, 3))
    d = O.morphology(e, 1, 0, (3, 3))
    for dev, ref in [(g_dev, g), (b_dev, b), (th_dev, th), (e_dev, e), (d_dev, d)]:
        assert_same(dev.cpu().numpy(), ref)


def test_device_in_place_and_views():
    import torch
    a = natural(64, 80, 3)
    t = torch.from_numpy(a).cuda()
    ref = O.gaussian_blur(a, (7, 7), 0)
    vb.gaussian_blur(t, (7, 7), 0, dst=t)  # src == dst on the device
    assert_same(t.cpu().numpy(), ref)
    big = torch.from_numpy(natural(100, 120, 1)).cuda()
    view = big[10:70, 5:90]
    out = vb.resize(view, (40, 30), 1)
    assert_same(out.cpu().numpy(), O.resize(np.ascontiguousarray(big.cpu().numpy()[10:70, 5:90]), (40, 30), 1))


def test_error_codes_match_oracle():
    a = natural(8, 8, 3)
    bad = [
        lambda m: m.cvt_color(a, 99),
        lambda m: m.gaussian_blur(a, (4, 4), 0),
        lambda m: m.gaussian_blur(a, (3, 3), 0, border=9),
        lambda m: m.gaussian_blur(a, (3, 3), 0, dst=np.empty((8, 9, 3), np.uint8)),
        lambda m: m.resize(a, (4, 4), 4),
        lambda m: m.morphology(a, 9, 0, (3, 3)),
        lambda m: m.morphology(a, 0, 0, (0, 3)),
        lambda m: m.threshold(a, 0, 255, 8),
        lambda m: m.warp_affine(a, np.zeros((2, 3)), (8, 8)),
        lambda m: m.sobel(a, np.int16, 1, 0, 4),
        lambda m: m.box_filter(a, (4, 3)),
        lambda m: m.cvt_color(natural(8, 8, 1), 6),
    ]
    for i, f in enumerate(bad):
        with pytest.raises(vb.VisarError) as e1:
            f(vb)
        with pytest.raises(O.OracleError) as e2:
            f(O)
        assert (e1.value.status, e1.value.name) == (e2.value.status, e2.value.name), f"case {i}"


# ------------------------------------------------- fast-path coverage

@pytest.mark.parametrize("cn", [1, 4])
@pytest.mark.parametrize("h,w", [(37, 53), (64, 130), (1, 9), (9, 1), (200, 257)])
def test_morphology_fast_shapes(cn, h, w):
    a = natural(h, w, cn)
    for shape in (0, 1, 2):
        for kw, kh in [(3, 3), (5, 5), (7, 7), (9, 9), (3, 5), (5, 3), (9, 3), (1, 7), (7, 1)]:
            for op in (0, 1, 2, 3):
                _both(vb.morphology, O.morphology, a, op, shape, (kw, kh), what=f"morph c{cn} op{op} sh{shape} {kw}x{kh}")


@pytest.mark.parametrize("cn", [1, 3, 4])
@pytest.mark.parametrize("h,w", [(33, 67), (8, 5), (130, 509)])
def test_fast_filters_odd_widths(cn, h, w):
    for dt in (np.uint8, np.float32):
        a = natural(h, w, cn, dt)
        for k in (3, 5, 7):
            for border in (0, 1, 2, 4):
                _both(vb.gaussian_blur, O.gaussian_blur, a, (k, k), 0, 0, border, exact_f32=True,
                      what=f"gauss fast {dt} c{cn} k{k} b{border} {w}x{h}")


def test_fast_paths_unaligned_views_fall_back():
    big = natural(90, 131, 1)
    v = big[3:80, 1:120]  # row starts not 4-byte aligned
    _both(vb.gaussian_blur, O.gaussian_blur, np.ascontiguousarray(v), (5, 5), 0, what="contig")
    _both(vb.gaussian_blur, O.gaussian_blur, v, (5, 5), 0, what="unaligned view")
    _both(vb.morphology, O.morphology, v, 2, 2, (5, 5), what="unaligned morph")
    _both(vb.resize, O.resize, v, (59, 38), 1, what="unaligned resize")


@pytest.mark.parametrize("cn", [1, 2, 3, 4])
def test_resize_half_and_linear_vector_paths(cn):
    for h, w in [(64, 128), (62, 130), (2, 8), (10, 18), (1081, 1921)]:
        a = natural(h, w, cn)
        _both(vb.resize, O.resize, a, (w // 2, h // 2), 1, what=f"half c{cn} {w}x{h}")
        _both(vb.resize, O.resize, a, (w // 2, h // 2), 3, what=f"area half c{cn} {w}x{h}")
        _both(vb.resize, O.resize, a, (max(1, w * 2 // 3), max(1, h * 2 // 3)), 1, what=f"lin c{cn} {w}x{h}")
