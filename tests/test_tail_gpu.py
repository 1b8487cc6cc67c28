"""The tracker's per-frame tail through the C ABI: equalizeHist,
adaptiveThreshold, the background model and connectedComponentsWithStats,
each equal to the oracle (labels, stats and centroids exactly) on host and
device images, on VISAR's test patterns, large masks and the refusals of
capi.zig."""
import numpy as np
import pytest

import pins_tail as PT
from conftest import natural
from oracle import oracle as O

vb = pytest.importorskip("visar_b200")
torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def host(x):
    return x.cpu().numpy() if hasattr(x, "cpu") else np.asarray(x)


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_equalize_hist():
    rng = np.random.default_rng(1)
    imgs = [np.array([[10, 10, 20, 30]], np.uint8), natural(480, 640, 1), rng.integers(40, 90, (37, 53), dtype=np.uint8),
            np.full((5, 7), 9, np.uint8), rng.integers(0, 256, (2160, 3840), dtype=np.uint8)]
    for img in imgs:
        want = O.equalize_hist(img)
        assert np.array_equal(vb.equalize_hist(img), want)
        assert np.array_equal(host(vb.equalize_hist(dev(img))), want)


def test_adaptive_threshold():
    g = natural(480, 640, 1)
    for method in (0, 1):
        for kind in (0, 1):
            for block, delta in [(3, 0.0), (11, 2.5), (31, -3.2), (5, 7.0)]:
                want = O.adaptive_threshold(g, 200.4, method, kind, block, delta)
                assert np.array_equal(vb.adaptive_threshold(g, 200.4, method, kind, block, delta), want)
                assert np.array_equal(host(vb.adaptive_threshold(dev(g), 200.4, method, kind, block, delta)), want)
    for h, w in [(1, 9), (7, 1), (1, 1)]:
        a = natural(h, w, 1)
        for method in (0, 1):
            assert np.array_equal(vb.adaptive_threshold(a, 255, method, 0, 5, 1.0), O.adaptive_threshold(a, 255, method, 0, 5, 1.0))


def test_adaptive_threshold_refusals():
    g = dev(natural(20, 30, 1))
    for args in [(255, 2, 0, 3, 0), (255, 0, 2, 3, 0), (255, 0, 0, 1, 0), (255, 0, 0, 4, 0)]:
        with pytest.raises(vb.VisarError) as e:
            vb.adaptive_threshold(g, *args)
        assert e.value.status == -1, args
    with pytest.raises(vb.VisarError) as e:
        vb.adaptive_threshold(dev(natural(20, 30, 3)), 255, 0, 0, 3, 0)
    assert e.value.status == -3


def test_background_model():
    rng = np.random.default_rng(5)
    for h, w in [(60, 80), (1080, 1920)]:
        frames = [np.clip(natural(h, w, 1).astype(int) + rng.integers(-40, 40, (h, w)), 0, 255).astype(np.uint8)
                  for _ in range(5)]
        for shift, t in [(4, 28), (0, 5)]:
            ob = O.Background(w, h, shift)
            gb = vb.Background(w, h, shift)
            gh = vb.Background(w, h, shift)
            for f in frames:
                want = ob.apply(f, t)
                assert np.array_equal(host(gb.apply(dev(f), t)), want)
                assert np.array_equal(gh.apply(f, t), want)
            gb.close()
            gh.close()
    bg = vb.Background(80, 60, 4)
    with pytest.raises(vb.VisarError) as e:
        bg.apply(dev(np.zeros((61, 80), np.uint8)), 10)
    assert e.value.status == -2
    with pytest.raises(vb.VisarError):
        vb.Background(8, 8, 16)


def check_cc(img, conn):
    n, lab, st, ce = O.connected_components(img, conn)
    for src in (img, dev(img)):
        n2, lab2, st2, ce2 = vb.connected_components(src, conn)
        assert n2 == n
        assert np.array_equal(host(lab2), lab)
        assert np.array_equal(st2, st)
        assert np.array_equal(np.isnan(ce2), np.isnan(ce)) and np.allclose(ce2, ce, rtol=0, atol=0, equal_nan=True)


@pytest.mark.parametrize("conn", [4, 8])
def test_components_reference_patterns(conn):
    rng = np.random.default_rng(42)
    for w, h in PT.CC_SIZES:
        for pat in PT.PATTERNS:
            check_cc(PT.cc_pattern(w, h, pat, rng), conn)


@pytest.mark.parametrize("conn", [4, 8])
def test_components_large_masks(conn):
    rng = np.random.default_rng(7)
    for w, h, pat in [(1920, 1080, "random"), (1920, 1080, "sparse"), (960, 540, "spiral"), (1023, 777, "checker")]:
        check_cc(PT.cc_pattern(w, h, pat, rng), conn)
    # A tracker-like mask: blobs from thresholding a blurred noise field.
    f = rng.standard_normal((1080, 1920)).astype(np.float32)
    b = O.gaussian_blur(f, (31, 31), 8.0, 0, 4)
    check_cc(((b > 0.02) * 255).astype(np.uint8), conn)


def test_components_stats_rows_and_refusals():
    img = PT.cc_pattern(64, 64, "random", np.random.default_rng(3))
    n, lab, st, ce = O.connected_components(img, 8)
    n2, lab2, st2, ce2 = vb.connected_components(dev(img), 8, max_stats=5)
    assert n2 == n and st2.shape == (5, 5) and np.array_equal(st2, st[:5])
    with pytest.raises(vb.VisarError) as e:
        vb.connected_components(dev(img), 8, labels=torch.zeros((64, 63), dtype=torch.int32, device="cuda"))
    assert e.value.status == -2
    with pytest.raises(vb.VisarError) as e:
        vb.connected_components(dev(img), 8, labels=torch.zeros((64, 64), dtype=torch.float32, device="cuda"))
    assert e.value.status == -3
