"""visar_pyr_down / visar_pyr_up (src/imgproc/pyramid.zig) through the C ABI:
equal to the oracle bit for bit (f32 included: same sums, same order) and to
the direct 5x5 definitions of VISAR's pyramid tests, for every type, channel
count 1-5 and 20, border, odd and even sizes, 4K frames, strided views, and
the refusals of capi.zig:234-249."""
import numpy as np
import pytest

import pins_pyr as PP
from oracle import oracle as O

vb = pytest.importorskip("visar_b200")
torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

TYPES = [np.uint8, np.uint16, np.int16, np.float32]


def host(x):
    return x.cpu().numpy() if hasattr(x, "cpu") else np.asarray(x)


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("dtype", TYPES)
def test_small_against_oracle_and_definition(dtype):
    for w, h in [(1, 1), (2, 3), (5, 4), (37, 19), (70, 9), (129, 7), (300, 41)]:
        for cn in (1, 2, 3, 4, 5, 20):
            src = PP.fill_random(dtype, w, h, cn, w * 31 + cn)
            for b in (4, 2, 1, 3):
                want = O.pyr_down(src, b)
                got = host(vb.pyr_down(src, b))
                assert np.array_equal(got, want), ("down", w, h, cn, b)
                assert np.array_equal(host(vb.pyr_down(dev(src), b)), want)
            want = O.pyr_up(src, 4)
            assert np.array_equal(host(vb.pyr_up(src, 4)), want), ("up", w, h, cn)
            assert np.array_equal(host(vb.pyr_up(dev(src), 4)), want)
            if w * h <= 100 and cn <= 5:
                d = host(vb.pyr_up(src, 4)).reshape(2 * h, 2 * w, cn).astype(np.float64)
                r = PP.ref_up(src)
                assert (np.abs(d - r).max() <= 1e-5) if dtype == np.float32 else np.array_equal(d, r)


@pytest.mark.parametrize("dtype", TYPES)
def test_4k(dtype):
    rng = np.random.default_rng(3)
    for cn in (1, 3):
        if dtype == np.float32:
            src = rng.standard_normal((2160, 3840, cn), dtype=np.float32)
        else:
            info = np.iinfo(dtype)
            src = rng.integers(info.min, info.max + 1, (2160, 3840, cn)).astype(dtype)
        src = src[..., 0] if cn == 1 else src
        d = dev(src)
        assert np.array_equal(host(vb.pyr_down(d, 4)), O.pyr_down(src, 4)), (dtype, cn)
        small = np.ascontiguousarray(src[:540, :960])
        assert np.array_equal(host(vb.pyr_up(dev(small), 4)), O.pyr_up(small, 4)), (dtype, cn)


def test_strided_views_and_odd_offsets():
    base = PP.fill_random(np.uint8, 257, 131, 3, 11)
    d = dev(base)
    for y0, x0 in [(1, 1), (0, 3), (5, 0)]:
        v = np.ascontiguousarray(base[y0:, x0:])
        assert np.array_equal(host(vb.pyr_down(d[y0:, x0:], 2)), O.pyr_down(v, 2))
        assert np.array_equal(host(vb.pyr_up(d[y0:y0 + 40, x0:x0 + 61], 4)), O.pyr_up(np.ascontiguousarray(v[:40, :61]), 4))
    out = torch.zeros((80, 300), dtype=torch.uint8, device="cuda")
    g = dev(PP.fill_random(np.uint8, 50, 30, 1, 5)[..., 0])
    vb.pyr_up(g, 4, dst=out[3:63, 7:107])
    assert np.array_equal(out[3:63, 7:107].cpu().numpy(), O.pyr_up(g.cpu().numpy(), 4))
    out[3:63, 7:107] = 0
    assert int(out.sum()) == 0


def test_refusals():
    src = torch.zeros((50, 101), dtype=torch.uint8, device="cuda")
    z = lambda *s: torch.zeros(s, dtype=torch.uint8, device="cuda")  # noqa: E731
    for fn, dst, border, want in [(vb.pyr_down, z(13, 26), 4, -2), (vb.pyr_down, z(25, 51), 0, -3),
                                  (vb.pyr_up, z(100, 202), 1, -3), (vb.pyr_up, z(100, 201), 4, -2),
                                  (vb.pyr_down, z(25, 51), 5, -3), (vb.pyr_down, z(25, 51, 3), 4, -2)]:
        with pytest.raises(vb.VisarError) as e:
            fn(src, border, dst=dst)
        assert e.value.status == want, (fn.__name__, tuple(dst.shape), border)
    with pytest.raises(vb.VisarError) as e:
        vb.pyr_down(src, 4, dst=torch.zeros((25, 51), dtype=torch.float32, device="cuda"))
    assert e.value.status == -3
