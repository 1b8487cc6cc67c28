"""visar_gray_downsample (src/videoio/frame.zig:169-335) through the C ABI:
bit-exact to the oracle for BGR and BGRA at every factor 1-16, on host and
device images, strided and unaligned views, a window of the output computed
alone (frame.zig:418-446's property), and the refusals of capi.zig:176-182."""
import numpy as np
import pytest

from oracle import oracle as O

vb = pytest.importorskip("visar_b200")
torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def rand(h, w, cn, seed):
    return np.random.default_rng(seed).integers(0, 256, (h, w, cn), dtype=np.uint8)


@pytest.mark.parametrize("cn", [3, 4])
def test_every_factor_small(cn):
    for k in range(1, 17):
        src = rand(9 * k + k // 2, 70 * k + 1 + k // 3, cn, seed=k * 10 + cn)
        want = O.gray_downsample(src, k)
        assert np.array_equal(vb.gray_downsample(src, k), want), (cn, k)
        d = vb.gray_downsample(torch.from_numpy(src).cuda(), k)
        assert np.array_equal(d.cpu().numpy(), want), (cn, k)


@pytest.mark.parametrize("cn", [3, 4])
def test_4k_frames(cn):
    src = rand(2160, 3840, cn, seed=cn)
    d_src = torch.from_numpy(src).cuda()
    for k in range(2, 17):
        want = O.gray_downsample(src, k)
        assert np.array_equal(vb.gray_downsample(d_src, k).cpu().numpy(), want), (cn, k)


def test_strided_and_unaligned_views():
    base = rand(301, 517, 4, seed=5)
    d_base = torch.from_numpy(base).cuda()
    for k in (1, 2, 3, 5, 16):
        for y0, x0 in [(0, 1), (3, 7), (1, 0)]:
            view = base[y0:, x0:]
            want = O.gray_downsample(np.ascontiguousarray(view), k)
            got = vb.gray_downsample(d_base[y0:, x0:], k)
            assert np.array_equal(got.cpu().numpy(), want), (k, y0, x0)
            assert np.array_equal(vb.gray_downsample(view, k), want), (k, y0, x0)
    bgr = rand(120, 333, 3, seed=6)
    for k in (2, 4, 7):
        out = torch.zeros((200, 256), dtype=torch.uint8, device="cuda")
        dst = out[7:7 + 120 // k, 3:3 + 333 // k]
        vb.gray_downsample(torch.from_numpy(bgr).cuda(), k, dst=dst)
        assert np.array_equal(dst.cpu().numpy(), O.gray_downsample(bgr, k))
        out[7:7 + 120 // k, 3:3 + 333 // k] = 0
        assert int(out.sum()) == 0  # nothing written outside the view


def test_window_equals_whole_image():
    # frame.zig:418-446: the k x k blocks under a window of the output give
    # that window of the whole-image result.
    rng = np.random.default_rng(9)
    for cn in (3, 4):
        for k in (1, 2, 3, 5, 6, 8):
            src = torch.from_numpy(rand(23 * k + 1, 61 * k + 3, cn, seed=k * 7 + cn)).cuda()
            whole = vb.gray_downsample(src, k)
            H, W = whole.shape
            for _ in range(10):
                x = int(rng.integers(0, W))
                y = int(rng.integers(0, H))
                w = 1 + int(rng.integers(0, W - x))
                h = 1 + int(rng.integers(0, H - y))
                got = vb.gray_downsample(src[y * k:(y + h) * k, x * k:(x + w) * k], k)
                assert torch.equal(got, whole[y:y + h, x:x + w]), (cn, k, x, y, w, h)


def test_refusals():
    src = torch.zeros((40, 50, 3), dtype=torch.uint8, device="cuda")
    for k, shape, want in [(0, (40, 50), -1), (-3, (40, 50), -1), (17, (2, 2), -2), (2, (20, 24), -2),
                           (2, (20, 25, 3), -2)]:
        with pytest.raises(vb.VisarError) as e:
            vb.gray_downsample(src, k, dst=torch.zeros(shape, dtype=torch.uint8, device="cuda"))
        assert e.value.status == want, (k, shape)
    with pytest.raises(vb.VisarError) as e:
        vb.gray_downsample(torch.zeros((40, 50), dtype=torch.uint8, device="cuda"), 2)
    assert e.value.status == -2
    with pytest.raises(vb.VisarError) as e:
        vb.gray_downsample(torch.zeros((40, 50, 3), dtype=torch.float32, device="cuda"), 2,
                           dst=torch.zeros((20, 25), dtype=torch.float32, device="cuda"))
    assert e.value.status == -3
