"""visar_undistort, visar_init_undistort_rectify_map and visar_remap
(src/calib3d/undistort.zig) through the C ABI: bit-exact to the oracle on
1-4 channels, odd sizes, 4K frames, several stripes, host and device images;
remap on the exact dyadic known answers; undistort and the maps against cv2
4.13 as in the oracle's pins; the refusals of capi_calib3d.zig."""
import numpy as np
import pytest

import pins_calib as PC
from oracle import oracle as O

vb = pytest.importorskip("visar_b200")
torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def host(x):
    return x.cpu().numpy() if hasattr(x, "cpu") else np.asarray(x)


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("cn", [1, 2, 3, 4])
def test_undistort_maps_remap_against_oracle(cn):
    rng = np.random.default_rng(10 + cn)
    for w, h in [(640, 480), (97, 61), (1500, 1000), (4100, 9), (1, 1), (3840, 2160)]:
        img = rng.integers(0, 256, (h, w, cn), dtype=np.uint8)
        img = img[..., 0] if cn == 1 else img
        d_img = dev(img)
        for K0, dist, nk in PC.CAMERAS:
            K = PC.scaled_camera(K0, w, h)
            want = O.undistort(img, K, dist, nk)
            assert np.array_equal(host(vb.undistort(d_img, K, dist, nk)), want), (cn, w, h, dist)
            if w * h < 2e6:
                assert np.array_equal(vb.undistort(img, K, dist, nk), want), (cn, w, h, dist)
            mx, my = O.init_undistort_rectify_map(K, dist, None, nk, (w, h))
            gx, gy = vb.init_undistort_rectify_map(K, dist, None, nk, (w, h), like=d_img)
            assert np.array_equal(host(gx), mx) and np.array_equal(host(gy), my), (w, h, dist)
            for value in (0.0, 200.4):
                want_r = O.remap(img, mx, my, value)
                assert np.array_equal(host(vb.remap(d_img, gx, gy, value)), want_r), (cn, w, h, dist, value)


def test_maps_with_rotation_and_host_buffers():
    K = PC.scaled_camera(PC.CAMERAS[2][0], 800, 600)
    R = np.array([[0.999, -0.01, 0.02], [0.011, 0.9995, -0.005], [-0.02, 0.006, 0.9992]])
    for dist in ([], [0.1, -0.05, 0.001, 0.002], PC.CAMERAS[2][1]):
        mx, my = O.init_undistort_rectify_map(K, dist, R, PC.CAMERAS[2][2], (800, 600))
        gx, gy = vb.init_undistort_rectify_map(K, dist, R, PC.CAMERAS[2][2], (800, 600))
        assert np.array_equal(gx, mx) and np.array_equal(gy, my)


def test_undistort_against_cv2():
    import cv2
    rng = np.random.default_rng(4)
    for w, h in [(640, 480), (1500, 1000)]:
        img = rng.integers(0, 256, (h, w, 3), dtype=np.uint8)
        for K0, dist, nk in PC.CAMERAS:
            K = PC.scaled_camera(K0, w, h)
            ours = host(vb.undistort(dev(img), K, dist, nk))
            ref = cv2.undistort(img, K, np.array(dist) if dist else None, newCameraMatrix=nk)
            for y, x in {(int(a), int(b)) for a, b in np.argwhere((ours != ref).any(axis=2))}:
                u, v = PC.undistort_coord(K, dist, nk, w, h, x, y)
                assert PC.near_tie(u) or PC.near_tie(v), (w, h, dist, x, y)


def test_remap_known_answers():
    bad = []
    for name, src, mx, my, v, exp in PC.remap_cases():
        if not np.array_equal(host(vb.remap(dev(src), dev(mx), dev(my), v)), exp):
            bad.append(name)
        if not np.array_equal(vb.remap(src, mx, my, v), exp):
            bad.append(name + "/host")
    assert not bad, bad[:10]


def test_remap_strided_maps_and_views():
    rng = np.random.default_rng(8)
    img = rng.integers(0, 256, (300, 400, 3), dtype=np.uint8)
    K = PC.scaled_camera(PC.CAMERAS[0][0], 400, 300)
    mx, my = O.init_undistort_rectify_map(K, PC.CAMERAS[0][1], None, None, (400, 300))
    bigx = torch.zeros((300, 512), dtype=torch.float32, device="cuda")
    bigy = torch.zeros((300, 512), dtype=torch.float32, device="cuda")
    bigx[:, 5:405] = dev(mx)
    bigy[:, 5:405] = dev(my)
    d_img = dev(img)
    out = torch.zeros((310, 420, 3), dtype=torch.uint8, device="cuda")
    vb.remap(d_img, bigx[:, 5:405], bigy[:, 5:405], 0.0, dst=out[3:303, 7:407])
    assert np.array_equal(host(out[3:303, 7:407]), O.remap(img, mx, my, 0.0))
    out[3:303, 7:407] = 0
    assert int(out.sum()) == 0


def test_refusals():
    img = torch.zeros((20, 30, 3), dtype=torch.uint8, device="cuda")
    K = [40, 0, 15, 0, 40, 10, 0, 0, 1]
    with pytest.raises(vb.VisarError) as e:
        vb.undistort(img, K, [0.1, 0.2])
    assert e.value.status == -1
    with pytest.raises(vb.VisarError) as e:
        vb.undistort(img, K, [], dst=torch.zeros((20, 31, 3), dtype=torch.uint8, device="cuda"))
    assert e.value.status == -2
    with pytest.raises(vb.VisarError) as e:
        vb.init_undistort_rectify_map([0] * 9, [], None, None, (30, 20))
    assert e.value.status == -1
    mx = torch.zeros((20, 30), dtype=torch.float32, device="cuda")
    with pytest.raises(vb.VisarError) as e:
        vb.remap(img, mx, torch.zeros((20, 29), dtype=torch.float32, device="cuda"))
    assert e.value.status == -2
    with pytest.raises(vb.VisarError) as e:
        vb.remap(img, mx, mx, dst=torch.zeros((20, 30), dtype=torch.uint8, device="cuda"))
    assert e.value.status == -3
    with pytest.raises(vb.VisarError) as e:
        vb.remap(img, mx.to(torch.float16), mx.to(torch.float16))
    assert e.value.status == -3


def test_undistort_singular_stripe_keeps_rows():
    """A new camera matrix whose stripe camera is singular for one stripe
    (det is linear in the principal point: 500 * (2 - a5) here, zero for the
    stripe whose first row is cy - 2 = 20): those rows are left as they are,
    the others follow the projective map (a camera with a perspective row).
    The device inverts each stripe's camera as the oracle does."""
    h, w = 64, 1024  # 4 rows per stripe
    rng = np.random.default_rng(77)
    img = rng.integers(0, 256, (h, w, 3), dtype=np.uint8)
    K = np.array([[500.0, 0, 510], [0, 500.0, 30], [0, 0, 1]])
    new_k = np.array([[500.0, 0, 510], [0, 2.0, 22.0], [0, 1.0, 1.0]])
    dist = [-0.1, 0.01, 0.0, 0.0]
    ref = O.undistort(img, K, dist, new_k, dst=np.full((h, w, 3), 77, np.uint8))
    assert np.all(ref[20:24] == 77) and not np.all(ref == 77)
    d_dst = dev(np.full((h, w, 3), 77, np.uint8))
    vb.undistort(dev(img), K, dist, new_k, dst=d_dst)
    assert np.array_equal(host(d_dst), ref)
    h_dst = np.full((h, w, 3), 77, np.uint8)
    vb.undistort(img, K, dist, new_k, dst=h_dst)
    assert np.array_equal(h_dst, ref)
