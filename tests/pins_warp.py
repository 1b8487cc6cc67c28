"""Analytic known answers for warpAffine / warpPerspective.

VISAR has no test of either warp. These cases are chosen so that every step
of its arithmetic is exact -- integer or dyadic source coordinates, weights
0, 1/2 or 1/4 -- and the result follows from the definitions alone
(geometry.zig:410-533 affine, :586-672 perspective):

* identity and integer translations: a copy of the source with the border
  rule applied per coordinate (constant border: the value);
* 90-degree rotations: numpy's rot90;
* half-pixel shifts and 2x zooms: averages of 2 or 4 samples rounded half to
  even (the affine fma chain and the perspective weight sum are both exact);
* a perspective matrix whose last row scales w (w = 2 or 1/2): the same
  zoom / decimation through the per-pixel divide;
* nearest neighbour on a half-pixel shift: the affine kernel rounds the
  coordinate half to even (sat.rint), the perspective one half away from zero
  (@round), so the two differ there on purpose.

`check_all(module)` runs every case through `module` (the oracle or the CUDA
binding, same call shapes) and returns a list of failures.
"""
import numpy as np


def border_map(p, n, b):
    """border.map (border.zig:22-37) in closed form (BORDER_CONSTANT: None)."""
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


def _sample(src, x, y, border, value):
    """src[y, x] with the border rule (float64 per channel)."""
    mx = border_map(x, src.shape[1], border)
    my = border_map(y, src.shape[0], border)
    c = 1 if src.ndim == 2 else src.shape[2]
    if mx is None or my is None:
        return np.full(c, value, np.float64)
    return np.asarray(src[my, mx], np.float64).reshape(c)


def _round_even(v, dtype):
    if dtype == np.float32:
        return v.astype(np.float32)
    info = np.iinfo(dtype)
    return np.clip(np.rint(v), info.min, info.max).astype(dtype)


def expected_linear(src, dw, dh, inv, border, value):
    """Bilinear at source coordinates sx = inv[0]*x + inv[1]*y + inv[2] (and sy
    likewise), with exact dyadic weights, rounded half to even."""
    c = 1 if src.ndim == 2 else src.shape[2]
    out = np.empty((dh, dw, c), np.float64)
    for y in range(dh):
        for x in range(dw):
            sx = inv[0] * x + inv[1] * y + inv[2]
            sy = inv[3] * x + inv[4] * y + inv[5]
            x0, y0 = int(np.floor(sx)), int(np.floor(sy))
            ax, ay = sx - x0, sy - y0
            if border == 0 and (x0 < -1 or y0 < -1 or x0 >= src.shape[1] or y0 >= src.shape[0]):
                out[y, x] = value
                continue
            p00 = _sample(src, x0, y0, border, value)
            p01 = _sample(src, x0 + 1, y0, border, value)
            p10 = _sample(src, x0, y0 + 1, border, value)
            p11 = _sample(src, x0 + 1, y0 + 1, border, value)
            out[y, x] = (p00 * (1 - ax) * (1 - ay) + p01 * ax * (1 - ay) + p10 * (1 - ax) * ay + p11 * ax * ay)
    out = _round_even(out, src.dtype)
    return out.reshape((dh, dw) if src.ndim == 2 else (dh, dw, c))


def expected_nearest(src, dw, dh, inv, border, value, half_even):
    c = 1 if src.ndim == 2 else src.shape[2]
    out = np.empty((dh, dw, c), np.float64)
    for y in range(dh):
        for x in range(dw):
            sx = inv[0] * x + inv[1] * y + inv[2]
            sy = inv[3] * x + inv[4] * y + inv[5]
            if half_even:
                ix, iy = int(np.rint(sx)), int(np.rint(sy))
            else:
                ix = int(np.sign(sx) * np.floor(abs(sx) + 0.5))
                iy = int(np.sign(sy) * np.floor(abs(sy) + 0.5))
            out[y, x] = _sample(src, ix, iy, border, value)
    out = out.astype(src.dtype)
    return out.reshape((dh, dw) if src.ndim == 2 else (dh, dw, c))


def affine(a, b, c, d, e, f):
    """A forward 2x3 matrix and its exact inverse (for the diagonal or
    permutation matrices used here)."""
    m = np.array([[a, b, c], [d, e, f]], np.float64)
    full = np.vstack([m, [0, 0, 1]])
    inv = np.linalg.inv(full)
    return m, inv[:2].ravel()


def _image(h, w, cn, dtype, seed):
    rng = np.random.default_rng(seed)
    if dtype == np.float32:
        x = rng.integers(-300, 300, size=(h, w, cn)).astype(np.float32) / 4.0
    elif dtype == np.uint16:
        x = rng.integers(0, 65536, size=(h, w, cn)).astype(np.uint16)
    else:
        x = rng.integers(0, 256, size=(h, w, cn)).astype(np.uint8)
    return x[..., 0] if cn == 1 else x


def cases():
    """(name, src, dsize, forward 2x3 (or None), forward 3x3 (or None),
    inverse as [6], interpolation, border, value, expected or None)."""
    out = []
    for cn, dtype in [(1, np.uint8), (3, np.uint8), (4, np.uint8), (1, np.float32), (3, np.uint16)]:
        src = _image(23, 31, cn, dtype, seed=cn * 7 + (dtype == np.float32))
        h, w = src.shape[:2]
        mats = [
            ("identity", affine(1, 0, 0, 0, 1, 0), (w, h)),
            ("shift+3-2", affine(1, 0, 3, 0, 1, -2), (w, h)),
            ("shift-5+4", affine(1, 0, -5, 0, 1, 4), (w, h)),
            ("rot90", affine(0, 1, 0, -1, 0, w - 1), (h, w)),
            ("rot270", affine(0, -1, h - 1, 1, 0, 0), (h, w)),
            ("half-x", affine(1, 0, 0.5, 0, 1, 0), (w, h)),
            ("half-xy", affine(1, 0, -0.5, 0, 1, 0.5), (w, h)),
            ("zoom2", affine(2, 0, 0, 0, 2, 0), (2 * w, 2 * h)),
            ("zoom2+shift", affine(2, 0, 0.5, 0, 2, -1.25), (2 * w + 3, 2 * h - 1)),
            ("half-scale", affine(0.5, 0, 0, 0, 0.5, 0), (w // 2, h // 2)),
        ]
        for name, (m, inv), (dw, dh) in mats:
            for border in (0, 1, 2, 3, 4):
                value = 0.0 if border else (77.0 if dtype != np.float32 else -2.5)
                exp = expected_linear(src, dw, dh, inv, border, value)
                H = np.vstack([m, [0, 0, 1]])
                out.append((f"{name}/c{cn}/{np.dtype(dtype).name}/b{border}", src, (dw, dh), m, H, 1, border, value, exp))
            exp_n = expected_nearest(src, dw, dh, inv, 1, 0.0, True)
            out.append((f"{name}/nearest-affine/c{cn}/{np.dtype(dtype).name}", src, (dw, dh), m, None, 0, 1, 0.0, exp_n))
            exp_p = expected_nearest(src, dw, dh, inv, 1, 0.0, False)
            H = np.vstack([m, [0, 0, 1]])
            out.append((f"{name}/nearest-persp/c{cn}/{np.dtype(dtype).name}", src, (dw, dh), None, H, 0, 1, 0.0, exp_p))
        # Perspective divides: H = diag(1, 1, s) maps (x, y) to (x/s, y/s).
        for s, (dw, dh), inv in [(0.5, (2 * w, 2 * h), [0.5, 0, 0, 0, 0.5, 0]), (2.0, (w // 2, h // 2), [2, 0, 0, 0, 2, 0])]:
            H = np.diag([1.0, 1.0, s])
            for border in (0, 1, 4):
                exp = expected_linear(src, dw, dh, inv, border, 0.0)
                out.append((f"persp-w{s}/c{cn}/{np.dtype(dtype).name}/b{border}", src, (dw, dh), None, H, 1, border, 0.0, exp))
    return out


def check_all(M):
    """Runs every case through module M; returns the failures (name, kind, n)."""
    bad = []
    for name, src, dsize, m, H, interp, border, value, exp in cases():
        if m is not None:
            got = M.warp_affine(src, m, dsize, interp, border, value)
            if not np.array_equal(np.asarray(got), exp):
                bad.append((name, "affine", int((np.asarray(got) != exp).sum())))
        if H is not None:
            got = M.warp_perspective(src, H, dsize, interp, border, value)
            if not np.array_equal(np.asarray(got), exp):
                bad.append((name, "perspective", int((np.asarray(got) != exp).sum())))
    return bad
