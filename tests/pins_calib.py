"""Cases for undistort / initUndistortRectifyMap / remap (src/calib3d/undistort.zig).

undistort and the f32 maps follow OpenCV's undistort / initUndistortRectifyMap
arithmetic (VISAR says bit for bit, undistort.zig:1-11), which cv2 4.13 shares,
so cv2 is their external pin. remap follows OpenCV 5's float kernel (OpenCV 4
remaps CV_32FC1 maps with INTER_BITS tables), so it is pinned by the exact
known answers of pins_warp through maps built from the same dyadic matrices."""
import numpy as np

import pins_warp

CAMERAS = [
    # (K, dist, new_k)
    (np.array([[500.0, 0, 320], [0, 510.0, 240], [0, 0, 1]]), [0.1, -0.05, 0.001, 0.002], None),
    (np.array([[500.0, 0, 320], [0, 510.0, 240], [0, 0, 1]]), [0.1, -0.05, 0.001, 0.002, 0.01], None),
    (np.array([[620.0, 0, 300.5], [0, 600.0, 250.25], [0, 0, 1]]), [-0.3, 0.12, -0.002, 0.001, -0.02, 0.05, -0.01, 0.003],
     np.array([[560.0, 0, 310], [0, 555.0, 245], [0, 0, 1]])),
    (np.array([[40.0, 0, 18], [0, 40.0, 11], [0, 0, 1]]), [], None),
]


def scaled_camera(K, w, h, w0=640, h0=480):
    """K for an image of w x h from one made for w0 x h0."""
    s = np.diag([w / w0, h / h0, 1.0])
    return s @ K


def remap_cases():
    """(name, src, mapx, mapy, value, expected) from pins_warp's dyadic affine
    cases with a constant border: map = the inverse matrix applied to (x, y)."""
    out = []
    for name, src, (dw, dh), m, H, interp, border, value, exp in pins_warp.cases():
        if m is None or interp != 1 or border != 0 or src.dtype != np.uint8:
            continue
        full = np.vstack([m, [0, 0, 1]])
        inv = np.linalg.inv(full)[:2]
        yy, xx = np.mgrid[0:dh, 0:dw].astype(np.float64)
        mx = (inv[0, 0] * xx + inv[0, 1] * yy + inv[0, 2]).astype(np.float32)
        my = (inv[1, 0] * xx + inv[1, 1] * yy + inv[1, 2]).astype(np.float32)
        v = int(round(value))
        out.append((name, src, mx, my, float(value), pins_warp.expected_linear(src, dw, dh, inv.ravel(), 0, float(v))))
    return out


def _inv3(a):
    a = list(np.asarray(a, np.float64).ravel())
    det = a[0] * (a[4] * a[8] - a[7] * a[5]) - a[1] * (a[3] * a[8] - a[6] * a[5]) + a[2] * (a[3] * a[7] - a[6] * a[4])
    d = 1 / det
    return [(a[4] * a[8] - a[5] * a[7]) * d, (a[2] * a[7] - a[1] * a[8]) * d, (a[1] * a[5] - a[2] * a[4]) * d,
            (a[5] * a[6] - a[3] * a[8]) * d, (a[0] * a[8] - a[2] * a[6]) * d, (a[2] * a[3] - a[0] * a[5]) * d,
            (a[3] * a[7] - a[4] * a[6]) * d, (a[1] * a[6] - a[0] * a[7]) * d, (a[0] * a[4] - a[1] * a[3]) * d]


def undistort_coord(K, dist, new_k, w, h, x, y, R=None, stripes=True):
    """The f64 source coordinate (u, v) undistort (stripes=True) or the map
    (stripes=False, rotation R) computes for destination pixel (x, y)
    (undistort.zig:44-81, 214-236), in Python floats (f64, each operation
    rounded on its own)."""
    K = list(np.asarray(K, np.float64).ravel())
    k = list(dist) + [0.0] * (8 - len(dist))
    ar = list(np.asarray(new_k if new_k is not None else K, np.float64).ravel())
    y0 = 0
    if stripes:
        stripe = min(max(1, 4096 // max(w, 1)), h)
        y0 = (y // stripe) * stripe
        ar[5] = ar[5] - float(y0)
    if R is not None:
        r = list(np.asarray(R, np.float64).ravel())
        ar = [ar[i * 3] * r[j] + ar[i * 3 + 1] * r[3 + j] + ar[i * 3 + 2] * r[6 + j] for i in range(3) for j in range(3)]
    ir = _inv3(ar)
    i, j = float(y - y0), float(x)
    X = (i * ir[1] + ir[2]) + j * ir[0]
    Y = (i * ir[4] + ir[5]) + j * ir[3]
    if not (ir[6] == 0 and ir[7] == 0 and ir[8] == 1):
        wv = 1.0 / ((i * ir[7] + ir[8]) + j * ir[6])
        X, Y = X * wv, Y * wv
    x2, y2 = X * X, Y * Y
    r2 = x2 + y2
    xy2 = 2 * X * Y
    kr = 1 + ((k[4] * r2 + k[1]) * r2 + k[0]) * r2
    if k[5] != 0 or k[6] != 0 or k[7] != 0:
        kr /= 1 + ((k[7] * r2 + k[6]) * r2 + k[5]) * r2
    xd = X * kr + k[2] * xy2 + k[3] * (r2 + 2 * x2)
    yd = Y * kr + k[2] * (r2 + 2 * y2) + k[3] * xy2
    return K[0] * xd + K[2], K[4] * yd + K[5]


def near_tie(c, eps=1e-6):
    """True when c * 32 lies within eps of a rounding boundary (n + 1/2)."""
    f = c * 32 - np.floor(c * 32)
    return abs(f - 0.5) < eps


def f32_tie(c, a, b):
    """True when the f64 value c lies within 1e-9 (relative) of the midpoint of
    the neighbouring f32 values a and b (either rounding is then one ulp)."""
    return abs(float(a) - float(b)) <= 2 * float(np.spacing(np.float32(max(abs(a), abs(b))))) and \
        abs(c - (float(a) + float(b)) / 2) <= 1e-9 * max(1.0, abs(c))
