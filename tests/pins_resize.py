"""Independent NumPy restatements used to pin resize and warp results.

Each kernel here is written from the formula it cites, with NumPy's IEEE
float32 operations standing in for Zig's unfused f32 arithmetic, so it checks
the C++ oracle and the CUDA library from outside both. Where OpenCV 4.13
(installed here) computes one step differently from VISAR, the same kernel is
given that step too: matching cv2 bit for bit with OpenCV's step and the
oracle bit for bit with VISAR's shows that the two differ only there.
"""
import numpy as np


def lcg_image(w, h, cn, seed):
    """VISAR's test images (resize.zig:657-663, :707-713): a u32 LCG
    seed = seed * 1103515245 + 12345, sample = (seed >> 16) & 0xFF, row-major."""
    n = w * h * cn
    out = np.empty(n, np.uint8)
    s = seed & 0xFFFFFFFF
    for i in range(n):
        s = (s * 1103515245 + 12345) & 0xFFFFFFFF
        out[i] = (s >> 16) & 0xFF
    return out.reshape((h, w) if cn == 1 else (h, w, cn))


def hash_image(w, h, cn):
    """resize.zig:687: sample i = ((i * 2654435761) mod 2^64 >> 7) & 0xFF."""
    i = np.arange(w * h * cn, dtype=np.uint64)
    v = ((i * np.uint64(2654435761)) >> np.uint64(7)) & np.uint64(0xFF)
    v = v.astype(np.uint8)
    return v.reshape((h, w) if cn == 1 else (h, w, cn))


# The destination sizes (w, h) of VISAR's resize property tests.
LINEAR_SIZES = [(75, 32), (300, 128), (113, 47), (120, 90), (112, 48), (37, 20), (20, 9), (9, 5), (199, 70),
                (151, 64), (1, 1), (2, 64), (112, 42), (100, 43), (225, 96), (141, 61), (6, 40)]  # resize.zig:668
NEAREST_SIZES = [(74, 22), (74, 31), (100, 40), (20, 5)]  # resize.zig:689
AREA_SIZES = [(53, 37), (64, 40), (30, 20), (13, 9), (11, 61), (97, 29), (7, 3), (1, 1), (2, 60), (96, 60)]  # :717


def _hwc(a):
    return a.reshape(a.shape[0], a.shape[1], -1)


def _back(r, like, h, w):
    return r.reshape((h, w) if like.ndim == 2 else (h, w, like.shape[2]))


def nearest_naive(src, dw, dh):
    """resize.zig:690-697: sx = min(w-1, floor(x * (w/dw))) in f64, same for y."""
    s = _hwc(src)
    h, w, _ = s.shape
    fx = w / dw
    fy = h / dh
    xs = np.minimum(w - 1, np.floor(np.arange(dw) * fx).astype(np.int64))
    ys = np.minimum(h - 1, np.floor(np.arange(dh) * fy).astype(np.int64))
    return _back(s[ys][:, xs], src, dh, dw)


def area_int_naive(src, fx, fy):
    """resize.zig:726-739: u32 block sum times f32(1 / (fx * fy)), cast with
    round half to even."""
    s = _hwc(src).astype(np.int64)
    h, w, cn = s.shape
    dh, dw = h // fy, w // fx
    tot = s[:dh * fy, :dw * fx].reshape(dh, fy, dw, fx, cn).sum(axis=(1, 3))
    scale = np.float32(1.0) / np.float32(fx * fy)
    v = (tot.astype(np.float32) * scale).astype(np.float32)
    return _back(np.clip(np.rint(v.astype(np.float64)), 0, 255).astype(np.uint8), src, dh, dw)


# ---------------------------------------------------------------- linear f32 / u16

def _linear_taps(dsize, ssize, f32_coords, pin):
    """Source index and weights per destination index. VISAR (linearCoord,
    resize.zig:155-178, Weights.coef :397-399): coordinate and fraction in f64,
    clamped at both ends on both axes, weights f32(1 - f), f32(f). OpenCV 4
    (f32_coords): the coordinate rounded to f32 first, weights 1.f - fx and fx
    in f32, and only x clamped (pin)."""
    scale = ssize / dsize
    idx = np.empty(dsize, np.int64)
    w0 = np.empty(dsize, np.float32)
    w1 = np.empty(dsize, np.float32)
    for d in range(dsize):
        if f32_coords:
            f = np.float32((d + 0.5) * scale - 0.5)
            s = int(np.floor(f))
            f = np.float32(f - np.float32(s))
            if pin and s < 0:
                s, f = 0, np.float32(0)
            if pin and s >= ssize - 1:
                s, f = ssize - 1, np.float32(0)
            idx[d], w0[d], w1[d] = s, np.float32(1) - f, f
        else:
            fx = (d + 0.5) * scale - 0.5
            s = int(np.floor(fx))
            f = fx - s
            if s < 0:
                s, f = 0, 0.0
            if s >= ssize - 1:
                s, f = ssize - 1, 0.0
            idx[d], w0[d], w1[d] = s, np.float32(1.0 - f), np.float32(f)
    return idx, w0, w1


def linear_generic(src, dw, dh, opencv4=False):
    """The generic bilinear kernel for f32 / u16 (resize.zig:284-423): hrow
    s0*a0 + s1*a1, vrow r0*b0 + r1*b1, each product and sum rounded to f32,
    then sat.cast. opencv4=True gives OpenCV 4's coordinates (see
    _linear_taps) and its copy of the edge sample where x is clamped."""
    s = _hwc(src).astype(np.float32)
    h, w, cn = s.shape
    xi, a0, a1 = _linear_taps(dw, w, opencv4, True)
    yi, b0, b1 = _linear_taps(dh, h, opencv4, False)
    x1 = np.minimum(xi + 1, w - 1)
    H = (s[:, xi] * a0[None, :, None]).astype(np.float32) + (s[:, x1] * a1[None, :, None]).astype(np.float32)
    H = H.astype(np.float32)
    if opencv4:
        cp = xi >= w - 1
        H[:, cp] = s[:, xi[cp]]
    r0 = np.clip(yi, 0, h - 1)
    r1 = np.clip(yi + 1, 0, h - 1)
    v = ((H[r0] * b0[:, None, None]).astype(np.float32) + (H[r1] * b1[:, None, None]).astype(np.float32)).astype(np.float32)
    if src.dtype == np.float32:
        out = v
    else:
        info = np.iinfo(src.dtype)
        out = np.clip(np.rint(v.astype(np.float64)), info.min, info.max).astype(src.dtype)
    return _back(out, src, dh, dw)


# ------------------------------------------------------------------- cubic u8

def _cubic_coeffs(x):
    """cubicCoeffs (resize.zig:632-640) in f32, A = -0.75."""
    f = np.float32
    x = f(x)
    A = f(-0.75)
    c0 = ((A * (x + f(1)) - f(5) * A) * (x + f(1)) + f(8) * A) * (x + f(1)) - f(4) * A
    c1 = ((A + f(2)) * x - (A + f(3))) * x * x + f(1)
    c2 = ((A + f(2)) * (f(1) - x) - (A + f(3))) * (f(1) - x) * (f(1) - x) + f(1)
    c3 = f(1) - c0 - c1 - c2
    return [f(c0), f(c1), f(c2), f(c3)]


def _cubic_tab(dsize, ssize):
    """cubicTab (resize.zig:262-277): f32 coordinate, 11-bit rounded weights,
    indices clamped to the image."""
    scale = 1.0 / (dsize / ssize)
    o = np.zeros((dsize, 4), np.int64)
    wt = np.zeros((dsize, 4), np.int64)
    for d in range(dsize):
        fx = np.float32((d + 0.5) * scale - 0.5)
        sx = np.floor(fx)
        fx = np.float32(fx - sx)
        cf = _cubic_coeffs(fx)
        for k in range(4):
            wt[d, k] = int(np.clip(np.rint(np.float64(np.float32(cf[k] * np.float32(2048)))), -32768, 32767))
            o[d, k] = min(max(int(sx) - 1 + k, 0), ssize - 1)
    return o, wt


def cubic_u8(src, dw, dh, vertical):
    """cubicU8: the integer horizontal pass, then the vertical pass chosen by
    `vertical`:
      "visar":  vcubic (resize_u8.zig:742-763), the fused f32 chain
                fma(s0, b0, fma(s1, b1, fma(s2, b2, s3 * b3))) with
                b = w * 2^-22, rounded half to even;
      "opencv4": OpenCV 4.13's portable build: the same chain without fusing
                over 16-sample groups, and (v + 2^21) >> 22 on the row's last
                rowLen % 16 samples."""
    s = _hwc(src).astype(np.int64)
    h, w, cn = s.shape
    xo, xw = _cubic_tab(dw, w)
    yo, yw = _cubic_tab(dh, h)
    H = sum(s[:, xo[:, k]] * xw[None, :, k, None] for k in range(4))
    S = [H[yo[:, k]] for k in range(4)]
    sc = np.float32(1.0 / (2048 * 2048))
    b = [(yw[:, k].astype(np.float32) * sc).astype(np.float32)[:, None, None] for k in range(4)]
    Sf = [x.astype(np.float32) for x in S]
    if vertical == "visar":
        # Every product of a sum below 2^24 and a weight that is a multiple of
        # 2^-22, and every partial sum, is exact in f64: one f32 rounding of
        # the f64 result is the fused multiply-add.
        v = (Sf[3].astype(np.float64) * b[3]).astype(np.float32)
        for k in (2, 1, 0):
            v = (Sf[k].astype(np.float64) * b[k].astype(np.float64) + v.astype(np.float64)).astype(np.float32)
        out = np.clip(np.rint(v.astype(np.float64)), 0, 255)
    else:
        v = (Sf[3] * b[3]).astype(np.float32)
        for k in (2, 1, 0):
            v = ((Sf[k] * b[k]).astype(np.float32) + v).astype(np.float32)
        body = np.clip(np.rint(v.astype(np.float64)), 0, 255).reshape(dh, dw * cn)
        V = sum(S[k] * yw[:, k, None, None] for k in range(4))
        tail = np.clip((V + (1 << 21)) >> 22, 0, 255).reshape(dh, dw * cn)
        cut = dw * cn - (dw * cn) % 16
        out = tail.copy()
        out[:, :cut] = body[:, :cut]
    return _back(out.astype(np.uint8), src, dh, dw)
