"""Direct definitions of pyrDown / pyrUp (pyramid.zig:583-605, the reference
functions of VISAR's own pyramid tests) and its test images."""
import numpy as np

K5 = np.array([1, 4, 6, 4, 1], np.float64)


def border_map(p, n, b):
    """border.map (border.zig:22-37), closed form; BORDER_CONSTANT is never used here."""
    if 0 <= p < n:
        return p
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


def fill_random(dtype, w, h, cn, seed0):
    """fillRandom (pyramid.zig:607-621): u32 LCG, r = (seed >> 12) & 0xFFFF."""
    n = w * h * cn
    out = np.empty(n, np.uint32)
    s = seed0 & 0xFFFFFFFF
    for i in range(n):
        s = (s * 1103515245 + 12345) & 0xFFFFFFFF
        out[i] = (s >> 12) & 0xFFFF
    if dtype == np.uint8:
        v = (out & 0xFF).astype(np.uint8)
    elif dtype == np.uint16:
        v = out.astype(np.uint16)
    elif dtype == np.int16:
        v = out.astype(np.uint16).view(np.int16)
    else:
        v = (out.astype(np.float32) / np.float32(65536.0)).astype(np.float32)
    return v.reshape(h, w, cn)


def ref_down(src, b):
    """refDown: the 5x5 sum over border-mapped source coordinates; integers
    floor((s + 128) / 256), f32 s / 256 (compared within 1e-5)."""
    h, w, cn = src.shape
    dh, dw = (h + 1) // 2, (w + 1) // 2
    ys = np.array([[border_map(2 * y + j - 2, h, b) for j in range(5)] for y in range(dh)])
    xs = np.array([[border_map(2 * x + i - 2, w, b) for i in range(5)] for x in range(dw)])
    S = src.astype(np.float64)[ys][:, :, xs]
    s = (S * K5[None, :, None, None, None] * K5[None, None, None, :, None]).sum(axis=(1, 3))
    return s / 256 if src.dtype == np.float32 else np.floor((s + 128) / 256)


def ref_up(src):
    """refUp: the 5x5 kernel over the zero-upsampled image reflected about its
    own edges (reflect101 in upsampled coordinates); integers floor((s + 32) / 64)."""
    h, w, cn = src.shape
    out = np.zeros((2 * h, 2 * w, cn), np.float64)
    f = src.astype(np.float64)
    for y in range(2 * h):
        uys = [border_map(y + j - 2, 2 * h, 4) for j in range(5)]
        for x in range(2 * w):
            uxs = [border_map(x + i - 2, 2 * w, 4) for i in range(5)]
            s = np.zeros(cn)
            for j, uy in enumerate(uys):
                if uy % 2:
                    continue
                for i, ux in enumerate(uxs):
                    if ux % 2:
                        continue
                    s += f[uy // 2, ux // 2] * K5[i] * K5[j]
            out[y, x] = s
    return out / 64 if src.dtype == np.float32 else np.floor((out + 32) / 64)


def down_f32_scalar(src, b):
    """pyramid.zig:646-672: the f32 scalar formula, every step in f32:
    p_i = ((r0 + r4) + (r1 + r3) * 4) + r2 * 6 per tap column, then the same
    over p, times 1/256."""
    h, w, cn = src.shape
    dh, dw = (h + 1) // 2, (w + 1) // 2
    f = np.float32
    ys = np.array([[border_map(2 * y + k - 2, h, b) for k in range(5)] for y in range(dh)])
    xs = np.array([[border_map(2 * x + i - 2, w, b) for i in range(5)] for x in range(dw)])
    r = [src[ys[:, k]][:, xs] for k in range(5)]  # (dh, dw, 5, cn)
    p = (((r[0] + r[4]).astype(f) + ((r[1] + r[3]).astype(f) * f(4)).astype(f)).astype(f) + (r[2] * f(6)).astype(f)).astype(f)
    q = [p[:, :, i] for i in range(5)]
    v = (((q[0] + q[4]).astype(f) + ((q[1] + q[3]).astype(f) * f(4)).astype(f)).astype(f) + (q[2] * f(6)).astype(f)).astype(f)
    return (v * f(1.0 / 256.0)).astype(f)
