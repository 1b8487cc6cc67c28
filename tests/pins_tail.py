"""Test images for the tracker tail: the mask patterns of VISAR's
connected-components test (components.zig:615-650: random, sparse, checker,
spiral, stripes, zeros, ones, diag) at its sizes, drawn with NumPy's RNG, and
a NumPy restatement of the background model (track.zig:33-81)."""
import numpy as np

CC_SIZES = [(1, 1), (1, 300), (300, 1), (37, 129), (200, 257), (64, 64), (33, 400)]  # (w, h)
PATTERNS = ["random", "sparse", "checker", "spiral", "stripes", "zeros", "ones", "diag"]


def cc_pattern(w, h, pat, rng):
    y, x = np.mgrid[0:h, 0:w]
    if pat == "random":
        m = rng.integers(0, 10, (h, w)) < 5
    elif pat == "sparse":
        m = rng.integers(0, 10, (h, w)) == 0
    elif pat == "checker":
        m = (x + y) % 2 == 0
    elif pat == "stripes":
        m = (x % 3 == 0) | (y % 50 == 0)
    elif pat == "zeros":
        m = np.zeros((h, w), bool)
    elif pat == "ones":
        m = np.ones((h, w), bool)
    elif pat == "diag":
        m = ((x + y) % 7 == 0) | ((x + 2 * h - y) % 11 == 0)
    else:  # spiral: concentric square rings with one gap each
        d = np.minimum(np.minimum(x, y), np.minimum(w - 1 - x, h - 1 - y))
        m = (d % 2 == 0) & ~((x == d + 1) & (y == d) & (d + 2 < w))
    return (m * 255).astype(np.uint8)


def _background(frames, shift, t):
    model = None
    out = []
    for f in frames:
        fv = f.astype(np.int64)
        if model is None:
            model = fv << 8
            out.append(np.zeros_like(f))
            continue
        fg = np.abs(fv - (model >> 8)) > t
        out.append(np.where(fg, 255, 0).astype(np.uint8))
        sh = np.where(fg, shift + 2, shift)
        model = model + (((fv << 8) - model) >> sh)
    return out, model.astype(np.uint16)


def background_ref(frames, shift, t):
    """The masks the model gives for a sequence of gray frames."""
    return _background(frames, shift, t)[0]


def background_model(frames, shift, t):
    """The model after a sequence of gray frames."""
    return _background(frames, shift, t)[1]
