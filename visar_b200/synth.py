"""Seeded synthetic images with the shapes and value distributions of the
benchmark workloads (VISAR publishes no dataset for this path).

base_image: a horizontal gradient 0..255 across the width (same in every
channel) plus uniform integer noise in [-20, 20], clamped to 0..255, with
filled axis-aligned rectangles of random colour, 20-160 px per side.
"""
import numpy as np


def base_image(h, w, c=3, nrect=8, seed=0, dtype=np.uint8):
    rng = np.random.default_rng(seed)
    x = np.arange(w, dtype=np.float64)
    grad = np.rint(x * 255.0 / max(w - 1, 1)).astype(np.int32)
    noise = rng.integers(-20, 21, size=(h, w, c), dtype=np.int32)
    img = np.clip(grad[None, :, None] + noise, 0, 255).astype(np.uint8)
    for _ in range(nrect):
        rw = int(rng.integers(20, 161))
        rh = int(rng.integers(20, 161))
        x0 = int(rng.integers(0, max(1, w - rw + 1)))
        y0 = int(rng.integers(0, max(1, h - rh + 1)))
        col = rng.integers(0, 256, size=c, dtype=np.int32).astype(np.uint8)
        img[y0:y0 + rh, x0:x0 + rw] = col
    if c == 1:
        img = img[:, :, 0]
    if dtype == np.uint8:
        return np.ascontiguousarray(img)
    if dtype == np.uint16:
        return img.astype(np.uint16) * 257
    if dtype == np.int16:
        return img.astype(np.int16) - 128
    if dtype == np.float32:
        return img.astype(np.float32) / 255.0
    raise ValueError(dtype)


def normal_f32(h, w, c=1, seed=0):
    """float32 N(0, 1) samples (the f32 Gaussian workload)."""
    rng = np.random.default_rng(seed)
    shape = (h, w) if c == 1 else (h, w, c)
    return rng.standard_normal(shape, dtype=np.float32)


def rotation_matrix_2d(cx, cy, angle_deg, scale):
    """OpenCV's getRotationMatrix2D (angle in degrees, counter-clockwise)."""
    a = angle_deg * np.pi / 180.0
    alpha = np.cos(a) * scale
    beta = np.sin(a) * scale
    return np.array([[alpha, beta, (1 - alpha) * cx - beta * cy],
                     [-beta, alpha, beta * cx + (1 - alpha) * cy]], np.float64)


def affine_params(w, h, seed):
    """A seeded rotation +-30 deg, scale 0.8-1.2 about the centre, plus +-50 px translation."""
    rng = np.random.default_rng(seed)
    ang = rng.uniform(-30, 30)
    sc = rng.uniform(0.8, 1.2)
    m = rotation_matrix_2d(w / 2.0, h / 2.0, ang, sc)
    m[0, 2] += rng.uniform(-50, 50)
    m[1, 2] += rng.uniform(-50, 50)
    return m


def homography_from_corners(src_pts, dst_pts):
    """The 3x3 homography mapping 4 source corners to 4 destination corners (f64 DLT solve)."""
    a = []
    b = []
    for (x, y), (u, v) in zip(src_pts, dst_pts):
        a.append([x, y, 1, 0, 0, 0, -u * x, -u * y])
        b.append(u)
        a.append([0, 0, 0, x, y, 1, -v * x, -v * y])
        b.append(v)
    h = np.linalg.solve(np.array(a, np.float64), np.array(b, np.float64))
    return np.append(h, 1.0).reshape(3, 3)


def perspective_params(w, h, seed, jitter=80.0):
    """Each image corner jittered uniformly by +-jitter px; the homography from the jittered corners."""
    rng = np.random.default_rng(seed)
    src = [(0.0, 0.0), (w - 1.0, 0.0), (w - 1.0, h - 1.0), (0.0, h - 1.0)]
    dst = [(x + rng.uniform(-jitter, jitter), y + rng.uniform(-jitter, jitter)) for x, y in src]
    return homography_from_corners(src, dst)


def mixed_shapes(n=256, seed=2, wmin=64, wmax=4096, hmin=64, hmax=2160, channels=(1, 3)):
    """(height, width, channels) of the mixed-size batch: uniform integer sides, channels drawn uniformly."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        w = int(rng.integers(wmin, wmax + 1))
        h = int(rng.integers(hmin, hmax + 1))
        c = int(channels[int(rng.integers(0, len(channels)))])
        out.append((h, w, c))
    return out


def base_image_torch(h, w, c=3, nrect=8, seed=0, device="cuda"):
    """base_image's recipe generated on the device (for large batches); a uint8 torch tensor."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    x = torch.arange(w, device=device, dtype=torch.float64)
    grad = torch.round(x * 255.0 / max(w - 1, 1)).to(torch.int32)
    noise = torch.randint(-20, 21, (h, w, c), generator=g, device=device, dtype=torch.int32)
    img = (grad[None, :, None] + noise).clamp_(0, 255).to(torch.uint8)
    rng = np.random.default_rng(seed)
    for _ in range(nrect):
        rw = int(rng.integers(20, 161))
        rh = int(rng.integers(20, 161))
        x0 = int(rng.integers(0, max(1, w - rw + 1)))
        y0 = int(rng.integers(0, max(1, h - rh + 1)))
        col = torch.as_tensor(rng.integers(0, 256, size=c).astype(np.uint8), device=device)
        img[y0:y0 + rh, x0:x0 + rw] = col
    if c == 1:
        img = img[:, :, 0]
    return img.contiguous()


class VideoScene:
    """The video workload's scene: a diagonal gradient background with
    per-frame Gaussian noise (sigma 4), and 16 filled rectangles and ellipses
    (sides uniform 40-400 px, random colours) moving at constant velocities
    of +-12 px/frame and bouncing off the frame borders. frame(k) renders
    frame k on the device (u8, H x W x 3)."""

    def __init__(self, h=2160, w=3840, nobj=16, seed=3):
        rng = np.random.default_rng(seed)
        self.h, self.w, self.seed = h, w, seed
        self.objs = []
        for _ in range(nobj):
            ow, oh = int(rng.integers(40, 401)), int(rng.integers(40, 401))
            self.objs.append({
                "ellipse": bool(rng.integers(0, 2)), "w": ow, "h": oh,
                "x0": float(rng.uniform(0, max(1, w - ow))), "y0": float(rng.uniform(0, max(1, h - oh))),
                "vx": float(rng.uniform(-12, 12)), "vy": float(rng.uniform(-12, 12)),
                "col": rng.integers(0, 256, size=3).astype(np.uint8)})
        self._bg = None

    @staticmethod
    def _bounce(p0, v, k, span):
        # Position after k frames of constant velocity, reflected at 0 and span.
        if span <= 0:
            return 0.0
        p = (p0 + v * k) % (2 * span)
        return p if p <= span else 2 * span - p

    def frame(self, k, device="cuda"):
        import torch
        h, w = self.h, self.w
        if self._bg is None:
            yy = torch.arange(h, device=device, dtype=torch.float32)[:, None]
            xx = torch.arange(w, device=device, dtype=torch.float32)[None, :]
            self._bg = (xx + yy) * (255.0 / max(1, w + h - 2))
        g = torch.Generator(device=device)
        g.manual_seed(self.seed * 100003 + k)
        noise = torch.randn((h, w, 3), generator=g, device=device, dtype=torch.float32) * 4.0
        img = (self._bg[:, :, None] + noise).round_().clamp_(0, 255).to(torch.uint8)
        for o in self.objs:
            x = int(self._bounce(o["x0"], o["vx"], k, w - o["w"]))
            y = int(self._bounce(o["y0"], o["vy"], k, h - o["h"]))
            col = torch.as_tensor(o["col"], device=device)
            if not o["ellipse"]:
                img[y:y + o["h"], x:x + o["w"]] = col
            else:
                ry, rx = o["h"] / 2.0, o["w"] / 2.0
                yy = torch.arange(o["h"], device=device, dtype=torch.float32)[:, None] + 0.5 - ry
                xx = torch.arange(o["w"], device=device, dtype=torch.float32)[None, :] + 0.5 - rx
                m = (yy / ry) ** 2 + (xx / rx) ** 2 <= 1.0
                sub = img[y:y + o["h"], x:x + o["w"]]
                sub[m[:sub.shape[0], :sub.shape[1]]] = col
        return img.contiguous()


SERVED_STAGES = ("gray", "gauss", "resize", "affine", "open")


def served_requests(n, seed=4, mp_min=0.1, mp_max=8.3):
    """The served workload's requests: pixel count log-uniform in
    [mp_min, mp_max] MP, aspect ratio uniform 0.5-2.0, 1 / 3 / 4 channels,
    u8 (80%) or f32 N(0,1) (20%), and a pipeline of 1-4 stages drawn
    uniformly from gray, GaussianBlur 5x5, resize linear 0.5x, warpAffine
    with a random +-30 degree rotation about the centre, and OPEN 3x3 rect.
    Returns dicts with h, w, c, dtype ('u8' / 'f32'), seed and stages, each a
    (name, params) pair."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        px = float(np.exp(rng.uniform(np.log(mp_min * 1e6), np.log(mp_max * 1e6))))
        aspect = float(rng.uniform(0.5, 2.0))
        w = max(8, int(round(np.sqrt(px * aspect))))
        h = max(8, int(round(px / w)))
        c = int(rng.choice([1, 3, 4]))
        dtype = "f32" if rng.uniform() < 0.2 else "u8"
        stages = []
        for _ in range(int(rng.integers(1, 5))):
            name = SERVED_STAGES[int(rng.integers(0, len(SERVED_STAGES)))]
            params = {}
            if name == "affine":
                params["angle"] = float(rng.uniform(-30, 30))
            stages.append((name, params))
        out.append({"h": h, "w": w, "c": c, "dtype": dtype, "seed": seed * 100003 + k, "stages": stages})
    return out


def served_image(r, device="cuda"):
    """The input image of a served_requests entry, on the device."""
    import torch
    if r["dtype"] == "u8":
        return base_image_torch(r["h"], r["w"], r["c"], nrect=4, seed=r["seed"], device=device)
    g = torch.Generator(device=device)
    g.manual_seed(int(r["seed"]))
    shape = (r["h"], r["w"]) if r["c"] == 1 else (r["h"], r["w"], r["c"])
    return torch.randn(shape, generator=g, device=device, dtype=torch.float32)
