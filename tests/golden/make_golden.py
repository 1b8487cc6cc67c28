"""Generates the golden fixtures in this directory from OpenCV (cv2 4.13, IPP).

VISAR's differential suite (tests/py/test_core_vs_opencv.py in VISAR) holds
VISAR equal to OpenCV with tolerance 0 for u8/u16 colour, Gaussian, area
resize, threshold and morphology, and within 1 level for u8 linear/cubic
resize. The fixtures record OpenCV's outputs on the seeded benchmark images:

  golden.json  SHA-256 digests of exact-tolerance outputs (large images)
  golden.npz   full arrays of small tolerance cases (inputs and outputs)

Run from the repository root:  python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def digest(a):
    a = np.ascontiguousarray(a)
    return {"shape": list(a.shape), "dtype": str(a.dtype), "sha256": hashlib.sha256(a.tobytes()).hexdigest()}


def cases():
    """(name, input builder, op) triples shared by the generator and the test.
    op(m, x) calls module m (cv2-like wrapper or oracle) on input x."""
    from visar_b200 import synth
    c0 = lambda: synth.base_image(480, 640, 3, nrect=8, seed=0)  # noqa: E731
    c1 = lambda: synth.base_image(1080, 1920, 3, nrect=32, seed=1)  # noqa: E731
    gray = lambda: synth.base_image(480, 640, 1, nrect=8, seed=5)  # noqa: E731
    u16 = lambda: synth.base_image(240, 320, 3, nrect=6, seed=6, dtype=np.uint16)  # noqa: E731
    return [
        ("c0_gray", c0, lambda m, x: m.cvt_color(x, 6)),
        ("c0_gauss5", c0, lambda m, x: m.gaussian_blur(m.cvt_color(x, 6), (5, 5), 0)),
        ("c0_thresh127", c0, lambda m, x: m.threshold(m.gaussian_blur(m.cvt_color(x, 6), (5, 5), 0), 127, 255, 0)[1]),
        ("c0_erode3", c0, lambda m, x: m.morphology(
            m.threshold(m.gaussian_blur(m.cvt_color(x, 6), (5, 5), 0), 127, 255, 0)[1], 0, 0, (3, 3))),
        ("c0_dilate3", c0, lambda m, x: m.morphology(m.morphology(
            m.threshold(m.gaussian_blur(m.cvt_color(x, 6), (5, 5), 0), 127, 255, 0)[1], 0, 0, (3, 3)), 1, 0, (3, 3))),
        ("c1_area_960x540", c1, lambda m, x: m.resize(x, (960, 540), 3)),
        ("c1_area_640x360", c1, lambda m, x: m.resize(x, (640, 360), 3)),
        ("c1_area_1000x600", c1, lambda m, x: m.resize(x, (1000, 600), 3)),
        ("c1_gauss5_bgr", c1, lambda m, x: m.gaussian_blur(x, (5, 5), 0)),
        ("c1_gauss_s2.5", c1, lambda m, x: m.gaussian_blur(x, (0, 0), 2.5)),
        ("c1_hsv", c1, lambda m, x: m.cvt_color(x, 40)),
        ("c1_ycrcb", c1, lambda m, x: m.cvt_color(x, 36)),
        ("gray_open_ellipse5", gray, lambda m, x: m.morphology(x, 2, 2, (5, 5))),
        ("gray_close_rect7", gray, lambda m, x: m.morphology(x, 3, 0, (7, 7))),
        ("gray_gradient_cross3", gray, lambda m, x: m.morphology(x, 4, 1, (3, 3))),
        ("gray_otsu", gray, lambda m, x: m.threshold(x, 0, 255, 8)[1]),
        ("gray_triangle", gray, lambda m, x: m.threshold(x, 0, 255, 16)[1]),
        ("gray_box7", gray, lambda m, x: m.box_filter(x, (7, 7))),
        ("gray_sobel_dx", gray, lambda m, x: m.sobel(x, np.int16, 1, 0, 3)),
        ("u16_gauss7", u16, lambda m, x: m.gaussian_blur(x, (7, 7), 0)),
        ("u16_gauss_s1.7", u16, lambda m, x: m.gaussian_blur(x, (0, 0), 1.7)),
    ]


class CvShim:
    """cv2 behind the binding's call shapes."""

    def __init__(self):
        import cv2
        self.cv2 = cv2

    def cvt_color(self, x, code):
        return self.cv2.cvtColor(x, code)

    def gaussian_blur(self, x, k, s, sy=0, border=4):
        return self.cv2.GaussianBlur(x, k, s, sigmaY=sy, borderType=border)

    def threshold(self, x, t, m, kind):
        return self.cv2.threshold(x, t, m, kind)

    def morphology(self, x, op, shape, k, iterations=1):
        return self.cv2.morphologyEx(x, op, self.cv2.getStructuringElement(shape, k), iterations=iterations)

    def resize(self, x, size, interp):
        return self.cv2.resize(x, size, interpolation=interp)

    def box_filter(self, x, k):
        return self.cv2.blur(x, k)

    def sobel(self, x, ddepth, dx, dy, ks):
        return self.cv2.Sobel(x, self.cv2.CV_16S if ddepth == np.int16 else self.cv2.CV_32F, dx, dy, ksize=ks)


def small_cases():
    """Tolerance cases (VISAR's suite: linear/cubic u8 within 1, f32 within 1e-5), stored whole."""
    from visar_b200 import synth
    a = synth.base_image(61, 97, 3, nrect=3, seed=9)
    f = synth.normal_f32(48, 64, 1, seed=10)
    return {
        "in_u8": a, "in_f32": f,
        "linear_53x37": ("in_u8", lambda m, x: m.resize(x, (53, 37), 1), 1.0),
        "linear_150x90": ("in_u8", lambda m, x: m.resize(x, (150, 90), 1), 1.0),
        "cubic_53x37": ("in_u8", lambda m, x: m.resize(x, (53, 37), 2), 1.0),
        "cubic_150x90": ("in_u8", lambda m, x: m.resize(x, (150, 90), 2), 1.0),
        "gauss_f32_7x7_s1.5": ("in_f32", lambda m, x: m.gaussian_blur(x, (7, 7), 1.5), 1e-5),
    }


def main():
    cv = CvShim()
    out = {"generator": "tests/golden/make_golden.py", "source": f"cv2 {cv.cv2.__version__}", "cases": {}}
    for name, build, op in cases():
        out["cases"][name] = digest(op(cv, build()))
    with open(os.path.join(HERE, "golden.json"), "w") as fh:
        json.dump(out, fh, indent=1, sort_keys=True)
    sc = small_cases()
    arrays = {"in_u8": sc["in_u8"], "in_f32": sc["in_f32"]}
    for k, v in sc.items():
        if k.startswith("in_"):
            continue
        src, op, _tol = v
        arrays[k] = op(cv, sc[src])
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **arrays)
    print(f"wrote {len(out['cases'])} digests and {len(arrays)} arrays")


if __name__ == "__main__":
    main()
