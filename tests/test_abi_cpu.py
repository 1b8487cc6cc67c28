"""The C-ABI library without a GPU: it loads, exports every function that
include/visar.h declares, and rejects bad arguments with VISAR's status codes
and error names (src/capi.zig:61-80) before touching the device."""
import ctypes
import os
import re

import numpy as np
import pytest

import visar_b200 as vb
from conftest import natural
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for fn in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not fn.endswith(".h"):
            continue
        txt = open(os.path.join(ROOT, "include", fn)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        names += re.findall(r"^[A-Za-z_][\w \*]*?\b(visar_\w+)\s*\(", txt, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_function():
    names = declared_functions()
    assert len(names) >= 18
    lib = ctypes.CDLL(vb.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_version_and_threads():
    assert vb.version()
    vb.set_num_threads(3)
    assert vb.lib.visar_get_num_threads() == 3
    vb.set_num_threads(0)
    assert vb.lib.visar_get_num_threads() >= 1


BAD = [
    ("cvt code", lambda m, a: m.cvt_color(a, 99)),
    ("cvt channels", lambda m, a: m.cvt_color(a[..., 0].copy(), 6)),
    ("cvt size", lambda m, a: m.cvt_color(a, 6, dst=np.empty((8, 9), np.uint8))),
    ("gauss even", lambda m, a: m.gaussian_blur(a, (4, 4), 0)),
    ("gauss big", lambda m, a: m.gaussian_blur(a, (129, 3), 0)),
    ("gauss border", lambda m, a: m.gaussian_blur(a, (3, 3), 0, border=9)),
    ("gauss neg", lambda m, a: m.gaussian_blur(a, (-1, 3), 0)),
    ("gauss size", lambda m, a: m.gaussian_blur(a, (3, 3), 0, dst=np.empty((8, 9, 3), np.uint8))),
    ("gauss depth", lambda m, a: m.gaussian_blur(a, (3, 3), 0, dst=np.empty((8, 8, 3), np.float32))),
    ("resize interp", lambda m, a: m.resize(a, (4, 4), 7)),
    ("resize lanczos", lambda m, a: m.resize(a, (4, 4), 4)),
    ("resize channels", lambda m, a: m.resize(a, (4, 4), 1, dst=np.empty((4, 4), np.uint8))),
    ("morph op", lambda m, a: m.morphology(a, 9, 0, (3, 3))),
    ("morph shape", lambda m, a: m.morphology(a, 0, 5, (3, 3))),
    ("morph size", lambda m, a: m.morphology(a, 0, 0, (0, 3))),
    ("morph 256", lambda m, a: m.morphology(a, 0, 0, (256, 3))),
    ("morph iter", lambda m, a: m.morphology(a, 0, 0, (3, 3), -1)),
    ("thresh otsu 3ch", lambda m, a: m.threshold(a, 0, 255, 8)),
    ("thresh type", lambda m, a: m.threshold(a, 0, 255, 6)),
    ("affine singular", lambda m, a: m.warp_affine(a, np.zeros((2, 3)), (8, 8))),
    ("affine border", lambda m, a: m.warp_affine(a, np.eye(2, 3), (8, 8), 1, 7)),
    ("persp singular", lambda m, a: m.warp_perspective(a, np.zeros((3, 3)), (8, 8))),
    ("sobel ksize", lambda m, a: m.sobel(a, np.int16, 1, 0, 4)),
    ("sobel order", lambda m, a: m.sobel(a, np.int16, 3, 0, 3)),
    ("sobel neg", lambda m, a: m.sobel(a, np.int16, -1, 0, 3)),
    ("sobel f32->i16", lambda m, a: m.sobel(a.astype(np.float32), np.int16, 1, 0, 3)),
    ("box even", lambda m, a: m.box_filter(a, (4, 3))),
    ("box zero", lambda m, a: m.box_filter(a, (0, 3))),
    ("sep even", lambda m, a: m.sep_filter_2d(a, np.uint8, [1, 1], [1])),
    ("depth i32", lambda m, a: m.gaussian_blur(a.astype(np.int32), (3, 3), 0)),
]


@pytest.mark.parametrize("name,f", BAD, ids=[b[0] for b in BAD])
def test_invalid_arguments_match_oracle(name, f):
    a = natural(8, 8, 3)
    with pytest.raises(O.OracleError) as ref:
        f(O, a)
    with pytest.raises(vb.VisarError) as ours:
        f(vb, a)
    assert (ours.value.status, ours.value.name) == (ref.value.status, ref.value.name)


def test_descriptor_checks():
    a = natural(8, 8, 3)
    d = vb.desc(a)
    null = vb.Image(8, 8, 3, 0, 24, None)
    assert vb.lib.visar_cvt_color(ctypes.byref(null), ctypes.byref(d), 6) == -1
    odd = vb.Image(8, 8, 1, 5, 33, a.ctypes.data)  # stride not a multiple of 4
    out = vb.Image(8, 8, 1, 5, 32, a.ctypes.data)
    assert vb.lib.visar_gaussian_blur(ctypes.byref(odd), ctypes.byref(out), 3, 3, ctypes.c_double(0), ctypes.c_double(0), 4) == -1
    short = vb.Image(8, 8, 3, 0, 10, a.ctypes.data)  # stride < row bytes
    assert vb.lib.visar_gaussian_blur(ctypes.byref(short), ctypes.byref(d), 3, 3, ctypes.c_double(0), ctypes.c_double(0), 4) == -1
    assert vb.lib.visar_last_error() == b"InvalidSize"


def test_no_cpu_fallback_without_gpu():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    a = natural(8, 8, 3)
    with pytest.raises(vb.VisarError) as e:
        vb.gaussian_blur(a, (3, 3), 0)
    assert e.value.status == -6 and e.value.name.startswith("CudaError")


def test_tuning_table_reader(tmp_path):
    """visar_tune_load reads the autotuner's flat JSON (string entries are
    descriptions and are skipped); NULL restores the built-in defaults."""
    from visar_b200 import batch as B
    p = tmp_path / "t.json"
    p.write_text('{"_device": "NVIDIA B200", "_sms": 148, "_workload": "w",\n'
                 ' "gauss_strip.u8.c1.k5.L.rows": 32, "gray.u8.c3.k0.M.vec": 8, "x.per_sm": -1}\n')
    try:
        B.tune_load(str(p))
        assert B.tune_get("gauss_strip.u8.c1.k5.L.rows") == 32
        assert B.tune_get("gray.u8.c3.k0.M.vec") == 8
        assert B.tune_get("x.per_sm") == -1
        assert B.tune_get("_sms") == 148
        assert B.tune_get("_device", 7) == 7
        B.tune_set("half.u8.c1.k0.S.vec", 8)
        assert B.tune_get("half.u8.c1.k0.S.vec") == 8
        B.tune_load(None)
        assert B.tune_get("gauss_strip.u8.c1.k5.L.rows", -5) == -5
        bad = tmp_path / "bad.json"
        bad.write_text('{"a": "unterminated')
        with pytest.raises(vb.VisarError):
            B.tune_load(str(bad))
        with pytest.raises(vb.VisarError):
            B.tune_load(str(tmp_path / "missing.json"))
    finally:
        B.tune_load(None)
