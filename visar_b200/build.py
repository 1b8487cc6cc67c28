"""Builds libvisar_b200.so (the C ABI of include/visar.h) in-tree for sm_100a.

Device code is compiled with --fmad=false so that no multiply-add is fused
unless the source asks for it (fmaf/fma), which keeps f32 results in VISAR's
operation order; host code gets -ffp-contract=off for the same reason.

Usage: python visar_b200/build.py [--force]   (the package import needs the built library)
"""
import os
import re
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libvisar_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "--fmad=false", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
                     "-Xptxas", "-O3", "--expt-relaxed-constexpr"]
CXX_FLAGS = ["-O2", "-fPIC", "-std=c++17", "-ffp-contract=off", "-fno-fast-math", "-I/usr/local/cuda/include"]


def _sources():
    out = []
    for f in sorted(os.listdir(CSRC)):
        if f.endswith((".cu", ".cpp")):
            out.append(os.path.join(CSRC, f))
    return out


_INCLUDE = re.compile(r'^\s*#\s*include\s+"([^"]+)"', re.M)


def _deps_mtime(src, seen=None):
    """Newest modification time of src and the local headers it includes (recursively)."""
    seen = set() if seen is None else seen
    m = os.path.getmtime(src)
    with open(src, errors="replace") as f:
        text = f.read()
    for name in _INCLUDE.findall(text):
        for d in (os.path.dirname(src), CSRC, os.path.join(HERE, "..", "include")):
            path = os.path.normpath(os.path.join(d, name))
            if os.path.exists(path):
                if path not in seen:
                    seen.add(path)
                    m = max(m, _deps_mtime(path, seen))
                break
    return m


def _compile(src, force):
    obj = os.path.join(OBJ, os.path.basename(src) + ".o")
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= _deps_mtime(src):
        return obj, None
    if src.endswith(".cu"):
        cmd = [NVCC] + NVCC_FLAGS + ["-c", src, "-o", obj]
    else:
        cmd = ["g++"] + CXX_FLAGS + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, f"$ {' '.join(cmd)}\n{r.stdout}{r.stderr}"
    return obj, None


def build(force=False, verbose=False):
    """Compiles every source under csrc/ and links libvisar_b200.so; returns its path."""
    os.makedirs(OBJ, exist_ok=True)
    srcs = _sources()
    # The slowest units first, so that they do not start last.
    srcs.sort(key=lambda f: -os.path.getsize(f) if "strip" not in f else -1e9)
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        results = list(ex.map(lambda s: _compile(s, force), srcs))
    errs = [e for _, e in results if e]
    if errs:
        raise RuntimeError("visar_b200 build failed:\n" + "\n".join(errs))
    objs = [o for o, _ in results]
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-Xcompiler", "-fPIC"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"visar_b200 link failed:\n$ {' '.join(cmd)}\n{r.stdout}{r.stderr}")
        if verbose:
            print("linked", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
