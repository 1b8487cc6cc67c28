"""The oracle against the committed golden fixtures (OpenCV outputs on the
seeded benchmark images, generated by tests/golden/make_golden.py). CPU only:
it pins the checker that the GPU parity tests rely on."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
import sys
sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
from make_golden import cases, digest, small_cases  # noqa: E402

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
GOLD = json.load(open(os.path.join(HERE, "golden.json")))["cases"]
NAMES = [c[0] for c in cases()]


@pytest.mark.parametrize("name", NAMES)
def test_oracle_matches_golden_digest(name):
    _, build, op = next(c for c in cases() if c[0] == name)
    assert digest(op(O, build())) == GOLD[name]


def test_oracle_matches_golden_arrays():
    arrs = np.load(os.path.join(HERE, "golden.npz"))
    sc = small_cases()
    assert np.array_equal(arrs["in_u8"], sc["in_u8"]) and np.array_equal(arrs["in_f32"], sc["in_f32"])
    for k, v in sc.items():
        if k.startswith("in_"):
            continue
        src, op, tol = v
        ours = op(O, arrs[src]).astype(np.float64)
        ref = arrs[k].astype(np.float64)
        err = np.abs(ours - ref)
        if tol < 1:
            err = err / np.maximum(1.0, np.abs(ref))
        assert err.max() <= tol, (k, err.max())
