"""The served form (include/visar_serve.h).

Every request's result must equal its pipeline run through the per-call
entry points (u8 bit for bit, f32 within 1e-5 relative), whether the request
ran alone or batched with others; the plain mode gives the same results;
admission keeps a small pool within bounds; trace replay completes every
request.
"""
import numpy as np
import pytest

import visar_b200 as vb
from visar_b200 import batch as B
from visar_b200 import serve as S
from visar_b200 import synth

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def rotation(r, angle):
    h, w = r["h"], r["w"]
    return synth.rotation_matrix_2d(w / 2.0, h / 2.0, angle, 1.0)


def stage_list(r):
    out = []
    for name, p in r["stages"]:
        if name == "gray":
            out.append(B.gray())
        elif name == "gauss":
            out.append(B.gaussian((5, 5), 0.0, 0.0, 4))
        elif name == "resize":
            out.append(B.resize(0.5, 0.5, 1))
        elif name == "affine":
            out.append(B.warp_affine(rotation(r, p["angle"]), 1, 0, 0.0))
        else:
            out.append(B.morphology(2, 0, (3, 3), 1))
    return out


def plain_pipeline(r, x):
    for name, p in r["stages"]:
        c = 1 if x.ndim == 2 else x.shape[2]
        if name == "gray":
            if c > 1:
                x = vb.cvt_color(x, 6 if c == 3 else 10)
        elif name == "gauss":
            x = vb.gaussian_blur(x, (5, 5), 0, 0, 4)
        elif name == "resize":
            h, w = max(1, x.shape[0] // 2), max(1, x.shape[1] // 2)
            if (h, w) != tuple(x.shape[:2]):
                x = vb.resize(x, (w, h), 1)
        elif name == "affine":
            x = vb.warp_affine(x, rotation(r, p["angle"]), (x.shape[1], x.shape[0]), 1, 0, 0.0)
        else:
            x = vb.morphology(x, 2, 0, (3, 3), 1)
    return x


def same(a, b, f32):
    if a.shape != b.shape:
        return False
    if not f32:
        return torch.equal(a, b)
    return bool(((a - b).abs() <= 1e-5 * b.abs().clamp(min=1.0)).all())


def check(reqs, imgs, outs):
    for r, x, y in zip(reqs, imgs, outs):
        ref = plain_pipeline(r, x)
        torch.cuda.synchronize()
        assert same(y, ref, r["dtype"] == "f32"), (r["h"], r["w"], r["c"], r["dtype"], r["stages"])


def small_requests(n, seed):
    return synth.served_requests(n, seed=seed, mp_min=0.01, mp_max=0.6)


def test_results_match_per_call_pipeline():
    reqs = small_requests(40, seed=11)
    imgs = [synth.served_image(r) for r in reqs]
    srv = S.Server(pool_bytes=2 << 30)
    try:
        ids = [srv.submit(x, stage_list(r)) for r, x in zip(reqs, imgs)]
        outs = [srv.wait(i).clone() for i in ids]
        for i in ids:
            srv.release(i)
        check(reqs, imgs, outs)
        st = srv.stats()
        assert st["completed"] == len(reqs) and st["released"] == len(reqs)
        assert st["launches"] > 0 and st["pool_used"] == 0
    finally:
        srv.close()


def test_same_result_alone_and_in_a_mix():
    reqs = small_requests(60, seed=12)
    imgs = [synth.served_image(r) for r in reqs]
    probe = list(range(len(reqs)))
    srv = S.Server(pool_bytes=2 << 30)
    try:
        alone = {}
        for k in probe:  # alone: nothing else in the server
            i = srv.submit(imgs[k], stage_list(reqs[k]))
            alone[k] = srv.wait(i).clone()
            srv.release(i)
        ids = [srv.submit(x, stage_list(r)) for r, x in zip(reqs, imgs)]  # the mix
        for k in probe:
            mixed = srv.wait(ids[k]).clone()
            assert same(mixed, alone[k], reqs[k]["dtype"] == "f32")
        for i in ids:
            srv.wait(i)
            srv.release(i)
        assert srv.stats()["mean_batch"] > 1.0  # requests did share launches
    finally:
        srv.close()


def test_plain_mode_matches():
    reqs = small_requests(16, seed=13)
    imgs = [synth.served_image(r) for r in reqs]
    srv = S.Server(pool_bytes=1 << 30, mode=S.PLAIN)
    try:
        ids = [srv.submit(x, stage_list(r)) for r, x in zip(reqs, imgs)]
        outs = [srv.wait(i).clone() for i in ids]
        for i in ids:
            srv.release(i)
        check(reqs, imgs, outs)
        assert srv.stats()["launches"] == 0
    finally:
        srv.close()


def test_admission_with_a_small_pool():
    reqs = small_requests(50, seed=14)
    imgs = [synth.served_image(r) for r in reqs]
    srv = S.Server(pool_bytes=64 << 20)
    try:
        ids = [srv.submit(x, stage_list(r)) for r, x in zip(reqs, imgs)]
        peak = 0
        outs = []
        for i in ids:
            outs.append(srv.wait(i).clone())
            peak = max(peak, srv.stats()["pool_used"])
            srv.release(i)
        assert peak <= 64 << 20
        check(reqs, imgs, outs)
    finally:
        srv.close()


def test_trace_replay_completes():
    reqs = small_requests(200, seed=15)
    imgs = [synth.served_image(r) for r in reqs]
    rng = np.random.default_rng(3)
    t = np.cumsum(rng.exponential(1.0 / 4000.0, size=len(reqs)))
    for mode in (S.BATCHED, S.PLAIN):
        srv = S.Server(pool_bytes=2 << 30, mode=mode)
        try:
            lat, el = srv.run_trace([(float(a), x, stage_list(r)) for a, x, r in zip(t, imgs, reqs)])
            assert (lat > 0).all() and el > 0
            st = srv.stats()
            assert st["completed"] == len(reqs) and st["released"] == len(reqs) and st["pool_used"] == 0
        finally:
            srv.close()


def test_device_error_fails_requests_and_later_submissions():
    # A completion check that returns a CUDA error (faked here: no GPU fault
    # is raised) fails every request not yet done with Internal and the
    # error's name, and every later submission the same way.
    reqs = small_requests(12, seed=16)
    imgs = [synth.served_image(r) for r in reqs]
    srv = S.Server(pool_bytes=1 << 30)
    try:
        srv.fake_round_error(700)  # cudaErrorIllegalAddress
        ids = [srv.submit(x, stage_list(r)) for r, x in zip(reqs, imgs)]
        failed = 0
        for i in ids:
            try:
                srv.wait(i)
            except vb.VisarError as e:
                assert e.status == -6 and "cudaErrorIllegalAddress" in e.name
                failed += 1
        assert failed >= 1
        late = srv.submit(imgs[0], stage_list(reqs[0]))
        with pytest.raises(vb.VisarError) as e:
            srv.wait(late)
        assert e.value.status == -6 and "cudaErrorIllegalAddress" in e.value.name
    finally:
        srv.close()
    # A new server on the same device is unaffected.
    srv = S.Server(pool_bytes=1 << 30)
    try:
        i = srv.submit(imgs[0], stage_list(reqs[0]))
        y = srv.wait(i).clone()
        srv.release(i)
        check(reqs[:1], imgs[:1], [y])
    finally:
        srv.close()
