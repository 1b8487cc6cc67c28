"""The batched form (include/visar_batch.h) against the per-call drop-in.

Every stage output of every image in a plan must equal, bit for bit, what
the per-call entry points give for that image alone (which the parity suite
holds equal to the oracle). Covers the mixed-size batch pipeline, a video
frame pipeline replayed through a CUDA graph with new frames, every depth and
channel count (including the images that take the per-call fallback), more
images than the shared-memory prefix cache holds, and every tuning choice.
"""
import numpy as np
import pytest

import visar_b200 as vb
from visar_b200 import batch as B
from visar_b200 import synth

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def dims_after_resize(h, w, fx, fy):
    return max(1, int(h * fy)), max(1, int(w * fx))


def plain_stage(x, spec):
    """One stage through the per-call entry points (the reference of the batch)."""
    kind, a = spec
    c = 1 if x.ndim == 2 else x.shape[2]
    if kind == "gray":
        return x if c == 1 else vb.cvt_color(x, 6 if c == 3 else 10)
    if kind == "gauss":
        return vb.gaussian_blur(x, a["k"], a.get("sx", 0.0), a.get("sy", 0.0), a.get("border", 4))
    if kind == "morph":
        return vb.morphology(x, a["op"], a["shape"], a["k"], a.get("it", 1))
    if kind == "resize":
        h, w = dims_after_resize(x.shape[0], x.shape[1], a["fx"], a["fy"])
        if (h, w) == tuple(x.shape[:2]):
            return x
        return vb.resize(x, (w, h), a.get("interp", 1))
    if kind == "thresh":
        return vb.threshold(x, a["t"], a["m"], a["type"])[1]
    if kind == "affine":
        return vb.warp_affine(x, a["m"][a["i"]], (x.shape[1], x.shape[0]), a.get("interp", 1), a.get("border", 0),
                              a.get("value", 0.0))
    if kind == "persp":
        return vb.warp_perspective(x, a["m"][a["i"]], (x.shape[1], x.shape[0]), a.get("interp", 1),
                                   a.get("border", 0), a.get("value", 0.0))
    raise ValueError(kind)


def batch_stage(spec):
    kind, a = spec
    if kind == "gray":
        return B.gray()
    if kind == "gauss":
        return B.gaussian(a["k"], a.get("sx", 0.0), a.get("sy", 0.0), a.get("border", 4))
    if kind == "morph":
        return B.morphology(a["op"], a["shape"], a["k"], a.get("it", 1))
    if kind == "resize":
        return B.resize(a["fx"], a["fy"], a.get("interp", 1))
    if kind == "thresh":
        return B.threshold(a["t"], a["m"], a["type"])
    if kind == "affine":
        return B.warp_affine(None, a.get("interp", 1), a.get("border", 0), a.get("value", 0.0),
                             per_image=np.stack(a["m"]))
    if kind == "persp":
        return B.warp_perspective(None, a.get("interp", 1), a.get("border", 0), a.get("value", 0.0),
                                  per_image=np.stack(a["m"]))
    raise ValueError(kind)


def check_plan(images, specs, graph=False, plan=None):
    plan = plan or B.Batch(images, [batch_stage(s) for s in specs])
    (plan.run_graph if graph else plan.run)()
    torch.cuda.synchronize()
    for i, x in enumerate(images):
        cur = x
        for k, s in enumerate(specs):
            if s[0] in ("affine", "persp"):
                s = (s[0], dict(s[1], i=i))
            cur = plain_stage(cur, s)
            got = plan.stage_output(k, i)
            assert tuple(got.shape) == tuple(cur.shape), (i, k, s[0])
            if not torch.equal(got, cur):
                bad = int((got != cur).sum())
                raise AssertionError(f"image {i} {tuple(x.shape)} {x.dtype} stage {k} {s[0]}: {bad} samples differ")
    return plan


def mixed_u8(n, seed, wmax=1200, hmax=700, channels=(1, 3)):
    shapes = synth.mixed_shapes(n, seed=seed, wmax=wmax, hmax=hmax, channels=channels)
    return [synth.base_image_torch(h, w, c, nrect=8, seed=seed * 1000 + k) for k, (h, w, c) in enumerate(shapes)]


C2 = [("gray", {}), ("gauss", {"k": (5, 5)}), ("morph", {"op": 2, "shape": 2, "k": (5, 5)}),
      ("resize", {"fx": 0.5, "fy": 0.5})]


def test_mixed_size_pipeline_matches_plain():
    imgs = mixed_u8(24, seed=3)
    # Degenerate and narrow shapes next to the large ones.
    imgs += [synth.base_image_torch(h, w, c, nrect=1, seed=50 + k)
             for k, (h, w, c) in enumerate([(1, 1, 1), (2, 3, 3), (64, 5, 1), (7, 300, 3), (3, 2, 1), (33, 17, 3)])]
    plan = check_plan(imgs, C2)
    info = plan.info()
    assert info["images"] == len(imgs) and info["stages"] == 4
    # One launch per shape class and pass: gray (3-ch), Gaussian (1-ch), erode + dilate, half + linear.
    assert info["launches"] <= 8
    check_plan(imgs, C2, graph=True, plan=plan)
    check_plan(imgs, C2, graph=True, plan=plan)


def test_mixed_batch_matches_oracle_directly():
    """The C2 pipeline's final outputs against the CPU oracle itself (not only
    through the per-call path), on a few uneven 1- and 3-channel images that
    include odd sizes (general bilinear) and even ones (exact halving)."""
    from oracle import oracle as O
    shapes = [(67, 91, 3), (120, 200, 1), (53, 64, 3), (96, 130, 1), (201, 77, 3)]
    imgs = [synth.base_image_torch(h, w, c, nrect=3, seed=700 + k) for k, (h, w, c) in enumerate(shapes)]
    plan = B.Batch(imgs, [batch_stage(s) for s in C2])
    plan.run_graph()
    torch.cuda.synchronize()
    for i, x in enumerate(imgs):
        a = x.cpu().numpy()
        y = a if a.ndim == 2 else O.cvt_color(a, 6)
        y = O.gaussian_blur(y, (5, 5), 0, 0, 4)
        y = O.morphology(y, 2, 2, (5, 5))
        h, w = dims_after_resize(y.shape[0], y.shape[1], 0.5, 0.5)
        if (h, w) != y.shape[:2]:
            y = O.resize(y, (w, h), 1)
        got = plan.output(i).cpu().numpy()
        assert got.shape == y.shape and np.array_equal(got, y), i


def test_video_frames_replayed_through_graph():
    h, w = 360, 640
    hom = synth.perspective_params(w, h, seed=7)
    specs = [("gray", {}), ("gauss", {"k": (5, 5)}), ("thresh", {"t": 100, "m": 255, "type": 0}),
             ("morph", {"op": 3, "shape": 0, "k": (7, 7)}), ("persp", {"m": [hom]})]
    plan = B.Batch([(h, w, 3, np.uint8)], [batch_stage(s) for s in specs])
    assert plan.info()["fallback_calls"] == 0
    for f in range(3):
        frame = synth.base_image_torch(h, w, 3, nrect=16, seed=100 + f)
        plan.input(0).copy_(frame)
        check_plan([frame], specs, graph=True, plan=plan)


def test_depths_channels_and_fallbacks():
    imgs, k = [], 0
    for dt in (np.uint8, np.uint16, np.float32):
        for c in (1, 3, 4):
            for (h, w) in ((57, 91), (130, 64)):
                x = synth.base_image(h, w, c, nrect=2, seed=200 + k, dtype=dt)
                if dt == np.float32:
                    x = synth.normal_f32(h, w, c, seed=200 + k)
                imgs.append(torch.from_numpy(np.ascontiguousarray(x)).cuda())
                k += 1
    rng = np.random.default_rng(5)
    mats = [synth.rotation_matrix_2d(x.shape[1] / 2, x.shape[0] / 2, rng.uniform(-30, 30), 1.0) for x in imgs]
    specs = [("gauss", {"k": (5, 5)}), ("affine", {"m": mats}), ("morph", {"op": 2, "shape": 0, "k": (3, 3)}),
             ("resize", {"fx": 0.5, "fy": 0.5}), ("gray", {})]
    check_plan(imgs, specs)


def test_thresholds_warps_and_borders():
    imgs = mixed_u8(10, seed=11, wmax=400, hmax=300, channels=(1, 3, 4))
    rng = np.random.default_rng(12)
    homs = [synth.perspective_params(x.shape[1], x.shape[0], seed=300 + i) for i, x in enumerate(imgs)]
    affs = [synth.affine_params(x.shape[1], x.shape[0], seed=400 + i) for i, x in enumerate(imgs)]
    for t, typ in ((127, 0), (30, 1), (200, 2), (-5, 3), (300, 4)):
        check_plan(imgs, [("thresh", {"t": t, "m": 255, "type": typ})])
    for interp in (0, 1):
        for border in (0, 1, 4):
            check_plan(imgs, [("persp", {"m": homs, "interp": interp, "border": border, "value": 17}),
                              ("affine", {"m": affs, "interp": interp, "border": border, "value": 250})])
    for op, shape, k in ((0, 1, (3, 3)), (1, 2, (7, 7)), (3, 0, (9, 9)), (4, 0, (3, 3)), (2, 0, (11, 11))):
        check_plan(imgs, [("morph", {"op": op, "shape": shape, "k": k, "it": 2})])
    for k in ((3, 3), (7, 7), (9, 9)):
        check_plan(imgs, [("gauss", {"k": k, "border": int(rng.integers(0, 5))})])
    check_plan(imgs, [("resize", {"fx": 0.37, "fy": 0.61}), ("resize", {"fx": 1.7, "fy": 1.3}),
                      ("resize", {"fx": 0.5, "fy": 0.5, "interp": 3})])


def test_gauss_strip_every_border_and_edge_geometry():
    """The binomial 3x3 / 5x5 strips under every border (wrap through the
    general kernel), on images whose rows end at every offset within a lane
    and a strip, down to 1-3 rows and columns, in 1, 3 and 4 channels, with
    every tile height."""
    rng = np.random.default_rng(71)
    shapes = [(1, 1), (2, 3), (3, 2), (3, 17), (5, 5), (9, 1), (1, 40)]
    shapes += [(int(rng.integers(4, 140)), int(w)) for w in list(range(236, 252)) + list(range(1, 20, 3))]
    shapes += [(300, 481), (257, 719), (64, 240), (65, 241)]
    imgs = [synth.base_image_torch(h, w, [1, 3, 4][k % 3], nrect=3, seed=700 + k) for k, (h, w) in enumerate(shapes)]
    try:
        for rows in (8, 32, 64):
            B.tune_load(None)
            for cn in (1, 3, 4):
                for k in (3, 5):
                    B.tune_set(f"gauss_strip.u8.c{cn}.k{k}.rows", rows)
            for k in (3, 5):
                for border in range(5):
                    plan = check_plan(imgs, [("gauss", {"k": (k, k), "border": border})])
                    # Wrap takes the general kernel (its border columns come from the row's far end).
                    assert any(st["name"].startswith("gauss_strip") for st in plan.launch_stats()) == (border != 3)
                    del plan
    finally:
        B.tune_load(None)


def test_strips_on_strided_views():
    """Caller images whose rows start 8-byte aligned but are not a multiple of
    8 bytes long (views into wider buffers): the plan repacks them before the
    strips, which read and write whole 8-byte words."""
    imgs = []
    for k, (h, w, c) in enumerate([(37, 19, 1), (70, 101, 3), (129, 45, 4), (64, 250, 1), (33, 7, 3)]):
        pitch = ((w * c + 63) // 64) * 64 + 64
        buf = torch.zeros((h, pitch), dtype=torch.uint8, device="cuda")
        x = synth.base_image_torch(h, w, c, nrect=3, seed=900 + k)
        v = buf[:, : w * c]
        v.copy_(x.reshape(h, w * c))
        imgs.append(v if c == 1 else v.view(h, w, c))
    for spec in ([("gauss", {"k": (5, 5)})], [("gauss", {"k": (3, 3), "border": 1})],
                 [("morph", {"op": 2, "shape": 2, "k": (5, 5)})], [("morph", {"op": 0, "shape": 0, "k": (3, 3)})]):
        check_plan(imgs, spec)


def test_every_strip_profile_fused_and_single():
    """Each compiled element profile (rect 3/5/7, cross 3/5, ellipse 5/7) as
    erode, dilate and the fused open / close, on 1-, 3- and 4-channel images."""
    imgs = mixed_u8(6, seed=61, wmax=500, hmax=300, channels=(1, 3, 4))
    for shape, k in ((0, 3), (0, 5), (0, 7), (1, 3), (1, 5), (2, 5), (2, 7)):
        for op in (0, 1, 2, 3):
            check_plan(imgs, [("morph", {"op": op, "shape": shape, "k": (k, k)})])


def test_more_images_than_prefix_cache():
    rng = np.random.default_rng(21)
    imgs = []
    for k in range(1100):
        h, w, c = int(rng.integers(1, 30)), int(rng.integers(1, 40)), int(rng.choice([1, 3, 4]))
        imgs.append(synth.base_image_torch(h, w, c, nrect=0, seed=k))
    specs = [("gauss", {"k": (3, 3)}), ("morph", {"op": 1, "shape": 1, "k": (3, 3)}),
             ("thresh", {"t": 90, "m": 200, "type": 0}), ("resize", {"fx": 0.5, "fy": 0.5})]
    check_plan(imgs, specs)


def test_tuning_choices_give_identical_results():
    """Every candidate the autotuner may pick (tile rows, samples per thread,
    CTAs per SM) gives the same bytes."""
    from visar_b200 import autotune
    imgs = mixed_u8(8, seed=31, wmax=900, hmax=500)
    specs = C2 + [("thresh", {"t": 128, "m": 255, "type": 0})]
    plan = check_plan(imgs, specs)
    keys = sorted({s["name"] for s in plan.launch_stats()})
    del plan
    assert {autotune.op_of(k) for k in keys} >= {"gray", "gauss_strip", "morph_strip", "lut"}
    try:
        for field in autotune.FIELDS:
            n = max(len(autotune.candidates(k, field)) for k in keys)
            for i in range(n):
                B.tune_load(None)
                for k in keys:
                    c = autotune.candidates(k, field)
                    if c:
                        B.tune_set(f"{k}.{field}", c[i % len(c)])
                check_plan(imgs, specs)
    finally:
        B.tune_load(None)


def test_warp_tile_heights_give_identical_results():
    """One-channel u8 linear warps run tiles 32 pixels wide and 32 to 256
    rows tall (a thread takes every 32nd row of its tile); every height gives
    the per-call bytes, partial tiles at the bottom included."""
    imgs = mixed_u8(6, seed=61, wmax=700, hmax=600, channels=(1,))
    homs = [synth.perspective_params(x.shape[1], x.shape[0], seed=500 + i) for i, x in enumerate(imgs)]
    affs = [synth.affine_params(x.shape[1], x.shape[0], seed=600 + i) for i, x in enumerate(imgs)]
    specs = [("persp", {"m": homs, "interp": 1, "border": 0, "value": 5}),
             ("affine", {"m": affs, "interp": 1, "border": 1, "value": 0})]
    plan = check_plan(imgs, specs)
    keys = sorted({s["name"] for s in plan.launch_stats()})
    del plan
    assert any(k.startswith("warp_perspective.u8.c1") for k in keys)
    assert any(k.startswith("warp_affine.u8.c1") for k in keys)
    try:
        for rows in (32, 64, 256):
            B.tune_load(None)
            for k in keys:
                B.tune_set(f"{k}.rows", rows)
            check_plan(imgs, specs)
    finally:
        B.tune_load(None)


def test_autotune_writes_a_table_the_library_reads(tmp_path):
    from visar_b200 import autotune
    imgs = mixed_u8(6, seed=51, wmax=600, hmax=400)
    path = str(tmp_path / "tune.json")
    try:
        table = autotune.ensure(path, imgs, [batch_stage(s) for s in C2], "test-c2", reps=1)
        doc = autotune.read(path)
        assert doc["_workload"] == "test-c2" and autotune.matches(doc, "test-c2")
        for k, v in table.items():
            cls, field = k.rsplit(".", 1)
            assert v in autotune.candidates(cls, field), k
            assert B.tune_get(k) == v
        check_plan(imgs, C2)
        # A second call reads the cache instead of tuning again.
        assert autotune.ensure(path, imgs, [], "test-c2") == table
    finally:
        B.tune_load(None)


def test_rebind_upload_download_and_profile():
    imgs = mixed_u8(6, seed=41, wmax=700, hmax=400)
    plan = B.Batch([(x.shape[0], x.shape[1], 1 if x.ndim == 2 else x.shape[2], np.uint8) for x in imgs],
                   [batch_stage(s) for s in C2])
    hosts = [torch.empty(tuple(x.shape), dtype=torch.uint8, pin_memory=True).numpy() for x in imgs]
    for h, x in zip(hosts, imgs):
        h[...] = x.cpu().numpy()
    plan.upload(hosts)
    plan.profile(True)
    check_plan(imgs, C2, plan=plan)
    stats = plan.launch_stats()
    assert len(stats) == plan.info()["launches"] and all(s["ms"] > 0 and s["grid"] > 0 for s in stats)
    assert sum(s["bytes"] for s in stats) == plan.info()["bytes_moved"]
    outs = [np.empty(tuple(plan.output(i).shape), np.uint8) for i in range(len(imgs))]
    plan.download(outs)
    for i, o in enumerate(outs):
        assert np.array_equal(o, plan.output(i).cpu().numpy())
    # Rebind input 0 to another device image with the plan input's row pitch.
    x0 = imgs[0]
    c0 = 1 if x0.ndim == 2 else x0.shape[2]
    new0 = synth.base_image_torch(x0.shape[0], x0.shape[1], c0, nrect=5, seed=999)
    pitch = plan.input(0).stride(0)
    big = torch.zeros((new0.shape[0], pitch), dtype=torch.uint8, device="cuda")
    view = big[:, :new0.shape[1] * c0]
    view.copy_(new0.reshape(new0.shape[0], -1))
    if c0 > 1:
        view = view.view(new0.shape[0], new0.shape[1], c0)
    plan.set_input(0, view)
    check_plan([new0] + imgs[1:], C2, graph=True, plan=plan)
