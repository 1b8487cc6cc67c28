"""Autotuner of the batched form's launch parameters.

The batch engine (include/visar_batch.h) runs every stage as one persistent
launch per shape class. Its tuning table holds, per class key
`<op>.<depth>.c<channels>.k<ksize>[.<element>][.<pass>].<size class>`
(the `name` of a launch in `Batch.launch_stats()`), integer fields:

  rows    tile height: rows per tile (strip ops: 8, 32, 64 or 128 rows per
          warp tile; one-channel u8 linear warps: 32 to 256 rows per 32-pixel
          wide tile; row-tiled ops: rows per thread, the tile being rows x
          the CTA's rows in flight)
  vec     samples (pixels) per thread, i.e. the vector width of the loads
          and stores: gray / threshold LUT 8 or 16 bytes, exact halving 4 or
          8 output pixels
  per_sm  CTAs per SM of the persistent grid (0: as many as fit)

`tune(images, stages)` builds the plan once per candidate value, times every
launch with the plan's per-launch CUDA events (median of `reps` runs after a
warm-up run) and keeps, for every class, the fastest candidate per field
(coordinate descent: rows, then vec, then per_sm, each starting from the best
so far); a candidate is written only if it beats the built-in adaptive
default by more than `margin`. The result is a flat JSON object that
`visar_tune_load` reads (string entries describe the run and are ignored by
the library):

    {"_device": "NVIDIA B200", "_sms": 148, "_workload": "...",
     "gauss_strip.u8.c1.k5.L.rows": 32, ...}

`ensure(path, images, stages, workload)` loads `path` when it was written for
this device and workload, else tunes and writes it. Results never depend on
the table: every candidate gives the same bytes (tests/test_batch_gpu.py).
"""
import json
import os

import numpy as np

from . import batch as B

# Candidate values per field, by op (the first word of a class key).
CANDIDATES = {
    "gauss_strip": {"rows": (8, 32, 64, 128), "per_sm": (2, 4, 5)},
    "morph_strip": {"rows": (8, 32, 64, 128), "per_sm": (2, 3, 4)},
    "gauss": {"rows": (8, 16, 32), "per_sm": (2, 4)},
    "morph": {"per_sm": (2, 4)},
    "gray": {"rows": (1, 2, 4, 8, 16), "vec": (8, 16), "per_sm": (2, 4, 6)},
    "lut": {"rows": (1, 2, 4, 8, 16), "vec": (8, 16), "per_sm": (2, 4, 6)},
    "half": {"rows": (1, 2, 4, 8, 16), "vec": (4, 8), "per_sm": (2, 4, 6)},
    "linear": {"rows": (2, 4, 8, 16, 32), "per_sm": (2, 4, 6)},
    "morph_f": {"rows": (1, 2, 4, 8, 16), "per_sm": (2, 4)},
    "copy": {"rows": (1, 2, 4, 8, 16), "per_sm": (2, 4)},
    "warp_affine": {"rows": (32, 64, 128, 256), "per_sm": (2, 4, 8)},
    "warp_perspective": {"rows": (32, 64, 128, 256), "per_sm": (2, 4, 8)},
}
FIELDS = ("rows", "vec", "per_sm")


def op_of(key):
    return key.split(".", 1)[0]


def candidates(key, field):
    return CANDIDATES.get(op_of(key), {}).get(field, ())


def _device():
    import torch
    p = torch.cuda.get_device_properties(torch.cuda.current_device())
    return p.name, p.multi_processor_count


def measure(images, stages, table, reps=5, fill=None):
    """Per-class milliseconds (summed over a plan's launches of the class) with
    `table` as the tuning table: median of `reps` profiled runs."""
    import torch
    B.tune_load(None)
    for k, v in table.items():
        B.tune_set(k, v)
    plan = B.Batch(images, stages)
    if fill is not None:
        fill(plan)
    plan.profile(True)
    runs = []
    for r in range(reps + 1):
        plan.run()
        torch.cuda.synchronize()
        if r == 0:
            continue
        per = {}
        for st in plan.launch_stats():
            per[st["name"]] = per.get(st["name"], 0.0) + st["ms"]
        runs.append(per)
    plan.profile(False)
    del plan
    return {k: float(np.median([p[k] for p in runs])) for k in runs[0]}


def tune(images, stages, reps=5, margin=0.02, fill=None, log=None):
    """Tuned table for a workload (dict of "<class>.<field>": value)."""
    base = measure(images, stages, {}, reps, fill)
    best = {k: ({}, ms) for k, ms in base.items()}  # class -> (its fields, ms)
    for field in FIELDS:
        values = sorted({v for k in base for v in candidates(k, field)})
        if not values:
            continue
        trials = {}
        for v in values:
            table = {}
            for k, (fields, _) in best.items():
                for f, fv in fields.items():
                    table[f"{k}.{f}"] = fv
                if v in candidates(k, field):
                    table[f"{k}.{field}"] = v
            ms = measure(images, stages, table, reps, fill)
            for k in base:
                if v in candidates(k, field) and k in ms:
                    trials.setdefault(k, []).append((ms[k], v))
            if log:
                log(f"{field}={v}: " + " ".join(f"{k}:{ms[k]:.3f}" for k in sorted(ms)))
        for k, res in trials.items():
            ms, v = min(res)
            if ms < best[k][1] * (1.0 - margin):
                best[k] = (dict(best[k][0], **{field: v}), ms)
    B.tune_load(None)
    out = {}
    for k, (fields, ms) in sorted(best.items()):
        for f, v in fields.items():
            out[f"{k}.{f}"] = int(v)
        if log:
            log(f"{k}: {base[k]:.3f} ms default -> {ms:.3f} ms {fields}")
    return out


def write(path, table, workload):
    name, sms = _device()
    doc = {"_device": name, "_sms": sms, "_workload": workload}
    doc.update(table)
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as fh:
        json.dump(doc, fh, indent=1, sort_keys=True)
        fh.write("\n")


def read(path):
    with open(path) as fh:
        return json.load(fh)


def matches(doc, workload):
    name, sms = _device()
    return doc.get("_device") == name and doc.get("_sms") == sms and doc.get("_workload") == workload


def ensure(path, images, stages, workload, reps=5, fill=None, log=None):
    """Loads the cached table at `path` if it was tuned for this device and
    workload; otherwise tunes, writes `path` and loads it. Returns the table."""
    if os.path.exists(path):
        doc = read(path)
        if matches(doc, workload):
            B.tune_load(path)
            return {k: v for k, v in doc.items() if not k.startswith("_")}
    table = tune(images, stages, reps=reps, fill=fill, log=log)
    write(path, table, workload)
    B.tune_load(path)
    return table
