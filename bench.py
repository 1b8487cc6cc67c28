"""Benchmark of the imgproc stencil-and-warp path on B200.

Workloads (`--workload`):

  batched-mixed (default): 256 uint8 images, width uniform 64-4096, height
      uniform 64-2160, 1 or 3 channels (p = 0.5 each), content as the
      640x480 case (gradient + noise + rectangles, seeded). Pipeline: gray
      (3-channel images) -> GaussianBlur 5x5 -> morphologyEx OPEN 5x5
      ELLIPSE -> resize INTER_LINEAR to half size. One step = the whole
      batch through the batched form (persistent tile-queue launches, one
      per stage pass and shape class, replayed as one CUDA graph). The plain
      per-call drop-in runs the same images call by call on the same GPU
      beside it, and the two results are compared.
  plain-1080p: one 1920x1080 u8 BGR frame through resize linear -> 720p,
      resize area -> 960x540, warpAffine, warpPerspective, plus one f32
      N(0,1) frame through GaussianBlur 7x7 sigma 1.5, call by call.

Gpix/s counts input pixels (width x height) once per image per step.

  value : inputs resident in HBM; CUDA events on the launching stream. The
          batched inputs (1.2 GB) are larger than L2; plain-1080p flushes L2
          (256 MiB write, then a 256 MiB read) before every timed step.
  e2e   : the same work through the public API from pinned host buffers:
          host->device copy of every input and device->host copy of every
          result inside each timed step.
  roofline : the dominant kernel (most time): its algorithmic bytes (every
          input and output byte once) / its CUDA-event duration, against
          MEASURED_PEAKS.json's HBM copy bandwidth.

`--impl reference` times VISAR's CPU path on the host cores instead: the
C++ restatement in oracle/ (VISAR itself is Zig and has no toolchain here).

Multi-GPU (torchrun, N>1): replicas only -- every rank runs the same
workload on its own GPU, no collective on the data path; rank 0 prints the
max-over-ranks time and the aggregate throughput.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Gpix/s bit-exact (served/batched vs per-call plain, 1 B200); p50/p99 latency"


# ------------------------------------------------------------------ common

def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic(workload, kernel):
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as fh:
        return json.load(fh).get(workload, {}).get(kernel)


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), f"visar_bench_clocks_{os.getpid()}_{id(self)}.csv")

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "100"], stdout=self.fh, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return None
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as fh:
            for line in fh:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx = float(parts[2])
                except ValueError:
                    continue
                for nm, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        reasons.add(nm)
        try:
            os.remove(self.path)
        except OSError:
            pass
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


_SYNTH = None


def load_synth():
    """visar_b200/synth.py loaded as a module of its own. The generators need
    only NumPy (and torch for device images); loading the file directly keeps
    the reference arm from importing the visar_b200 package, whose import maps
    the CUDA library."""
    global _SYNTH
    if _SYNTH is None:
        import importlib.util
        spec = importlib.util.spec_from_file_location("visar_bench_synth", os.path.join(ROOT, "visar_b200", "synth.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        _SYNTH = mod
    return _SYNTH


def dist_setup(n):
    if n <= 1 or "RANK" not in os.environ:
        return 0, 1, None
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    rank = int(os.environ["RANK"])
    world = int(os.environ["WORLD_SIZE"])
    local = int(os.environ.get("LOCAL_RANK", rank))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    return rank, world, dist


class Ctx:
    """Per-process GPU context: a dedicated stream shared by torch, the events
    and the library (torch's default stream has a NULL handle, which the
    library reads as "use your own stream"), barriers and max-over-ranks."""

    def __init__(self, args):
        import torch
        self.torch = torch
        self.rank, self.world, self.dist = dist_setup(args.gpus)
        if self.dist is None:
            torch.cuda.set_device(0)
        import visar_b200 as vb
        self.vb = vb
        self.dev = torch.cuda.current_device()
        self.stream = torch.cuda.Stream()
        torch.cuda.set_stream(self.stream)
        vb.set_stream(self.stream)

    def barrier(self):
        self.torch.cuda.synchronize()
        if self.dist is not None:
            self.dist.barrier()

    def max_over_ranks(self, x):
        if self.dist is None:
            return x
        t = self.torch.tensor([x], dtype=self.torch.float64, device="cuda")
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def timed(self, fn, steps, before=None):
        """Total ms of `steps` calls of fn, CUDA events on the stream around each."""
        torch = self.torch
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for i in range(steps):
            if before is not None:
                before(i)
            ev[i][0].record(self.stream)
            fn()
            ev[i][1].record(self.stream)
        torch.cuda.synchronize()
        return sum(a.elapsed_time(b) for a, b in ev)

    def close(self):
        if self.dist is not None:
            self.dist.barrier()
            self.dist.destroy_process_group()


class L2Flush:
    """Evicts L2 (126 MB) before a timed step: a 256 MiB write, then a 256 MiB
    read of another buffer, so that the step starts on clean lines instead of
    writing back the flush's own dirty ones inside its timed region."""

    def __init__(self, torch):
        self.w = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
        self.r = torch.zeros(64 << 20, dtype=torch.int32, device="cuda")

    def __call__(self, i):
        self.w.fill_(i & 0xFF)
        self.r.max()


# ----------------------------------------------------------- batched-mixed

N_IMAGES = 256
IMAGE_LIMIT = 0  # --images: the first N images only (reduced plans for profiling captures)
E2E_DEPTH = 2  # plans in flight in the end-to-end measurement
MIX_SEED = 2


def mixed_shapes():
    synth = load_synth()
    shapes = synth.mixed_shapes(N_IMAGES, seed=MIX_SEED)
    return shapes[:IMAGE_LIMIT] if IMAGE_LIMIT else shapes


def c2_stages(B):
    return [B.gray(), B.gaussian((5, 5), 0.0, 0.0, 4), B.morphology(2, 2, (5, 5), 1), B.resize(0.5, 0.5, 1)]


def half_dims(h, w):
    return max(1, h // 2), max(1, w // 2)


def c2_oracle_image(O, x):
    """The pipeline of one image through module O (the oracle)."""
    y = x if x.ndim == 2 else O.cvt_color(x, 6)
    y = O.gaussian_blur(y, (5, 5), 0, 0, 4)
    y = O.morphology(y, 2, 2, (5, 5))
    h, w = half_dims(y.shape[0], y.shape[1])
    return y if (h, w) == y.shape[:2] else O.resize(y, (w, h), 1)


def oracle_run(fn, items, threads, budget_s, keep=False):
    """Times fn(O, item) over items with the oracle on `threads` host threads
    (0 = all) until the items or the time budget run out (one untimed call of
    the first item first). Returns (items done, seconds, threads, outputs)."""
    from oracle import oracle as O
    O.set_num_threads(threads)
    fn(O, items[0])
    outs = []
    n, dt = 0, 0.0
    oracle_run.times = []
    for it in items:
        t0 = time.perf_counter()
        y = fn(O, it)
        t1 = time.perf_counter() - t0
        dt += t1
        oracle_run.times.append(t1)
        if keep:
            outs.append(y)
        n += 1
        if dt > budget_s:
            break
    cores = O.get_num_threads()
    O.set_num_threads(0)
    return n, dt, cores, outs


def cv2_c2_image(cv2, x):
    """The C2 pipeline through OpenCV (context timing only: OpenCV 4's arithmetic
    is not VISAR's everywhere)."""
    y = x if x.ndim == 2 else cv2.cvtColor(x, cv2.COLOR_BGR2GRAY)
    y = cv2.GaussianBlur(y, (5, 5), 0, borderType=cv2.BORDER_REFLECT_101)
    y = cv2.morphologyEx(y, cv2.MORPH_OPEN, cv2.getStructuringElement(cv2.MORPH_ELLIPSE, (5, 5)))
    h, w = half_dims(y.shape[0], y.shape[1])
    return y if (h, w) == y.shape[:2] else cv2.resize(y, (w, h), interpolation=cv2.INTER_LINEAR)


def cv2_context(fn, items, px_of, budget_s):
    """OpenCV (all its threads) over a bounded prefix of items: Gpix/s, or None without cv2."""
    try:
        import cv2
    except Exception:
        return None
    fn(cv2, items[0])
    n, px, dt = 0, 0, 0.0
    for it in items:
        t0 = time.perf_counter()
        fn(cv2, it)
        dt += time.perf_counter() - t0
        n += 1
        px += px_of(it)
        if dt > budget_s:
            break
    return {"value": px / dt / 1e9, "unit": "Gpix/s", "threads": cv2.getNumThreads(), "version": cv2.__version__,
            "sample": f"{n} items, {px / 1e6:.1f} MP in {dt:.1f} s"}


def c2_cpu_baselines(hosts, keep):
    """The oracle on the C2 images: all host threads over the whole batch (its
    outputs kept for the parity check when `keep`), then 1 thread and OpenCV
    on bounded prefixes. Returns (cpu_baseline dict, outputs)."""
    n, dt, cores, outs = oracle_run(c2_oracle_image, hosts, 0, 60.0, keep=keep)
    px = sum(x.shape[0] * x.shape[1] for x in hosts[:n])
    n1, dt1, _, _ = oracle_run(c2_oracle_image, hosts, 1, 15.0)
    px1 = sum(x.shape[0] * x.shape[1] for x in hosts[:n1])
    cpu = {"value": px / dt / 1e9, "unit": "Gpix/s", "cores": cores, "kind": "port",
           "sample": f"{n} of the {len(hosts)} images ({px / 1e6:.1f} MP) through the 4-stage pipeline in {dt:.1f} s",
           "one_thread": {"value": px1 / dt1 / 1e9, "unit": "Gpix/s", "cores": 1,
                          "sample": f"first {n1} images ({px1 / 1e6:.1f} MP) in {dt1:.1f} s"},
           "cv2_context": cv2_context(cv2_c2_image, hosts, lambda x: x.shape[0] * x.shape[1], 10.0)}
    return cpu, outs


def tune_workload(args, ctx, workload, images, stages, fill=None):
    """Loads the workload's tuned launch table (`--tuning`, by default
    visar_b200/tuned/<workload>.json) when it was written for this device,
    else runs the autotuner and writes it there. Returns the table."""
    from visar_b200 import autotune
    if args.no_tune:
        return None
    path = args.tuning or os.path.join(ROOT, "visar_b200", "tuned", f"{workload}.json")
    log = (lambda m: print(f"[tune {workload}] {m}", file=sys.stderr)) if ctx.rank == 0 else None
    return autotune.ensure(path, images, stages, workload, fill=fill, log=log)


def bench_batched(args, ctx):
    torch, vb = ctx.torch, ctx.vb
    from visar_b200 import batch as B
    synth = load_synth()
    shapes = mixed_shapes()
    bases = [synth.base_image_torch(h, w, c, nrect=8, seed=10_000 + k) for k, (h, w, c) in enumerate(shapes)]

    def fill(p):
        for k, x in enumerate(bases):
            p.input(k).copy_(x)

    tuned = tune_workload(args, ctx, "batched-mixed", [(h, w, c, np.uint8) for (h, w, c) in shapes], c2_stages(B),
                          fill)
    if args.rows:  # the full plan's strip tile height on a reduced plan (profiler captures)
        for key in ("gauss_strip.u8.c1.k5.rows", "morph_strip.u8.c1.k5.ell5.open.rows"):
            B.tune_set(key, args.rows)
    plan = B.Batch([(h, w, c, np.uint8) for (h, w, c) in shapes], c2_stages(B))
    fill(plan)
    del bases
    info = plan.info()
    px_step = info["pixels_in"]
    ins = [plan.input(k) for k in range(len(shapes))]
    vb.set_async(True)

    # ------------------------------------------------ value: graph replay
    for _ in range(args.warmup):
        plan.run_graph()
    ctx.barrier()
    with Clocks(ctx.dev) as clk:
        ms = ctx.timed(plan.run_graph, args.steps)
    ctx.barrier()
    ms_step = ctx.max_over_ranks(ms) / args.steps
    value = px_step * ctx.world / (ms_step / 1e3) / 1e9
    clocks = clk.summary()

    # --------------------------------------- plain per-call drop-in, same GPU
    outs = []
    for x in ins:
        c = 1 if x.ndim == 2 else x.shape[2]
        h, w = x.shape[:2]
        hh, ww = half_dims(h, w)
        outs.append((torch.empty((h, w), dtype=torch.uint8, device="cuda") if c == 3 else None,
                     torch.empty((h, w), dtype=torch.uint8, device="cuda"),
                     torch.empty((h, w), dtype=torch.uint8, device="cuda"),
                     torch.empty((hh, ww), dtype=torch.uint8, device="cuda")))

    def plain_step():
        for x, (g, gb, op, rs) in zip(ins, outs):
            y = vb.cvt_color(x, 6, dst=g) if g is not None else x
            vb.gaussian_blur(y, (5, 5), 0, 0, 4, dst=gb)
            vb.morphology(gb, 2, 2, (5, 5), 1, dst=op)
            if rs.shape != op.shape:
                vb.resize(op, (rs.shape[1], rs.shape[0]), 1, dst=rs)

    plain_step()
    ctx.barrier()
    p_steps = max(2, min(args.steps, 5))
    p_ms = ctx.max_over_ranks(ctx.timed(plain_step, p_steps)) / p_steps
    plain = px_step * ctx.world / (p_ms / 1e3) / 1e9
    for k in range(len(ins)):  # the two arms agree bit for bit
        ref = outs[k][3] if outs[k][3].shape != outs[k][2].shape else outs[k][2]
        if not torch.equal(ref, plan.output(k)):
            raise AssertionError(f"batched and per-call outputs differ for image {k}")

    # ------------------------------- per-launch timing for the roofline (eager)
    plan.profile(True)
    per = {}
    for r in range(max(3, args.steps // 2)):
        plan.run()
        torch.cuda.synchronize()
        if r == 0:
            continue
        for st in plan.launch_stats():
            key = f"s{st['stage']}:{st['name']}"
            d = per.setdefault(key, {"ms": [], "bytes": st["bytes"], "images": st["images"], "tiles": st["tiles"],
                                     "grid": st["grid"]})
            d["ms"].append(st["ms"])
    plan.profile(False)
    kernels = {k: {"ms": float(np.mean(v["ms"])), "bytes": v["bytes"], "images": v["images"], "tiles": v["tiles"],
                   "grid": v["grid"], "gbs": v["bytes"] / (np.mean(v["ms"]) / 1e3) / 1e9} for k, v in per.items()}
    dom = max(kernels, key=lambda k: kernels[k]["ms"])
    peak, peak_kind = load_peaks()
    achieved = kernels[dom]["gbs"]
    all_ms = sum(v["ms"] for v in kernels.values())
    pipeline_gbs = info["bytes_moved"] / (ms_step / 1e3) / 1e9

    # ---------------------------------------------- e2e through the public API
    hosts = [torch.empty(tuple(x.shape), dtype=torch.uint8, pin_memory=True).numpy() for x in ins]
    for h, x in zip(hosts, ins):
        h[...] = x.cpu().numpy()
    houts = [torch.empty(tuple(plan.output(k).shape), dtype=torch.uint8, pin_memory=True).numpy()
             for k in range(len(ins))]
    h2d = sum(h.nbytes for h in hosts)
    d2h = sum(h.nbytes for h in houts)

    # E2E_DEPTH plans on as many streams take the steps in turn, so one step's
    # upload overlaps the previous step's graph and download (a streaming
    # client); every step still uploads its inputs and downloads its results.
    e_plans = [plan] + [B.Batch([(h, w, c, np.uint8) for (h, w, c) in shapes], c2_stages(B))
                        for _ in range(E2E_DEPTH - 1)]
    e_streams = [torch.cuda.Stream() for _ in e_plans]
    e_outs = [houts] + [[torch.empty(tuple(plan.output(k).shape), dtype=torch.uint8, pin_memory=True).numpy()
                         for k in range(len(ins))] for _ in range(E2E_DEPTH - 1)]

    def e2e_step(k):
        i = k % E2E_DEPTH
        vb.set_stream(e_streams[i])
        e_plans[i].upload(hosts)
        e_plans[i].run_graph()
        e_plans[i].download(e_outs[i])

    for k in range(E2E_DEPTH):
        e2e_step(k)
    torch.cuda.synchronize()
    ctx.barrier()
    e_steps = max(4, min(args.steps, 8))
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(ctx.stream)
    for s_ in e_streams:
        s_.wait_event(ev0)
    for k in range(e_steps):
        e2e_step(k)
    for s_ in e_streams:
        ctx.stream.wait_stream(s_)
    vb.set_stream(ctx.stream)
    ev1.record(ctx.stream)
    torch.cuda.synchronize()
    e_ms = ctx.max_over_ranks(ev0.elapsed_time(ev1)) / e_steps
    e2e = px_step * ctx.world / (e_ms / 1e3) / 1e9
    vb.set_async(False)
    for i in range(E2E_DEPTH):
        if not np.array_equal(e_outs[i][0], plan.output(0).cpu().numpy()):
            raise AssertionError("downloaded output differs from the device result")
    del e_plans[1:]

    # CPU baselines on the same images; the oracle's outputs for the whole
    # batch are compared with the batched results (outside any timed region).
    cpu, parity = None, None
    if ctx.rank == 0 and ctx.world == 1 and not args.no_cpu_baseline:
        host_in = [x.cpu().numpy() for x in ins]
        cpu, ref_outs = c2_cpu_baselines(host_in, keep=True)
        bad = [k for k, y in enumerate(ref_outs) if not np.array_equal(y, plan.output(k).cpu().numpy())]
        parity = {"checked": len(ref_outs), "of": len(ins), "bit_exact": len(ref_outs) - len(bad),
                  "summary": f"{len(ref_outs) - len(bad)}/{len(ins)} images bit-exact against the oracle",
                  "first_mismatch": bad[0] if bad else None}
        del host_in, ref_outs
    return {
        "metric": METRIC, "value": value, "unit": "Gpix/s", "n_gpus": ctx.world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": "batched-mixed", "images": len(shapes), "shapes": "w U[64,4096], h U[64,2160], 1|3 ch",
                   "stages": ["gray", "gaussian 5x5", "open 5x5 ellipse", "resize linear 0.5x"],
                   "pixels_per_step": px_step, "bytes_per_step": info["bytes_moved"],
                   "pipeline_gbs": pipeline_gbs, "pipeline_frac": pipeline_gbs / peak,
                   "launches_per_step": info["launches"], "fallback_calls": info["fallback_calls"],
                   "plain_gpix_s": plain, "plain_ms_per_step": p_ms, "speedup_vs_plain": value / plain,
                   "exec": "one CUDA graph per step (persistent tile-queue kernels)", "tuning": tuned,
                   "l2": "inputs (1.2 GB) larger than L2", "parallelism": f"replicas{ctx.world}",
                   "kernels": kernels},
        "e2e": {"value": e2e, "unit": "Gpix/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": e_ms,
                "plans_in_flight": E2E_DEPTH, "host": "pinned, contiguous rows (staged 1-D copies)"},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "traffic": load_traffic("batched-mixed", dom.split(":", 1)[1]),
                     "alg_bytes_per_launch": kernels[dom]["bytes"], "share_of_kernel_time": kernels[dom]["ms"] / all_ms},
        "cpu_baseline": cpu,
        "parity": parity,
        "clocks": clocks,
        "gpu_launches": info["launches"] * args.steps,
    }


def reference_batched(args):
    """VISAR's CPU path (the oracle port) on all host threads: every step runs
    the whole 256-image batch through the 4-stage pipeline, for the same warm-up
    and step counts as the GPU arm."""
    from oracle import oracle as O
    synth = load_synth()
    O.set_num_threads(0)
    shapes = mixed_shapes()
    images = [synth.base_image(h, w, c, nrect=8, seed=10_000 + k) for k, (h, w, c) in enumerate(shapes)]
    px = sum(h * w for (h, w, c) in shapes)
    for _ in range(args.warmup):
        for x in images:
            c2_oracle_image(O, x)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for x in images:
            c2_oracle_image(O, x)
    dt = time.perf_counter() - t0
    v = px * args.steps / dt / 1e9
    return {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "Gpix/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": "batched-mixed", "images": N_IMAGES, "pixels_per_step": px,
                   "impl": "VISAR CPU path (C++ restatement, oracle/), all host threads"},
        "cpu_baseline": {"value": v, "unit": "Gpix/s", "cores": O.get_num_threads(), "kind": "port",
                         "sample": f"all {len(images)} images ({px / 1e6:.1f} MP) per step"},
        "e2e": {"value": v, "unit": "Gpix/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


# ---------------------------------------------------------------- video-4k

V_FRAMES, V_H, V_W = 300, 2160, 3840
V_INSTANCES = 4
V_BYTES_PER_FRAME = V_W * V_H * 3 + V_W * V_H + 2 * V_W * V_H + 2 * V_W * V_H + 2 * 2 * V_W * V_H + 2 * V_W * V_H


def video_homography():
    synth = load_synth()
    return synth.perspective_params(V_W, V_H, seed=7)


def video_stages(B):
    return [B.gray(), B.gaussian((5, 5), 0.0, 0.0, 4), B.threshold(100, 255, 0), B.morphology(3, 0, (7, 7), 1),
            B.warp_perspective(video_homography(), 1, 0, 0.0)]


def video_plain(vb, x, outs):
    """The per-frame pipeline call by call (the plain drop-in)."""
    g, b, t, c, w = outs
    vb.cvt_color(x, 6, dst=g)
    vb.gaussian_blur(g, (5, 5), 0, 0, 4, dst=b)
    vb.threshold(b, 100, 255, 0, dst=t)
    vb.morphology(t, 3, 0, (7, 7), 1, dst=c)
    vb.warp_perspective(c, video_homography(), (V_W, V_H), 1, 0, 0.0, dst=w)


def video_oracle(O, x):
    y = O.cvt_color(x, 6)
    y = O.gaussian_blur(y, (5, 5), 0, 0, 4)
    y = O.threshold(y, 100, 255, 0)[1]
    y = O.morphology(y, 3, 0, (7, 7))
    return O.warp_perspective(y, video_homography(), (V_W, V_H), 1, 0, 0.0)


def cv2_video_frame(cv2, x):
    """The video pipeline through OpenCV (context timing only)."""
    y = cv2.cvtColor(x, cv2.COLOR_BGR2GRAY)
    y = cv2.GaussianBlur(y, (5, 5), 0, borderType=cv2.BORDER_REFLECT_101)
    _, y = cv2.threshold(y, 100, 255, cv2.THRESH_BINARY)
    y = cv2.morphologyEx(y, cv2.MORPH_CLOSE, cv2.getStructuringElement(cv2.MORPH_RECT, (7, 7)))
    return cv2.warpPerspective(y, video_homography(), (V_W, V_H), flags=cv2.INTER_LINEAR, borderValue=0)


def bench_video(args, ctx):
    torch, vb = ctx.torch, ctx.vb
    from visar_b200 import batch as B
    synth = load_synth()
    scene = synth.VideoScene(V_H, V_W, nobj=16, seed=3)
    frames = [scene.frame(k) for k in range(V_FRAMES)]  # 7.5 GB in HBM, outside timing
    torch.cuda.synchronize()
    tuned = tune_workload(args, ctx, "video-4k", [frames[0]], video_stages(B))
    # V_INSTANCES graph instances on as many streams take the frames in turn,
    # so one frame's launches overlap the tails of the previous frame's.
    plans = [B.Batch([(V_H, V_W, 3, np.uint8)], video_stages(B)) for _ in range(V_INSTANCES)]
    streams = [torch.cuda.Stream() for _ in plans]
    plan = plans[0]
    assert plan.info()["fallback_calls"] == 0
    vb.set_async(True)

    def frame_step(k):
        i = k % V_INSTANCES
        vb.set_stream(streams[i])
        plans[i].set_input(0, frames[k % V_FRAMES])
        plans[i].run_graph()

    def fork(ev):
        for s in streams:
            s.wait_event(ev)

    def join():
        for s in streams:
            ctx.stream.wait_stream(s)
        vb.set_stream(ctx.stream)

    for k in range(max(args.warmup, V_INSTANCES)):
        frame_step(k)
    join()
    torch.cuda.synchronize()
    ctx.barrier()
    nf = V_FRAMES
    with Clocks(ctx.dev) as clk:
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(ctx.stream)
        fork(ev0)
        for k in range(nf):
            frame_step(k)
        join()
        ev1.record(ctx.stream)
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1)
    ctx.barrier()
    ms = ctx.max_over_ranks(ms)
    fps = nf * ctx.world / (ms / 1e3)
    value = fps * V_W * V_H / 1e9
    clocks = clk.summary()
    # The last frame's result against the per-call path.
    outs = [torch.empty((V_H, V_W), dtype=torch.uint8, device="cuda") for _ in range(5)]
    video_plain(vb, frames[(nf - 1) % V_FRAMES], outs)
    torch.cuda.synchronize()
    if not torch.equal(outs[4], plans[(nf - 1) % V_INSTANCES].output(0)):
        raise AssertionError("video: graph result differs from the per-call pipeline")

    # per-call drop-in, same GPU
    p_n = 30
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(ctx.stream)
    for k in range(p_n):
        video_plain(vb, frames[k % V_FRAMES], outs)
    e1.record(ctx.stream)
    torch.cuda.synchronize()
    p_ms = ctx.max_over_ranks(e0.elapsed_time(e1))
    plain_fps = p_n * ctx.world / (p_ms / 1e3)

    # per-launch timing (eager runs)
    plan.profile(True)
    per = {}
    for r in range(6):
        plan.set_input(0, frames[r % V_FRAMES])
        plan.run()
        torch.cuda.synchronize()
        if r == 0:
            continue
        for st in plan.launch_stats():
            d = per.setdefault(f"s{st['stage']}:{st['name']}", {"ms": [], "bytes": st["bytes"]})
            d["ms"].append(st["ms"])
    plan.profile(False)
    kernels = {k: {"ms": float(np.mean(v["ms"])), "bytes": v["bytes"],
                   "gbs": v["bytes"] / (np.mean(v["ms"]) / 1e3) / 1e9} for k, v in per.items()}
    dom = max(kernels, key=lambda k: kernels[k]["ms"])
    peak, peak_kind = load_peaks()

    # e2e: each frame from pinned host memory, the result back to the host
    nh = 8
    hosts = []
    for k in range(nh):
        h = torch.empty((V_H, V_W, 3), dtype=torch.uint8, pin_memory=True).numpy()
        h[...] = frames[k % V_FRAMES].cpu().numpy()
        hosts.append(h)
    houts = [torch.empty((V_H, V_W), dtype=torch.uint8, pin_memory=True).numpy() for _ in range(V_INSTANCES)]
    # Each instance's own input buffer receives its uploads; instance i's
    # upload, graph and download are ordered on its stream, and the instances
    # overlap (copy engines and SMs).
    owns = [B.Batch([(V_H, V_W, 3, np.uint8)], video_stages(B)) for _ in range(V_INSTANCES)]

    def e2e_frame(k):
        i = k % V_INSTANCES
        vb.set_stream(streams[i])
        owns[i].upload([hosts[k % nh]])
        owns[i].run_graph()
        owns[i].download([houts[i]])

    for k in range(max(3, V_INSTANCES)):
        e2e_frame(k)
    join()
    torch.cuda.synchronize()
    ctx.barrier()
    e_n = 60
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(ctx.stream)
    fork(e0)
    for k in range(e_n):
        e2e_frame(k)
    join()
    e1.record(ctx.stream)
    torch.cuda.synchronize()
    e_ms = ctx.max_over_ranks(e0.elapsed_time(e1)) / e_n
    vb.set_async(False)

    # CPU baselines on the first frames; the oracle's results for those frames
    # are compared with the graph's (outside any timed region).
    cpu, parity = None, None
    if ctx.rank == 0 and ctx.world == 1 and not args.no_cpu_baseline:
        nchk = 4
        xs = [frames[k % V_FRAMES].cpu().numpy() for k in range(8)]
        n, dt, cores, ref = oracle_run(video_oracle, xs, 0, 8.0, keep=True)
        n1, dt1, _, _ = oracle_run(video_oracle, xs, 1, 8.0)
        cpu = {"value": n * V_W * V_H / dt / 1e9, "unit": "Gpix/s", "cores": cores, "kind": "port",
               "sample": f"{n} frames through the 5-stage pipeline in {dt:.1f} s ({n / dt:.2f} frames/s)",
               "one_thread": {"value": n1 * V_W * V_H / dt1 / 1e9, "unit": "Gpix/s", "cores": 1,
                              "sample": f"{n1} frames in {dt1:.1f} s"},
               "cv2_context": cv2_context(cv2_video_frame, xs, lambda x: V_W * V_H, 5.0)}
        good = 0
        for k in range(min(nchk, len(ref))):
            plan.set_input(0, frames[k % V_FRAMES])
            plan.run()
            torch.cuda.synchronize()
            good += bool(np.array_equal(plan.output(0).cpu().numpy(), ref[k]))
        parity = {"checked": min(nchk, len(ref)), "bit_exact": good,
                  "summary": f"{good}/{min(nchk, len(ref))} frames bit-exact against the oracle"}
        del xs, ref
    return {
        "metric": METRIC, "value": value, "unit": "Gpix/s", "n_gpus": ctx.world, "steps": nf, "warmup": args.warmup,
        "ms_per_step": ms / nf, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
        "data": "synthetic",
        "config": {"workload": "video-4k", "frames": nf, "frame": f"{V_W}x{V_H}x3 u8",
                   "stages": ["gray", "gaussian 5x5", "threshold 100", "close 7x7 rect", "warpPerspective linear"],
                   "fps": fps, "hbm_gbs_algorithmic": V_BYTES_PER_FRAME * fps / 1e9,
                   "frac_of_peak": V_BYTES_PER_FRAME * fps / 1e9 / peak, "bytes_per_frame": V_BYTES_PER_FRAME,
                   "plain_fps": plain_fps, "speedup_vs_plain": fps / plain_fps,
                   "exec": f"one CUDA graph per frame; input rebound per frame by a one-thread kernel; "
                           f"{V_INSTANCES} graph instances on {V_INSTANCES} streams take the frames in turn",
                   "tuning": tuned,
                   "l2": "frames (24.9 MB each, 7.5 GB in all) stream from HBM", "parallelism": f"replicas{ctx.world}",
                   "kernels": kernels},
        "e2e": {"value": V_W * V_H / (e_ms / 1e3) / 1e9 * ctx.world, "unit": "Gpix/s",
                "h2d_bytes_per_step": V_W * V_H * 3, "d2h_bytes_per_step": V_W * V_H, "ms_per_step": e_ms},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": kernels[dom]["gbs"], "peak": peak, "unit": "GB/s",
                     "frac": kernels[dom]["gbs"] / peak, "peak_kind": peak_kind,
                     "traffic": load_traffic("video-4k", dom.split(":", 1)[1]),
                     "alg_bytes_per_launch": kernels[dom]["bytes"]},
        "cpu_baseline": cpu,
        "parity": parity,
        "clocks": clocks,
        "gpu_launches": (plan.info()["launches"] + 1) * nf,
    }


def reference_video(args):
    """The oracle port on all host threads: each step is one 4K frame through the
    5-stage pipeline (frames rendered on the host, outside timing)."""
    from oracle import oracle as O
    synth = load_synth()
    O.set_num_threads(0)
    scene = synth.VideoScene(V_H, V_W, nobj=16, seed=3)
    frames = [scene.frame(k, device="cpu").numpy() for k in range(4)]
    for k in range(args.warmup):
        video_oracle(O, frames[k % 4])
    t0 = time.perf_counter()
    for k in range(args.steps):
        video_oracle(O, frames[k % 4])
    dt = time.perf_counter() - t0
    v = args.steps * V_W * V_H / dt / 1e9
    return {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "Gpix/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": "video-4k", "frame": f"{V_W}x{V_H}x3 u8", "fps": args.steps / dt,
                   "impl": "VISAR CPU path (C++ restatement, oracle/), all host threads"},
        "cpu_baseline": {"value": v, "unit": "Gpix/s", "cores": O.get_num_threads(), "kind": "port",
                         "sample": f"{args.steps} frames of the video pipeline"},
        "e2e": {"value": v, "unit": "Gpix/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


# ------------------------------------------------------------------ served

S_RATES = (500, 2000, 8000, 20000)
S_CORPUS = 384


def served_stage_list(B, r):
    synth = load_synth()
    out = []
    for name, p in r["stages"]:
        if name == "gray":
            out.append(B.gray())
        elif name == "gauss":
            out.append(B.gaussian((5, 5), 0.0, 0.0, 4))
        elif name == "resize":
            out.append(B.resize(0.5, 0.5, 1))
        elif name == "affine":
            out.append(B.warp_affine(synth.rotation_matrix_2d(r["w"] / 2.0, r["h"] / 2.0, p["angle"], 1.0), 1, 0, 0.0))
        else:
            out.append(B.morphology(2, 0, (3, 3), 1))
    return out


def served_oracle(O, item):
    """One served request's pipeline through module O (the oracle): gray is a
    pass-through on one-channel images and the halving on 1-pixel sides, as
    in the server."""
    synth = load_synth()
    r, x = item
    for name, p in r["stages"]:
        c = 1 if x.ndim == 2 else x.shape[2]
        if name == "gray":
            if c > 1:
                x = O.cvt_color(x, 6 if c == 3 else 10)
        elif name == "gauss":
            x = O.gaussian_blur(x, (5, 5), 0, 0, 4)
        elif name == "resize":
            h, w = max(1, x.shape[0] // 2), max(1, x.shape[1] // 2)
            if (h, w) != tuple(x.shape[:2]):
                x = O.resize(x, (w, h), 1)
        elif name == "affine":
            m = synth.rotation_matrix_2d(r["w"] / 2.0, r["h"] / 2.0, p["angle"], 1.0)
            x = O.warp_affine(x, m, (x.shape[1], x.shape[0]), 1, 0, 0.0)
        else:
            x = O.morphology(x, 2, 0, (3, 3))
    return x


def served_cpu_baseline(corpus, hosts, keep):
    """The oracle over the corpus's requests in arrival order, one request at a
    time on all host threads (VISAR's own per-call threading): Gpix/s of
    request input pixels and the per-request service time (no queueing)."""
    items = list(zip(corpus, hosts))
    n, dt, cores, outs = oracle_run(served_oracle, items, 0, 15.0, keep=keep)
    t = np.array(oracle_run.times) * 1e3
    px = sum(r["h"] * r["w"] for r in corpus[:n])
    n1, dt1, _, _ = oracle_run(served_oracle, items, 1, 10.0)
    px1 = sum(r["h"] * r["w"] for r in corpus[:n1])
    return {"value": px / dt / 1e9, "unit": "Gpix/s", "cores": cores, "kind": "port",
            "sample": f"first {n} requests of the corpus ({px / 1e6:.1f} MP) one after another in {dt:.1f} s",
            "service_p50_ms": float(np.percentile(t, 50)), "service_p99_ms": float(np.percentile(t, 99)),
            "max_rate_req_s": n / dt,
            "one_thread": {"value": px1 / dt1 / 1e9, "unit": "Gpix/s", "cores": 1,
                           "sample": f"first {n1} requests in {dt1:.1f} s"}}, outs


def bench_served(args, ctx):
    torch = ctx.torch
    import ctypes
    from visar_b200 import batch as B
    from visar_b200 import serve as S
    synth = load_synth()
    from visar_b200 import desc
    corpus = synth.served_requests(S_CORPUS, seed=4)
    imgs = [synth.served_image(r) for r in corpus]  # device-resident payloads
    arrs = [S._stage_array(served_stage_list(B, r)) for r in corpus]
    descs = [desc(x) for x in imgs]
    torch.cuda.synchronize()
    dur = args.duration
    rng = np.random.default_rng(5)
    results = []
    # (rate, requests): the spec rates for `dur` seconds each, then a
    # saturation run (every request queued at t = 0) that measures capacity.
    runs = [(rate, int(rate * dur)) for rate in S_RATES] + [(0, int(S_RATES[-1] * dur))]
    clk = Clocks(ctx.dev).__enter__()  # sampled over every rate and both modes
    for rate, n in [(2000, 400)] + runs:  # the first run warms both modes up and is not reported
        if rate > 0:
            t = np.cumsum(rng.exponential(1.0 / rate, size=n))
        else:
            t = np.zeros(n)
        idx = rng.integers(0, S_CORPUS, size=n)
        reqs = (S.TraceRequest * n)()
        px = 0
        for i in range(n):
            k = int(idx[i])
            reqs[i].arrival_s = float(t[i])
            reqs[i].input = descs[k]
            reqs[i].stages = ctypes.cast(arrs[k][0], ctypes.POINTER(S.Stage))
            reqs[i].nstages = len(corpus[k]["stages"])
            px += corpus[k]["h"] * corpus[k]["w"]
        row = {"rate": rate, "requests": n}
        for mode, tag in ((S.BATCHED, ""), (S.PLAIN, "plain_")):
            srv = S.Server(pool_bytes=64 << 30, mode=mode)
            try:
                lat = (ctypes.c_double * n)()
                el = ctypes.c_double()
                rc = S.lib.visar_server_run_trace(srv._h, reqs, n, lat, ctypes.byref(el))
                S._check(rc)
                la = np.array(lat[:n])
                st = srv.stats()
            finally:
                srv.close()
            row[tag + "gpix_s"] = px / el.value / 1e9
            row[tag + "p50_ms"] = float(np.percentile(la, 50))
            row[tag + "p99_ms"] = float(np.percentile(la, 99))
            row[tag + "elapsed_s"] = el.value
            if mode == S.BATCHED:
                row["mean_batch"] = st["mean_batch"]
                row["rounds"] = st["rounds"]
                row["launches"] = st["launches"]
                row["fallback_calls"] = st["fallback_calls"]
                row["deferred"] = st["deferred"]
                row["solo"] = st["solo"]
                row["schedule_s"] = st["schedule_s"]
        results.append(row)
    clk.__exit__(None, None, None)
    clocks = clk.summary()
    results = results[1:]  # drop the warm-up run
    cpu, parity = None, None
    if ctx.rank == 0 and ctx.world == 1 and not args.no_cpu_baseline:
        nchk = 96
        hosts = [x.cpu().numpy() for x in imgs[:nchk]]
        cpu, ref = served_cpu_baseline(corpus[:nchk], hosts, keep=True)
        # The oracle's results against the server's for the same requests,
        # all submitted at once so that they share launches.
        srv = S.Server(pool_bytes=16 << 30)
        try:
            ids = [srv.submit(imgs[k], served_stage_list(B, corpus[k])) for k in range(len(ref))]
            good = 0
            for k, i in enumerate(ids):
                y = srv.wait(i).cpu().numpy()
                if corpus[k]["dtype"] == "u8":
                    good += bool(y.shape == ref[k].shape and np.array_equal(y, ref[k]))
                else:
                    good += bool(y.shape == ref[k].shape and np.all(
                        np.abs(y.astype(np.float64) - ref[k]) <= 1e-5 * np.maximum(1.0, np.abs(ref[k].astype(np.float64)))))
                srv.release(i)
            mb = srv.stats()["mean_batch"]
        finally:
            srv.close()
        parity = {"checked": len(ref), "matching": good, "mean_batch": mb,
                  "summary": f"{good}/{len(ref)} requests equal to the oracle (u8 bit-exact, f32 within 1e-5 relative), "
                             f"served together"}
        del hosts, ref
    sat = results[-1]
    sat["rate"] = "saturation"
    results = results[:-1]
    top = results[-1]
    return {
        "metric": METRIC, "value": top["gpix_s"], "unit": "Gpix/s", "n_gpus": ctx.world, "steps": len(S_RATES),
        "warmup": 0, "ms_per_step": top["elapsed_s"] * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8+f32", "data": "synthetic",
        "config": {"workload": "served", "rates_req_s": list(S_RATES), "duration_s_per_rate": dur,
                   "corpus": S_CORPUS, "requests": "px log-uniform 0.1-8.3 MP, aspect 0.5-2, 1|3|4 ch, u8 80% / f32 20%, "
                   "1-4 stages of gray / gauss 5x5 / resize 0.5 / warpAffine +-30 deg / open 3x3",
                   "payloads": "device-resident corpus (the request rates exceed PCIe)", "pool_bytes": 64 << 30,
                   "per_rate": results, "saturation": sat,
                   "capacity_vs_plain": sat["gpix_s"] / sat["plain_gpix_s"],
                   "value_is": "Gpix/s at the highest rate (the offered load when the server keeps up); "
                               "p50/p99 per rate in per_rate; capacity in saturation"},
        "e2e": None,
        "roofline": None,
        "cpu_baseline": cpu,
        "parity": parity,
        "clocks": clocks,
        "gpu_launches": int(sum(r["launches"] for r in results)),
    }


def reference_served(args):
    """VISAR has no request server: its CPU path serves the corpus's requests
    one after another on all host threads (images generated on the host)."""
    synth = load_synth()
    corpus = synth.served_requests(S_CORPUS, seed=4)[:96]
    hosts = [synth.served_image(r, device="cpu").numpy() for r in corpus]
    cpu, _ = served_cpu_baseline(corpus, hosts, keep=False)
    v = cpu["value"]
    return {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "Gpix/s", "n_gpus": args.gpus, "steps": 1,
        "warmup": 1, "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u8+f32", "data": "synthetic",
        "config": {"workload": "served", "impl": "VISAR CPU path (C++ restatement, oracle/), one request at a time",
                   "service_p50_ms": cpu["service_p50_ms"], "service_p99_ms": cpu["service_p99_ms"],
                   "max_rate_req_s": cpu["max_rate_req_s"]},
        "cpu_baseline": cpu,
        "e2e": {"value": v, "unit": "Gpix/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


# ------------------------------------------------------------- plain-1080p

W, H = 1920, 1080
OPS = [
    # name, input bytes, output bytes, input pixels
    ("resize_linear_720p", W * H * 3, 1280 * 720 * 3, W * H),
    ("resize_area_half", W * H * 3, 960 * 540 * 3, W * H),
    ("warp_affine", W * H * 3, W * H * 3, W * H),
    ("warp_perspective", W * H * 3, W * H * 3, W * H),
    ("gaussian_f32_7x7", W * H * 4, W * H * 4, W * H),
]
PIX_PER_STEP = sum(o[3] for o in OPS)
ALG_BYTES = {o[0]: o[1] + o[2] for o in OPS}
H2D_BYTES = 4 * W * H * 3 + W * H * 4
D2H_BYTES = sum(o[2] for o in OPS)


def make_inputs():
    synth = load_synth()
    img = synth.base_image(H, W, 3, nrect=32, seed=1)
    f = synth.normal_f32(H, W, 1, seed=2)
    maff = synth.affine_params(W, H, seed=3)
    mper = synth.perspective_params(W, H, seed=4)
    return img, f, maff, mper


def op_call(m, name, img, f, maff, mper, outs):
    i = [o[0] for o in OPS].index(name)
    if i == 0:
        m.resize(img, (1280, 720), 1, dst=outs[0])
    elif i == 1:
        m.resize(img, (960, 540), 3, dst=outs[1])
    elif i == 2:
        m.warp_affine(img, maff, (W, H), 1, 0, 0.0, dst=outs[2])
    elif i == 3:
        m.warp_perspective(img, mper, (W, H), 1, 0, 0.0, dst=outs[3])
    else:
        m.gaussian_blur(f, (7, 7), 1.5, 0, 4, dst=outs[4])


def run_step(m, img, f, maff, mper, outs):
    """The five calls of one step, through module `m` (the CUDA binding or the oracle)."""
    for name, _, _, _ in OPS:
        op_call(m, name, img, f, maff, mper, outs)


def alloc_outs(torch=None, pinned=False):
    shapes = [((720, 1280, 3), np.uint8), ((540, 960, 3), np.uint8), ((H, W, 3), np.uint8), ((H, W, 3), np.uint8),
              ((H, W), np.float32)]
    outs = []
    for shp, dt in shapes:
        if torch is not None and not pinned:
            outs.append(torch.empty(shp, dtype=torch.uint8 if dt == np.uint8 else torch.float32, device="cuda"))
        elif torch is not None and pinned:
            outs.append(torch.empty(shp, dtype=torch.uint8 if dt == np.uint8 else torch.float32, pin_memory=True).numpy())
        else:
            outs.append(np.empty(shp, dt))
    return outs


def plain_oracle_step(O, item):
    img, f, maff, mper = item
    outs = alloc_outs()
    run_step(O, img, f, maff, mper, outs)
    return outs


def cv2_plain_step(cv2, item):
    """The plain-1080p calls through OpenCV (context timing only)."""
    img, f, maff, mper = item
    cv2.resize(img, (1280, 720), interpolation=cv2.INTER_LINEAR)
    cv2.resize(img, (960, 540), interpolation=cv2.INTER_AREA)
    cv2.warpAffine(img, maff, (W, H), flags=cv2.INTER_LINEAR, borderValue=0)
    cv2.warpPerspective(img, mper, (W, H), flags=cv2.INTER_LINEAR, borderValue=0)
    cv2.GaussianBlur(f, (7, 7), 1.5, borderType=cv2.BORDER_REFLECT_101)


def plain_cpu_baseline(img, f, maff, mper, budget_s=12.0, max_steps=20):
    """The oracle with all host threads (and with one) on a bounded number of
    steps; returns (cpu_baseline, the oracle's outputs of one step)."""
    items = [(img, f, maff, mper)] * max_steps
    n, dt, cores, outs = oracle_run(plain_oracle_step, items, 0, budget_s, keep=True)
    n1, dt1, _, _ = oracle_run(plain_oracle_step, items, 1, 6.0)
    return ({"value": PIX_PER_STEP * n / dt / 1e9, "unit": "Gpix/s", "cores": cores, "kind": "port",
             "sample": f"{n} steps of the plain-1080p workload ({n * 5} calls, {PIX_PER_STEP * n / 1e6:.1f} MP) in {dt:.1f} s",
             "one_thread": {"value": PIX_PER_STEP * n1 / dt1 / 1e9, "unit": "Gpix/s", "cores": 1,
                            "sample": f"{n1} steps in {dt1:.1f} s"},
             "cv2_context": cv2_context(cv2_plain_step, items, lambda it: PIX_PER_STEP, 3.0)}, outs[0])


def bench_plain(args, ctx):
    torch, vb = ctx.torch, ctx.vb
    img, f, maff, mper = make_inputs()
    d_img = torch.from_numpy(img).cuda()
    d_f = torch.from_numpy(f).cuda()
    d_outs = alloc_outs(torch)
    flush = L2Flush(torch)
    vb.set_async(True)
    for _ in range(args.warmup):
        run_step(vb, d_img, d_f, maff, mper, d_outs)
    ctx.barrier()
    n0 = vb.launch_count()
    with Clocks(ctx.dev) as clk:
        ms = ctx.timed(lambda: run_step(vb, d_img, d_f, maff, mper, d_outs), args.steps,
                       before=flush)
    launches = vb.launch_count() - n0
    ctx.barrier()
    ms_step = ctx.max_over_ranks(ms) / args.steps
    value = PIX_PER_STEP * ctx.world / (ms_step / 1e3) / 1e9
    clocks = clk.summary()

    per_op = {}
    for name, _, _, _ in OPS:
        for _ in range(3):
            op_call(vb, name, d_img, d_f, maff, mper, d_outs)
        n = max(5, args.steps // 2)
        per_op[name] = ctx.timed(lambda: op_call(vb, name, d_img, d_f, maff, mper, d_outs), n,
                                 before=flush) / n
    vb.set_async(False)
    dom = max(per_op, key=lambda k: per_op[k])
    peak, peak_kind = load_peaks()
    achieved = ALG_BYTES[dom] / (per_op[dom] / 1e3) / 1e9

    h_img = torch.empty(img.shape, dtype=torch.uint8, pin_memory=True).numpy()
    h_img[...] = img
    h_f = torch.empty(f.shape, dtype=torch.float32, pin_memory=True).numpy()
    h_f[...] = f
    h_outs = alloc_outs(torch, pinned=True)
    for _ in range(args.warmup):
        run_step(vb, h_img, h_f, maff, mper, h_outs)
    ctx.barrier()
    e_ms = ctx.max_over_ranks(ctx.timed(lambda: run_step(vb, h_img, h_f, maff, mper, h_outs), args.steps,
                                        before=flush)) / args.steps
    e2e = PIX_PER_STEP * ctx.world / (e_ms / 1e3) / 1e9
    ctx.barrier()
    cpu, parity = None, None
    if ctx.rank == 0 and ctx.world == 1 and not args.no_cpu_baseline:
        cpu, ref = plain_cpu_baseline(img, f, maff, mper)
        run_step(vb, d_img, d_f, maff, mper, d_outs)
        torch.cuda.synchronize()
        good = 0
        for (name, _, _, _), y, r in zip(OPS, d_outs, ref):
            y = y.cpu().numpy()
            if y.dtype == np.float32:
                good += bool(np.all(np.abs(y.astype(np.float64) - r) <= 1e-5 * np.maximum(1.0, np.abs(r.astype(np.float64)))))
            else:
                good += bool(np.array_equal(y, r))
        parity = {"checked": len(OPS), "matching": good,
                  "summary": f"{good}/{len(OPS)} calls equal to the oracle (u8 bit-exact, f32 within 1e-5 relative)"}
    return {
        "metric": METRIC, "value": value, "unit": "Gpix/s", "n_gpus": ctx.world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8+f32", "data": "synthetic",
        "config": {"workload": "plain-1080p", "frame": f"{W}x{H}x3 u8 + {W}x{H}x1 f32",
                   "ops": [o[0] for o in OPS], "pixels_per_step": PIX_PER_STEP,
                   "l2": "flushed before every timed step (256 MiB write, then a 256 MiB read)", "parallelism": f"replicas{ctx.world}",
                   "per_op_ms": per_op},
        "e2e": {"value": e2e, "unit": "Gpix/s", "h2d_bytes_per_step": H2D_BYTES, "d2h_bytes_per_step": D2H_BYTES,
                "ms_per_step": e_ms},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind, "traffic": load_traffic("plain-1080p", dom),
                     "alg_bytes_per_launch": ALG_BYTES[dom]},
        "cpu_baseline": cpu,
        "parity": parity,
        "clocks": clocks,
        "gpu_launches": launches,
    }


def reference_plain(args):
    from oracle import oracle as O
    O.set_num_threads(0)
    img, f, maff, mper = make_inputs()
    outs = alloc_outs()
    for _ in range(args.warmup):
        run_step(O, img, f, maff, mper, outs)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        run_step(O, img, f, maff, mper, outs)
    dt = time.perf_counter() - t0
    v = PIX_PER_STEP * args.steps / dt / 1e9
    return {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "Gpix/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8+f32", "data": "synthetic",
        "config": {"workload": "plain-1080p", "frame": f"{W}x{H}x3 u8 + {W}x{H}x1 f32",
                   "ops": [o[0] for o in OPS], "impl": "VISAR CPU path (C++ restatement, oracle/), all host threads"},
        "cpu_baseline": {"value": v, "unit": "Gpix/s", "cores": O.get_num_threads(), "kind": "port",
                         "sample": f"{args.steps} steps of plain-1080p"},
        "e2e": {"value": v, "unit": "Gpix/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


# ------------------------------------------------------------------ c0-640

C0_H, C0_W = 480, 640
C0_NAMES = ["gray", "gaussian 5x5", "threshold 127", "erode 3x3 rect", "dilate 3x3 rect"]
C0_BYTES = C0_H * C0_W * 3 + C0_H * C0_W + 4 * 2 * C0_H * C0_W  # in + out of each call


def c0_pipeline(m, x, outs=None):
    """The 640x480 pipeline through module m (the CUDA binding or the oracle);
    returns every intermediate."""
    o = outs or [None] * 5
    g = m.cvt_color(x, 6, dst=o[0])
    b = m.gaussian_blur(g, (5, 5), 0, 0, 4, dst=o[1])
    t = m.threshold(b, 127, 255, 0, dst=o[2])
    t = t[1] if isinstance(t, tuple) else t
    e = m.morphology(t, 0, 0, (3, 3), 1, dst=o[3])
    d = m.morphology(e, 1, 0, (3, 3), 1, dst=o[4])
    return [g, b, t, e, d]


def c0_input():
    return load_synth().base_image(C0_H, C0_W, 3, nrect=8, seed=0)


def bench_c0(args, ctx):
    """The 640x480 BGR pipeline, call by call through the C ABI on device
    images (value) and on host images (e2e), and as one batch plan replayed
    as a CUDA graph (graph_us)."""
    torch, vb = ctx.torch, ctx.vb
    from visar_b200 import batch as B
    x = c0_input()
    d_x = torch.from_numpy(x).cuda()
    d_outs = [torch.empty((C0_H, C0_W), dtype=torch.uint8, device="cuda") for _ in range(5)]
    flush = L2Flush(torch)
    vb.set_async(True)
    steps = max(args.steps, 50)
    for _ in range(args.warmup):
        c0_pipeline(vb, d_x, d_outs)
    ctx.barrier()
    n0 = vb.launch_count()
    with Clocks(ctx.dev) as clk:
        ms = ctx.timed(lambda: c0_pipeline(vb, d_x, d_outs), steps, before=flush)
    launches = vb.launch_count() - n0
    ctx.barrier()
    ms_step = ctx.max_over_ranks(ms) / steps
    clocks = clk.summary()
    px = C0_H * C0_W
    value = px * ctx.world / (ms_step / 1e3) / 1e9
    # The same pipeline as a batch plan of one image, replayed as a graph.
    plan = B.Batch([(C0_H, C0_W, 3, np.uint8)],
                   [B.gray(), B.gaussian((5, 5), 0.0, 0.0, 4), B.threshold(127, 255, 0), B.morphology(0, 0, (3, 3), 1),
                    B.morphology(1, 0, (3, 3), 1)])
    plan.input(0).copy_(d_x)
    for _ in range(args.warmup):
        plan.run_graph()
    g_ms = ctx.max_over_ranks(ctx.timed(plan.run_graph, steps, before=flush)) / steps
    vb.set_async(False)
    # e2e: host images in pinned memory through the per-call C ABI.
    h_x = torch.empty(x.shape, dtype=torch.uint8, pin_memory=True).numpy()
    h_x[...] = x
    h_outs = [torch.empty((C0_H, C0_W), dtype=torch.uint8, pin_memory=True).numpy() for _ in range(5)]
    for _ in range(args.warmup):
        c0_pipeline(vb, h_x, h_outs)
    e_ms = ctx.max_over_ranks(ctx.timed(lambda: c0_pipeline(vb, h_x, h_outs), steps)) / steps
    cpu, parity = None, None
    if ctx.rank == 0 and ctx.world == 1 and not args.no_cpu_baseline:
        items = [x] * 400
        n, dt, cores, ref = oracle_run(lambda O, it: c0_pipeline(O, it), items, 0, 3.0, keep=True)
        n1, dt1, _, _ = oracle_run(lambda O, it: c0_pipeline(O, it), items, 1, 3.0)
        cpu = {"value": n * px / dt / 1e9, "unit": "Gpix/s", "cores": cores, "kind": "port",
               "sample": f"{n} runs of the pipeline in {dt:.2f} s ({dt / n * 1e3:.3f} ms each)",
               "one_thread": {"value": n1 * px / dt1 / 1e9, "unit": "Gpix/s", "cores": 1,
                              "sample": f"{n1} runs in {dt1:.2f} s ({dt1 / n1 * 1e3:.3f} ms each)"}}
        got = c0_pipeline(vb, d_x, d_outs)
        torch.cuda.synchronize()
        ok = [bool(np.array_equal(a.cpu().numpy(), b)) for a, b in zip(got, ref[0])]
        ok_graph = bool(np.array_equal(plan.output(0).cpu().numpy(), ref[0][4]))
        ok_host = [bool(np.array_equal(a, b)) for a, b in zip(h_outs, ref[0])]
        parity = {"intermediates_bit_exact": dict(zip(C0_NAMES, ok)), "graph_bit_exact": ok_graph,
                  "host_calls_bit_exact": all(ok_host),
                  "summary": f"{sum(ok)}/5 intermediates bit-exact against the oracle"}
    return {
        "metric": METRIC, "value": value, "unit": "Gpix/s", "n_gpus": ctx.world, "steps": steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": "c0-640x480", "image": f"{C0_W}x{C0_H}x3 u8, seed 0, 8 rectangles", "stages": C0_NAMES,
                   "latency_us": ms_step * 1e3, "graph_us": g_ms * 1e3, "graph_gpix_s": px / (g_ms / 1e3) / 1e9,
                   "alg_bytes_per_step": C0_BYTES, "l2": "flushed before every timed step (256 MiB write, then a 256 MiB read)"},
        "e2e": {"value": px * ctx.world / (e_ms / 1e3) / 1e9, "unit": "Gpix/s", "h2d_bytes_per_step": C0_BYTES // 2,
                "d2h_bytes_per_step": 5 * px, "ms_per_step": e_ms},
        "cpu_baseline": cpu,
        "parity": parity,
        "clocks": clocks,
        "gpu_launches": launches,
    }


def reference_c0(args):
    from oracle import oracle as O
    O.set_num_threads(0)
    x = c0_input()
    steps = max(args.steps, 50)
    for _ in range(args.warmup):
        c0_pipeline(O, x)
    t0 = time.perf_counter()
    for _ in range(steps):
        c0_pipeline(O, x)
    dt = time.perf_counter() - t0
    v = steps * C0_H * C0_W / dt / 1e9
    return {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "Gpix/s", "n_gpus": args.gpus, "steps": steps,
        "warmup": args.warmup, "ms_per_step": dt / steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": "c0-640x480", "impl": "VISAR CPU path (C++ restatement, oracle/), all host threads"},
        "cpu_baseline": {"value": v, "unit": "Gpix/s", "cores": O.get_num_threads(), "kind": "port",
                         "sample": f"{steps} runs of the pipeline"},
        "e2e": {"value": v, "unit": "Gpix/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


# ------------------------------------------------------ next rows (f1-f3)

N_W, N_H = 3840, 2160


def timed_op(ctx, fn, n, flush):
    """Mean ms of fn over n launches, L2 flushed (256 MiB write, then a 256 MiB read) before each."""
    for _ in range(3):
        fn()
    return ctx.timed(fn, n, before=flush) / n


def bench_next(args, ctx):
    """The rows after the core path: fused gray + integer shrink
    (visar_gray_downsample) on 4K BGR / BGRA frames, pyrDown / pyrUp on 4K,
    undistort and remap on 1080p BGR. Per call: device-image time (CUDA
    events, L2 flushed), algorithmic GB/s against the HBM peak, the oracle on
    the host cores, and the results against the oracle."""
    torch, vb = ctx.torch, ctx.vb
    from oracle import oracle as O
    synth = load_synth()
    peak, peak_kind = load_peaks()
    flush = L2Flush(torch)
    n = max(10, args.steps)
    cpu_ok = ctx.rank == 0 and ctx.world == 1 and not args.no_cpu_baseline
    out = {}
    vb.set_async(True)

    def row(name, fn, nbytes, px, oracle_fn=None, got=None, cpu_items=None):
        ms = ctx.max_over_ranks(timed_op(ctx, fn, n, flush))
        r = {"ms": ms, "gpix_s": px / (ms / 1e3) / 1e9, "alg_bytes": nbytes, "gbs": nbytes / (ms / 1e3) / 1e9,
             "frac": nbytes / (ms / 1e3) / 1e9 / peak}
        if cpu_ok and oracle_fn is not None:
            nn, dt, cores, ref = oracle_run(lambda O_, it: oracle_fn(), [0] * 20, 0, 3.0, keep=True)
            n1, dt1, _, _ = oracle_run(lambda O_, it: oracle_fn(), [0] * 4, 1, 3.0)
            r["cpu_baseline"] = {"value": nn * px / dt / 1e9, "unit": "Gpix/s", "cores": cores, "kind": "port",
                                 "one_thread_gpix_s": n1 * px / dt1 / 1e9}
            g = got()
            r["bit_exact_vs_oracle"] = bool(np.array_equal(g, ref[0]))
        return r

    # f1: gray + integer shrink
    for cn in (3, 4):
        img = synth.base_image(N_H, N_W, cn, nrect=32, seed=20 + cn)
        d_img = torch.from_numpy(img).cuda()
        for k in (2, 3, 4, 8, 16):
            dst = torch.empty((N_H // k, N_W // k), dtype=torch.uint8, device="cuda")
            nbytes = N_W * N_H * cn + (N_W // k) * (N_H // k)
            out[f"gray_downsample.c{cn}.k{k}"] = row(
                f"gd{cn}{k}", lambda: vb.gray_downsample(d_img, k, dst=dst), nbytes, N_W * N_H,
                oracle_fn=lambda: O.gray_downsample(img, k), got=lambda: dst.cpu().numpy())
        # e2e: pinned host frame in, result out, through the C ABI
        torch.cuda.synchronize()
        h_img = torch.empty(img.shape, dtype=torch.uint8, pin_memory=True).numpy()
        h_img[...] = img
        h_dst = torch.empty((N_H // 2, N_W // 2), dtype=torch.uint8, pin_memory=True).numpy()
        e_ms = ctx.timed(lambda: vb.gray_downsample(h_img, 2, dst=h_dst), n) / n
        out[f"gray_downsample.c{cn}.k2"]["e2e_gpix_s"] = N_W * N_H / (e_ms / 1e3) / 1e9
    # f2: pyramids
    img = synth.base_image(N_H, N_W, 3, nrect=32, seed=31)
    d_img = torch.from_numpy(img).cuda()
    dd = torch.empty((N_H // 2, N_W // 2, 3), dtype=torch.uint8, device="cuda")
    out["pyr_down.u8.c3.4k"] = row("pd", lambda: vb.pyr_down(d_img, 4, dst=dd), N_W * N_H * 3 * 5 // 4, N_W * N_H,
                                   oracle_fn=lambda: O.pyr_down(img, 4), got=lambda: dd.cpu().numpy())
    half = np.ascontiguousarray(img[::2, ::2])
    d_half = torch.from_numpy(half).cuda()
    du = torch.empty((N_H, N_W, 3), dtype=torch.uint8, device="cuda")
    out["pyr_up.u8.c3.to4k"] = row("pu", lambda: vb.pyr_up(d_half, 4, dst=du), N_W * N_H * 3 * 5 // 4, N_W * N_H // 4,
                                   oracle_fn=lambda: O.pyr_up(half, 4), got=lambda: du.cpu().numpy())
    f = synth.normal_f32(N_H, N_W, 1, seed=32)
    d_f = torch.from_numpy(f).cuda()
    dfd = torch.empty((N_H // 2, N_W // 2), dtype=torch.float32, device="cuda")
    out["pyr_down.f32.c1.4k"] = row("pdf", lambda: vb.pyr_down(d_f, 4, dst=dfd), N_W * N_H * 4 * 5 // 4, N_W * N_H,
                                    oracle_fn=lambda: O.pyr_down(f, 4), got=lambda: dfd.cpu().numpy())
    # f3: undistort / maps / remap on 1080p BGR
    W1, H1 = 1920, 1080
    img = synth.base_image(H1, W1, 3, nrect=32, seed=33)
    d_img = torch.from_numpy(img).cuda()
    K = np.array([[1000.0, 0, 959.5], [0, 1000.0, 539.5], [0, 0, 1]])
    dist = [-0.28, 0.09, 0.0008, -0.0004, -0.012]
    du = torch.empty_like(d_img)
    out["undistort.u8.c3.1080p"] = row("ud", lambda: vb.undistort(d_img, K, dist, None, dst=du), 2 * W1 * H1 * 3, W1 * H1,
                                       oracle_fn=lambda: O.undistort(img, K, dist), got=lambda: du.cpu().numpy())
    mx = torch.empty((H1, W1), dtype=torch.float32, device="cuda")
    my = torch.empty((H1, W1), dtype=torch.float32, device="cuda")
    out["init_undistort_map.1080p"] = row(
        "um", lambda: vb.init_undistort_rectify_map(K, dist, None, None, (W1, H1), mapx=mx, mapy=my), 8 * W1 * H1, W1 * H1,
        oracle_fn=lambda: O.init_undistort_rectify_map(K, dist, None, None, (W1, H1))[0], got=lambda: mx.cpu().numpy())
    dr = torch.empty_like(d_img)
    hmx, hmy = mx.cpu().numpy(), my.cpu().numpy()
    out["remap.u8.c3.1080p"] = row("rm", lambda: vb.remap(d_img, mx, my, 0.0, dst=dr), 2 * W1 * H1 * 3 + 8 * W1 * H1, W1 * H1,
                                   oracle_fn=lambda: O.remap(img, hmx, hmy, 0.0), got=lambda: dr.cpu().numpy())
    torch.cuda.synchronize()
    vb.set_async(False)
    return {"workload": "next-rows", "peak_gbs": peak, "peak_kind": peak_kind,
            "timing": "device images, CUDA events, L2 flushed (256 MiB write, then a 256 MiB read) before each launch",
            "alg_bytes": "source + destination bytes once (remap adds its two f32 maps)", "calls": out}


# -------------------------------------------------------------------- main

WORKLOADS = {"batched-mixed": (bench_batched, reference_batched), "plain-1080p": (bench_plain, reference_plain),
             "video-4k": (bench_video, reference_video), "served": (bench_served, reference_served),
             "c0": (bench_c0, reference_c0), "next-rows": (bench_next, None)}
# The other configs, reported as sub-objects of the batched-mixed line's
# config when it runs on one GPU (the headline stays batched-mixed).
SUBS = [("c0", "c0"), ("plain_1080p", "plain-1080p"), ("video_4k", "video-4k"), ("served", "served"),
        ("next_rows", "next-rows")]
SUB_DROP = ("metric", "n_gpus", "higher_is_better", "scaling", "vs_baseline", "data")


def sub_line(line):
    if "metric" not in line:
        return line
    return {k: v for k, v in line.items() if k not in SUB_DROP}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="batched-mixed", choices=sorted(WORKLOADS))
    ap.add_argument("--only", action="store_true",
                    help="batched-mixed alone (by default a 1-GPU run adds the other configs under config)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="built-in launch defaults instead of the tuned table")
    ap.add_argument("--tuning", default=None, help="tuned table to load, or to write when it was made elsewhere")
    ap.add_argument("--duration", type=float, default=20.0, help="seconds per arrival rate (served workload)")
    ap.add_argument("--images", type=int, default=0,
                    help="batched-mixed: the first N images only (a reduced plan for profiler captures; not a bench line)")
    ap.add_argument("--rows", type=int, default=0, choices=[0, 8, 32, 64, 128],
                    help="batched-mixed: strip tile height (with --images: the full plan's 64 on a reduced plan)")
    ap.add_argument("--frames", type=int, default=0,
                    help="video-4k: N frames in HBM instead of 300 (a reduced case for profiler captures; not a bench line)")
    ap.add_argument("--instances", type=int, default=0,
                    help="video-4k: graph instances (and streams) taking the frames in turn (default 4)")
    args = ap.parse_args()
    global IMAGE_LIMIT, V_FRAMES, V_INSTANCES
    IMAGE_LIMIT = max(0, args.images)
    if args.frames > 0:
        V_FRAMES = args.frames
    if args.instances > 0:
        V_INSTANCES = args.instances
    ours, ref = WORKLOADS[args.workload]
    subs = args.workload == "batched-mixed" and not args.only and args.gpus == 1
    if args.impl == "reference":
        if int(os.environ.get("RANK", "0")) != 0:
            return 0
        if ref is None:
            print(json.dumps({"impl": "reference", "unavailable": f"{args.workload}: timed against the oracle inside "
                              "the GPU arm's line"}), flush=True)
            return 0
        line = ref(args)
        if subs:
            for key, wl in SUBS:
                if WORKLOADS[wl][1] is not None:
                    line["config"][key] = sub_line(WORKLOADS[wl][1](args))
        print(json.dumps(line), flush=True)
        return 0
    args.warmup = max(3, args.warmup)
    ctx = Ctx(args)
    line = ours(args, ctx)
    if "metric" not in line:  # a section of the full line run on its own
        line = {"metric": METRIC, "config": line}
    if subs and ctx.world == 1:
        sub_args = argparse.Namespace(**vars(args))
        sub_args.tuning = None
        for key, wl in SUBS:
            import gc
            gc.collect()
            ctx.torch.cuda.synchronize()
            ctx.torch.cuda.empty_cache()
            line["config"][key] = sub_line(WORKLOADS[wl][0](sub_args, ctx))
    ctx.barrier()
    if ctx.rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
