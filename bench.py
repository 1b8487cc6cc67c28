"""Benchmark of the imgproc stencil-and-warp path on B200.

Workload (default, `plain-1080p`): one 1920x1080 u8 BGR frame (gradient +
noise + 32 rectangles, seeded) run through the plain per-call C ABI:
resize INTER_LINEAR -> 1280x720, resize INTER_AREA -> 960x540 (exact half),
warpAffine INTER_LINEAR BORDER_CONSTANT 0 (seeded rotation +-30 deg, scale
0.8-1.2, translation +-50 px), warpPerspective INTER_LINEAR (corners jittered
+-80 px), plus one 1920x1080 f32 N(0,1) frame through GaussianBlur 7x7
sigma 1.5. One step = those five calls. Gpix/s counts input pixels
(width x height) once per call.

  value : inputs resident in HBM, CUDA events on the launching stream,
          L2 flushed (256 MiB write) before every timed step
  e2e   : the same calls on pinned host buffers through the C ABI, so every
          step includes the host->device and device->host copies
  roofline : the dominant kernel (most total time), algorithmic bytes
          (input + output image bytes) / its average event-timed duration,
          against MEASURED_PEAKS.json's HBM copy bandwidth

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
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

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
    from visar_b200 import synth
    img = synth.base_image(H, W, 3, nrect=32, seed=1)
    f = synth.normal_f32(H, W, 1, seed=2)
    maff = synth.affine_params(W, H, seed=3)
    mper = synth.perspective_params(W, H, seed=4)
    return img, f, maff, mper


def run_step(m, img, f, maff, mper, outs):
    """The five calls of one step, through module `m` (the CUDA binding or the oracle)."""
    m.resize(img, (1280, 720), 1, dst=outs[0])
    m.resize(img, (960, 540), 3, dst=outs[1])
    m.warp_affine(img, maff, (W, H), 1, 0, 0.0, dst=outs[2])
    m.warp_perspective(img, mper, (W, H), 1, 0, 0.0, dst=outs[3])
    m.gaussian_blur(f, (7, 7), 1.5, 0, 4, dst=outs[4])


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


def alloc_outs(like_u8, like_f32, torch=None, pinned=False):
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


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = os.path.join(ROOT, "gpurun_out" if os.path.isdir(os.path.join(ROOT, "gpurun_out")) else ".",
                                 f".clocks_{os.getpid()}.csv")

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


def cpu_baseline(img, f, maff, mper, budget_s=12.0, max_steps=20):
    """The oracle (C++ restatement of VISAR's CPU path) with all host threads, on a bounded sample."""
    from oracle import oracle as O
    O.set_num_threads(0)
    outs = alloc_outs(None, None)
    run_step(O, img, f, maff, mper, outs)  # warm-up
    t0 = time.perf_counter()
    n = 0
    while n < max_steps and (time.perf_counter() - t0) < budget_s:
        run_step(O, img, f, maff, mper, outs)
        n += 1
    dt = time.perf_counter() - t0
    return {"value": PIX_PER_STEP * n / dt / 1e9, "unit": "Gpix/s", "cores": O.get_num_threads(), "kind": "port",
            "sample": f"{n} steps of the plain-1080p workload ({n * 5} calls, {PIX_PER_STEP * n / 1e6:.1f} MP) in {dt:.1f} s"}


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


def bench_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import oracle as O
    O.set_num_threads(0)
    img, f, maff, mper = make_inputs()
    outs = alloc_outs(None, None)
    for _ in range(max(1, min(args.warmup, 2))):
        run_step(O, img, f, maff, mper, outs)
    steps = max(1, min(args.steps, 10))
    t0 = time.perf_counter()
    for _ in range(steps):
        run_step(O, img, f, maff, mper, outs)
    dt = time.perf_counter() - t0
    v = PIX_PER_STEP * steps / dt / 1e9
    line = {
        "impl": "reference", "metric": "Gpix/s (plain per-call, bit-exact)", "value": v, "unit": "Gpix/s",
        "n_gpus": args.gpus, "steps": steps, "warmup": args.warmup, "ms_per_step": dt / steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8+f32", "data": "synthetic",
        "config": {"workload": "plain-1080p", "frame": f"{W}x{H}x3 u8 + {W}x{H}x1 f32",
                   "ops": [o[0] for o in OPS], "impl": "VISAR CPU path (C++ restatement, oracle/), all host threads"},
        "cpu_baseline": {"value": v, "unit": "Gpix/s", "cores": O.get_num_threads(), "kind": "port",
                         "sample": f"{steps} steps of plain-1080p"},
        "e2e": {"value": v, "unit": "Gpix/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        return bench_reference(args)
    args.warmup = max(3, args.warmup)

    import torch
    rank, world, dist = dist_setup(args.gpus)
    if dist is None:
        torch.cuda.set_device(0)
    import visar_b200 as vb
    dev = torch.cuda.current_device()
    # A real stream (torch's default stream has a NULL handle, which the
    # library reads as "use your own stream"): events, the L2 flush and the
    # library's kernels are all ordered on it.
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    vb.set_stream(stream)

    img, f, maff, mper = make_inputs()
    d_img = torch.from_numpy(img).cuda()
    d_f = torch.from_numpy(f).cuda()
    d_outs = alloc_outs(None, None, torch=torch)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # ---------------------------------------------------------- value (HBM-resident)
    vb.set_async(True)
    for _ in range(args.warmup):
        run_step(vb, d_img, d_f, maff, mper, d_outs)
    barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    n0 = vb.launch_count()
    with Clocks(dev) as clk:
        for i in range(args.steps):
            flush.fill_(i & 0xFF)
            ev[i][0].record(stream)
            run_step(vb, d_img, d_f, maff, mper, d_outs)
            ev[i][1].record(stream)
        torch.cuda.synchronize()
    launches = vb.launch_count() - n0
    barrier()
    ms_total = sum(a.elapsed_time(b) for a, b in ev)
    ms_total = max_over_ranks(ms_total)
    ms_step = ms_total / args.steps
    value = PIX_PER_STEP * world / (ms_step / 1e3) / 1e9
    clocks = clk.summary()

    # ------------------------------------------------- per-kernel roofline (device)
    per_op = {}
    for name, _, _, _ in OPS:
        for _ in range(3):
            op_call(vb, name, d_img, d_f, maff, mper, d_outs)
        es = []
        for i in range(max(5, args.steps // 2)):
            flush.fill_(i & 0xFF)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            op_call(vb, name, d_img, d_f, maff, mper, d_outs)
            b.record(stream)
            es.append((a, b))
        torch.cuda.synchronize()
        per_op[name] = float(np.mean([a.elapsed_time(b) for a, b in es]))
    vb.set_async(False)
    dom = max(per_op, key=lambda k: per_op[k])
    peak, peak_kind = load_peaks()
    achieved = ALG_BYTES[dom] / (per_op[dom] / 1e3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as fh:
            traffic = json.load(fh).get("plain-1080p", {}).get(dom)

    # ------------------------------------------------------- e2e (pinned host buffers)
    h_img = torch.empty(img.shape, dtype=torch.uint8, pin_memory=True).numpy()
    h_img[...] = img
    h_f = torch.empty(f.shape, dtype=torch.float32, pin_memory=True).numpy()
    h_f[...] = f
    h_outs = alloc_outs(None, None, torch=torch, pinned=True)
    for _ in range(args.warmup):
        run_step(vb, h_img, h_f, maff, mper, h_outs)
    barrier()
    e_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for i in range(args.steps):
        flush.fill_(i & 0xFF)
        e_ev[i][0].record(stream)
        run_step(vb, h_img, h_f, maff, mper, h_outs)
        e_ev[i][1].record(stream)
    torch.cuda.synchronize()
    e_ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in e_ev)) / args.steps
    e2e = PIX_PER_STEP * world / (e_ms / 1e3) / 1e9
    barrier()

    if rank == 0:
        cpu = None if args.no_cpu_baseline or world > 1 else cpu_baseline(img, f, maff, mper)
        line = {
            "metric": "Gpix/s (plain per-call, bit-exact)", "value": value, "unit": "Gpix/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8+f32", "data": "synthetic",
            "config": {"workload": "plain-1080p", "frame": f"{W}x{H}x3 u8 + {W}x{H}x1 f32",
                       "ops": [o[0] for o in OPS], "pixels_per_step": PIX_PER_STEP,
                       "l2": "flushed before every timed step (256 MiB write)", "parallelism": f"replicas{world}",
                       "per_op_ms": per_op},
            "e2e": {"value": e2e, "unit": "Gpix/s", "h2d_bytes_per_step": H2D_BYTES, "d2h_bytes_per_step": D2H_BYTES,
                    "ms_per_step": e_ms},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic,
                         "alg_bytes_per_launch": ALG_BYTES[dom]},
            "cpu_baseline": cpu,
            "clocks": clocks,
            "gpu_launches": launches,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
