#!/usr/bin/env python
"""Benchmark of the compensated BLAS-1 hot path on B200.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload solver|dot2]

Workloads (synthetic, seeded, in the shapes of the reference's configs):
  dot2    Dot2 of two float64 GenDot vectors, n = 1,048,576, cond ~ 1e20+;
          a step = one Dot2 over one pair; 16 resident pairs (268 MB, above
          the 126 MB L2) are rotated so every step streams from HBM.
  solver  (default) BiCGStab(4) in float64 with Dot2 reductions on the 2-D
          5-point convection-diffusion matrix, 1024x1024 grid, Peclet 50,
          RHS U[-1,1], to a 1e-10 true relative residual; a step = one solve.

Multi-GPU (torchrun): replicas -- every rank runs the same workload on its
own GPU with no data-path collective; ranks meet at a barrier around the
timed region and the reported time is the max over ranks.

--impl reference times the reference's own CPU implementation (compiled from
its sources into oracle/_ref) on the host cores of this box, rank 0 only.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402

PEAKS_FILE = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0
L2_BYTES = 126 * 1024 * 1024


# ----------------------------------------------------------------- helpers
def peaks():
    try:
        d = json.loads(PEAKS_FILE.read_text())
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None
        time.sleep(0.15)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.flush()
        rows = []
        for line in Path(self.f.name).read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_init(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


# ------------------------------------------------------------ reference arm
def run_reference(args, ws, rank):
    """The reference's own CPU implementation, rank 0 only."""
    if rank != 0:
        return
    import oracle
    ref = oracle.ref()
    cores = os.cpu_count() or 1
    if ref is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU code (oracle/_ref) was not built"}))
        return
    if args.workload == "dot2":
        res = ref_dot2(ref, args, cores)
    else:
        res = ref_solver(args, cores)
    print(json.dumps(res))


def ref_dot2(ref, args, cores):
    from high_precision_blas1_b200 import _lib
    n = 1 << 20
    x = np.zeros(n)
    y = np.zeros(n)
    _lib.lib.hpb_gendot_f64(1, n, 1e20, x.ctypes.data, y.ctypes.data, None)
    per_step = 200  # threaded Dot2 calls per step (~0.1-0.3 s of CPU work)
    for _ in range(args.warmup):
        ref.ref_threaded_dot_f64_loop(n, x.ctypes.data, y.ctypes.data, 0, 5)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ref.ref_threaded_dot_f64_loop(n, x.ctypes.data, y.ctypes.data, 0, per_step)
    dt = time.perf_counter() - t0
    gbs = 16.0 * n * per_step * args.steps / dt / 1e9
    return {
        "impl": "reference", "metric": "dot2_hbm_gbs", "value": gbs, "unit": "GB/s", "higher_is_better": True,
        "n_gpus": 0, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": "dot2 f64 GenDot n=1048576 cond~1e20"},
        "cpu_baseline": {"value": gbs, "unit": "GB/s", "cores": cores, "kind": "reference",
                         "sample": f"{per_step} threaded_reduction<double>::dot calls per step, "
                                   f"hardware_concurrency threads"},
        "e2e": {"value": gbs, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def ref_solver(args, cores):
    raise SystemExit("solver workload not built yet")


# ------------------------------------------------------------------ our arm
def bench_dot2(args, ws, rank, local, torch, dist):
    from high_precision_blas1_b200 import Context, _lib
    L = _lib.lib
    n = 1 << 20
    x = np.zeros(n)
    y = np.zeros(n)
    L.hpb_gendot_f64(1 + rank, n, 1e20, x.ctypes.data, y.ctypes.data, None)
    R = max(4, int(np.ceil(2.0 * L2_BYTES / (16.0 * n))))  # rotated pairs, > L2
    xs = [torch.from_numpy(x).cuda() for _ in range(R)]
    ys = [torch.from_numpy(y).cuda() for _ in range(R)]
    out = torch.zeros(4 * (args.steps + args.warmup + 8), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    with Context(local, stream.cuda_stream) as ctx:
        for i in range(args.warmup):
            ctx.check(L.hpb_dot2_f64(ctx.h, n, xs[i % R].data_ptr(), ys[i % R].data_ptr(), out.data_ptr()))
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        clk = ClockSampler(local)
        clk.start()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        t_all0 = torch.cuda.Event(enable_timing=True)
        t_all1 = torch.cuda.Event(enable_timing=True)
        launches0 = L.hpb_launch_count()
        t_all0.record(stream)
        for i in range(args.steps):
            evs[i][0].record(stream)
            ctx.check(L.hpb_dot2_f64(ctx.h, n, xs[i % R].data_ptr(), ys[i % R].data_ptr(),
                                     out.data_ptr() + 32 * (i % 8)))
            evs[i][1].record(stream)
        t_all1.record(stream)
        torch.cuda.synchronize()
        launches = L.hpb_launch_count() - launches0
        clocks = clk.stop()
        total_ms = t_all0.elapsed_time(t_all1)
        per_launch_ms = [a.elapsed_time(b) for a, b in evs]
        if dist:
            tt = torch.tensor([total_ms], device="cuda")
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            total_ms = tt.item()

        # e2e: pinned host inputs -> H2D -> Dot2 -> D2H of (hi, lo), every step
        hx = torch.from_numpy(x).pin_memory()
        hy = torch.from_numpy(y).pin_memory()
        hres = torch.zeros(4, dtype=torch.float64).pin_memory()
        dx, dy = xs[0], ys[0]
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        for _ in range(2):
            dx.copy_(hx, non_blocking=True)
            dy.copy_(hy, non_blocking=True)
            ctx.check(L.hpb_dot2_f64(ctx.h, n, dx.data_ptr(), dy.data_ptr(), out.data_ptr()))
            hres.copy_(out[:4], non_blocking=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            dx.copy_(hx, non_blocking=True)
            dy.copy_(hy, non_blocking=True)
            ctx.check(L.hpb_dot2_f64(ctx.h, n, dx.data_ptr(), dy.data_ptr(), out.data_ptr()))
            hres.copy_(out[:4], non_blocking=True)
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_ms = e0.elapsed_time(e1)
        result = float(hres[0])

    bytes_step = 16.0 * n
    value = bytes_step * args.steps * ws / (total_ms * 1e-3) / 1e9
    kern_ms = float(np.mean(per_launch_ms))
    hbm, src = peaks()
    achieved = bytes_step / (kern_ms * 1e-3) / 1e9
    return {
        "metric": "dot2_hbm_gbs", "value": value, "unit": "GB/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "dot2 f64 GenDot n=1048576 cond~1e20", "n": n, "rotated_pairs": R,
                   "l2": "inputs rotated over 16.8 MB x R > L2", "parallelism": f"replicas{ws}"},
        "roofline": {"kernel": "reduce_kernel<double,DOT2>", "bound": "hbm", "achieved": achieved, "peak": hbm,
                     "peak_source": src, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": None, "algorithmic_bytes_per_launch": bytes_step,
                     "avg_launch_us": kern_ms * 1e3},
        "e2e": {"value": bytes_step * args.steps / (e2e_ms * 1e-3) / 1e9, "unit": "GB/s",
                "h2d_bytes_per_step": int(2 * 8 * n), "d2h_bytes_per_step": 32},
        "gpu_launches": int(launches),
        "clocks": clocks,
        "result_check": result,
    }


def cpu_baseline_dot2():
    import oracle
    ref = oracle.ref()
    from high_precision_blas1_b200 import _lib
    n = 1 << 20
    x = np.zeros(n)
    y = np.zeros(n)
    _lib.lib.hpb_gendot_f64(1, n, 1e20, x.ctypes.data, y.ctypes.data, None)
    cores = os.cpu_count() or 1
    if ref is not None:
        reps = 10
        t0 = time.perf_counter()
        tot = 0
        while time.perf_counter() - t0 < 5.0:
            ref.ref_threaded_dot_f64_loop(n, x.ctypes.data, y.ctypes.data, 0, reps)
            tot += reps
        dt = time.perf_counter() - t0
        return {"value": 16.0 * n * tot / dt / 1e9, "unit": "GB/s", "cores": cores, "kind": "reference",
                "sample": f"{tot} threaded_reduction<double>::dot calls (n=2^20, {cores} threads), ~5 s"}
    t0 = time.perf_counter()
    tot = 0
    while time.perf_counter() - t0 < 5.0:
        oracle.dot2_seq(x, y)
        tot += 1
    dt = time.perf_counter() - t0
    return {"value": 16.0 * n * tot / dt / 1e9, "unit": "GB/s", "cores": 1, "kind": "port",
            "sample": f"{tot} sequential Dot2 calls (n=2^20), ~5 s"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--warmup", type=int, default=None)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["solver", "dot2"], default="dot2")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.steps is None:
        args.steps = 200 if args.workload == "dot2" else 3
    if args.warmup is None:
        args.warmup = 20 if args.workload == "dot2" else 3
    args.warmup = max(args.warmup, 3)
    ws, rank, local = dist_init(args)

    if args.impl == "reference":
        run_reference(args, ws, rank)
        return

    import torch
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(local)
    try:
        if args.workload == "dot2":
            res = bench_dot2(args, ws, rank, local, torch, dist)
        else:
            raise SystemExit("solver workload not built yet")
        if rank == 0:
            if not args.no_cpu_baseline:
                res["cpu_baseline"] = cpu_baseline_dot2()
            print(json.dumps(res))
    finally:
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
