"""Run the reference's own CPU BiCGStab(4) (oracle/_ref: bicgstabl.h over
cpu_vector_operations<double> with Dot2, an OpenMP CSR operator with one FMA
per nonzero in index order) to convergence on the benchmark's solver system
(2-D convection-diffusion, 1024x1024, Peclet 50, RHS U[-1,1] seed 2024,
tol 1e-10) and record:

* the monitor's per-cycle residual history (default_monitor.h:202-212,
  ||r_0|| once per BiCGStab(4) cycle) and iteration count with ONE Dot2
  thread -- the only deterministic configuration of the reference's CPU
  path: its threaded Dot2 (common/threaded_reduction.h:220-349) merges each
  thread's (s, c) pair into shared accumulators under a mutex in the order
  the threads finish, so with more than one thread the last bits of every
  inner product, and with them the iterates, change from run to run;
* runs with 2, 4, 8 and 16 Dot2 threads (four each): their iteration counts
  (iters_by_run) and how far their residual histories drift from the
  one-thread history -- the reference's own run-to-run spread under
  last-bit changes of its reductions.  The drift is measured on the running
  minimum of the relative residual (the convergence envelope; single cycles
  of BiCGStab(l) on this non-normal operator spike by orders of magnitude
  wherever a near-breakdown lands): envelope_spread_log10 is the largest
  |log10(env_run / env_1)| over the cycles where both exceed 1e-8.

The benchmark's CPU baseline times a few reference cycles on the GPU box's
host and scales by iters_median.  Takes about twenty minutes on 8 cores.

    python tests/golden/make_solver_calibration.py
"""
import json
import os
import platform
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

import oracle  # noqa: E402
from high_precision_blas1_b200 import problems  # noqa: E402

RUNS = tuple((f"{t}{c}", t) for t in (2, 4, 8, 16) for c in "abcd")
FLOOR = 1e-8


def envelope(h, bn):
    return np.minimum.accumulate(h[:, 1] / bn)


def main():
    A = problems.convdiff2d(1024, peclet=50.0)
    b = problems.rhs_uniform(A.n, 2024)
    bn = float(np.linalg.norm(b))
    ok, it, res, sec, x, hist = oracle.ref_cpu_solve_history(0, A, b, np.zeros(A.n), 4, 1e-10, 20000, 1, 1)
    r = b - A.matvec(x)
    e1 = envelope(hist, bn)
    counts = {"1": it}
    spread = 0.0
    for name, t in RUNS:
        okt, itt, _, _, _, ht = oracle.ref_cpu_solve_history(0, A, b, np.zeros(A.n), 4, 1e-10, 20000, 1, t)
        counts[name] = itt if okt else None
        et = envelope(ht, bn)
        k = min(et.size, e1.size)
        m = (et[:k] > FLOOR) & (e1[:k] > FLOOR)
        spread = max(spread, float(np.abs(np.log10(et[:k][m] / e1[:k][m])).max()))
        print("threads", t, "iters", itt, "envelope spread", spread, flush=True)
    vals = [v for v in counts.values() if v]
    out = {"system": "convdiff2d N=1024 Pe=50, rhs seed 2024", "solver": "reference bicgstabl.h L=4, Dot2",
           "dot2_threads": 1, "converged": ok, "iters": it, "monitor_resid": res, "rhs_norm": bn,
           "true_rel_residual": float(np.linalg.norm(r) / bn), "seconds": sec,
           "host_cores": os.cpu_count(), "host": platform.processor() or platform.machine(),
           "when": time.strftime("%Y-%m-%d"),
           "iters_by_run": counts, "iters_median": int(np.median(vals)), "iters_min": min(vals),
           "iters_max": max(vals), "envelope_floor": FLOOR, "envelope_spread_log10": spread,
           "history": [[int(i), float(v)] for i, v in hist]}
    (HERE / "ref_solver_calibration.json").write_text(json.dumps(out, indent=1) + "\n")
    print({k: v for k, v in out.items() if k != "history"})


if __name__ == "__main__":
    main()
