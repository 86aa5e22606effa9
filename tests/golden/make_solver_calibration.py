"""Run the reference's own CPU BiCGStab(4) (oracle/_ref: bicgstabl.h over
cpu_vector_operations<double> with Dot2) to convergence on the benchmark's
solver system (2-D convection-diffusion, 1024x1024, Peclet 50, RHS U[-1,1]
seed 2024, tol 1e-10) and record its iteration count.  The benchmark's CPU
baseline times a few reference cycles on the GPU box's host and scales by
this count.  Takes about a minute on 8 cores.

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


def main():
    A = problems.convdiff2d(1024, peclet=50.0)
    b = problems.rhs_uniform(A.n, 2024)
    ok, it, res, sec, x = oracle.ref_cpu_solve(0, A, b, np.zeros(A.n), 4, 1e-10, 20000, 1, -1)
    r = b - A.matvec(x)
    out = {"system": "convdiff2d N=1024 Pe=50, rhs seed 2024", "solver": "reference bicgstabl.h L=4, Dot2",
           "converged": ok, "iters": it, "monitor_resid": res,
           "true_rel_residual": float(np.linalg.norm(r) / np.linalg.norm(b)),
           "seconds": sec, "host_cores": os.cpu_count(), "host": platform.processor() or platform.machine(),
           "when": time.strftime("%Y-%m-%d")}
    (HERE / "ref_solver_calibration.json").write_text(json.dumps(out, indent=1) + "\n")
    print(out)


if __name__ == "__main__":
    main()
