"""GPU Krylov solvers through the C ABI (the plain drop-in path) against the
reference's own CPU solvers (bicgstabl.h / gmres.h over
cpu_vector_operations, compiled from the reference sources into
oracle/_ref) and against the oracle's exact residual.

Tolerances: the true relative residual ||b - A x|| / ||b|| of every
converged solve is <= 1.05 * rel_tol (the monitor tests the recurrence
residual); iteration counts of the GPU BiCGStab(l) / GMRES(m) equal the
reference CPU counts to within one cycle (the solvers run the same
recurrences; Dot2 results differ only in the last bits between the GPU tree
and the CPU sequential order)."""
import ctypes as C

import numpy as np
import pytest

import oracle
from gpu_utils import dev, host
from high_precision_blas1_b200 import _lib, problems

pytestmark = pytest.mark.gpu

DT = {"f32": np.float32, "f64": np.float64, "c64": np.complex64, "c128": np.complex128}


def solve(ctx, torch, t, A, b, params, x0=None, hist_cap=0, host_api=False):
    x0 = np.zeros(A.n, dtype=DT[t]) if x0 is None else x0.astype(DT[t])
    rep = _lib.hpb_solver_report()
    hist = np.zeros(2 * max(hist_cap, 1))
    if host_api:
        x = x0.copy()
        arrs = [np.ascontiguousarray(a) for a in (A.row_ptr, A.col_ind, A.val.astype(DT[t]), b.astype(DT[t]))]
        st = getattr(_lib.lib, f"hpb_csr_solve_{t}_host")(C.byref(params), A.n, A.nnz, *[a.ctypes.data for a in arrs],
                                                          x.ctypes.data, C.byref(rep), hist.ctypes.data, hist_cap)
    else:
        d = [dev(torch, a) for a in (A.row_ptr, A.col_ind, A.val.astype(DT[t]), b.astype(DT[t]), x0)]
        st = getattr(_lib.lib, f"hpb_csr_solve_{t}")(C.byref(params), A.n, A.nnz, *[a.data_ptr() for a in d],
                                                     C.byref(rep), hist.ctypes.data, hist_cap)
        torch.cuda.synchronize()
        x = host(d[4])
    return st, rep, x, hist[:2 * rep.history_len].reshape(-1, 2)


def true_rel(A, b, x):
    r = b.astype(np.complex128 if np.iscomplexobj(x) else np.float64) - A.matvec(x.astype(np.complex128 if np.iscomplexobj(x) else np.float64))
    return np.linalg.norm(r) / np.linalg.norm(b)


@pytest.mark.parametrize("N,L", [(32, 4), (64, 4), (48, 2)])
def test_bicgstabl_f64_matches_reference_cpu(gpu, N, L):
    ctx, torch = gpu
    A = problems.convdiff2d(N)
    b = problems.rhs_uniform(A.n, 7)
    p = _lib.solver_params("bicgstabl", basis=L, rel_tol=1e-10, max_iters=20000)
    st, rep, x, hist = solve(ctx, torch, "f64", A, b, p, hist_cap=4096)
    assert st == 0 and rep.converged == 1
    assert true_rel(A, b, x) <= 1.05e-10
    assert rep.true_resid_norm / rep.true_rhs_norm <= 1.05e-10
    assert hist.shape[0] == rep.iters // L + 1
    ref = oracle.ref_cpu_solve(0, A, b, np.zeros(A.n), L, 1e-10, 20000)
    if ref is None:
        pytest.skip("reference CPU solver not built")
    ok, it, res, sec, xr = ref
    assert ok
    assert abs(rep.iters - it) <= L, (rep.iters, it)
    # same solution to the accuracy the tolerance implies
    assert np.linalg.norm(x - xr) / np.linalg.norm(xr) < 1e-6


def test_gmres_f64_matches_reference_cpu(gpu):
    ctx, torch = gpu
    A = problems.poisson3d_aniso(12, eps=(1.0, 1e-2, 1e-4))
    b = problems.rhs_uniform(A.n, 3)
    p = _lib.solver_params("gmres", basis=30, rel_tol=1e-8, max_iters=20000)
    st, rep, x, _ = solve(ctx, torch, "f64", A, b, p)
    assert st == 0 and true_rel(A, b, x) <= 1.05e-8
    ref = oracle.ref_cpu_solve(1, A, b, np.zeros(A.n), 30, 1e-8, 20000)
    if ref is None:
        pytest.skip("reference CPU solver not built")
    ok, it, res, sec, xr = ref
    assert ok and abs(rep.iters - it) <= 30, (rep.iters, it)


def test_bicgstab_and_jacobi(gpu):
    ctx, torch = gpu
    A = problems.diffusion3d_lognormal(14, seed=2, sigma=1.0, corr=3.0)
    b = problems.rhs_uniform(A.n, 5)
    p = _lib.solver_params("bicgstab", rel_tol=1e-9, max_iters=20000)
    st, rep, x, _ = solve(ctx, torch, "f64", A, b, p)
    assert st == 0 and true_rel(A, b, x) <= 2e-9
    pj = _lib.solver_params("bicgstab", rel_tol=1e-9, max_iters=20000, precond="jacobi")
    st2, rep2, x2, _ = solve(ctx, torch, "f64", A, b, pj)
    assert st2 == 0
    # left preconditioning: the monitor tests ||D^-1 r||; check the true residual loosely
    assert true_rel(A, b, x2) <= 1e-6
    assert rep2.iters < rep.iters


def test_host_api_matches_device_api(gpu):
    ctx, torch = gpu
    A = problems.convdiff2d(40)
    b = problems.rhs_uniform(A.n, 9)
    p = _lib.solver_params("bicgstabl", basis=4, rel_tol=1e-10)
    st1, rep1, x1, _ = solve(ctx, torch, "f64", A, b, p)
    st2, rep2, x2, _ = solve(ctx, torch, "f64", A, b, p, host_api=True)
    assert st1 == st2 == 0 and rep1.iters == rep2.iters
    assert np.array_equal(x1, x2)  # deterministic kernels: identical iterates


@pytest.mark.parametrize("t", ["f32", "c64", "c128"])
def test_other_types_converge(gpu, t):
    ctx, torch = gpu
    if t.startswith("c"):
        A = problems.helmholtz2d(40, ppw=10.0)
        b = problems.rhs_uniform(A.n, 4, complex_=True)
        tol = 1e-5 if t == "c64" else 1e-10
    else:
        A = problems.convdiff2d(40)
        b = problems.rhs_uniform(A.n, 4)
        tol = 1e-5
    p = _lib.solver_params("bicgstabl", basis=2, rel_tol=tol, max_iters=50000)
    st, rep, x, _ = solve(ctx, torch, t, A, b, p)
    assert st == 0, (st, rep.iters, rep.resid_norm)
    assert true_rel(A, b, x) <= 20 * tol
    pg = _lib.solver_params("gmres", basis=40, rel_tol=tol, max_iters=50000, early_exit=True)
    st, rep, x, _ = solve(ctx, torch, t, A, b, pg)
    assert st == 0 and true_rel(A, b, x) <= 20 * tol


def test_not_converged_and_bad_args(gpu):
    ctx, torch = gpu
    A = problems.convdiff2d(64)
    b = problems.rhs_uniform(A.n, 1)
    p = _lib.solver_params("bicgstabl", basis=2, rel_tol=1e-14, max_iters=4)
    st, rep, x, _ = solve(ctx, torch, "f64", A, b, p)
    assert st == -7 and rep.converged == 0 and rep.iters == 4
    bad = _lib.solver_params("bicgstabl")
    bad.method = 9
    st, rep, x, _ = solve(ctx, torch, "f64", A, b, bad)
    assert st == -4


def test_nan_rhs_is_reported(gpu):
    """A non-finite input stops the solve at the monitor's finiteness check."""
    ctx, torch = gpu
    A = problems.convdiff2d(16)
    b = problems.rhs_uniform(A.n, 1)
    b[5] = np.nan
    p = _lib.solver_params("bicgstabl", basis=2, rel_tol=1e-10, max_iters=100)
    st, rep, x, _ = solve(ctx, torch, "f64", A, b, p)
    assert st != 0 and rep.converged == 0
