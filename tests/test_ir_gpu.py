"""Mixed-precision iterative refinement (precision form): binary32 inner
solves with Dot2 reductions inside a binary64 refinement loop whose residual
is a compensated row sum.  The bar: the true relative residual, recomputed
here in float64/complex128 by numpy, is <= 1.05 * 1e-10 (a hair above the
library's own compensated test, numpy's product rounds once per term); the
solution agrees with a binary64 solve of the same system to within
cond-scaled rounding (relative difference <= 1e-6 here)."""
import ctypes as C

import numpy as np
import pytest

from gpu_utils import dev, host
from high_precision_blas1_b200 import _lib, problems

pytestmark = pytest.mark.gpu


def ir(torch, A, b, params, complex_=False, M=None, cap=64):
    dt = np.complex128 if complex_ else np.float64
    d = [dev(torch, a) for a in (A.row_ptr, A.col_ind, A.val.astype(dt), b.astype(dt), np.zeros(A.n, dtype=dt))]
    m = [None, None, None, 0]
    if M is not None:
        dm = [dev(torch, a) for a in (M.row_ptr, M.col_ind, M.val.astype(np.complex64 if complex_ else np.float32))]
        m = [dm[0].data_ptr(), dm[1].data_ptr(), dm[2].data_ptr(), M.nnz]
    rep = _lib.hpb_ir_report()
    hist = np.zeros(2 * cap)
    f = _lib.lib.hpb_ir_solve_c128 if complex_ else _lib.lib.hpb_ir_solve_f64
    st = f(C.byref(params), A.n, A.nnz, d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), None, m[0], m[1], m[2],
           m[3], d[3].data_ptr(), d[4].data_ptr(), C.byref(rep), hist.ctypes.data, cap)
    torch.cuda.synchronize()
    return st, rep, host(d[4]), hist[:2 * rep.history_len].reshape(-1, 2)


def rel_res(A, b, x):
    return np.linalg.norm(b - A.matvec(x)) / np.linalg.norm(b)


def test_ir_gmres_f32_inner_reaches_1e10_aniso_poisson(gpu):
    ctx, torch = gpu
    A = problems.poisson3d_aniso(24, eps=(1.0, 1e-2, 1e-4))
    b = problems.rhs_uniform(A.n, 5)
    p = _lib.ir_params("gmres", basis=50, inner_rel_tol=1e-5, rel_tol=1e-10)
    st, rep, x, hist = ir(torch, A, b, p)
    assert st == 0 and rep.converged == 1, (st, rep.refinements, rep.true_resid_norm / rep.rhs_norm)
    assert rel_res(A, b, x) <= 1.05e-10
    assert rep.refinements >= 2  # binary32 alone cannot reach 1e-10
    assert np.all(np.diff(hist[:, 1]) < 0)  # every refinement reduces the residual
    # against a binary64 fused GMRES solve of the same system
    p64 = _lib.solver_params("gmres", basis=50, rel_tol=1e-12, max_iters=100000, fused=True)
    rep64 = _lib.hpb_solver_report()
    d = [dev(torch, a) for a in (A.row_ptr, A.col_ind, A.val, b, np.zeros(A.n))]
    assert _lib.lib.hpb_csr_solve_f64(C.byref(p64), A.n, A.nnz, *[a.data_ptr() for a in d], C.byref(rep64), None, 0) == 0
    torch.cuda.synchronize()
    x64 = host(d[4])
    assert np.linalg.norm(x - x64) / np.linalg.norm(x64) < 1e-6


def test_ir_one_cycle_refinement_keeps_gmres_iteration_count(gpu):
    """inner_max_iters = 0: each refinement is one binary32 GMRES(m) cycle with
    binary64 restart residual and solution -- restarted GMRES(m) at binary32
    cost; its iteration count stays within two cycles of binary64 GMRES(m)."""
    ctx, torch = gpu
    A = problems.poisson3d_aniso(24, eps=(1.0, 1e-2, 1e-4))
    b = problems.rhs_uniform(A.n, 9)
    p = _lib.ir_params("gmres", basis=30, inner_rel_tol=0.0, inner_max_iters=0, rel_tol=1e-10, max_refinements=500)
    st, rep, x, hist = ir(torch, A, b, p, cap=600)
    assert st == 0 and rel_res(A, b, x) <= 1.05e-10
    assert rep.inner_iters == 30 * rep.refinements
    p64 = _lib.solver_params("gmres", basis=30, rel_tol=1e-10, max_iters=100000, fused=True)
    rep64 = _lib.hpb_solver_report()
    d = [dev(torch, a) for a in (A.row_ptr, A.col_ind, A.val, b, np.zeros(A.n))]
    assert _lib.lib.hpb_csr_solve_f64(C.byref(p64), A.n, A.nnz, *[a.data_ptr() for a in d], C.byref(rep64), None, 0) == 0
    assert rep.inner_iters <= rep64.iters + 60, (rep.inner_iters, rep64.iters)


def test_ir_jacobi_and_matrix_preconditioner_agree(gpu):
    ctx, torch = gpu
    A = problems.diffusion3d_lognormal(16, seed=7, sigma=2.3, corr=4.0)
    b = problems.rhs_uniform(A.n, 2)
    pj = _lib.ir_params("gmres", basis=30, inner_rel_tol=1e-5, precond="jacobi")
    st1, r1, x1, _ = ir(torch, A, b, pj)
    # M = D^{-1} given as an explicit CSR matrix
    diag = np.array([A.val[A.row_ptr[i]:A.row_ptr[i + 1]][A.col_ind[A.row_ptr[i]:A.row_ptr[i + 1]] == i][0]
                     for i in range(A.n)])
    M = problems.CSR(A.n, np.arange(A.n + 1, dtype=np.int32), np.arange(A.n, dtype=np.int32), 1.0 / diag)
    pm = _lib.ir_params("gmres", basis=30, inner_rel_tol=1e-5, precond="matrix")
    st2, r2, x2, _ = ir(torch, A, b, pm, M=M)
    assert st1 == 0 and st2 == 0
    assert rel_res(A, b, x1) <= 1.05e-10 and rel_res(A, b, x2) <= 1.05e-10
    assert abs(r1.inner_iters - r2.inner_iters) <= 30


def test_ir_complex_bicgstab2_c64_inner_helmholtz(gpu):
    ctx, torch = gpu
    A = problems.helmholtz2d(64, ppw=10.0)
    b = problems.rhs_uniform(A.n, 3, complex_=True)
    p = _lib.ir_params("bicgstabl", basis=2, inner_rel_tol=1e-4, rel_tol=1e-10)
    st, rep, x, _ = ir(torch, A, b, p, complex_=True)
    assert st == 0, (st, rep.refinements, rep.true_resid_norm / rep.rhs_norm)
    assert rel_res(A, b, x) <= 1.05e-10


def test_ir_rejects_matrix_preconditioner_without_matrix(gpu):
    ctx, torch = gpu
    A = problems.convdiff2d(8)
    b = problems.rhs_uniform(A.n, 1)
    p = _lib.ir_params("gmres", precond="matrix")
    st, rep, x, _ = ir(torch, A, b, p)
    assert st == -1


@pytest.mark.parametrize("sweeps", [0, 2])
def test_ir_ilu0_preconditioner(gpu, sweeps):
    """ILU(0) of the binary32 matrix as the right preconditioner of the
    binary32 GMRES(30) inner cycles (exact triangular solves, or 2 Jacobi
    sweeps per factor): the binary64 refinement still reaches a 1e-10 true
    residual, with fewer inner iterations than Jacobi; a BiCGStab(l) inner
    solver refuses it."""
    ctx, torch = gpu
    A = problems.diffusion3d_lognormal(24, seed=7, sigma=1.5, corr=4.0)
    b = problems.rhs_uniform(A.n, 3)
    pj = _lib.ir_params("gmres", basis=30, inner_rel_tol=0.0, inner_max_iters=0, precond="jacobi",
                        max_refinements=2000)
    st, rj, _, _ = ir(torch, A, b, pj)
    assert st == 0
    pi = _lib.ir_params("gmres", basis=30, inner_rel_tol=0.0, inner_max_iters=0, precond="ilu0",
                        max_refinements=2000, ilu_sweeps=sweeps)
    st, ri, x, _ = ir(torch, A, b, pi)
    assert st == 0 and ri.converged == 1
    assert rel_res(A, b, x) <= 1.05e-10
    assert ri.inner_iters < rj.inner_iters, (ri.inner_iters, rj.inner_iters)
    pb = _lib.ir_params("bicgstabl", basis=2, precond="ilu0")
    st, _, _, _ = ir(torch, A, b, pb)
    assert st == -4
