"""The device-resident (fused) BiCGStab(l) against the drop-in path and the
reference's CPU solver.  Same recurrences and stopping test, different
reduction trees: iteration counts agree to within one cycle (l iterations),
and every converged solve meets the tolerance on the true residual
(||b - A x|| / ||b|| <= 1.05 tol, or 20 tol for binary32 storage whose
rounding floor sits near 1e-7)."""
import ctypes as C

import numpy as np
import pytest

import oracle
from gpu_utils import dev, host
from high_precision_blas1_b200 import _lib, problems

pytestmark = pytest.mark.gpu

DT = {"f32": np.float32, "f64": np.float64, "c64": np.complex64, "c128": np.complex128}


def solve(torch, t, A, b, params, hist_cap=0):
    rep = _lib.hpb_solver_report()
    hist = np.zeros(2 * max(hist_cap, 1))
    d = [dev(torch, a) for a in (A.row_ptr, A.col_ind, A.val.astype(DT[t]), b.astype(DT[t]),
                                 np.zeros(A.n, dtype=DT[t]))]
    st = getattr(_lib.lib, f"hpb_csr_solve_{t}")(C.byref(params), A.n, A.nnz, *[a.data_ptr() for a in d],
                                                 C.byref(rep), hist.ctypes.data, hist_cap)
    torch.cuda.synchronize()
    return st, rep, host(d[4]), hist[:2 * rep.history_len].reshape(-1, 2)


def true_rel(A, b, x):
    w = np.complex128 if np.iscomplexobj(x) else np.float64
    r = b.astype(w) - A.matvec(x.astype(w))
    return np.linalg.norm(r) / np.linalg.norm(b)


@pytest.mark.parametrize("N,L", [(64, 4), (48, 2), (40, 1), (40, 8)])
def test_fused_matches_dropin_f64(gpu, N, L):
    ctx, torch = gpu
    A = problems.convdiff2d(N)
    b = problems.rhs_uniform(A.n, 13)
    pf = _lib.solver_params("bicgstabl", basis=L, rel_tol=1e-10, max_iters=50000, fused=True)
    pp = _lib.solver_params("bicgstabl", basis=L, rel_tol=1e-10, max_iters=50000)
    st1, r1, x1, h1 = solve(torch, "f64", A, b, pf, hist_cap=10000)
    st2, r2, x2, h2 = solve(torch, "f64", A, b, pp, hist_cap=10000)
    assert st1 == 0 and st2 == 0
    assert abs(r1.iters - r2.iters) <= L, (r1.iters, r2.iters)
    assert true_rel(A, b, x1) <= 1.05e-10
    assert r1.true_resid_norm / r1.true_rhs_norm <= 1.05e-10
    assert h1.shape[0] == r1.iters // L + 1 and h1[0, 0] == 0
    # the residual histories agree while far from the rounding floor
    k = min(h1.shape[0], h2.shape[0], 5)
    assert np.allclose(h1[:k, 1], h2[:k, 1], rtol=1e-6)
    ref = oracle.ref_cpu_solve(0, A, b, np.zeros(A.n), L, 1e-10, 50000)
    if ref is not None:
        assert abs(r1.iters - ref[1]) <= L


def test_fused_config2_shape_small(gpu):
    """Config-2 operator at reduced size, reference iteration count."""
    ctx, torch = gpu
    A = problems.convdiff2d(128, peclet=50.0)
    b = problems.rhs_uniform(A.n, 2024)
    p = _lib.solver_params("bicgstabl", basis=4, rel_tol=1e-10, max_iters=50000, fused=True)
    st, rep, x, _ = solve(torch, "f64", A, b, p)
    assert st == 0 and true_rel(A, b, x) <= 1.05e-10
    ref = oracle.ref_cpu_solve(0, A, b, np.zeros(A.n), 4, 1e-10, 50000)
    if ref is not None:
        assert abs(rep.iters - ref[1]) <= 4, (rep.iters, ref[1])


def test_fused_jacobi(gpu):
    ctx, torch = gpu
    A = problems.diffusion3d_lognormal(16, seed=4, sigma=1.5, corr=3.0)
    b = problems.rhs_uniform(A.n, 6)
    pf = _lib.solver_params("bicgstabl", basis=2, rel_tol=1e-9, max_iters=50000, precond="jacobi", fused=True)
    pp = _lib.solver_params("bicgstabl", basis=2, rel_tol=1e-9, max_iters=50000, precond="jacobi")
    st1, r1, x1, _ = solve(torch, "f64", A, b, pf)
    st2, r2, x2, _ = solve(torch, "f64", A, b, pp)
    assert st1 == 0 and st2 == 0 and abs(r1.iters - r2.iters) <= 2
    assert r1.rhs_norm == pytest.approx(r2.rhs_norm, rel=1e-13)  # ||D^-1 b||
    assert np.linalg.norm(x1 - x2) / np.linalg.norm(x2) < 1e-6


@pytest.mark.parametrize("t", ["f32", "c64", "c128"])
def test_fused_other_types(gpu, t):
    ctx, torch = gpu
    if t.startswith("c"):
        A = problems.helmholtz2d(48)
        b = problems.rhs_uniform(A.n, 8, complex_=True)
    else:
        A = problems.convdiff2d(48)
        b = problems.rhs_uniform(A.n, 8)
    tol = 1e-10 if t == "c128" else 1e-6
    p = _lib.solver_params("bicgstabl", basis=2, rel_tol=tol, max_iters=50000, fused=True)
    st, rep, x, _ = solve(torch, t, A, b, p)
    assert st == 0, (st, rep.iters, rep.resid_norm)
    assert true_rel(A, b, x) <= (1.05 if t == "c128" else 20) * tol


@pytest.mark.parametrize("t,L,precond", [("c128", 1, "none"), ("c128", 3, "jacobi"), ("f32", 1, "jacobi"),
                                          ("c64", 5, "none"), ("f64", 3, "jacobi"), ("f64", 7, "none")])
def test_fused_deferred_updates_match_dropin(gpu, t, L, precond):
    """The cycle's deferred r updates (each BiCG step's r_j applied by the
    next step's kernel, the last step's by the second MR sweep or, for
    l = 1, by the closing update) and the first MR sweep's sums formed in
    the last step's kernel, across element types, basis sizes and the
    Jacobi scaling: the fused solve against the drop-in path.  The
    residual histories agree while far from the rounding floor; the
    iteration counts within two cycles or 3 % (with l = 1 the indefinite
    complex Helmholtz operator, and binary32 storage near its rounding
    floor, drift by two iterations between reduction orders)."""
    ctx, torch = gpu
    if t.startswith("c"):
        A = problems.helmholtz2d(40)
        b = problems.rhs_uniform(A.n, 21, complex_=True)
    else:
        A = problems.convdiff2d(40)
        b = problems.rhs_uniform(A.n, 21)
    tol = 1e-6 if t in ("f32", "c64") else 1e-10
    pf = _lib.solver_params("bicgstabl", basis=L, rel_tol=tol, max_iters=50000, precond=precond, fused=True)
    pp = _lib.solver_params("bicgstabl", basis=L, rel_tol=tol, max_iters=50000, precond=precond)
    st1, r1, x1, h1 = solve(torch, t, A, b, pf, hist_cap=10000)
    st2, r2, x2, h2 = solve(torch, t, A, b, pp, hist_cap=10000)
    assert st1 == 0 and st2 == 0, (st1, st2, r1.iters, r2.iters)
    k = min(h1.shape[0], h2.shape[0], 4)
    assert np.allclose(h1[:k, 1], h2[:k, 1], rtol=1e-3 if t in ("f32", "c64") else 1e-6), (h1[:k], h2[:k])
    assert abs(r1.iters - r2.iters) <= max(2 * L, 0.03 * r2.iters), (r1.iters, r2.iters)
    # binary64: the tolerance on the true residual; binary32 storage: no
    # further from it than the drop-in solve (whose recursive residual drifts
    # from the true one the same way at large l)
    if t in ("f32", "c64"):
        assert true_rel(A, b, x1) <= max(20 * tol, 2 * true_rel(A, b, x2))
    else:
        assert true_rel(A, b, x1) <= 1.05 * tol


def test_fused_not_converged_and_unsupported(gpu):
    ctx, torch = gpu
    A = problems.convdiff2d(32)
    b = problems.rhs_uniform(A.n, 1)
    p = _lib.solver_params("bicgstabl", basis=4, rel_tol=1e-14, max_iters=8, fused=True)
    st, rep, x, _ = solve(torch, "f64", A, b, p)
    assert st == -7 and rep.iters == 8 and rep.converged == 0
    bad = _lib.solver_params("bicgstab", fused=True)
    st, rep, x, _ = solve(torch, "f64", A, b, bad)
    assert st == -4
    bad = _lib.solver_params("bicgstabl", basis=9, fused=True)
    st, rep, x, _ = solve(torch, "f64", A, b, bad)
    assert st == -4


def test_fused_nonfinite_rhs_stops(gpu):
    ctx, torch = gpu
    A = problems.convdiff2d(16)
    b = problems.rhs_uniform(A.n, 1)
    b[3] = np.inf
    p = _lib.solver_params("bicgstabl", basis=2, rel_tol=1e-10, max_iters=100, fused=True)
    st, rep, x, _ = solve(torch, "f64", A, b, p)
    assert st != 0 and rep.converged == 0


def test_fused_gmres_f64_matches_dropin(gpu):
    """Fused GMRES(m) (CGS2, binary64 Hessenberg on the GPU) vs the drop-in
    GMRES (MGS, host Hessenberg): same restart length, both test the true
    residual once per cycle, so the cycle counts agree within one cycle."""
    ctx, torch = gpu
    A = problems.poisson3d_aniso(14, eps=(1.0, 1e-2, 1e-4))
    b = problems.rhs_uniform(A.n, 3)
    m = 30
    pf = _lib.solver_params("gmres", basis=m, rel_tol=1e-10, max_iters=100000, fused=True)
    pp = _lib.solver_params("gmres", basis=m, rel_tol=1e-10, max_iters=100000)
    st1, r1, x1, h1 = solve(torch, "f64", A, b, pf, hist_cap=1000)
    st2, r2, x2, _ = solve(torch, "f64", A, b, pp)
    assert st1 == 0 and st2 == 0
    assert abs(r1.iters - r2.iters) <= m, (r1.iters, r2.iters)
    assert true_rel(A, b, x1) <= 1.05e-10
    assert h1.shape[0] == r1.iters // m + 1


@pytest.mark.parametrize("t,precond", [("f32", "none"), ("f64", "jacobi"), ("c128", "none"), ("c64", "jacobi")])
def test_fused_gmres_types_and_jacobi(gpu, t, precond):
    ctx, torch = gpu
    if t.startswith("c"):
        A = problems.helmholtz2d(32)
        b = problems.rhs_uniform(A.n, 2, complex_=True)
    else:
        A = problems.diffusion3d_lognormal(12, seed=1, sigma=1.0, corr=3.0)
        b = problems.rhs_uniform(A.n, 2)
    tol = 1e-10 if t in ("f64", "c128") else 1e-6
    p = _lib.solver_params("gmres", basis=40, rel_tol=tol, max_iters=100000, precond=precond, fused=True)
    st, rep, x, _ = solve(torch, t, A, b, p)
    assert st == 0, (st, rep.iters, rep.resid_norm / rep.rhs_norm)
    assert true_rel(A, b, x) <= (1.05 if tol == 1e-10 else 20) * tol


@pytest.mark.parametrize("t", ["f64", "f32", "c128", "c64"])
def test_fused_gmres_ilu0(gpu, t):
    """Fused GMRES(30) with ILU(0) as right preconditioner (two sparse
    triangular solves inside the captured cycle): converges to the tolerance
    on the true residual in fewer iterations than with Jacobi, and leaves
    the caller's matrix values untouched (the factors are a copy)."""
    ctx, torch = gpu
    if t.startswith("c"):
        A = problems.helmholtz2d(48)
        b = problems.rhs_uniform(A.n, 3, complex_=True)
    else:
        A = problems.convdiff2d(96)
        b = problems.rhs_uniform(A.n, 3)
    tol = 1e-10 if t in ("f64", "c128") else 1e-6
    its = {}
    for precond in ("jacobi", "ilu0"):
        p = _lib.solver_params("gmres", basis=30, rel_tol=tol, max_iters=100000, precond=precond, fused=True)
        st, rep, x, _ = solve(torch, t, A, b, p)
        assert st == 0, (precond, st, rep.iters)
        assert true_rel(A, b, x) <= (1.05 if tol == 1e-10 else 20) * tol
        its[precond] = rep.iters
    assert its["ilu0"] < its["jacobi"], its


@pytest.mark.parametrize("t", ["f64", "f32"])
def test_fused_gmres_ilu0_sweeps(gpu, t):
    """ILU(0) factors applied by Jacobi sweeps (ilu_sweeps = 2) inside the
    fused GMRES: converges on the true residual, with fewer iterations than
    Jacobi; the drop-in path refuses the option (it applies factors exactly)."""
    ctx, torch = gpu
    A = problems.convdiff2d(96)
    b = problems.rhs_uniform(A.n, 8)
    tol = 1e-10 if t == "f64" else 1e-6
    pj = _lib.solver_params("gmres", basis=30, rel_tol=tol, max_iters=100000, precond="jacobi", fused=True)
    st, rj, x, _ = solve(torch, t, A, b, pj)
    assert st == 0
    ps = _lib.solver_params("gmres", basis=30, rel_tol=tol, max_iters=100000, precond="ilu0", fused=True,
                            ilu_sweeps=2)
    st, rs, x, _ = solve(torch, t, A, b, ps)
    assert st == 0 and rs.iters < rj.iters, (rs.iters, rj.iters)
    assert true_rel(A, b, x) <= (1.05 if tol == 1e-10 else 20) * tol
    pd = _lib.solver_params("gmres", basis=30, rel_tol=tol, max_iters=100, precond="ilu0", ilu_sweeps=2)
    st, _, _, _ = solve(torch, t, A, b, pd)
    assert st == -4


def _diag(values):
    n = len(values)
    return problems.CSR(n, np.arange(n + 1, dtype=np.int32), np.arange(n, dtype=np.int32), np.asarray(values))


@pytest.mark.parametrize("t", ["f64", "c128", "f32"])
def test_fused_gmres_invariant_krylov_space(gpu, t):
    """Krylov spaces that stop growing: A = 2 I (dimension 1) and a diagonal
    A with three distinct values (dimension 3).  Past that dimension the
    delayed re-orthogonalisation meets vectors of rounding size (nu near
    zero, the Pythagorean scale at its fallback, or an exact breakdown that
    zeroes the remaining slots); the first restart cycle must still return
    a finite solution that meets the tolerance."""
    ctx, torch = gpu
    n = 4000
    cplx = t.startswith("c")
    b = problems.rhs_uniform(n, 11, complex_=cplx)
    tol = 1e-10 if t in ("f64", "c128") else 1e-6
    for vals in (np.full(n, 2.0), np.array([1.0, 3.0, 7.0] * (n // 3) + [1.0] * (n % 3))):
        A = _diag(vals.astype(np.complex128) if cplx else vals)
        p = _lib.solver_params("gmres", basis=30, rel_tol=tol, max_iters=3000, fused=True)
        st, rep, x, _ = solve(torch, t, A, b, p)
        assert st == 0, (st, rep.iters)
        assert np.isfinite(x).all()
        assert true_rel(A, b, x) <= (1.05 if tol == 1e-10 else 20) * tol
        assert rep.iters <= 30, rep.iters


@pytest.mark.parametrize("t", ["f32", "f64", "c64", "c128"])
def test_fused_gmres_odd_sizes(gpu, t):
    """Vector lengths that are not a multiple of the 16-byte pack (1089 =
    33^2 rows, odd) take the element-wise forms of the DCGS2 reduction and
    update; the solve converges on the true residual as the packed forms
    do, for every storage type."""
    ctx, torch = gpu
    if t.startswith("c"):
        A = problems.helmholtz2d(33)
        b = problems.rhs_uniform(A.n, 5, complex_=True)
    else:
        A = problems.convdiff2d(33)
        b = problems.rhs_uniform(A.n, 5)
    assert A.n % 4 == 1
    tol = 1e-10 if t in ("f64", "c128") else 1e-6
    for precond in ("none", "jacobi"):
        p = _lib.solver_params("gmres", basis=20, rel_tol=tol, max_iters=100000, precond=precond, fused=True)
        st, rep, x, _ = solve(torch, t, A, b, p)
        assert st == 0, (precond, st, rep.iters)
        assert true_rel(A, b, x) <= (1.05 if tol == 1e-10 else 20) * tol


@pytest.mark.parametrize("t,m", [("f64", 64), ("f32", 64), ("c128", 64), ("f64", 1), ("f64", 2)])
def test_fused_gmres_basis_extremes(gpu, t, m):
    """The largest basis the fused GMRES takes (m = 64: 131 inner products
    per step, the whole Hessenberg band in shared memory) and the smallest
    ones (m = 1, 2: the closing reduction right after the first steps)."""
    ctx, torch = gpu
    if t.startswith("c"):
        A = problems.helmholtz2d(40)
        b = problems.rhs_uniform(A.n, 9, complex_=True)
    else:
        A = problems.convdiff2d(40)
        b = problems.rhs_uniform(A.n, 9)
    tol = 1e-10 if t in ("f64", "c128") else 1e-6
    p = _lib.solver_params("gmres", basis=m, rel_tol=tol, max_iters=200000, precond="jacobi", fused=True)
    st, rep, x, _ = solve(torch, t, A, b, p)
    assert st == 0, (st, rep.iters)
    assert true_rel(A, b, x) <= (1.05 if tol == 1e-10 else 20) * tol
