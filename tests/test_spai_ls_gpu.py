"""The least-squares SPAI builder (hpb_spai_ls_*, through the C ABI) against
a numpy restatement: for every column j, the least-squares solution of
min ||A(:, J_j) m - e_j|| over the rows A's columns J_j reach (J_j = the
rows of A's column j), by numpy.linalg.lstsq in binary64.  Tolerance: the
builder solves the normal equations by Cholesky in binary64 (condition
number squared), so its columns agree to about sqrt(eps) times the
columns' condition -- 1e-8 relative to the largest entry here -- and the
binary32 build to binary32 rounding.  Also: the Frobenius norm of A M - I is
below Jacobi's, and GMRES(30) with it as a right preconditioner needs fewer
iterations than with Jacobi."""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

from gpu_utils import dev, host
from high_precision_blas1_b200 import _lib, problems, spai

pytestmark = pytest.mark.gpu


def ls_columns(A):
    As = sp.csr_matrix((A.val, A.col_ind, A.row_ptr), shape=(A.n, A.n)).tocsc()
    M = np.zeros(A.nnz)
    Ar = sp.csr_matrix((np.arange(A.nnz, dtype=np.float64) + 1, A.col_ind, A.row_ptr), shape=(A.n, A.n))
    pos = Ar.tocsc()  # CSR position + 1 of every entry, by column
    for j in range(A.n):
        J = As.indices[As.indptr[j]:As.indptr[j + 1]]
        B = As[:, J].toarray()
        rows = np.nonzero(np.abs(B).sum(1))[0]
        e = (rows == j).astype(float)
        m = np.linalg.lstsq(B[rows], e, rcond=None)[0]
        k = pos[:, j].toarray().ravel()[J].astype(np.int64) - 1
        M[k] = m
    return M


@pytest.mark.parametrize("case", ["lognormal8", "convdiff16"])
@pytest.mark.parametrize("t", ["f64", "f32"])
def test_spai_ls_matches_numpy(gpu, case, t):
    ctx, torch = gpu
    A = spai.family(8, seed=11) if case == "lognormal8" else problems.convdiff2d(16, peclet=50.0)
    dt = np.float64 if t == "f64" else np.float32
    want = ls_columns(problems.CSR(A.n, A.row_ptr, A.col_ind, A.val.astype(dt).astype(np.float64)))
    rp, ci, va = dev(torch, A.row_ptr), dev(torch, A.col_ind), dev(torch, A.val.astype(dt))
    m = torch.zeros(A.nnz, dtype=torch.float64 if t == "f64" else torch.float32, device="cuda")
    f = getattr(_lib.lib, f"hpb_spai_ls_{t}")
    ctx.check(f(ctx.h, A.n, A.nnz, rp.data_ptr(), ci.data_ptr(), va.data_ptr(), m.data_ptr()), "spai_ls")
    got = host(m).astype(np.float64)
    tol = 1e-8 if t == "f64" else 2e-6
    assert np.max(np.abs(got - want)) <= tol * np.max(np.abs(want)), np.max(np.abs(got - want)) / np.max(np.abs(want))
    As = sp.csr_matrix((A.val, A.col_ind, A.row_ptr), shape=(A.n, A.n))
    Ms = sp.csr_matrix((got, A.col_ind, A.row_ptr), shape=(A.n, A.n))
    I = sp.identity(A.n)
    assert sp.linalg.norm(As @ Ms - I) < sp.linalg.norm(As @ sp.diags(1.0 / As.diagonal()) - I)


def test_spai_ls_preconditions_gmres(gpu):
    """binary32 GMRES(30) + Dot2 in binary64 refinement on a 24^3 lognormal
    system: the least-squares SPAI reaches 1e-10 in fewer inner iterations
    than Jacobi."""
    ctx, torch = gpu
    A = spai.family(24, seed=77)
    b = problems.rhs_uniform(A.n, 3)
    d = [dev(torch, a) for a in (A.row_ptr, A.col_ind, A.val, b, np.zeros(A.n))]
    va32 = dev(torch, A.val.astype(np.float32))
    M = torch.zeros(A.nnz, dtype=torch.float32, device="cuda")
    ctx.check(_lib.lib.hpb_spai_ls_f32(ctx.h, A.n, A.nnz, d[0].data_ptr(), d[1].data_ptr(), va32.data_ptr(),
                                       M.data_ptr()), "spai_ls")
    its = {}
    for pc in ("jacobi", "matrix"):
        d[4].zero_()
        p = _lib.ir_params("gmres", basis=30, inner_rel_tol=0.0, inner_max_iters=0, precond=pc, rel_tol=1e-10,
                           max_refinements=1000)
        rep = _lib.hpb_ir_report()
        mp = [None, None, None, 0] if pc == "jacobi" else [d[0].data_ptr(), d[1].data_ptr(), M.data_ptr(), A.nnz]
        st = _lib.lib.hpb_ir_solve_f64(C.byref(p), A.n, A.nnz, d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(),
                                       None, mp[0], mp[1], mp[2], mp[3], d[3].data_ptr(), d[4].data_ptr(),
                                       C.byref(rep), None, 0)
        torch.cuda.synchronize()
        assert st == 0
        x = host(d[4])
        assert np.linalg.norm(b - A.matvec(x)) <= 1.05e-10 * np.linalg.norm(b)
        its[pc] = rep.inner_iters
    assert its["matrix"] < its["jacobi"], its
