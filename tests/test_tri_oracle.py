"""CPU checks of the triangular-solve and ILU(0) restatement (oracle/tri.c)
before it is used to check the GPU kernels: the solves agree with scipy's
sparse triangular solver, and the ILU(0) factors satisfy the defining
property (L U)_ij = A_ij on A's pattern (and are the exact LU when the
pattern admits no fill)."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as sla

import oracle
from high_precision_blas1_b200 import problems

TOL = {np.float32: 2e-5, np.float64: 1e-13, np.complex64: 2e-5, np.complex128: 1e-13}


def random_dominant(n, density, dtype, seed):
    rng = np.random.default_rng(seed)
    M = sp.random(n, n, density=density, random_state=seed, format="csr")
    if np.issubdtype(dtype, np.complexfloating):
        M = M + 1j * sp.random(n, n, density=density, random_state=seed + 1, format="csr")
    M = (M + sp.eye(n) * (4.0 + rng.random())).astype(dtype).tocsr()
    M.sort_indices()
    return M


@pytest.mark.parametrize("dtype", [np.float64, np.float32, np.complex128, np.complex64])
def test_trsv_matches_scipy(dtype):
    n = 200
    M = random_dominant(n, 0.05, dtype, 1)
    rng = np.random.default_rng(2)
    b = rng.standard_normal(n).astype(dtype)
    wide = np.complex128 if np.issubdtype(dtype, np.complexfloating) else np.float64
    for upper in (False, True):
        for unit in (False, True):
            x = oracle.csr_trsv(M.indptr, M.indices, M.data, b, upper, unit, alpha=1.5)
            T = sp.triu(M, 1) if upper else sp.tril(M, -1)
            D = sp.eye(n) if unit else sp.diags(M.diagonal())
            want = sla.spsolve_triangular((T + D).tocsr().astype(wide), 1.5 * b.astype(wide), lower=not upper)
            assert np.abs(x - want).max() <= TOL[dtype] * np.abs(want).max()


@pytest.mark.parametrize("dtype", [np.float64, np.float32, np.complex128, np.complex64])
def test_ilu0_reproduces_a_on_its_pattern(dtype):
    n = 300
    M = random_dominant(n, 0.03, dtype, 3)
    lu, zero_row = oracle.csr_ilu0(M.indptr, M.indices, M.data)
    assert zero_row == -1 and lu.dtype == M.data.dtype
    F = sp.csr_matrix((lu, M.indices, M.indptr), shape=M.shape)
    L = sp.tril(F, -1) + sp.eye(n)
    U = sp.triu(F)
    P = (L @ U).toarray()
    A = M.toarray()
    mask = A != 0
    assert np.abs(P[mask] - A[mask]).max() <= 20 * TOL[dtype] * np.abs(A).max()


def test_ilu0_exact_without_fill():
    """A 5-point matrix on a 1-wide strip is tridiagonal: no fill, ILU(0) = LU."""
    A = problems.convdiff2d(8)
    M = sp.csr_matrix((A.val, A.col_ind, A.row_ptr))
    band = sp.diags([M.diagonal(-1), M.diagonal(), M.diagonal(1)], [-1, 0, 1]).tocsr()
    band.sort_indices()
    lu, _ = oracle.csr_ilu0(band.indptr, band.indices, band.data)
    x = np.random.default_rng(0).standard_normal(band.shape[0])
    b = band @ x
    y = oracle.csr_trsv(band.indptr, band.indices, lu, b, upper=False, unit=True)
    z = oracle.csr_trsv(band.indptr, band.indices, lu, y, upper=True, unit=False)
    assert np.abs(z - x).max() < 1e-12


def test_zero_pivot_and_missing_diagonal():
    rp = np.array([0, 2, 4], np.int32)
    ci = np.array([0, 1, 0, 1], np.int32)
    _, zero_row = oracle.csr_ilu0(rp, ci, np.ones(4))
    assert zero_row == 1
    with pytest.raises(ValueError):
        oracle.csr_ilu0(np.array([0, 1, 2], np.int32), np.array([0, 0], np.int32), np.ones(2))
    with pytest.raises(ValueError):
        oracle.csr_trsv(np.array([0, 1, 2], np.int32), np.array([0, 0], np.int32), np.ones(2), np.ones(2),
                        upper=False, unit=False)
