"""The delayed re-orthogonalisation (DCGS2) of the fused GMRES, restated in
numpy with the kernels' formulas (csrc/hpb_fused_gmres.cu: one reduction
a = Q^H u, b = Q^H w, <u,u>, <u,w>, <w,w> per step; nu = sqrt(<u,u> - |a|^2);
column i-1 completed by + alpha a and alpha nu; column i = (t - H a) / nu
with t = (b, (<u,w> - a^H b) / nu); the next vector (w - Q t) / (nu alpha')
with a Pythagorean alpha'; a closing reduction for column m-1), checked
against classical Gram-Schmidt with two full passes (CGS2) in binary64:
same Hessenberg matrix and residual estimate to rounding, an orthonormal
basis, and the same restarted-GMRES iteration count."""
import numpy as np
import pytest

from high_precision_blas1_b200 import problems


def arnoldi_cgs2(A, r, m):
    n = r.shape[0]
    beta = np.linalg.norm(r)
    Q = np.zeros((m + 1, n), dtype=r.dtype)
    H = np.zeros((m + 1, m), dtype=r.dtype)
    Q[0] = r / beta
    for i in range(m):
        w = A @ Q[i]
        h1 = Q[: i + 1].conj() @ w
        w = w - Q[: i + 1].T @ h1
        h2 = Q[: i + 1].conj() @ w
        w = w - Q[: i + 1].T @ h2
        H[: i + 1, i] = h1 + h2
        H[i + 1, i] = np.linalg.norm(w)
        Q[i + 1] = w / H[i + 1, i]
    return Q[:m], H, beta


def arnoldi_dcgs2(A, r, m):
    n = r.shape[0]
    beta = np.linalg.norm(r)
    V = np.zeros((m + 1, n), dtype=r.dtype)
    H = np.zeros((m + 1, m), dtype=r.dtype)
    V[0] = r / beta
    alpha = 1.0
    for i in range(m + 1):
        u = V[i].copy()
        Q = V[:i]
        last = i == m
        a = Q.conj() @ u
        uu = np.vdot(u, u).real
        if not last:
            w = A @ u
            b = Q.conj() @ w
            uw = np.vdot(u, w)
            ww = np.vdot(w, w).real
        nu = 1.0 if i == 0 else np.sqrt(uu - np.sum(np.abs(a) ** 2))
        if i > 0:  # complete column i-1
            H[:i, i - 1] += alpha * a
            H[i, i - 1] = alpha * nu
        if last:
            break
        t = np.append(b, (uw - np.vdot(a, b)) / nu)
        Ha = H[: i + 1, :i] @ a if i > 0 else np.zeros(1, dtype=r.dtype)
        H[: i + 1, i] = (t - Ha) / nu
        a2 = (ww - np.sum(np.abs(t) ** 2)) / nu ** 2
        alpha_next = np.sqrt(a2) if a2 > 0 else np.sqrt(ww) / nu * 1e-8
        q = (u - Q.T @ a) / nu if i > 0 else u
        V[i] = q
        V[i + 1] = (w - Q.T @ b - t[i] * q) / (nu * alpha_next)
        alpha = alpha_next
    return V[:m], H, beta


def lsq_residual(H, beta):
    e1 = np.zeros(H.shape[0], dtype=H.dtype)
    e1[0] = beta
    y, *_ = np.linalg.lstsq(H, e1, rcond=None)
    return np.linalg.norm(e1 - H @ y), y


@pytest.mark.parametrize("kind", ["convdiff", "helmholtz"])
def test_dcgs2_matches_cgs2_one_cycle(kind):
    if kind == "convdiff":
        A = problems.convdiff2d(24)
        b = problems.rhs_uniform(A.n, 7)
    else:
        A = problems.helmholtz2d(20)
        b = problems.rhs_uniform(A.n, 7, complex_=True)
    import scipy.sparse as sp
    As = sp.csr_matrix((A.val, A.col_ind, A.row_ptr), shape=(A.n, A.n))
    m = 30
    Q1, H1, beta = arnoldi_cgs2(As, b, m)
    Q2, H2, _ = arnoldi_dcgs2(As, b, m)
    scale = np.abs(H1).max()
    assert np.abs(H1 - H2).max() <= 1e-10 * scale
    I = np.eye(m)
    assert np.abs(Q2.conj() @ Q2.T - I).max() <= 1e-12
    assert np.abs(Q1 - Q2).max() <= 1e-10
    r1, _ = lsq_residual(H1, beta)
    r2, _ = lsq_residual(H2, beta)
    assert abs(r1 - r2) <= 1e-10 * beta


def restarted(As, b, m, tol, arnoldi, max_cycles=200):
    x = np.zeros_like(b)
    nb = np.linalg.norm(b)
    for c in range(max_cycles):
        r = b - As @ x
        if np.linalg.norm(r) <= tol * nb:
            return c * m
        Q, H, beta = arnoldi(As, r, m)
        _, y = lsq_residual(H, beta)
        x = x + Q.T @ y
    return max_cycles * m


def test_dcgs2_restarted_iterations_match_cgs2():
    import scipy.sparse as sp
    A = problems.convdiff2d(32)
    b = problems.rhs_uniform(A.n, 3)
    As = sp.csr_matrix((A.val, A.col_ind, A.row_ptr), shape=(A.n, A.n))
    i1 = restarted(As, b, 20, 1e-10, arnoldi_cgs2)
    i2 = restarted(As, b, 20, 1e-10, arnoldi_dcgs2)
    assert i1 == i2 and i1 < 200 * 20
