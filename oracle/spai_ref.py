"""TEST INFRASTRUCTURE ONLY: float64 CPU restatement of the learned SPAI's
features, MLP forward pass, SPAI assembly, loss and parameter gradient
(the kernels in high_precision_blas1_b200/csrc/hpb_spai.cu), used to check
the GPU forward/backward kernels.  The reference has no learned component;
this oracle restates this repository's own definition:

  scaled matrix     : Ah = D^{-1/2} A D^{-1/2} (unit diagonal), D = diag(A)
  features of row i : Ah_{i,s} (off-diagonal slots), log(a_jj / a_ii) of each
                      neighbour slot, log|a_ii| - mean log|diag|, 1; padded to 16
  MLP               : h1 = relu(x W1 + b1), h2 = relu(h1 W2 + b2), o = h2 W3 + b3
                      with bf16-rounded weights
  Mh (symmetric, on A's pattern, diagonally dominant hence SPD):
                      S_ij = (tanh(o_{i,s}) + tanh(o_{j,s'})) / 4 for the edge i-j
                      (slot s of row i, slot s' of row j),
                      Mh_ij = S_ij,  Mh_ii = 1 + tanh(o_{i,d}) / 2 + sum_j |S_ij|;
                      o = 0 gives Mh = I (Jacobi);  M = D^{-1/2} Mh D^{-1/2}
  loss              = w_F ||Ah Mh - I||_F^2 / n
                      + w_R mean_s ||Ah Mh rh_s - rh_s||^2 / ||rh_s||^2,  rh_s = D^{-1/2} r_s
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

KF, KH, KO = 16, 64, 8
W1, B1 = 0, KF * KH
W2 = B1 + KH
B2 = W2 + KH * KH
W3 = B2 + KH
B3 = W3 + KH * KO
NP = B3 + KO


def bf16(w: np.ndarray) -> np.ndarray:
    """Round float32 to bfloat16 (nearest, ties to even), returned as float64."""
    u = np.ascontiguousarray(w, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def slots(A, offsets):
    """slot index of every CSR entry (-1 if its offset is not a stencil slot)."""
    rows = np.repeat(np.arange(A.n), np.diff(A.row_ptr))
    d = A.col_ind.astype(np.int64) - rows
    s = np.full(A.nnz, -1, dtype=np.int64)
    for k, o in enumerate(offsets):
        s[d == o] = k
    return rows, s


def scaled(A, diag):
    """Ah values on A's pattern: a_ij / sqrt(a_ii a_jj) (binary32 inputs)."""
    val = A.val.astype(np.float32).astype(np.float64)
    rows = np.repeat(np.arange(A.n), np.diff(A.row_ptr))
    return val / np.sqrt(np.abs(diag[rows] * diag[A.col_ind]))


def features(A, offsets, dslot):
    val = A.val.astype(np.float32).astype(np.float64)
    rows, s = slots(A, offsets)
    diag = np.zeros(A.n)
    diag[rows[s == dslot]] = val[s == dslot]
    ah = scaled(A, diag)
    ns = len(offsets)
    a = np.zeros((A.n, ns))
    dj = np.zeros((A.n, ns))
    ok = s >= 0
    a[rows[ok], s[ok]] = ah[ok]
    dj[rows[ok], s[ok]] = np.log(np.abs(diag[A.col_ind[ok]] / diag[rows[ok]]))
    X = np.zeros((A.n, KF))
    others = [k for k in range(ns) if k != dslot]
    for j, k in enumerate(others):
        X[:, j] = a[:, k]
        X[:, j + ns - 1] = dj[:, k]
    ml = np.mean(np.log(np.abs(diag)))
    X[:, 2 * (ns - 1)] = np.log(np.abs(diag)) - ml
    X[:, 2 * (ns - 1) + 1] = 1.0
    return X, diag


def unpack(w):
    wb = bf16(w)
    return (wb[W1:B1].reshape(KF, KH), wb[B1:W2], wb[W2:B2].reshape(KH, KH), wb[B2:W3],
            wb[W3:B3].reshape(KH, KO), wb[B3:NP])


def forward(w, X):
    w1, b1, w2, b2, w3, b3 = unpack(w)
    z1 = X @ w1 + b1
    h1 = np.maximum(z1, 0)
    z2 = h1 @ w2 + b2
    h2 = np.maximum(z2, 0)
    out = h2 @ w3 + b3
    return h1, h2, out


def edges(A, offsets, dslot):
    """rows, slot, and the CSR position of the transposed entry of every entry."""
    rows, s = slots(A, offsets)
    pos = {(int(i), int(j)): k for k, (i, j) in enumerate(zip(rows, A.col_ind))}
    tr = np.array([pos.get((int(j), int(i)), -1) for i, j in zip(rows, A.col_ind)])
    return rows, s, tr


def assemble_scaled(A, offsets, out, dslot):
    """Mh on A's pattern."""
    rows, s, tr = edges(A, offsets, dslot)
    t = np.tanh(out)
    m = np.zeros(A.nnz)
    off = (s >= 0) & (s != dslot) & (tr >= 0)
    S = np.zeros(A.nnz)
    S[off] = 0.25 * (t[rows[off], s[off]] + t[A.col_ind[off], s[tr[off]]])
    m[off] = S[off]
    d = (s == dslot)
    rowsum = np.bincount(rows, weights=np.abs(S), minlength=A.n)
    m[d] = 1.0 + 0.5 * t[rows[d], dslot] + rowsum[rows[d]]
    return m


def assemble(A, offsets, dslot, out, diag):
    """M = D^{-1/2} Mh D^{-1/2} on A's pattern (the preconditioner)."""
    rows = np.repeat(np.arange(A.n), np.diff(A.row_ptr))
    return assemble_scaled(A, offsets, out, dslot) / np.sqrt(np.abs(diag[rows] * diag[A.col_ind]))


def loss_and_grad(A, offsets, dslot, w, residuals, w_frob=1.0, w_resid=1.0):
    """Returns (total, frobenius, residual, grad[NP]) in float64."""
    n = A.n
    X, diag = features(A, offsets, dslot)
    h1, h2, out = forward(w, X)
    m = assemble_scaled(A, offsets, out, dslot)
    ah = scaled(A, diag)
    As = sp.csr_matrix((ah, A.col_ind, A.row_ptr), shape=(n, n))
    Ms = sp.csr_matrix((m, A.col_ind, A.row_ptr), shape=(n, n))
    G = (As @ Ms - sp.identity(n)).tocsr()
    lf = float(G.multiply(G).sum()) / n
    rows = np.repeat(np.arange(n), np.diff(A.row_ptr))
    dMf = (2.0 * (As.T @ G)).tocsr()
    dm = np.asarray(dMf[rows, A.col_ind]).ravel() * (w_frob / n)
    lr = 0.0
    nres = len(residuals)
    for r in residuals:
        r = np.asarray(r, dtype=np.float32).astype(np.float64) / np.sqrt(np.abs(diag))
        rr = r @ r
        z = As @ (Ms @ r) - r
        lr += (z @ z) / rr / nres
        g = As.T @ z
        dm += w_resid * 2.0 * g[rows] * r[A.col_ind] / (rr * nres)
    # dout[i][s] = dL/do_{i,s} through S (both entries, both diagonals) and the diagonal
    rows_, s, tr = edges(A, offsets, dslot)
    t = np.tanh(out)
    dpos = np.full(n, -1)
    dpos[rows_[s == dslot]] = np.nonzero(s == dslot)[0]
    dout = np.zeros((n, KO))
    off = (s >= 0) & (s != dslot) & (tr >= 0)
    S = np.zeros(A.nnz)
    S[off] = 0.25 * (t[rows_[off], s[off]] + t[A.col_ind[off], s[tr[off]]])
    dS = np.zeros(A.nnz)
    dS[off] = dm[off] + dm[tr[off]] + np.sign(S[off]) * (dm[dpos[rows_[off]]] + dm[dpos[A.col_ind[off]]])
    dout[rows_[off], s[off]] = 0.25 * (1 - t[rows_[off], s[off]] ** 2) * dS[off]
    d = s == dslot
    dout[rows_[d], dslot] = 0.5 * (1 - t[rows_[d], dslot] ** 2) * dm[d]
    # backprop
    w1, b1, w2, b2, w3, b3 = unpack(w)
    grad = np.zeros(NP)
    grad[W3:B3] = (h2.T @ dout).ravel()
    grad[B3:NP] = dout.sum(0)
    dh2 = (dout @ w3.T) * (h2 > 0)
    grad[W2:B2] = (h1.T @ dh2).ravel()
    grad[B2:W3] = dh2.sum(0)
    dh1 = (dh2 @ w2.T) * (h1 > 0)
    grad[W1:B1] = (X.T @ dh1).ravel()
    grad[B1:W2] = dh1.sum(0)
    return w_frob * lf + w_resid * lr, lf, lr, grad
