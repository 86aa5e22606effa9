"""TEST INFRASTRUCTURE ONLY: float64 CPU restatement of the learned SPAI's
features, MLP forward pass, SPAI assembly, loss and parameter gradient
(the kernels in high_precision_blas1_b200/csrc/hpb_spai.cu), used to check
the GPU forward/backward kernels.  The reference has no learned component;
this oracle restates this repository's own definition:

  features of row i : a_{i,s}/a_ii (off-diagonal slots), a_jj/a_ii of each
                      neighbour slot, log|a_ii| - mean log|diag|, 1; padded to 16
  MLP               : h1 = relu(x W1 + b1), h2 = relu(h1 W2 + b2), o = h2 W3 + b3
                      with bf16-rounded weights
  M_{i, i+off_s}    = o_s / a_ii on A's pattern
  loss              = w_F ||A M - I||_F^2 / n + w_R mean_s ||A M r_s - r_s||^2 / ||r_s||^2
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


def features(A, offsets, dslot):
    val = A.val.astype(np.float32).astype(np.float64)
    rows, s = slots(A, offsets)
    diag = np.zeros(A.n)
    diag[rows[s == dslot]] = val[s == dslot]
    ns = len(offsets)
    a = np.zeros((A.n, ns))
    dj = np.zeros((A.n, ns))
    ok = s >= 0
    a[rows[ok], s[ok]] = val[ok] / diag[rows[ok]]
    dj[rows[ok], s[ok]] = diag[A.col_ind[ok]] / diag[rows[ok]]
    X = np.zeros((A.n, KF))
    others = [k for k in range(ns) if k != dslot]
    for j, k in enumerate(others):
        X[:, j] = a[:, k]
        X[:, j + ns - 1] = dj[:, k]
    ml = np.mean(np.log(np.abs(diag.astype(np.float32).astype(np.float64))))
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


def assemble(A, offsets, out, diag):
    rows, s = slots(A, offsets)
    m = np.zeros(A.nnz)
    ok = s >= 0
    m[ok] = out[rows[ok], s[ok]] / diag[rows[ok]]
    return m


def loss_and_grad(A, offsets, dslot, w, residuals, w_frob=1.0, w_resid=1.0):
    """Returns (total, frobenius, residual, grad[NP]) in float64."""
    n = A.n
    X, diag = features(A, offsets, dslot)
    h1, h2, out = forward(w, X)
    m = assemble(A, offsets, out, diag)
    Av = A.val.astype(np.float32).astype(np.float64)
    As = sp.csr_matrix((Av, A.col_ind, A.row_ptr), shape=(n, n))
    Ms = sp.csr_matrix((m, A.col_ind, A.row_ptr), shape=(n, n))
    G = (As @ Ms - sp.identity(n)).tocsr()
    lf = float(G.multiply(G).sum()) / n
    dMf = (2.0 * (As.T @ G)).tocsr()
    dm = np.asarray(dMf[np.repeat(np.arange(n), np.diff(A.row_ptr)), A.col_ind]).ravel() * (w_frob / n)
    lr = 0.0
    nres = len(residuals)
    for r in residuals:
        r = np.asarray(r, dtype=np.float64)
        rr = r @ r
        z = As @ (Ms @ r) - r
        lr += (z @ z) / rr / nres
        g = As.T @ z
        rows = np.repeat(np.arange(n), np.diff(A.row_ptr))
        dm += w_resid * 2.0 * g[rows] * r[A.col_ind] / (rr * nres)
    # dout[i][s] = dM_{i,i+off_s} / a_ii
    rows, s = slots(A, offsets)
    dout = np.zeros((n, KO))
    ok = s >= 0
    dout[rows[ok], s[ok]] = dm[ok] / diag[rows[ok]]
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
