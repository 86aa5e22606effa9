"""Seeded synthetic linear systems in the shapes of the benchmark configs.

All matrices are square CSR (int32 row pointers / column indices, sorted
columns, 0-based) on a uniform grid of interior points with homogeneous
Dirichlet boundaries, natural (x fastest) ordering, spacing h = 1/(N+1).

* convdiff2d   -- 2-D 5-point convection-diffusion  a.grad u - (1/Re) lap u,
                  first-order upwind convection, central diffusion; the 2-D
                  form of the reference's 1-D test operator
                  (linear_operator.hpp:28-56).  Peclet = |a| L Re with
                  a = (1, 1)/sqrt(2), L = 1.  1024^2: n = 1,048,576,
                  nnz = 5,238,784.
* poisson3d_aniso -- 3-D 7-point -(ex u_xx + ey u_yy + ez u_zz), scaled by
                  h^2 (entries O(1)).  128^3: nnz = 14,581,760.
* helmholtz2d  -- 2-D 5-point -lap u - k^2 u + 0.5i k^2 u (damped), k chosen
                  for `ppw` points per wavelength (k h = 2 pi / ppw), scaled
                  by h^2; complex.  2048^2: nnz = 20,963,328.
* diffusion3d_lognormal -- 3-D 7-point -div(kappa grad u), kappa = exp(g),
                  g a Gaussian random field (separable Gaussian smoothing of
                  white noise, correlation length `corr` cells, rescaled to
                  standard deviation `sigma`), harmonic-mean face
                  coefficients, scaled by h^2.  96^3: nnz = 6,137,856.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


@dataclass
class CSR:
    n: int
    row_ptr: np.ndarray  # int32 [n+1]
    col_ind: np.ndarray  # int32 [nnz]
    val: np.ndarray      # float64 / complex128 [nnz]

    @property
    def nnz(self) -> int:
        return int(self.col_ind.shape[0])

    def astype(self, dtype) -> "CSR":
        return CSR(self.n, self.row_ptr, self.col_ind, self.val.astype(dtype))

    def matvec(self, x: np.ndarray) -> np.ndarray:
        """Reference product for tests (numpy, float64/complex128)."""
        prod = self.val * x[self.col_ind]
        rows = np.repeat(np.arange(self.n), np.diff(self.row_ptr))
        if np.iscomplexobj(prod):
            return (np.bincount(rows, weights=prod.real, minlength=self.n)
                    + 1j * np.bincount(rows, weights=prod.imag, minlength=self.n))
        return np.bincount(rows, weights=prod, minlength=self.n)


def _assemble(n: int, cols: np.ndarray, vals: np.ndarray) -> CSR:
    """cols/vals: [n, k] stencil slots in increasing column order; col < 0 = absent."""
    mask = cols >= 0
    counts = mask.sum(axis=1).astype(np.int64)
    rp = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(counts, out=rp[1:])
    return CSR(n, rp.astype(np.int32), cols[mask].astype(np.int32), vals[mask])


def convdiff2d(N: int = 1024, peclet: float = 50.0, a=(1.0 / math.sqrt(2.0), 1.0 / math.sqrt(2.0))) -> CSR:
    h = 1.0 / (N + 1)
    re = peclet  # |a| = 1, L = 1
    ax, ay = a
    n = N * N
    idx = np.arange(n, dtype=np.int64)
    i = idx % N
    j = idx // N
    d = 1.0 / (re * h * h)
    cols = np.full((n, 5), -1, dtype=np.int64)
    vals = np.zeros((n, 5))
    # slots in column order: south (j-1), west (i-1), centre, east (i+1), north (j+1)
    cols[:, 0] = np.where(j > 0, idx - N, -1)
    vals[:, 0] = -ay / h - d
    cols[:, 1] = np.where(i > 0, idx - 1, -1)
    vals[:, 1] = -ax / h - d
    cols[:, 2] = idx
    vals[:, 2] = (ax + ay) / h + 4.0 * d
    cols[:, 3] = np.where(i < N - 1, idx + 1, -1)
    vals[:, 3] = -d
    cols[:, 4] = np.where(j < N - 1, idx + N, -1)
    vals[:, 4] = -d
    return _assemble(n, cols, vals)


def _stencil7(N: int, cx, cy, cz, diag) -> CSR:
    """7-point operator with per-row face coefficients (arrays or scalars)."""
    n = N ** 3
    idx = np.arange(n, dtype=np.int64)
    i = idx % N
    j = (idx // N) % N
    k = idx // (N * N)
    cols = np.full((n, 7), -1, dtype=np.int64)
    vals = np.zeros((n, 7))
    cxm, cxp = cx
    cym, cyp = cy
    czm, czp = cz
    cols[:, 0] = np.where(k > 0, idx - N * N, -1)
    vals[:, 0] = -czm
    cols[:, 1] = np.where(j > 0, idx - N, -1)
    vals[:, 1] = -cym
    cols[:, 2] = np.where(i > 0, idx - 1, -1)
    vals[:, 2] = -cxm
    cols[:, 3] = idx
    vals[:, 3] = diag
    cols[:, 4] = np.where(i < N - 1, idx + 1, -1)
    vals[:, 4] = -cxp
    cols[:, 5] = np.where(j < N - 1, idx + N, -1)
    vals[:, 5] = -cyp
    cols[:, 6] = np.where(k < N - 1, idx + N * N, -1)
    vals[:, 6] = -czp
    return _assemble(n, cols, vals)


def poisson3d_aniso(N: int = 128, eps=(1.0, 1e-2, 1e-4)) -> CSR:
    ex, ey, ez = eps
    return _stencil7(N, (ex, ex), (ey, ey), (ez, ez), 2.0 * (ex + ey + ez))


def helmholtz2d(N: int = 2048, ppw: float = 10.0, damping: float = 0.5) -> CSR:
    h = 1.0 / (N + 1)
    kh = 2.0 * math.pi / ppw
    shift = complex(-kh * kh, damping * kh * kh)  # (-k^2 + i*damping*k^2) * h^2
    n = N * N
    idx = np.arange(n, dtype=np.int64)
    i = idx % N
    j = idx // N
    cols = np.full((n, 5), -1, dtype=np.int64)
    vals = np.zeros((n, 5), dtype=np.complex128)
    cols[:, 0] = np.where(j > 0, idx - N, -1)
    vals[:, 0] = -1.0
    cols[:, 1] = np.where(i > 0, idx - 1, -1)
    vals[:, 1] = -1.0
    cols[:, 2] = idx
    vals[:, 2] = 4.0 + shift
    cols[:, 3] = np.where(i < N - 1, idx + 1, -1)
    vals[:, 3] = -1.0
    cols[:, 4] = np.where(j < N - 1, idx + N, -1)
    vals[:, 4] = -1.0
    return _assemble(n, cols, vals)


def _gauss_kernel(corr: float) -> np.ndarray:
    r = int(math.ceil(3 * corr))
    t = np.arange(-r, r + 1, dtype=np.float64)
    w = np.exp(-0.5 * (t / corr) ** 2)
    return w / w.sum()


def lognormal_field(N: int, seed: int, sigma: float = 2.3, corr: float = 8.0) -> np.ndarray:
    """log-coefficient g on the N^3 cells (array [k, j, i]), std = sigma."""
    rng = np.random.default_rng(seed)
    g = rng.standard_normal((N, N, N))
    w = _gauss_kernel(corr)
    for ax in range(3):  # separable periodic smoothing
        g = sum(np.roll(g, s, axis=ax) * w[s + len(w) // 2] for s in range(-(len(w) // 2), len(w) // 2 + 1))
    g = (g - g.mean()) / g.std() * sigma
    return g


def diffusion3d_lognormal(N: int = 96, seed: int = 0, sigma: float = 2.3, corr: float = 8.0) -> CSR:
    kap = np.exp(lognormal_field(N, seed, sigma, corr))  # [k, j, i]

    def hm(a, b):
        return 2.0 * a * b / (a + b)

    # face coefficients; boundary faces use the cell's own kappa
    kxm = np.concatenate([kap[:, :, :1], hm(kap[:, :, 1:], kap[:, :, :-1])], axis=2)
    kxp = np.concatenate([hm(kap[:, :, :-1], kap[:, :, 1:]), kap[:, :, -1:]], axis=2)
    kym = np.concatenate([kap[:, :1, :], hm(kap[:, 1:, :], kap[:, :-1, :])], axis=1)
    kyp = np.concatenate([hm(kap[:, :-1, :], kap[:, 1:, :]), kap[:, -1:, :]], axis=1)
    kzm = np.concatenate([kap[:1], hm(kap[1:], kap[:-1])], axis=0)
    kzp = np.concatenate([hm(kap[:-1], kap[1:]), kap[-1:]], axis=0)
    f = lambda a: a.reshape(-1)  # noqa: E731
    diag = f(kxm + kxp + kym + kyp + kzm + kzp)
    return _stencil7(N, (f(kxm), f(kxp)), (f(kym), f(kyp)), (f(kzm), f(kzp)), diag)


def rhs_uniform(n: int, seed: int, complex_: bool = False) -> np.ndarray:
    rng = np.random.default_rng(seed)
    if complex_:
        return rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    return rng.uniform(-1, 1, n)


def read_matrix_market(path) -> CSR:
    """A Matrix Market coordinate file as a CSR matrix (host arrays), read by
    the library's parser (hpb_mm_read_csr: the reference's
    csr::matrix_market_reader semantics -- symmetric files mirrored, entries
    in stable (row, column) order, duplicates kept, pattern entries 1).
    Raises ValueError with the parser's message on a rejected file."""
    import ctypes as C
    from . import _lib
    m = _lib.hpb_mm_csr()
    st = _lib.lib.hpb_mm_read_csr(str(path).encode(), C.byref(m))
    if st != 0:
        raise ValueError(_lib.lib.hpb_mm_last_error().decode())
    try:
        n, nnz = m.rows, m.nnz
        rp = np.ctypeslib.as_array(m.row_ptr, shape=(n + 1,)).copy()
        ci = np.ctypeslib.as_array(m.col_ind, shape=(max(nnz, 1),))[:nnz].copy()
        if m.is_complex:
            v = np.ctypeslib.as_array(m.val, shape=(max(2 * nnz, 2),))[:2 * nnz].copy()
            val = v[0::2] + 1j * v[1::2]
        else:
            val = np.ctypeslib.as_array(m.val, shape=(max(nnz, 1),))[:nnz].copy()
        if m.cols != m.rows:
            raise ValueError(f"matrix is {m.rows} x {m.cols}; the CSR type here holds square operators")
        return CSR(n, rp.astype(np.int32), ci.astype(np.int32), val)
    finally:
        _lib.lib.hpb_mm_free(C.byref(m))
