"""GPU parity of the CSR SpMV (through the C ABI) against a numpy
float64/complex128 restatement.  Tolerance per row:
|gpu - ref| <= 4 (nnz_row + 2) eps(type) (|alpha| sum_k |a_k||x_k| + |beta||y|)."""
import numpy as np
import pytest

from gpu_utils import EPS, dev, host
from high_precision_blas1_b200 import _lib, problems

pytestmark = pytest.mark.gpu

DT = {"f32": np.float32, "f64": np.float64, "c64": np.complex64, "c128": np.complex128}
WIDE = {"f32": np.float64, "f64": np.float64, "c64": np.complex128, "c128": np.complex128}


def random_csr(rng, rows, cols, density, long_rows=(), empty_rows=()):
    rp = [0]
    ci = []
    for r in range(rows):
        if r in empty_rows:
            k = 0
        elif r in long_rows:
            k = cols
        else:
            k = rng.binomial(cols, density)
        c = np.sort(rng.choice(cols, size=k, replace=False)) if k else np.zeros(0, dtype=np.int64)
        ci.extend(c.tolist())
        rp.append(len(ci))
    return problems.CSR(rows, np.array(rp, dtype=np.int32), np.array(ci, dtype=np.int32),
                        rng.standard_normal(len(ci)))


def spmv(ctx, torch, t, A, alpha, x, beta, y):
    d = [dev(torch, a) for a in (A.row_ptr, A.col_ind, A.val.astype(DT[t]), x.astype(DT[t]), y.astype(DT[t]))]
    st = getattr(_lib.lib, f"hpb_csr_spmv_{t}")(ctx.h, A.n, x.shape[0], A.nnz, d[0].data_ptr(), d[1].data_ptr(),
                                               d[2].data_ptr(), _lib.scalar(t, alpha), d[3].data_ptr(),
                                               _lib.scalar(t, beta), d[4].data_ptr())
    ctx.check(st, "spmv")
    torch.cuda.synchronize()
    return host(d[4])


def check(A, t, alpha, x, beta, y, got):
    W = WIDE[t]
    v = A.val.astype(DT[t]).astype(W)
    xs = x.astype(DT[t]).astype(W)
    ys = y.astype(DT[t]).astype(W)
    want = alpha * problems.CSR(A.n, A.row_ptr, A.col_ind, v).matvec(xs) + (beta * ys if beta != 0 else 0)
    absA = problems.CSR(A.n, A.row_ptr, A.col_ind, np.abs(v)).matvec(np.abs(xs))
    rowlen = np.diff(A.row_ptr)
    tol = 4 * (rowlen + 2) * EPS[t] * (abs(alpha) * absA + (abs(beta) * np.abs(ys) if beta != 0 else 0)) + 1e-300
    err = np.abs(got.astype(W) - want)
    assert np.all(err <= tol), (t, float(np.max(err / tol)))


@pytest.mark.parametrize("t", ["f32", "f64", "c64", "c128"])
def test_spmv_stencils(gpu, t):
    ctx, torch = gpu
    rng = np.random.default_rng(1)
    for A in (problems.convdiff2d(37), problems.poisson3d_aniso(11), problems.diffusion3d_lognormal(12, seed=3)):
        cplx = t.startswith("c")
        if cplx:
            A = problems.CSR(A.n, A.row_ptr, A.col_ind, A.val * (1 + 0.3j))
        x = rng.standard_normal(A.n) + (1j * rng.standard_normal(A.n) if cplx else 0)
        y = rng.standard_normal(A.n) + (1j * rng.standard_normal(A.n) if cplx else 0)
        for alpha, beta in ((1.0, 0.0), (2.5, -0.75), (-1.0, 1.0)):
            if cplx:
                alpha, beta = complex(alpha, 0.5), complex(beta, -0.25) if beta else 0.0
            got = spmv(ctx, torch, t, A, alpha, x, beta, y)
            check(A, t, alpha, x, beta, y, got)


@pytest.mark.parametrize("t", ["f64", "c128", "f32"])
def test_spmv_ragged_empty_and_long_rows(gpu, t):
    """Empty rows, rows longer than the shared-memory staging capacity, and
    a row count that is not a multiple of the block's 256 rows."""
    ctx, torch = gpu
    rng = np.random.default_rng(5)
    A = random_csr(rng, 1000, 3000, 0.002, long_rows=(3, 700), empty_rows=(0, 1, 999))
    if t.startswith("c"):
        A = problems.CSR(A.n, A.row_ptr, A.col_ind, A.val + 1j * rng.standard_normal(A.nnz))
    x = rng.standard_normal(3000) + (1j * rng.standard_normal(3000) if t.startswith("c") else 0)
    y = rng.standard_normal(1000) + (1j * rng.standard_normal(1000) if t.startswith("c") else 0)
    got = spmv(ctx, torch, t, A, 1.5, x, -0.5, y)
    check(A, t, 1.5, x, -0.5, y, got)


def test_spmv_beta_zero_ignores_y(gpu):
    ctx, torch = gpu
    A = problems.convdiff2d(20)
    x = np.ones(A.n)
    y = np.full(A.n, np.nan)
    got = spmv(ctx, torch, "f64", A, 1.0, x, 0.0, y)
    assert np.all(np.isfinite(got))
    assert np.allclose(got, A.matvec(x))


def test_spmv_zero_rows_and_bad_args(gpu):
    ctx, torch = gpu
    L = _lib.lib
    assert L.hpb_csr_spmv_f64(ctx.h, 0, 0, 0, None, None, None, 1.0, None, 0.0, None) == 0
    assert L.hpb_csr_spmv_f64(ctx.h, -1, 0, 0, None, None, None, 1.0, None, 0.0, None) == -1
    assert L.hpb_csr_spmv_f64(ctx.h, 4, 4, 4, None, None, None, 1.0, None, 0.0, None) == -1


def test_csr_diagonal(gpu):
    ctx, torch = gpu
    A = problems.convdiff2d(16)
    d = dev(torch, np.zeros(A.n))
    rp, ci, va = dev(torch, A.row_ptr), dev(torch, A.col_ind), dev(torch, A.val)
    ctx.check(_lib.lib.hpb_csr_diag_f64(ctx.h, A.n, rp.data_ptr(), ci.data_ptr(), va.data_ptr(), d.data_ptr()))
    torch.cuda.synchronize()
    want = np.array([A.val[A.row_ptr[r]:A.row_ptr[r + 1]][A.col_ind[A.row_ptr[r]:A.row_ptr[r + 1]] == r][0]
                     for r in range(A.n)])
    assert np.array_equal(host(d), want)


def spmv_dot2(ctx, torch, t, A, x, w):
    d = [dev(torch, a) for a in (A.row_ptr, A.col_ind, A.val.astype(DT[t]), x.astype(DT[t]), np.zeros(A.n, DT[t]),
                                 w.astype(DT[t]))]
    out = torch.full((4,), np.nan, dtype=torch.float64, device="cuda")
    st = getattr(_lib.lib, f"hpb_csr_spmv_dot2_{t}")(ctx.h, A.n, x.shape[0], A.nnz, d[0].data_ptr(),
                                                    d[1].data_ptr(), d[2].data_ptr(), d[3].data_ptr(),
                                                    d[4].data_ptr(), d[5].data_ptr(), out.data_ptr())
    ctx.check(st, "spmv_dot2")
    torch.cuda.synchronize()
    return host(d[4]), host(out)


@pytest.mark.parametrize("t", ["f32", "f64", "c64", "c128"])
def test_spmv_dot2_fused(gpu, t):
    """y bit-identical to hpb_csr_spmv (alpha 1, beta 0); <w, y> within the
    compensated Dot2 bound of the exact dot of the rounded y (oracle)."""
    import oracle
    ctx, torch = gpu
    rng = np.random.default_rng(5)
    for A in (problems.convdiff2d(300), random_csr(rng, 3001, 2900, 0.003, long_rows=(7,), empty_rows=(0, 11)),
              problems.convdiff2d(1024)):
        x = rng.standard_normal(2900 if A.n == 3001 else A.n)
        w = rng.standard_normal(A.n)
        if t in ("c64", "c128"):
            x = x + 1j * rng.standard_normal(x.shape[0])
            w = w + 1j * rng.standard_normal(A.n)
        y, out = spmv_dot2(ctx, torch, t, A, x, w)
        y_ref = spmv(ctx, torch, t, A, 1.0, x, 0.0, np.zeros(A.n))
        assert np.array_equal(y.view(np.uint8), y_ref.view(np.uint8))
        wd, yd = w.astype(DT[t]).astype(WIDE[t]), y.astype(WIDE[t])
        if t in ("f32", "f64"):
            hi, _ = oracle.exact_dot(wd, yd)
            scale = float(np.sum(np.abs(wd * yd)))
            assert abs(out[0] - hi) <= oracle.bound_dot2(A.n, scale / abs(hi)) * abs(hi) + 2 * np.spacing(abs(hi))
        else:
            hc, _ = oracle.exact_dot(wd, yd)
            hr, hi_ = hc.real, hc.imag
            scale = float(np.sum(np.abs(wd) * np.abs(yd)))
            b = oracle.bound_dot2(A.n, 1.0, complex_=True) * scale
            assert abs(out[0] - hr) <= b + 2 * np.spacing(abs(hr)) and abs(out[1] - hi_) <= b + 2 * np.spacing(abs(hi_))


def test_spmv_dot2_bad_args(gpu):
    ctx, torch = gpu
    A = problems.convdiff2d(8)
    d = [dev(torch, a) for a in (A.row_ptr, A.col_ind, A.val, np.ones(A.n), np.zeros(A.n), np.ones(A.n))]
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    f = _lib.lib.hpb_csr_spmv_dot2_f64
    p = [a.data_ptr() for a in d]
    assert f(ctx.h, A.n, A.n, A.nnz, p[0], p[1], p[2], p[3], p[4], p[5], None) == -1
    assert f(ctx.h, -1, A.n, A.nnz, p[0], p[1], p[2], p[3], p[4], p[5], out.data_ptr()) == -1
    assert f(ctx.h, A.n, A.n, A.nnz, p[0], p[1], p[2] + 4, p[3], p[4], p[5], out.data_ptr()) == -1
    # zero rows: out is the empty sum
    assert f(ctx.h, 0, 0, 0, p[0], None, None, None, None, None, out.data_ptr()) == 0


@pytest.mark.parametrize("name,t", [("general_real", "f64"), ("symmetric_real", "f32"), ("complex_general", "c128")])
def test_spmv_of_matrix_market_file(gpu, name, t):
    """A Matrix Market file read by the library's parser, multiplied on the
    GPU: equals scipy's product of scipy's own reading of the file."""
    import scipy.io
    from conftest import GOLDEN
    ctx, torch = gpu
    A = problems.read_matrix_market(GOLDEN / "mm" / f"{name}.mtx")
    ref = scipy.io.mmread(str(GOLDEN / "mm" / f"{name}.mtx")).tocsr()
    rng = np.random.default_rng(2)
    x = rng.standard_normal(A.n) + (1j * rng.standard_normal(A.n) if t.startswith("c") else 0)
    y = spmv(ctx, torch, t, A, 1.0, x, 0.0, np.zeros(A.n))
    want = ref @ x.astype(WIDE[t])
    assert np.allclose(y, want, rtol=4e-6 if t in ("f32", "c64") else 1e-14, atol=1e-6 if t == "f32" else 1e-14)


@pytest.mark.parametrize("shape", [(300, 200), (200, 300), (1024, 1024)])
def test_transpose_pattern_matches_scipy(gpu, shape):
    """hpb_csr_transpose_pattern: A^T's row pointers and column indices equal
    scipy's transpose (sorted indices), and the gathered values
    (hpb_gather_f64 with perm) equal its values; rectangular and square."""
    import scipy.sparse as sp
    ctx, torch = gpu
    rows, cols = shape
    A = sp.random(rows, cols, density=0.02, random_state=rows + cols, format="csr")
    A.sort_indices()
    T = sp.csr_matrix(A.T)
    T.sort_indices()
    d = [dev(torch, a) for a in (A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data)]
    rp_t = torch.zeros(cols + 1, dtype=torch.int32, device="cuda")
    ci_t = torch.zeros(max(A.nnz, 1), dtype=torch.int32, device="cuda")
    perm = torch.zeros(max(A.nnz, 1), dtype=torch.int32, device="cuda")
    ctx.check(_lib.lib.hpb_csr_transpose_pattern(ctx.h, rows, cols, A.nnz, d[0].data_ptr(), d[1].data_ptr(),
                                                 rp_t.data_ptr(), ci_t.data_ptr(), perm.data_ptr()), "transpose")
    vt = torch.zeros(max(A.nnz, 1), dtype=torch.float64, device="cuda")
    ctx.check(_lib.lib.hpb_gather_f64(ctx.h, A.nnz, perm.data_ptr(), d[2].data_ptr(), vt.data_ptr()), "gather")
    torch.cuda.synchronize()
    assert np.array_equal(host(rp_t), T.indptr) and np.array_equal(host(ci_t)[:A.nnz], T.indices)
    assert np.array_equal(host(vt)[:A.nnz], T.data)


def test_transpose_pattern_rejects_bad_columns(gpu):
    ctx, torch = gpu
    rp = dev(torch, np.array([0, 2], np.int32))
    ci = dev(torch, np.array([0, 7], np.int32))
    out = [torch.zeros(4, dtype=torch.int32, device="cuda") for _ in range(3)]
    st = _lib.lib.hpb_csr_transpose_pattern(ctx.h, 1, 3, 2, rp.data_ptr(), ci.data_ptr(), *[o.data_ptr() for o in out])
    assert st == -1


def test_dropin_transposed_operations(gpu):
    """csr::gpu_matrix with transpose_ = true (compiled into the drop-in test
    library): A^T x against scipy, L^T and U^T solves bit for bit against
    substitution on scipy's transpose (oracle/tri.c)."""
    import ctypes as C
    import oracle
    import scipy.sparse as sp
    ctx, torch = gpu
    so = oracle.HERE / "_ref" / "libhpb_ref_dropin.so"
    if not so.exists():
        pytest.skip("oracle/_ref/libhpb_ref_dropin.so not built")
    lib = C.CDLL(str(so))
    lib.ref_dropin_transposed_ops_f64.argtypes = [C.c_int, C.c_int64] + [C.c_void_p] * 7
    A = problems.convdiff2d(48)
    rows = np.repeat(np.arange(A.n), np.diff(A.row_ptr))
    diag = A.val[A.col_ind == rows]
    A = problems.CSR(A.n, A.row_ptr, A.col_ind, A.val / diag[rows])  # row-scaled: bounded unit solves
    rng = np.random.default_rng(4)
    x = rng.standard_normal(A.n)
    d = [dev(torch, a) for a in (A.row_ptr, A.col_ind, A.val, x, np.zeros(A.n), np.zeros(A.n), np.zeros(A.n))]
    assert lib.ref_dropin_transposed_ops_f64(A.n, A.nnz, *[a.data_ptr() for a in d]) == 1
    torch.cuda.synchronize()
    M = sp.csr_matrix((A.val, A.col_ind, A.row_ptr), shape=(A.n, A.n))
    T = sp.csr_matrix(M.T)
    T.sort_indices()
    assert np.allclose(host(d[4]), T @ x, rtol=1e-14, atol=1e-14 * np.abs(T).dot(np.abs(x)).max())
    z = oracle.csr_trsv(T.indptr, T.indices, T.data, x, upper=True, unit=True)    # (L)^T = unit upper of A^T
    w = oracle.csr_trsv(T.indptr, T.indices, T.data, x, upper=False, unit=False)  # (U)^T = lower of A^T
    assert np.array_equal(host(d[5]), z) and np.array_equal(host(d[6]), w)
