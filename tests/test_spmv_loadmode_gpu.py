"""The load modes of the sparse products (csrc/hpb_common.cuh, load_mode):
evict-first or cached streaming of the matrix by its size against L2, and
one access per complex element when the arrays are aligned to it.  The
modes change only how bytes move.  The large cases (2048^2, 252 MB of
binary64 and 419 MB of complex<double> matrix) take the cached mode on
B200's 126 MB L2, the small ones stay evict-first: each matches the numpy
restatement within the SpMV tolerance.  An 8-byte-offset complex<double>
value array takes the two-access form, which must give the same bits as
the one-access form of the same matrix."""
import numpy as np
import pytest

from gpu_utils import host
from high_precision_blas1_b200 import _lib, problems
from test_spmv_gpu import check

pytestmark = pytest.mark.gpu


def spmv_ptrs(ctx, torch, t, A, rp, ci, val_ptr, x, y):
    st = getattr(_lib.lib, f"hpb_csr_spmv_{t}")(ctx.h, A.n, A.n, A.nnz, rp.data_ptr(), ci.data_ptr(), val_ptr,
                                               _lib.scalar(t, 1.0), x.data_ptr(), _lib.scalar(t, 0.0), y.data_ptr())
    ctx.check(st, "spmv")
    torch.cuda.synchronize()
    return host(y)


@pytest.mark.parametrize("t,N", [("f64", 2048), ("c128", 2048), ("f64", 256), ("c128", 256)])
def test_load_modes_same_bits(gpu, t, N):
    ctx, torch = gpu
    cplx = t == "c128"
    A = problems.helmholtz2d(N) if cplx else problems.convdiff2d(N)
    rng = np.random.default_rng(N)
    x = rng.uniform(-1, 1, A.n) + (1j * rng.uniform(-1, 1, A.n) if cplx else 0)
    tdt = torch.complex128 if cplx else torch.float64
    rp = torch.from_numpy(A.row_ptr).cuda()
    ci = torch.from_numpy(A.col_ind).cuda()
    val = torch.from_numpy(A.val.astype(np.complex128 if cplx else np.float64)).cuda()
    dx = torch.from_numpy(x.astype(np.complex128 if cplx else np.float64)).cuda()
    y1 = torch.empty(A.n, dtype=tdt, device="cuda")
    got = spmv_ptrs(ctx, torch, t, A, rp, ci, val.data_ptr(), dx, y1)
    check(A, t, 1.0, x, 0.0, np.zeros(A.n), got)
    if cplx:
        # the same values from an array that is 8- but not 16-byte aligned
        raw = torch.zeros(2 * A.nnz + 1, dtype=torch.float64, device="cuda")
        raw[1:].copy_(torch.view_as_real(val).reshape(-1))
        y2 = torch.empty(A.n, dtype=tdt, device="cuda")
        got2 = spmv_ptrs(ctx, torch, t, A, rp, ci, raw.data_ptr() + 8, dx, y2)
        assert np.array_equal(got.view(np.float64), got2.view(np.float64))
    del val, dx, rp, ci
    torch.cuda.empty_cache()
