"""The reference's own bicgstabl.h / gmres.h / default_monitor.h, compiled
unchanged against the C++ drop-in (oracle/_ref/libhpb_ref_dropin.so), run
beside the library's solvers on the same device arrays.  Real data: the
inner products are symmetric, so both run the same recurrences on the same
kernels and must agree bit for bit (iteration count and iterate)."""
import ctypes as C

import numpy as np
import pytest

import oracle
from gpu_utils import dev, host, red
from high_precision_blas1_b200 import _lib, problems

pytestmark = pytest.mark.gpu


def ref_dropin():
    so = oracle.HERE / "_ref" / "libhpb_ref_dropin.so"
    if not so.exists():
        pytest.skip("oracle/_ref/libhpb_ref_dropin.so not built")
    lib = C.CDLL(str(so))
    lib.ref_dropin_solve_f64.argtypes = [C.c_int, C.c_int, C.c_int64] + [C.c_void_p] * 5 + [
        C.c_int, C.c_double, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double)]
    lib.ref_dropin_solve_prec_f64.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int64] + [C.c_void_p] * 5 + [
        C.c_int, C.c_double, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double)]
    return lib


@pytest.mark.parametrize("method,basis,N", [(0, 4, 64), (0, 2, 40), (1, 30, 24)])
def test_reference_solver_over_dropin_matches_library_solver(gpu, method, basis, N):
    ctx, torch = gpu
    lib = ref_dropin()
    A = problems.convdiff2d(N)
    b = problems.rhs_uniform(A.n, 11)
    tol = 1e-10 if method == 0 else 1e-8
    d = [dev(torch, a) for a in (A.row_ptr, A.col_ind, A.val, b)]
    x_ref = dev(torch, np.zeros(A.n))
    it = C.c_int()
    res = C.c_double()
    ok = lib.ref_dropin_solve_f64(method, A.n, A.nnz, d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(),
                                  d[3].data_ptr(), x_ref.data_ptr(), basis, tol, 100000, 1, C.byref(it),
                                  C.byref(res))
    assert ok == 1
    x = dev(torch, np.zeros(A.n))
    rep = _lib.hpb_solver_report()
    p = _lib.solver_params("bicgstabl" if method == 0 else "gmres", basis=basis, rel_tol=tol, max_iters=100000)
    st = _lib.lib.hpb_csr_solve_f64(C.byref(p), A.n, A.nnz, d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(),
                                    d[3].data_ptr(), x.data_ptr(), C.byref(rep), None, 0)
    torch.cuda.synchronize()
    assert st == 0
    assert rep.iters == it.value
    if method == 0:
        assert np.array_equal(host(x), host(x_ref))
    else:
        # GMRES: host-side Givens/triangular solve in the reference runs in T,
        # here in binary64 for every T -- identical for T = double
        assert np.allclose(host(x), host(x_ref), rtol=1e-12, atol=1e-14)
    assert rep.resid_norm == pytest.approx(res.value, rel=1e-12)


@pytest.mark.parametrize("method,basis,N", [(0, 4, 64), (1, 30, 48)])
def test_reference_solver_with_ilu0_matches_library_solver(gpu, method, basis, N):
    """csr::gpu_ilu0_preconditioner (ILU(0) factors, two sparse triangular
    solves per application) under the reference's bicgstabl.h / gmres.h,
    against the library's plain path with HPB_PRECOND_ILU0: same factors,
    same kernels, same iterates.  ILU(0) needs fewer iterations than no
    preconditioner on the convection-diffusion system."""
    ctx, torch = gpu
    lib = ref_dropin()
    A = problems.convdiff2d(N)
    b = problems.rhs_uniform(A.n, 5)
    tol = 1e-10 if method == 0 else 1e-8
    d = [dev(torch, a) for a in (A.row_ptr, A.col_ind, A.val, b)]
    val0 = host(d[2]).copy()
    its = {}
    for pc in (0, 1):
        x_ref = dev(torch, np.zeros(A.n))
        it = C.c_int()
        res = C.c_double()
        ok = lib.ref_dropin_solve_prec_f64(method, pc, A.n, A.nnz, d[0].data_ptr(), d[1].data_ptr(),
                                           d[2].data_ptr(), d[3].data_ptr(), x_ref.data_ptr(), basis, tol, 100000, 1,
                                           C.byref(it), C.byref(res))
        assert ok == 1
        its[pc] = it.value
    assert its[1] < its[0]
    assert np.array_equal(host(d[2]), val0)  # the preconditioner factors a copy
    x = dev(torch, np.zeros(A.n))
    rep = _lib.hpb_solver_report()
    p = _lib.solver_params("bicgstabl" if method == 0 else "gmres", basis=basis, rel_tol=tol, max_iters=100000,
                           precond="ilu0")
    st = _lib.lib.hpb_csr_solve_f64(C.byref(p), A.n, A.nnz, d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(),
                                    d[3].data_ptr(), x.data_ptr(), C.byref(rep), None, 0)
    torch.cuda.synchronize()
    assert st == 0
    assert rep.iters == its[1]
    if method == 0:
        assert np.array_equal(host(x), host(x_ref))
    else:
        assert np.allclose(host(x), host(x_ref), rtol=1e-12, atol=1e-14)
    # left preconditioning: the monitor tests the preconditioned residual
    assert rep.true_resid_norm <= 1e-6 * rep.true_rhs_norm


@pytest.mark.parametrize("code,dtype,n", [(0, np.float32, 100_003), (1, np.float64, 1 << 20), (1, np.float64, 77),
                                          (2, np.complex64, 50_001), (3, np.complex128, 65_537)])
def test_dropin_reducer_class_returns_the_c_abi_bits(gpu, code, dtype, n):
    """gpu_reduction_ogita<T, T*> from the drop-in headers (the class the
    reference's drivers build directly, test_vector_operations.cpp:61/:100)
    returns the C ABI's hi for dot / sum / asum / norm, bit for bit."""
    ctx, torch = gpu
    so = oracle.HERE / "_ref" / "libhpb_ref_dropin.so"
    if not so.exists():
        pytest.skip("oracle/_ref/libhpb_ref_dropin.so not built")
    lib = C.CDLL(str(so))
    lib.ref_dropin_reducer.argtypes = [C.c_int, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p]
    rng = np.random.default_rng(code * 1000 + n)
    if np.issubdtype(dtype, np.complexfloating):
        x = (rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)).astype(dtype)
        y = (rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)).astype(dtype)
    else:
        x = rng.uniform(-1, 1, n).astype(dtype)
        y = rng.uniform(-1, 1, n).astype(dtype)
    dx, dy = dev(torch, x), dev(torch, y)
    out = np.zeros(6)
    torch.cuda.synchronize()
    assert lib.ref_dropin_reducer(code, n, dx.data_ptr(), dy.data_ptr(), out.ctypes.data) == 0
    real = np.float32 if dtype in (np.float32, np.complex64) else np.float64
    cplx = np.issubdtype(dtype, np.complexfloating)
    dot = red(ctx, "dot2", dx, dy)
    s = red(ctx, "sum2", dx)
    a = red(ctx, "asum2", dx)
    nr = red(ctx, "nrm2", dx)
    assert real(out[0]) == real(dot[0]) and real(out[2]) == real(s[0])
    if cplx:
        assert real(out[1]) == real(dot[1]) and real(out[3]) == real(s[1])
    assert real(out[4]) == real(a[0]) and real(out[5]) == real(nr[0])
