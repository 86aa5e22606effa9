"""TEST INFRASTRUCTURE ONLY: ctypes loaders for the oracle.

* ``oro()``  -- liboro.so, the CPU restatement of the reference's Dot2/Sum2
  and the exact (fixed-point) accumulator, built from oro.c.
* ``ref()``  -- _ref/libhpb_ref.so, the reference's own CPU code compiled
  from the reference sources (None when it was not built on this host).

Only tests/, the smoke check and the benchmark's CPU-baseline leg use these.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_ORO = None
_REF = None

D = C.c_double
I64 = C.c_int64
PD = C.POINTER(C.c_double)
P = C.c_void_p


def build() -> None:
    """Build liboro.so (and _ref/ when the reference sources exist)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True, capture_output=True)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(P)


def oro():
    global _ORO
    if _ORO is None:
        so = HERE / "liboro.so"
        if not so.exists():
            build()
        lib = C.CDLL(str(so))
        for name in ("oro_dot2_seq_f64", "oro_dot2_seq_f32", "oro_dot2_seq_c128", "oro_dot2_seq_c64",
                     "oro_dot_naive_f64", "oro_exact_dot_f64", "oro_exact_dot_f32", "oro_exact_dot_c128",
                     "oro_exact_dot_c64", "oro_exact_absdot_f64"):
            getattr(lib, name).argtypes = [I64, P, P, P]
            getattr(lib, name).restype = None
        for name in ("oro_sum2_seq_f64", "oro_sum2_seq_f32"):
            getattr(lib, name).argtypes = [I64, P, C.c_int, P]
            getattr(lib, name).restype = None
        lib.oro_dot2_threaded_f64.argtypes = [I64, P, P, C.c_int, P]
        for name in ("oro_exact_sum_f64", "oro_exact_sum_f32"):
            getattr(lib, name).argtypes = [I64, P, C.c_int, C.c_int, P]
        lib.oro_exact_sumsq_f64.argtypes = [I64, P, C.c_int, P]
        lib.oro_abs_err_dot_f64.argtypes = [I64, P, P, D, D, P]
        for name in ("oro_bound_dot2_real", "oro_bound_dot2_complex", "oro_bound_sum2", "oro_bound_dot_naive_real"):
            getattr(lib, name).argtypes = [D, D, D]
            getattr(lib, name).restype = D
        lib.oro_bound_dot2_block_real.argtypes = [D, D, D, D]
        lib.oro_bound_dot2_block_real.restype = D
        lib.oro_gendot_dev_f64.argtypes = [C.c_uint64, I64, D, P, P]
        lib.oro_gendot_dev_f64.restype = I64
        for suf in ("f32", "f64", "c64", "c128"):
            f = getattr(lib, "oro_csr_trsv_" + suf)
            f.argtypes = [C.c_int32, P, P, P, C.c_int, C.c_int, P, P, P]
            f.restype = C.c_int
            f = getattr(lib, "oro_csr_ilu0_" + suf)
            f.argtypes = [C.c_int32, P, P, P]
            f.restype = C.c_int32
            f = getattr(lib, "oro_csr_trsv_sweeps_" + suf)
            f.argtypes = [C.c_int32, P, P, P, C.c_int, C.c_int, P, P, C.c_int, P, P]
            f.restype = C.c_int
        _ORO = lib
    return _ORO


_REF_GPU = None


def ref_gpu():
    """The reference's own GPU compensated reductions (built for sm_100a), or
    None if _ref was not built.  Needs a CUDA device at call time."""
    global _REF_GPU
    if _REF_GPU is None:
        so = HERE / "_ref" / "libhpb_ref_gpu.so"
        if not so.exists():
            return None
        lib = C.CDLL(str(so))
        for name, args in (("ref_gpu_dot2_f64", [I64, P, P, P]), ("ref_gpu_sum2_f64", [I64, P, P]),
                           ("ref_gpu_dot2_c128", [I64, P, P, P])):
            f = getattr(lib, name)
            f.argtypes = args
            f.restype = C.c_int
        _REF_GPU = lib
    return _REF_GPU


def ref():
    """The reference's own CPU reductions, or None if _ref was not built."""
    global _REF
    if _REF is None:
        so = HERE / "_ref" / "libhpb_ref.so"
        if not so.exists():
            return None
        lib = C.CDLL(str(so))
        lib.ref_dot_ogita_f64.argtypes = [I64, P, P]
        lib.ref_dot_ogita_f64.restype = D
        lib.ref_dot_naive_f64.argtypes = [I64, P, P]
        lib.ref_dot_naive_f64.restype = D
        lib.ref_dot_ogita_f32.argtypes = [I64, P, P]
        lib.ref_dot_ogita_f32.restype = C.c_float
        for name in ("ref_dot_ogita_c128", "ref_dot_ogita_c64", "ref_dot_naive_c128"):
            getattr(lib, name).argtypes = [I64, P, P, P]
        lib.ref_threaded_dot_f64.argtypes = [I64, P, P, C.c_int, C.c_int]
        lib.ref_threaded_dot_f64.restype = D
        lib.ref_threaded_dot_f32.argtypes = [I64, P, P, C.c_int, C.c_int]
        lib.ref_threaded_dot_f32.restype = C.c_float
        lib.ref_threaded_sum_f64.argtypes = [I64, P, C.c_int, C.c_int, C.c_int]
        lib.ref_threaded_sum_f64.restype = D
        lib.ref_threaded_dot_f64_loop.argtypes = [I64, P, P, C.c_int, C.c_int]
        lib.ref_threaded_dot_f64_loop.restype = D
        for name in ("ref_bounds_dot_real_f64", "ref_bounds_dot_complex_f64", "ref_bounds_sum_real_f64"):
            getattr(lib, name).argtypes = [I64, D, I64, P]
        _REF = lib
    return _REF


_REF_SOLVER = None


def ref_solver():
    """The reference's own CPU Krylov solvers (oracle/_ref), or None."""
    global _REF_SOLVER
    if _REF_SOLVER is None:
        so = HERE / "_ref" / "libhpb_ref_solver.so"
        if not so.exists():
            return None
        lib = C.CDLL(str(so))
        lib.ref_cpu_solve_f64.argtypes = [C.c_int, C.c_int, P, P, P, P, P, C.c_int, D, C.c_int, C.c_int, C.c_int,
                                          C.POINTER(C.c_int), PD, PD]
        lib.ref_cpu_solve_f64.restype = C.c_int
        if hasattr(lib, "ref_cpu_solve_hist_f64"):
            lib.ref_cpu_solve_hist_f64.argtypes = [C.c_int, C.c_int, P, P, P, P, P, C.c_int, D, C.c_int, C.c_int,
                                                   C.c_int, C.POINTER(C.c_int), PD, PD, P, C.c_int,
                                                   C.POINTER(C.c_int)]
            lib.ref_cpu_solve_hist_f64.restype = C.c_int
        _REF_SOLVER = lib
    return _REF_SOLVER


def ref_cpu_solve(method: int, A, b: np.ndarray, x0: np.ndarray, basis: int, rel_tol: float, max_iters: int,
                  high_prec: int = 1, threads: int = -1):
    """Run the reference's bicgstabl (method 0) / gmres (method 1) on the CPU.
    Returns (converged, iters, monitor residual norm, seconds, x)."""
    lib = ref_solver()
    if lib is None:
        return None
    x = np.ascontiguousarray(x0, dtype=np.float64).copy()
    bb = np.ascontiguousarray(b, dtype=np.float64).copy()
    it = C.c_int()
    res = C.c_double()
    sec = C.c_double()
    ok = lib.ref_cpu_solve_f64(method, A.n, _ptr(A.row_ptr), _ptr(A.col_ind), _ptr(A.val), _ptr(bb), _ptr(x), basis,
                               rel_tol, max_iters, high_prec, threads, C.byref(it), C.byref(res), C.byref(sec))
    return bool(ok), it.value, res.value, sec.value, x


def ref_cpu_solve_history(method: int, A, b: np.ndarray, x0: np.ndarray, basis: int, rel_tol: float,
                          max_iters: int, high_prec: int = 1, threads: int = -1):
    """As ref_cpu_solve, plus the reference monitor's convergence history:
    returns (converged, iters, residual, seconds, x, history) with history an
    (k, 2) array of (iteration, ||r||) pairs, one per monitor check."""
    lib = ref_solver()
    if lib is None or not hasattr(lib, "ref_cpu_solve_hist_f64"):
        return None
    x = np.ascontiguousarray(x0, dtype=np.float64).copy()
    bb = np.ascontiguousarray(b, dtype=np.float64).copy()
    it = C.c_int()
    res = C.c_double()
    sec = C.c_double()
    cap = max_iters + 2
    hist = np.zeros(2 * cap)
    hl = C.c_int()
    ok = lib.ref_cpu_solve_hist_f64(method, A.n, _ptr(A.row_ptr), _ptr(A.col_ind), _ptr(A.val), _ptr(bb), _ptr(x),
                                    basis, rel_tol, max_iters, high_prec, threads, C.byref(it), C.byref(res),
                                    C.byref(sec), _ptr(hist), cap, C.byref(hl))
    return bool(ok), it.value, res.value, sec.value, x, hist[:2 * hl.value].reshape(-1, 2)


# ----------------------------------------------------------------- helpers
def exact_dot(x: np.ndarray, y: np.ndarray) -> tuple:
    """Exact sum conj(x_i) y_i as (hi, lo) (real) or (hi, lo) complex pairs."""
    lib = oro()
    n = x.shape[0]
    if x.dtype == np.float64:
        out = np.zeros(2)
        lib.oro_exact_dot_f64(n, _ptr(x), _ptr(y), _ptr(out))
        return out[0], out[1]
    if x.dtype == np.float32:
        out = np.zeros(2)
        lib.oro_exact_dot_f32(n, _ptr(x), _ptr(y), _ptr(out))
        return out[0], out[1]
    out = np.zeros(4)
    if x.dtype == np.complex128:
        lib.oro_exact_dot_c128(n, _ptr(x), _ptr(y), _ptr(out))
    else:
        lib.oro_exact_dot_c64(n, _ptr(x), _ptr(y), _ptr(out))
    return complex(out[0], out[1]), complex(out[2], out[3])


def exact_sum(x: np.ndarray, absolute: bool = False) -> tuple:
    lib = oro()
    n = x.shape[0]
    ncomp = 2 if np.iscomplexobj(x) else 1
    out = np.zeros(4)
    if x.dtype in (np.float64, np.complex128):
        lib.oro_exact_sum_f64(n, _ptr(x), ncomp, 1 if absolute else 0, _ptr(out))
    else:
        lib.oro_exact_sum_f32(n, _ptr(x), ncomp, 1 if absolute else 0, _ptr(out))
    if ncomp == 2 and not absolute:
        return complex(out[0], out[1]), complex(out[2], out[3])
    return out[0], out[1]


def exact_sumsq(x: np.ndarray) -> tuple:
    lib = oro()
    xd = np.ascontiguousarray(x.astype(np.complex128 if np.iscomplexobj(x) else np.float64))
    out = np.zeros(2)
    lib.oro_exact_sumsq_f64(x.shape[0], _ptr(xd), 2 if np.iscomplexobj(x) else 1, _ptr(out))
    return out[0], out[1]


def condition_dot(x: np.ndarray, y: np.ndarray) -> float:
    """cond = sum|x_i y_i| / |sum x_i y_i| (real float64 inputs), exactly."""
    lib = oro()
    a = np.zeros(2)
    lib.oro_exact_absdot_f64(x.shape[0], _ptr(x), _ptr(y), _ptr(a))
    hi, _ = exact_dot(x, y)
    return float("inf") if hi == 0 else a[0] / abs(hi)


def dot2_seq(x: np.ndarray, y: np.ndarray):
    """The reference's sequential Dot2 restated (dot_product<T>::dot_ogita)."""
    lib = oro()
    n = x.shape[0]
    if x.dtype == np.float64:
        out = np.zeros(3)
        lib.oro_dot2_seq_f64(n, _ptr(x), _ptr(y), _ptr(out))
        return out[0]
    if x.dtype == np.float32:
        out = np.zeros(3)
        lib.oro_dot2_seq_f32(n, _ptr(x), _ptr(y), _ptr(out))
        return np.float32(out[0])
    out = np.zeros(6)
    if x.dtype == np.complex128:
        lib.oro_dot2_seq_c128(n, _ptr(x), _ptr(y), _ptr(out))
        return complex(out[0], out[1])
    lib.oro_dot2_seq_c64(n, _ptr(x), _ptr(y), _ptr(out))
    return np.complex64(complex(out[0], out[1]))


def dot2_threaded(x: np.ndarray, y: np.ndarray, parts: int) -> float:
    out = np.zeros(1)
    oro().oro_dot2_threaded_f64(x.shape[0], _ptr(x), _ptr(y), parts, _ptr(out))
    return out[0]


def sum2_seq(x: np.ndarray, absolute: bool = False):
    lib = oro()
    out = np.zeros(3)
    if x.dtype == np.float64:
        lib.oro_sum2_seq_f64(x.shape[0], _ptr(x), 1 if absolute else 0, _ptr(out))
        return out[0]
    lib.oro_sum2_seq_f32(x.shape[0], _ptr(x), 1 if absolute else 0, _ptr(out))
    return np.float32(out[0])


def bound_dot2(n: int, cond: float, complex_: bool = False, eps: float = 2.0 ** -52) -> float:
    """Relative a priori bound of compensated Dot2 (error_bounds.hpp)."""
    lib = oro()
    if complex_:
        return lib.oro_bound_dot2_complex(float(n), float(cond), eps)
    return lib.oro_bound_dot2_real(float(n), float(cond), eps)


def bound_sum2(n: int, cond: float, eps: float = 2.0 ** -52) -> float:
    return oro().oro_bound_sum2(float(max(n, 2)), float(cond), eps)


_TRI_SUFFIX = {np.dtype(np.float32): "f32", np.dtype(np.float64): "f64", np.dtype(np.complex64): "c64",
               np.dtype(np.complex128): "c128"}


def csr_trsv(row_ptr: np.ndarray, col_ind: np.ndarray, val: np.ndarray, b: np.ndarray, upper: bool, unit: bool,
             alpha=1.0) -> np.ndarray:
    """x = T^-1 (alpha b) for the lower (upper=False) or upper triangle of a
    CSR matrix, by forward / backward substitution (oracle/tri.c)."""
    suf = _TRI_SUFFIX[val.dtype]
    rp = np.ascontiguousarray(row_ptr, dtype=np.int32)
    ci = np.ascontiguousarray(col_ind, dtype=np.int32)
    v = np.ascontiguousarray(val)
    bb = np.ascontiguousarray(b, dtype=val.dtype)
    x = np.zeros_like(bb)
    a = np.array([alpha], dtype=val.dtype)
    st = getattr(oro(), "oro_csr_trsv_" + suf)(len(rp) - 1, _ptr(rp), _ptr(ci), _ptr(v), int(upper), int(unit),
                                               _ptr(a), _ptr(bb), _ptr(x))
    if st != 0:
        raise ValueError("a row stores no diagonal")
    return x


def csr_ilu0(row_ptr: np.ndarray, col_ind: np.ndarray, val: np.ndarray):
    """ILU(0) factors on A's pattern (L unit lower, U upper, stored in one
    array like the input), and the first zero-pivot row (-1 if none)."""
    suf = _TRI_SUFFIX[val.dtype]
    rp = np.ascontiguousarray(row_ptr, dtype=np.int32)
    ci = np.ascontiguousarray(col_ind, dtype=np.int32)
    lu = np.array(val, copy=True)
    r = getattr(oro(), "oro_csr_ilu0_" + suf)(len(rp) - 1, _ptr(rp), _ptr(ci), _ptr(lu))
    if r == -2:
        raise ValueError("a row stores no diagonal")
    return lu, int(r)


def gendot_dev(seed: int, n: int, cond: float):
    """The device GenDot generator restated on the CPU: (x, y, N_fix)."""
    x = np.zeros(n)
    y = np.zeros(n)
    nfix = oro().oro_gendot_dev_f64(seed, n, cond, _ptr(x), _ptr(y))
    return x, y, int(nfix)


def csr_trsv_sweeps(row_ptr, col_ind, val, b, upper: bool, unit: bool, sweeps: int, alpha=1.0) -> np.ndarray:
    """Jacobi-sweep approximation of T^-1 (alpha b) (oracle/tri.c)."""
    suf = _TRI_SUFFIX[val.dtype]
    rp = np.ascontiguousarray(row_ptr, dtype=np.int32)
    ci = np.ascontiguousarray(col_ind, dtype=np.int32)
    v = np.ascontiguousarray(val)
    bb = np.ascontiguousarray(b, dtype=val.dtype)
    x = np.zeros_like(bb)
    tmp = np.zeros_like(bb)
    a = np.array([alpha], dtype=val.dtype)
    st = getattr(oro(), "oro_csr_trsv_sweeps_" + suf)(len(rp) - 1, _ptr(rp), _ptr(ci), _ptr(v), int(upper),
                                                      int(unit), _ptr(a), _ptr(bb), int(sweeps), _ptr(x), _ptr(tmp))
    if st != 0:
        raise ValueError("a row stores no diagonal")
    return x


def shard_merge(parts, is_complex: bool) -> np.ndarray:
    """Merge of per-rank (hi, lo) reduction results in rank order (the
    sharded reductions' combine), restated in plain Python binary64: per
    real component s = TwoSum(s, hi_k, t), c = c + (t + lo_k), then
    (hi, lo) = TwoSum(s, c) -- the (value, error) recurrence of the
    reference's compensated pass, common/ogita/gpu_reduction_ogita_impl.cuh:
    274-276.  parts: count x 2 (real) or count x 4 (complex: hi.re, hi.im,
    lo.re, lo.im)."""
    comps = 2 if is_complex else 1
    a = [float(v) for v in np.asarray(parts, dtype=np.float64).reshape(-1)]

    def two_sum(x, y):
        s = x + y
        bv = s - x
        av = s - bv
        return s, (y - bv) + (x - av)

    out = np.zeros(2 * comps)
    for q in range(comps):
        s = c = 0.0
        for k in range(len(a) // (2 * comps)):
            s, t = two_sum(s, a[k * 2 * comps + q])
            c = c + (t + a[k * 2 * comps + comps + q])
        hi, lo = two_sum(s, c)
        out[q], out[comps + q] = hi, lo
    return out
