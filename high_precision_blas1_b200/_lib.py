"""ctypes binding of libhpblas1.so (the C ABI declared in include/hpblas1.h).

The library is built in-tree by ``high_precision_blas1_b200.build``.  There
is no fallback: if the shared object is missing or fails to load, importing
this module raises, so no caller can silently run without the CUDA kernels.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libhpblas1.so"

TYPES = ("f32", "f64", "c64", "c128")


class hpb_c64(C.Structure):
    _fields_ = [("re", C.c_float), ("im", C.c_float)]


class hpb_c128(C.Structure):
    _fields_ = [("re", C.c_double), ("im", C.c_double)]


SCALAR = {"f32": C.c_float, "f64": C.c_double, "c64": hpb_c64, "c128": hpb_c128}

STATUS = {
    0: "HPB_SUCCESS",
    -1: "HPB_ERROR_INVALID_VALUE",
    -2: "HPB_ERROR_CUDA",
    -3: "HPB_ERROR_OUT_OF_MEMORY",
    -4: "HPB_ERROR_NOT_SUPPORTED",
    -5: "HPB_ERROR_BREAKDOWN",
    -6: "HPB_ERROR_NOT_FINITE",
    -7: "HPB_ERROR_NOT_CONVERGED",
    -8: "HPB_ERROR_SIZE_LIMIT",
    -9: "HPB_ERROR_TIMEOUT",
}


class HpbError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class _TypedCDLL(C.CDLL):
    """CDLL that only hands out the functions declared below (with their
    argtypes).  A plain CDLL creates a fresh, untyped function object when
    __getattr__ is called directly, which would pass 64-bit device pointers
    as 32-bit ints; here an undeclared name raises instead."""

    def __getattr__(self, name):
        d = self.__dict__
        if name in d:  # a direct __getattr__ call returns the typed function too
            return d[name]
        if name.startswith("hpb_") and "_declared" in d:
            raise AttributeError(f"{name} is not declared in high_precision_blas1_b200/_lib.py")
        return super().__getattr__(name)


def _load() -> C.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m high_precision_blas1_b200.build` "
            "(there is no CPU fallback)")
    return _TypedCDLL(str(LIB_PATH))


lib = _load()

P = C.c_void_p
I64 = C.c_int64
I32 = C.c_int32


def _sig(name, res, args):
    f = C.CDLL.__getattr__(lib, name)
    f.restype = res
    f.argtypes = args
    lib.__dict__.setdefault("_declared", set()).add(name)
    lib.__dict__[name] = f
    return f


# context / errors
_sig("hpb_create", C.c_int, [C.POINTER(P), C.c_int, P])
_sig("hpb_destroy", C.c_int, [P])
_sig("hpb_set_stream", C.c_int, [P, P])
_sig("hpb_get_stream", P, [P])
_sig("hpb_synchronize", C.c_int, [P])
_sig("hpb_status_string", C.c_char_p, [C.c_int])
_sig("hpb_last_error", C.c_char_p, [P])
_sig("hpb_version", C.c_int, [C.POINTER(C.c_int)] * 3)
_sig("hpb_launch_count", C.c_uint64, [])
_sig("hpb_shard_merge", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p])
_sig("hpb_shard_merge_cpu", C.c_int, [C.c_int, C.c_int, C.c_void_p, C.c_void_p])

# reductions
for t in TYPES:
    for op in ("dot2", "dot"):
        _sig(f"hpb_{op}_{t}", C.c_int, [P, I64, P, P, P])
        _sig(f"hpb_{op}_{t}_host", C.c_int, [P, I64, P, P, P])
    for op in ("sum2", "asum2", "nrm2", "asum", "nrm2plain"):
        _sig(f"hpb_{op}_{t}", C.c_int, [P, I64, P, P])
        _sig(f"hpb_{op}_{t}_host", C.c_int, [P, I64, P, P])

_sig("hpb_dot2_f64_noalloc", C.c_int, [I64, P, P, P, P])
NOALLOC_MAX_N = 16777216

# elementwise
for t in TYPES:
    S = SCALAR[t]
    _sig(f"hpb_axpy_{t}", C.c_int, [P, I64, S, P, P])
    _sig(f"hpb_axpby_{t}", C.c_int, [P, I64, S, P, S, P])
    _sig(f"hpb_lincomb2_{t}", C.c_int, [P, I64, S, P, S, P, P])
    _sig(f"hpb_axpbypcz_{t}", C.c_int, [P, I64, S, P, S, P, S, P])
    _sig(f"hpb_axpbypcwpdz_{t}", C.c_int, [P, I64, S, P, S, P, S, P, S, P])
    _sig(f"hpb_lincomb4_{t}", C.c_int, [P, I64, S, P, S, P, S, P, S, P, P])
    _sig(f"hpb_scal_{t}", C.c_int, [P, I64, S, P, P])
    _sig(f"hpb_add_scalar_{t}", C.c_int, [P, I64, S, S, P])
    _sig(f"hpb_fill_{t}", C.c_int, [P, I64, S, P])
    _sig(f"hpb_mul_pointwise_{t}", C.c_int, [P, I64, S, P, S, P, P])
    _sig(f"hpb_div_pointwise_{t}", C.c_int, [P, I64, S, P, S, P, P])
    _sig(f"hpb_abs_{t}", C.c_int, [P, I64, P, P])
    _sig(f"hpb_isfinite_{t}", C.c_int, [P, I64, P, C.POINTER(C.c_int)])
    _sig(f"hpb_csr_spmv_{t}", C.c_int, [P, I32, I32, I64, P, P, P, S, P, S, P])
    _sig(f"hpb_csr_spmv_dot2_{t}", C.c_int, [P, I32, I32, I64, P, P, P, P, P, P, P])
    _sig(f"hpb_csr_diag_{t}", C.c_int, [P, I32, P, P, P, P])
    _sig(f"hpb_random_{t}", C.c_int, [P, I64, C.c_uint64, S, S, P])
# Matrix Market reader (host)
class hpb_mm_csr(C.Structure):
    _fields_ = [("rows", C.c_int32), ("cols", C.c_int32), ("nnz", C.c_int64), ("is_complex", C.c_int),
                ("symmetric", C.c_int), ("row_ptr", C.POINTER(C.c_int32)), ("col_ind", C.POINTER(C.c_int32)),
                ("val", C.POINTER(C.c_double))]


_sig("hpb_mm_read_csr", C.c_int, [C.c_char_p, C.POINTER(hpb_mm_csr)])
_sig("hpb_mm_free", None, [C.POINTER(hpb_mm_csr)])
_sig("hpb_mm_last_error", C.c_char_p, [])

_sig("hpb_csr_transpose_pattern", C.c_int, [P, I32, I32, I64, P, P, P, P, P])
for t in TYPES:
    _sig(f"hpb_gather_{t}", C.c_int, [P, I64, P, P, P])

# sparse triangular solves and ILU(0)
_sig("hpb_csr_tri_create", C.c_int, [P, C.c_int, I32, I64, P, P, C.POINTER(P)])
_sig("hpb_csr_tri_destroy", C.c_int, [P])
_sig("hpb_csr_tri_info", C.c_int, [P, C.POINTER(I32), C.POINTER(I32), C.POINTER(I64), C.POINTER(C.c_int)])
_sig("hpb_csr_tri_check", C.c_int, [P, P])
_sig("hpb_csr_tri_set_wait_limit", C.c_int, [P, C.c_uint64])
_sig("hpb_csr_tri_test_withhold_row", C.c_int, [P, I32])
for t in TYPES:
    _sig(f"hpb_csr_trsv_{t}", C.c_int, [P, P, C.c_int, P, SCALAR[t], P, P])
    _sig(f"hpb_csr_ilu0_{t}", C.c_int, [P, P, P])
    _sig(f"hpb_csr_trsv_sweeps_{t}", C.c_int, [P, P, C.c_int, P, SCALAR[t], P, P, C.c_int])
_sig("hpb_gendot_f64", C.c_int, [C.c_uint64, I64, C.c_double, P, P, C.POINTER(C.c_int64)])
_sig("hpb_gendot_c128", C.c_int, [C.c_uint64, I64, C.c_double, P, P])
_sig("hpb_gendot_f64_dev", C.c_int, [P, C.c_uint64, I64, C.c_double, P, P, C.POINTER(C.c_int64)])
_sig("hpb_gendot_c128_dev", C.c_int, [P, C.c_uint64, I64, C.c_double, P, P])
_sig("hpb_copy", C.c_int, [P, I64, C.c_size_t, P, P])
_sig("hpb_swap", C.c_int, [P, I64, C.c_size_t, P, P])


class hpb_solver_params(C.Structure):
    _fields_ = [("method", C.c_int), ("basis", C.c_int), ("rel_tol", C.c_double), ("abs_tol", C.c_double),
                ("max_iters", C.c_int), ("precond", C.c_int), ("high_precision", C.c_int),
                ("resid_recalc_freq", C.c_int), ("early_exit", C.c_int), ("reorthogonalize", C.c_int),
                ("fused", C.c_int), ("ilu_sweeps", C.c_int)]


class hpb_solver_report(C.Structure):
    _fields_ = [("converged", C.c_int), ("iters", C.c_int), ("breakdown", C.c_int), ("history_len", C.c_int),
                ("rhs_norm", C.c_double), ("resid_norm", C.c_double), ("true_resid_norm", C.c_double),
                ("true_rhs_norm", C.c_double), ("seconds", C.c_double)]


SOLVER = {"bicgstabl": 0, "gmres": 1, "bicgstab": 2}
PRECOND = {"none": 0, "jacobi": 1, "matrix": 2, "ilu0": 3}


class hpb_ir_params(C.Structure):
    _fields_ = [("inner_method", C.c_int), ("inner_basis", C.c_int), ("inner_rel_tol", C.c_double),
                ("inner_max_iters", C.c_int), ("precond", C.c_int), ("rel_tol", C.c_double),
                ("max_refinements", C.c_int), ("ilu_sweeps", C.c_int)]


class hpb_ir_report(C.Structure):
    _fields_ = [("converged", C.c_int), ("refinements", C.c_int), ("inner_iters", C.c_int),
                ("history_len", C.c_int), ("rhs_norm", C.c_double), ("true_resid_norm", C.c_double),
                ("seconds", C.c_double)]

_sig("hpb_solver_params_default", C.c_int, [C.POINTER(hpb_solver_params)])
for t in TYPES:
    for suf in ("", "_host"):
        _sig(f"hpb_csr_solve_{t}{suf}", C.c_int,
             [C.POINTER(hpb_solver_params), I32, I64, P, P, P, P, P, C.POINTER(hpb_solver_report), P, C.c_int])


_sig("hpb_solver_memory_release", C.c_int, [])
_sig("hpb_ir_params_default", C.c_int, [C.POINTER(hpb_ir_params)])
for _n in ("hpb_ir_solve_f64", "hpb_ir_solve_c128"):
    _sig(_n, C.c_int, [C.POINTER(hpb_ir_params), I32, I64, P, P, P, P, P, P, P, I64, P, P,
                       C.POINTER(hpb_ir_report), P, C.c_int])


class hpb_spai_system(C.Structure):
    _fields_ = [("rows", C.c_int32), ("nnz", C.c_int64), ("row_ptr", P), ("col_ind", P), ("val", P),
                ("nres", C.c_int), ("residuals", P)]


_sig("hpb_spai_ls_f32", C.c_int, [P, I32, I64, P, P, P, P])
_sig("hpb_spai_ls_f64", C.c_int, [P, I32, I64, P, P, P, P])
_sig("hpb_spai_create", C.c_int, [C.POINTER(P), C.c_int, C.c_int, C.POINTER(C.c_int), C.c_uint64])
_sig("hpb_spai_destroy", C.c_int, [P])
_sig("hpb_spai_num_params", C.c_int, [])
_sig("hpb_spai_set_weights", C.c_int, [P, P])
_sig("hpb_spai_get_weights", C.c_int, [P, P])
_sig("hpb_spai_assemble", C.c_int, [P, C.POINTER(hpb_spai_system), P])
_sig("hpb_spai_loss_grad", C.c_int, [P, C.POINTER(hpb_spai_system), C.c_float, C.c_float, P, P])
_sig("hpb_spai_loss", C.c_int, [P, C.POINTER(hpb_spai_system), C.c_float, C.c_float, P])
_sig("hpb_spai_adam", C.c_int, [P, C.c_float, C.c_float])
_sig("hpb_spai_forward", C.c_int, [P, I32, P, P, C.c_int])


def ir_params(inner="gmres", basis=50, inner_rel_tol=1e-5, inner_max_iters=5000, precond="none", rel_tol=1e-10,
              max_refinements=30, ilu_sweeps=0):
    p = hpb_ir_params()
    lib.hpb_ir_params_default(C.byref(p))
    p.inner_method = SOLVER[inner]
    p.inner_basis = basis
    p.inner_rel_tol = inner_rel_tol
    p.inner_max_iters = inner_max_iters
    p.precond = PRECOND[precond]
    p.rel_tol = rel_tol
    p.max_refinements = max_refinements
    p.ilu_sweeps = ilu_sweeps
    return p


def solver_params(method="bicgstabl", basis=2, rel_tol=1e-10, abs_tol=0.0, max_iters=10000, precond="none",
                  high_precision=True, resid_recalc_freq=0, early_exit=False, reorthogonalize=False, fused=False,
                  ilu_sweeps=0):
    p = hpb_solver_params()
    lib.hpb_solver_params_default(C.byref(p))
    p.method = SOLVER[method]
    p.basis = basis
    p.rel_tol = rel_tol
    p.abs_tol = abs_tol
    p.max_iters = max_iters
    p.precond = PRECOND[precond]
    p.high_precision = 1 if high_precision else 0
    p.resid_recalc_freq = resid_recalc_freq
    p.early_exit = 1 if early_exit else 0
    p.reorthogonalize = 1 if reorthogonalize else 0
    p.fused = 1 if fused else 0
    p.ilu_sweeps = ilu_sweeps
    return p


def scalar(t: str, v):
    """Convert a Python number to the C scalar type of element type t."""
    if t in ("c64", "c128"):
        v = complex(v)
        return SCALAR[t](v.real, v.imag)
    return SCALAR[t](float(v))


def exported_symbols() -> list[str]:
    """Names declared in include/hpblas1.h (parsed from the header)."""
    import re
    hdr = Path(__file__).resolve().parent.parent / "include" / "hpblas1.h"
    txt = hdr.read_text()
    return sorted(set(re.findall(r"^\s*(?:int|void\*|void|const char\*|uint64_t)\s+(hpb_\w+)\s*\(", txt, re.M)))
