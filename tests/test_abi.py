"""CPU tests of the C ABI: the library loads, exports every symbol that
include/hpblas1.h declares, and rejects bad arguments without touching a GPU."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent


def test_library_loads_and_exports_every_declared_symbol():
    from high_precision_blas1_b200 import _lib
    declared = _lib.exported_symbols()
    assert len(declared) > 100
    missing = [s for s in declared if not hasattr(_lib.lib, s)]
    assert not missing, missing
    # and nm agrees: each declared name is a defined dynamic symbol
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)], capture_output=True, text=True).stdout
    defined = set(re.findall(r"\s[TW]\s(hpb_\w+)", out))
    assert set(declared) <= defined, sorted(set(declared) - defined)


def test_no_undeclared_exports():
    """Every exported hpb_ symbol is declared in a public header."""
    from high_precision_blas1_b200 import _lib
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)], capture_output=True, text=True).stdout
    defined = set(re.findall(r"\s[TW]\s(hpb_\w+)", out))
    declared = set(_lib.exported_symbols())
    assert defined <= declared, sorted(defined - declared)


def test_status_strings_and_version():
    from high_precision_blas1_b200 import _lib
    assert _lib.lib.hpb_status_string(0) == b"HPB_SUCCESS"
    assert _lib.lib.hpb_status_string(-7) == b"HPB_ERROR_NOT_CONVERGED"
    a, b, c = C.c_int(), C.c_int(), C.c_int()
    assert _lib.lib.hpb_version(C.byref(a), C.byref(b), C.byref(c)) == 0
    assert (a.value, b.value) == (0, 1)


def test_null_context_is_rejected():
    from high_precision_blas1_b200 import _lib
    out = np.zeros(4)
    assert _lib.lib.hpb_dot2_f64(None, 10, None, None, out.ctypes.data) == -1
    assert _lib.lib.hpb_axpy_f64(None, 10, 1.0, None, None) == -1
    assert _lib.lib.hpb_csr_spmv_f64(None, 1, 1, 1, None, None, None, 1.0, None, 0.0, None) == -1
    assert _lib.lib.hpb_create(None, 0, None) == -1


def test_generator_rejects_bad_arguments():
    from high_precision_blas1_b200 import _lib
    x = np.zeros(4)
    assert _lib.lib.hpb_gendot_f64(1, -1, 1e10, x.ctypes.data, x.ctypes.data, None) == -1
    assert _lib.lib.hpb_gendot_f64(1, 4, 0.5, x.ctypes.data, x.ctypes.data, None) == -1


def test_generator_is_seeded_and_reaches_condition():
    import oracle
    from high_precision_blas1_b200 import _lib
    n = 20000
    a, b, c, d = (np.zeros(n) for _ in range(4))
    assert _lib.lib.hpb_gendot_f64(3, n, 1e20, a.ctypes.data, b.ctypes.data, None) == 0
    assert _lib.lib.hpb_gendot_f64(3, n, 1e20, c.ctypes.data, d.ctypes.data, None) == 0
    assert np.array_equal(a, c) and np.array_equal(b, d)
    cond = oracle.condition_dot(a, b)
    assert 1e18 < cond < 1e24
