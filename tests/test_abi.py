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


def _header_prototypes():
    h = (ROOT / "include" / "hpblas1.h").read_text()
    h = re.sub(r"/\*.*?\*/", " ", h, flags=re.S)
    h = re.sub(r"//[^\n]*", " ", h)
    h = re.sub(r"#[^\n]*", " ", h)
    h = re.sub(r"\s+", " ", h)
    out = {}
    for ret, name, args in re.findall(r"([A-Za-z_][\w\s\*]*?)\s*\b(hpb_\w+)\s*\(([^)]*)\)\s*;", h):
        ts = []
        for a in args.split(","):
            a = a.strip()
            if not a or a == "void":
                continue
            t = a if a.endswith("*") else re.sub(r"\b\w+$", "", a)
            ts.append(re.sub(r"\bconst\b", "", t).replace(" ", ""))
        out[name] = (re.sub(r"\bconst\b", "", ret).replace(" ", ""), ts)
    return out


def _c_kind(t: str):
    """(kind, bytes) of a C parameter or return type of the header."""
    if t.endswith("*"):
        return ("ptr", 8)
    return {"int": ("int", 4), "int32_t": ("int", 4), "int64_t": ("int", 8), "uint64_t": ("uint", 8),
            "size_t": ("uint", 8), "double": ("float", 8), "float": ("float", 4), "void": ("void", 0),
            "hpb_c64": ("struct", 8), "hpb_c128": ("struct", 16)}[t]


def _ctypes_kind(ct):
    if ct is None:
        return ("void", 0)
    if isinstance(ct, type) and issubclass(ct, (C._Pointer, C.c_void_p, C.c_char_p)):
        return ("ptr", 8)
    if isinstance(ct, type) and issubclass(ct, C.Structure):
        return ("struct", C.sizeof(ct))
    code = getattr(ct, "_type_", None)
    kinds = {"i": "int", "l": "int", "q": "int", "I": "uint", "L": "uint", "Q": "uint", "d": "float", "f": "float",
             "P": "ptr", "z": "ptr"}
    return (kinds[code], C.sizeof(ct))


def test_ctypes_declarations_match_the_header():
    """Every ctypes declaration in _lib.py has the prototype's arity and, per
    argument, its kind and width (a 32-bit int where the C side takes a
    64-bit pointer or size would corrupt the call)."""
    from high_precision_blas1_b200 import _lib
    protos = _header_prototypes()
    assert set(protos) == set(_lib.exported_symbols())
    bad = []
    for name, (ret, args) in protos.items():
        f = _lib.lib.__dict__.get(name)
        assert f is not None, name
        got = [_ctypes_kind(a) for a in (f.argtypes or [])]
        want = [_c_kind(a) for a in args]
        if got != want:
            bad.append((name, want, got))
        if _ctypes_kind(f.restype) != _c_kind(ret) and not (ret in ("char*", "void*") and
                                                             _ctypes_kind(f.restype)[0] == "ptr"):
            bad.append((name, "restype", ret, f.restype))
    assert not bad, bad[:5]
