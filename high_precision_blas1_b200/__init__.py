"""B200-native compensated BLAS-1 (Ogita-Rump-Oishi Sum2/Dot2, axpy family,
CSR SpMV) behind a C ABI (include/hpblas1.h), with a C++ drop-in of the
reference's gpu_vector_operations / csr::gpu_matrix / csr::linear_operator
interface (include/hpblas1_dropin/).

This Python package holds the build script, a ctypes binding used by the
tests and the benchmark, and the seeded input generators.  It carries no
compute path of its own: every operation runs in libhpblas1.so.
"""
from __future__ import annotations

__all__ = ["load", "Context"]


def load():
    """Import the ctypes binding (raises if libhpblas1.so is missing)."""
    from . import _lib
    return _lib


class Context:
    """RAII wrapper of an hpb_context bound to a CUDA stream (integer handle)."""

    def __init__(self, device: int = 0, stream: int | None = None):
        import ctypes as C
        self._lib = load()
        self.h = C.c_void_p()
        st = self._lib.lib.hpb_create(C.byref(self.h), device, stream)
        if st != 0:
            raise self._lib.HpbError(st, "hpb_create failed")

    @property
    def handle(self):
        return self.h

    def check(self, status: int, what: str = ""):
        if status != 0:
            msg = self._lib.lib.hpb_last_error(self.h).decode(errors="replace")
            raise self._lib.HpbError(status, f"{what}: {msg}")

    def close(self):
        if self.h:
            self._lib.lib.hpb_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
