"""Helpers for the GPU tests: device buffers through torch, calls through
the C ABI (libhpblas1.so via ctypes)."""
import ctypes as C

import numpy as np

from high_precision_blas1_b200 import _lib

NP2T = {np.dtype(np.float32): "f32", np.dtype(np.float64): "f64",
        np.dtype(np.complex64): "c64", np.dtype(np.complex128): "c128"}
EPS = {"f32": 2.0 ** -23, "f64": 2.0 ** -52, "c64": 2.0 ** -23, "c128": 2.0 ** -52}


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda")


def host(t):
    return t.detach().cpu().numpy()


def red(ctx, op, x, y=None, n=None):
    """Run hpb_<op>_<type>_host on device tensors; returns the 4-double output."""
    t = NP2T[np.dtype(str(x.dtype).replace("torch.", ""))]
    n = x.numel() if n is None else n
    out = np.zeros(4)
    f = getattr(_lib.lib, f"hpb_{op}_{t}_host")
    if y is None:
        st = f(ctx.h, n, x.data_ptr(), out.ctypes.data)
    else:
        st = f(ctx.h, n, x.data_ptr(), y.data_ptr(), out.ctypes.data)
    ctx.check(st, f"hpb_{op}_{t}_host")
    return out


def red_ptr(ctx, op, t, n, xp, yp=None):
    out = np.zeros(4)
    f = getattr(_lib.lib, f"hpb_{op}_{t}_host")
    st = f(ctx.h, n, xp, out.ctypes.data) if yp is None else f(ctx.h, n, xp, yp, out.ctypes.data)
    ctx.check(st, f"hpb_{op}_{t}_host")
    return out


def ulp(v: float) -> float:
    v = abs(float(v))
    return np.spacing(v) if v > 0 else np.spacing(0.0)


def gendot(seed, n, cond):
    x = np.zeros(n)
    y = np.zeros(n)
    assert _lib.lib.hpb_gendot_f64(seed, n, cond, x.ctypes.data, y.ctypes.data, None) == 0
    return x, y
