"""GPU parity of the elementwise BLAS-1 kernels (through the C ABI) against a
plain numpy float64/complex128 restatement of the same formula.
Tolerance: |gpu - ref| <= 8 eps(type) * (sum of |terms|) per entry."""
import numpy as np
import pytest

from gpu_utils import EPS, dev, host
from high_precision_blas1_b200 import _lib

pytestmark = pytest.mark.gpu

DT = {"f32": np.float32, "f64": np.float64, "c64": np.complex64, "c128": np.complex128}
WIDE = {"f32": np.float64, "f64": np.float64, "c64": np.complex128, "c128": np.complex128}


def rnd(rng, t, n):
    if t.startswith("c"):
        return (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(DT[t])
    return rng.standard_normal(n).astype(DT[t])


def coef(rng, t):
    v = complex(rng.standard_normal(), rng.standard_normal()) if t.startswith("c") else float(rng.standard_normal())
    return v


def close(got, want, scale, t):
    return np.all(np.abs(got.astype(WIDE[t]) - want) <= 8 * EPS[t] * scale + 1e-300)


@pytest.mark.parametrize("t", ["f32", "f64", "c64", "c128"])
@pytest.mark.parametrize("n", [0, 1, 3, 1025, 300007])
def test_axpy_family(gpu, t, n):
    ctx, torch = gpu
    L = _lib.lib
    rng = np.random.default_rng(n + 7)
    x, y, z, w, v = (rnd(rng, t, n) for _ in range(5))
    a, b, c, d = (coef(rng, t) for _ in range(4))
    S = lambda q: _lib.scalar(t, q)  # noqa: E731
    W = lambda q: q.astype(WIDE[t])  # noqa: E731
    cases = [
        ("axpy", lambda X, Y, Z, Wd, V: getattr(L, f"hpb_axpy_{t}")(ctx.h, n, S(a), X, Y), "y",
         a * W(x) + W(y), abs(a) * np.abs(W(x)) + np.abs(W(y))),
        ("axpby", lambda X, Y, Z, Wd, V: getattr(L, f"hpb_axpby_{t}")(ctx.h, n, S(a), X, S(b), Y), "y",
         a * W(x) + b * W(y), abs(a) * np.abs(W(x)) + abs(b) * np.abs(W(y))),
        ("lincomb2", lambda X, Y, Z, Wd, V: getattr(L, f"hpb_lincomb2_{t}")(ctx.h, n, S(a), X, S(b), Y, Z), "z",
         a * W(x) + b * W(y), abs(a) * np.abs(W(x)) + abs(b) * np.abs(W(y))),
        ("axpbypcz", lambda X, Y, Z, Wd, V: getattr(L, f"hpb_axpbypcz_{t}")(ctx.h, n, S(a), X, S(b), Y, S(c), Z),
         "z", a * W(x) + b * W(y) + c * W(z), abs(a) * np.abs(W(x)) + abs(b) * np.abs(W(y)) + abs(c) * np.abs(W(z))),
        ("axpbypcwpdz",
         lambda X, Y, Z, Wd, V: getattr(L, f"hpb_axpbypcwpdz_{t}")(ctx.h, n, S(a), X, S(b), Y, S(c), Wd, S(d), Z),
         "z", a * W(x) + b * W(y) + c * W(w) + d * W(z),
         abs(a) * np.abs(W(x)) + abs(b) * np.abs(W(y)) + abs(c) * np.abs(W(w)) + abs(d) * np.abs(W(z))),
        ("lincomb4",
         lambda X, Y, Z, Wd, V: getattr(L, f"hpb_lincomb4_{t}")(ctx.h, n, S(a), X, S(b), Y, S(c), V, S(d), Wd, Z),
         "z", a * W(x) + b * W(y) + c * W(v) + d * W(w),
         abs(a) * np.abs(W(x)) + abs(b) * np.abs(W(y)) + abs(c) * np.abs(W(v)) + abs(d) * np.abs(W(w))),
        ("scal", lambda X, Y, Z, Wd, V: getattr(L, f"hpb_scal_{t}")(ctx.h, n, S(a), X, Z), "z", a * W(x),
         abs(a) * np.abs(W(x))),
        ("add_scalar", lambda X, Y, Z, Wd, V: getattr(L, f"hpb_add_scalar_{t}")(ctx.h, n, S(b), S(a), Z), "z",
         a * W(z) + b, abs(a) * np.abs(W(z)) + abs(b)),
        ("fill", lambda X, Y, Z, Wd, V: getattr(L, f"hpb_fill_{t}")(ctx.h, n, S(a), Z), "z",
         np.full(n, a, dtype=WIDE[t]), np.full(n, abs(a))),
        ("mul_pointwise", lambda X, Y, Z, Wd, V: getattr(L, f"hpb_mul_pointwise_{t}")(ctx.h, n, S(a), X, S(b), Y, Z),
         "z", (a * W(x)) * (b * W(y)), np.abs(a * W(x)) * np.abs(b * W(y)) * 2),
        ("div_pointwise", lambda X, Y, Z, Wd, V: getattr(L, f"hpb_div_pointwise_{t}")(ctx.h, n, S(a), X, S(b), Y, Z),
         "z", (a * W(x)) / (b * W(y)), np.abs((a * W(x)) / (b * W(y))) * 4),
    ]
    for name, call, out, want, scale in cases:
        X, Y, Z, Wd, V = (dev(torch, q) for q in (x, y, z, w, v))
        ctx.check(call(X.data_ptr(), Y.data_ptr(), Z.data_ptr(), Wd.data_ptr(), V.data_ptr()), name)
        torch.cuda.synchronize()
        got = host({"y": Y, "z": Z}[out])
        assert close(got, want, scale, t), (name, t, n)


@pytest.mark.parametrize("t", ["f32", "f64", "c64", "c128"])
def test_unaligned_pointers_use_scalar_path(gpu, t):
    """Pointers aligned to the real component but not to 16 bytes."""
    ctx, torch = gpu
    rng = np.random.default_rng(2)
    n = 1001
    real = np.float32 if t in ("f32", "c64") else np.float64
    k = 2 if t.startswith("c") else 1
    xr = rng.standard_normal(k * n + 1).astype(real)
    yr = rng.standard_normal(k * n + 1).astype(real)
    X, Y = dev(torch, xr), dev(torch, yr)
    off = np.dtype(real).itemsize  # one real component
    a = coef(rng, t)
    ctx.check(getattr(_lib.lib, f"hpb_axpy_{t}")(ctx.h, n, _lib.scalar(t, a), X.data_ptr() + off,
                                                  Y.data_ptr() + off))
    torch.cuda.synchronize()
    x = xr[1:].view(DT[t])
    y = yr[1:].view(DT[t])
    want = a * x.astype(WIDE[t]) + y.astype(WIDE[t])
    got = host(Y)[1:].view(DT[t])
    assert close(got, want, np.abs(a) * np.abs(x.astype(WIDE[t])) + np.abs(y.astype(WIDE[t])), t)


@pytest.mark.parametrize("t", ["f32", "f64", "c64", "c128"])
def test_abs_copy_swap_isfinite_random(gpu, t):
    ctx, torch = gpu
    L = _lib.lib
    rng = np.random.default_rng(9)
    n = 4099
    x, y = rnd(rng, t, n), rnd(rng, t, n)
    X, Y = dev(torch, x), dev(torch, y)
    # abs: complex -> |re| + |im|
    Z = dev(torch, np.zeros_like(x))
    ctx.check(getattr(L, f"hpb_abs_{t}")(ctx.h, n, X.data_ptr(), Z.data_ptr()))
    torch.cuda.synchronize()
    want = (np.abs(x.real) + np.abs(x.imag)) if t.startswith("c") else np.abs(x)
    assert np.allclose(host(Z).real, want, rtol=4 * EPS[t]) and np.all(host(Z).imag == 0)
    # copy / swap
    ctx.check(L.hpb_copy(ctx.h, n, x.itemsize, X.data_ptr(), Z.data_ptr()))
    ctx.check(L.hpb_swap(ctx.h, n, x.itemsize, Z.data_ptr(), Y.data_ptr()))
    torch.cuda.synchronize()
    assert np.array_equal(host(Y), x) and np.array_equal(host(Z), y)
    # isfinite (complex: isfinite(re + im), the reference's test)
    import ctypes as C
    r = C.c_int(-1)
    ctx.check(getattr(L, f"hpb_isfinite_{t}")(ctx.h, n, X.data_ptr(), C.byref(r)))
    assert r.value == 1
    for bad in (np.nan, np.inf, -np.inf):
        xb = x.copy()
        xb[n // 2] = bad
        ctx.check(getattr(L, f"hpb_isfinite_{t}")(ctx.h, n, dev(torch, xb).data_ptr(), C.byref(r)))
        assert r.value == 0
    ctx.check(getattr(L, f"hpb_isfinite_{t}")(ctx.h, 0, X.data_ptr(), C.byref(r)))
    assert r.value == 1
    # seeded random fill in [a, b)
    a, b = (complex(-1, 2), complex(3, 5)) if t.startswith("c") else (-2.0, 3.0)
    R1, R2 = dev(torch, np.zeros_like(x)), dev(torch, np.zeros_like(x))
    ctx.check(getattr(L, f"hpb_random_{t}")(ctx.h, n, 42, _lib.scalar(t, a), _lib.scalar(t, b), R1.data_ptr()))
    ctx.check(getattr(L, f"hpb_random_{t}")(ctx.h, n, 42, _lib.scalar(t, a), _lib.scalar(t, b), R2.data_ptr()))
    torch.cuda.synchronize()
    r1 = host(R1)
    assert np.array_equal(r1, host(R2))
    assert np.all(r1.real >= np.real(a)) and np.all(r1.real <= np.real(b))
    if t.startswith("c"):
        assert np.all(r1.imag >= np.imag(a)) and np.all(r1.imag <= np.imag(b))
    assert abs(np.mean(r1.real) - (np.real(a) + np.real(b)) / 2) < 0.1
