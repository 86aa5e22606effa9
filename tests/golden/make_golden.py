"""Generate the golden vectors in tests/golden/ (run in a container where the
reference sources are present, after `make -C oracle`).

For every case the inputs are seeded, and the expected outputs come from the
reference's OWN CPU code compiled from its sources (oracle/_ref, i.e.
dot_product<T>::dot_ogita, threaded_reduction<T>::dot/sum and
error_bounds<T>), plus the exact value from the oracle's fixed-point
accumulator.  The reference has no golden vectors or known-answer tests of
its own, so these fixtures pin both the oracle restatement and the GPU
kernels to the reference's arithmetic.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import ctypes as C
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from high_precision_blas1_b200 import _lib  # noqa: E402  (host-side generator only)

SIZES = [0, 1, 2, 3, 7, 31, 32, 33, 255, 256, 1000, 1023, 4097, 16384]


def gendot(seed: int, n: int, cond: float):
    x = np.zeros(n)
    y = np.zeros(n)
    nf = C.c_int64()
    st = _lib.lib.hpb_gendot_f64(seed, n, cond, x.ctypes.data, y.ctypes.data, C.byref(nf))
    assert st == 0
    return x, y


def real_cases(rng):
    cases = []
    for n in SIZES:
        x = rng.standard_normal(n) * np.exp2(rng.integers(-20, 20, n))
        y = rng.standard_normal(n)
        cases.append(("random", n, x, y))
    for n, cond in [(64, 1e8), (1000, 1e16), (4096, 1e20), (4096, 1e30), (16384, 1e25)]:
        x, y = gendot(1000 + n + int(np.log10(cond)), n, cond)
        cases.append((f"gendot{cond:.0e}", n, x, y))
    # exact cancellation: [a, -a] pairs -> exact dot 0 plus a tiny tail
    a = rng.standard_normal(500) * np.exp2(rng.integers(0, 40, 500))
    b = rng.standard_normal(500)
    x = np.concatenate([a, a, [1e-10]])
    y = np.concatenate([b, -b, [3.0]])
    cases.append(("cancel", x.size, x, y))
    return cases


def save(name, cases, extra):
    arrays = {}
    meta = []
    for i, (kind, n, x, y) in enumerate(cases):
        arrays[f"x__{i}"] = x
        arrays[f"y__{i}"] = y
        for k, v in extra(i, x, y).items():
            arrays[f"{k}__{i}"] = np.asarray(v)
        meta.append({"kind": kind, "n": int(n)})
    arrays["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(HERE / name, **arrays)
    print("wrote", name, len(cases), "cases")


def main():
    ref = oracle.ref()
    if ref is None:
        raise SystemExit("oracle/_ref/libhpb_ref.so missing: run `make -C oracle` with the reference sources present")
    rng = np.random.default_rng(20240601)
    P = lambda a: a.ctypes.data  # noqa: E731

    # ---- float64 Dot2 ------------------------------------------------------
    def ext_f64(i, x, y):
        n = x.size
        hi, lo = oracle.exact_dot(x, y)
        return {
            "ref_ogita": ref.ref_dot_ogita_f64(n, P(x), P(y)),
            "ref_naive": ref.ref_dot_naive_f64(n, P(x), P(y)),
            "ref_threaded1": ref.ref_threaded_dot_f64(n, P(x), P(y), 1, 1),
            "exact": [hi, lo],
            "cond": oracle.condition_dot(x, y) if n else 1.0,
        }
    save("dot2_f64.npz", real_cases(rng), ext_f64)

    # ---- float32 Dot2 ------------------------------------------------------
    cases32 = []
    for n in SIZES:
        x = (rng.standard_normal(n) * np.exp2(rng.integers(-10, 10, n))).astype(np.float32)
        y = rng.standard_normal(n).astype(np.float32)
        cases32.append(("random", n, x, y))
    # ill-conditioned float pairs: [a, -a] halves plus small terms
    a = (rng.standard_normal(2000) * np.exp2(rng.integers(0, 20, 2000))).astype(np.float32)
    b = rng.standard_normal(2000).astype(np.float32)
    t = rng.standard_normal(50).astype(np.float32)
    cases32.append(("cancel", 4050, np.concatenate([a, a, t]), np.concatenate([b, -b, t])))

    def ext_f32(i, x, y):
        n = x.size
        hi, lo = oracle.exact_dot(x, y)
        return {"ref_ogita": np.float32(ref.ref_dot_ogita_f32(n, P(x), P(y))), "exact": [hi, lo]}
    save("dot2_f32.npz", cases32, ext_f32)

    # ---- complex128 / complex64 Dot2 ---------------------------------------
    cases_c = []
    for n in SIZES:
        x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        y = (rng.standard_normal(n) + 1j * rng.standard_normal(n)) * np.exp2(rng.integers(-15, 15, n))
        cases_c.append(("random", n, x, y))
    for n, cond in [(2048, 1e16), (4096, 1e24)]:
        xr = np.zeros(2 * n)
        yr = np.zeros(2 * n)
        assert _lib.lib.hpb_gendot_c128(77 + n, n, cond, P(xr), P(yr)) == 0
        cases_c.append((f"gendot{cond:.0e}", n, xr.view(np.complex128), yr.view(np.complex128)))

    def ext_c128(i, x, y):
        n = x.size
        out = np.zeros(2)
        ref.ref_dot_ogita_c128(n, P(x), P(y), P(out))
        hi, lo = oracle.exact_dot(x, y)
        return {"ref_ogita": complex(out[0], out[1]), "exact": [hi, lo]}
    save("dot2_c128.npz", cases_c, ext_c128)

    cases_c64 = [(k, n, x.astype(np.complex64), y.astype(np.complex64)) for (k, n, x, y) in cases_c[:len(SIZES)]]

    def ext_c64(i, x, y):
        n = x.size
        out = np.zeros(2)
        ref.ref_dot_ogita_c64(n, P(x), P(y), P(out))
        hi, lo = oracle.exact_dot(x, y)
        return {"ref_ogita": complex(out[0], out[1]), "exact": [hi, lo]}
    save("dot2_c64.npz", cases_c64, ext_c64)

    # ---- float64 Sum2 / asum2 ----------------------------------------------
    cases_s = []
    for n in SIZES:
        x = rng.standard_normal(n) * np.exp2(rng.integers(-30, 30, n))
        cases_s.append(("random", n, x, x))
    a = rng.standard_normal(3000) * np.exp2(rng.integers(0, 50, 3000))
    cases_s.append(("cancel", 6001, np.concatenate([a, -a[::-1], [0.125]]), np.zeros(1)))

    def ext_sum(i, x, _y):
        n = x.size
        s_hi, s_lo = oracle.exact_sum(x)
        a_hi, a_lo = oracle.exact_sum(x, absolute=True)
        return {
            "ref_sum2": ref.ref_threaded_sum_f64(n, P(x), 1, 1, 0),
            "ref_asum2": ref.ref_threaded_sum_f64(n, P(x), 1, 1, 1),
            "exact_sum": [s_hi, s_lo],
            "exact_asum": [a_hi, a_lo],
        }
    save("sum2_f64.npz", cases_s, ext_sum)

    # ---- error bounds from the reference's error_bounds<double> -------------
    rows = []
    for n in (1, 1000, 1 << 20):
        for cond in (1.0, 1e8, 1e16, 1e20):
            o = np.zeros(4)
            ref.ref_bounds_dot_real_f64(n, cond, 512, P(o))
            oc = np.zeros(4)
            ref.ref_bounds_dot_complex_f64(n, cond, 512, P(oc))
            os_ = np.zeros(4)
            ref.ref_bounds_sum_real_f64(max(n, 2), cond, 512, P(os_))
            rows.append([n, cond, *o, *oc, *os_])
    np.save(HERE / "bounds_f64.npy", np.array(rows))
    print("wrote bounds_f64.npy")


if __name__ == "__main__":
    main()
