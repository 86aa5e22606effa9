"""CPU tests of the oracle: the restatement is pinned bit for bit to the
reference's own CPU code through the committed golden vectors, and the exact
accumulator is checked against Python's exact rationals."""
from fractions import Fraction

import numpy as np
import pytest

import oracle
from conftest import load_golden, GOLDEN


def test_exact_dot_matches_fractions():
    rng = np.random.default_rng(5)
    for trial in range(300):
        n = int(rng.integers(0, 40))
        if trial % 3 == 0:  # full exponent range incl. subnormal products
            x = np.ldexp(rng.uniform(-1, 1, n), rng.integers(-1074, 900, n))
            y = np.ldexp(rng.uniform(-1, 1, n), rng.integers(-900, 100, n))
        else:
            x = rng.uniform(-1, 1, n) * np.exp2(rng.integers(-60, 60, n))
            y = rng.uniform(-1, 1, n) * np.exp2(rng.integers(-60, 60, n))
        ex = sum((Fraction(a) * Fraction(b) for a, b in zip(x, y)), Fraction(0))
        hi, lo = oracle.exact_dot(x, y)
        assert hi == float(ex)  # float(Fraction) rounds to nearest-even
        if hi != 0 and np.isfinite(hi):
            assert lo == float(ex - Fraction(hi))


def test_exact_dot_complex_matches_fractions():
    rng = np.random.default_rng(6)
    for _ in range(50):
        n = int(rng.integers(0, 30))
        x = (rng.standard_normal(n) + 1j * rng.standard_normal(n)) * np.exp2(rng.integers(-30, 30, n))
        y = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        re = sum((Fraction(a.real) * Fraction(b.real) + Fraction(a.imag) * Fraction(b.imag) for a, b in zip(x, y)),
                 Fraction(0))
        im = sum((Fraction(a.real) * Fraction(b.imag) - Fraction(a.imag) * Fraction(b.real) for a, b in zip(x, y)),
                 Fraction(0))
        hi, _ = oracle.exact_dot(x, y)
        assert hi.real == float(re) and hi.imag == float(im)


def test_exact_sum_matches_fractions():
    rng = np.random.default_rng(7)
    for _ in range(100):
        n = int(rng.integers(0, 60))
        x = rng.standard_normal(n) * np.exp2(rng.integers(-200, 200, n))
        hi, lo = oracle.exact_sum(x)
        ex = sum((Fraction(v) for v in x), Fraction(0))
        assert hi == float(ex)
        ahi, _ = oracle.exact_sum(x, absolute=True)
        assert ahi == float(sum((abs(Fraction(v)) for v in x), Fraction(0)))


@pytest.mark.parametrize("name", ["dot2_f64.npz", "dot2_f32.npz", "dot2_c128.npz", "dot2_c64.npz"])
def test_restatement_matches_reference_golden(name):
    """oro.c's sequential Dot2 == reference dot_product<T>::dot_ogita, bit for bit."""
    for meta, d in load_golden(name):
        got = oracle.dot2_seq(d["x"], d["y"])
        want = d["ref_ogita"][()]
        if np.iscomplexobj(d["x"]):
            assert complex(got) == complex(want), meta
        else:
            assert got == want or (np.isnan(got) and np.isnan(want)), meta


def test_threaded_restatement_matches_reference_golden():
    for meta, d in load_golden("dot2_f64.npz"):
        assert oracle.dot2_threaded(d["x"], d["y"], 1) == d["ref_threaded1"][()], meta


def test_exact_oracle_matches_golden_exact():
    for name in ("dot2_f64.npz", "dot2_f32.npz", "dot2_c128.npz", "dot2_c64.npz"):
        for meta, d in load_golden(name):
            hi, lo = oracle.exact_dot(d["x"], d["y"])
            ex = d["exact"]
            assert complex(hi) == complex(ex[0]) and complex(lo) == complex(ex[1]), (name, meta)


def test_sum2_restatement_matches_reference_golden():
    for meta, d in load_golden("sum2_f64.npz"):
        assert oracle.sum2_seq(d["x"]) == d["ref_sum2"][()], meta
        assert oracle.sum2_seq(d["x"], absolute=True) == d["ref_asum2"][()], meta


def test_reference_dot2_within_ogita_bound():
    """The reference's own Dot2 results respect the bound the GPU tests use."""
    for meta, d in load_golden("dot2_f64.npz"):
        n = meta["n"]
        if n == 0:
            continue
        hi = float(d["exact"][0])
        if hi == 0:
            continue
        err = abs(float(d["ref_ogita"]) - hi) / abs(hi)
        assert err <= oracle.bound_dot2(n, float(d["cond"])), (meta, err)


def test_bounds_match_reference_error_bounds():
    rows = np.load(GOLDEN / "bounds_f64.npy")
    for n, cond, seq, blk, pw, naive, cseq, cblk, cpw, cnaive, sseq, sblk, spw, snaive in rows:
        assert oracle.bound_dot2(n, cond) == pytest.approx(seq, rel=1e-12)
        assert oracle.bound_dot2(n, cond, complex_=True) == pytest.approx(cseq, rel=1e-12)
        assert oracle.bound_sum2(max(n, 2), cond) == pytest.approx(sseq, rel=1e-12)


def test_oracle_detects_planted_error():
    """A mistake planted in the oracle's input is caught by the exact check."""
    d = load_golden("dot2_f64.npz")[10][1]
    x = d["x"].copy()
    x[3] = x[3] * 1.5 + 1.0
    hi, _ = oracle.exact_dot(x, d["y"])
    assert hi != d["exact"][0]


def test_reference_golden_live_if_available():
    """When oracle/_ref was built here, regenerate a few reference outputs live."""
    ref = oracle.ref()
    if ref is None:
        pytest.skip("reference CPU code not built on this host")
    for meta, d in load_golden("dot2_f64.npz")[:8]:
        x, y = d["x"], d["y"]
        assert ref.ref_dot_ogita_f64(x.size, x.ctypes.data, y.ctypes.data) == d["ref_ogita"][()]
