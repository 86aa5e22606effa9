"""GPU parity of the compensated reductions (through the C ABI) against the
oracle and the reference's own CPU results (golden vectors).

Tolerances (stated per check):
  * bound:  |gpu - exact| <= B(n, cond) * |exact| with B the reference's a
    priori Dot2/Sum2 bound (high_prec/error_bounds.hpp, eps = 2^-52 for
    binary64 data, 2^-23 for binary32 data); where exact == 0 the bound is
    taken against sum|x_i y_i|.
  * 2 ulp:  |gpu - reference Dot2| <= 2 ulp(reference), wherever
    cond <= 1e8 (both results faithful there).
  * determinism: two launches give identical bits.
"""
import numpy as np
import pytest

import oracle
from conftest import load_golden
from gpu_utils import EPS, NP2T, dev, gendot, red, red_ptr, ulp

pytestmark = pytest.mark.gpu


def _abs_scale(x, y):
    return float(np.sum(np.abs(x.astype(np.complex128) if np.iscomplexobj(x) else x.astype(np.float64)) *
                        np.abs(y.astype(np.complex128) if np.iscomplexobj(y) else y.astype(np.float64))))


@pytest.mark.parametrize("name", ["dot2_f64.npz", "dot2_f32.npz", "dot2_c128.npz", "dot2_c64.npz"])
def test_dot2_golden(gpu, name):
    ctx, torch = gpu
    for meta, d in load_golden(name):
        x, y = d["x"], d["y"]
        n = meta["n"]
        t = NP2T[x.dtype]
        cplx = t in ("c64", "c128")
        xd, yd = dev(torch, x), dev(torch, y)
        out = red(ctx, "dot2", xd, yd)
        out2 = red(ctx, "dot2", xd, yd)
        assert np.array_equal(out, out2), ("nondeterministic", meta)
        got = complex(out[0], out[1]) if cplx else out[0]
        exact = complex(d["exact"][0]) if cplx else float(d["exact"][0])
        ref = complex(d["ref_ogita"][()]) if cplx else float(d["ref_ogita"][()])
        if n == 0:
            assert got == 0
            continue
        scale = _abs_scale(x, y)
        cond = scale / abs(exact) if exact != 0 else np.inf
        bnd = oracle.bound_dot2(n, min(cond, 1e300), complex_=cplx, eps=EPS[t])
        err = abs(got - exact)
        assert err <= bnd * abs(exact) + (bnd * scale if exact == 0 else 0.0), (meta, err, bnd)
        # per-component condition numbers (a complex GenDot pair cancels in
        # its real part only)
        xx = x.astype(np.complex128 if cplx else np.float64)
        yy = y.astype(np.complex128 if cplx else np.float64)
        re_scale = float(np.sum(np.abs(xx.real * yy.real) + np.abs(xx.imag * yy.imag)))
        im_scale = float(np.sum(np.abs(xx.real * yy.imag) + np.abs(xx.imag * yy.real)))
        comps = [(np.real(got), np.real(ref), re_scale / abs(np.real(exact)) if np.real(exact) else np.inf)]
        if cplx:
            comps.append((np.imag(got), np.imag(ref), im_scale / abs(np.imag(exact)) if np.imag(exact) else np.inf))
        for part_got, part_ref, ccond in comps:
            if ccond <= 1e8:
                if t in ("f32", "c64"):
                    # the reference rounds its float result to binary32; ours is binary64
                    assert abs(np.float32(part_got) - part_ref) <= 2 * np.spacing(np.float32(abs(part_ref))), meta
                else:
                    assert abs(part_got - part_ref) <= 2 * ulp(part_ref), (meta, part_got, part_ref)


def test_dot2_lo_is_rounding_error_of_hi(gpu):
    ctx, torch = gpu
    for meta, d in load_golden("dot2_f64.npz"):
        if meta["n"] == 0:
            continue
        out = red(ctx, "dot2", dev(torch, d["x"]), dev(torch, d["y"]))
        assert abs(out[1]) <= 0.5 * ulp(out[0]), meta


def test_dot2_matches_reference_golden_within_bound(gpu):
    """GPU Dot2 vs the reference's Dot2: both within the bound of exact."""
    ctx, torch = gpu
    for meta, d in load_golden("dot2_f64.npz"):
        n = meta["n"]
        if n == 0:
            continue
        out = red(ctx, "dot2", dev(torch, d["x"]), dev(torch, d["y"]))
        exact = float(d["exact"][0])
        bnd = oracle.bound_dot2(n, float(d["cond"]))
        assert abs(out[0] - float(d["ref_ogita"])) <= 2 * bnd * abs(exact) + 1e-300, meta


@pytest.mark.parametrize("n", [1 << 20, (1 << 20) + 3, 3 * 1000 * 1000 + 1])
def test_dot2_gendot_cond1e20_large(gpu, n):
    """Config-1 shape: GenDot f64, n ~ 1M, cond ~ 1e20..1e23."""
    ctx, torch = gpu
    x, y = gendot(11, n, 1e20)
    hi, _ = oracle.exact_dot(x, y)
    cond = oracle.condition_dot(x, y)
    out = red(ctx, "dot2", dev(torch, x), dev(torch, y))
    rel = abs(out[0] - hi) / abs(hi)
    assert rel <= oracle.bound_dot2(n, cond)
    # a plain dot loses everything at this condition number; Dot2 keeps
    # roughly u^2 * cond * (tree depth) relative accuracy
    plain = red(ctx, "dot", dev(torch, x), dev(torch, y))
    assert rel < 1e-3 and abs(plain[0] - hi) / abs(hi) > 1.0
    # and within the reference's own sequential Dot2 accuracy class
    seq = oracle.dot2_seq(x, y)
    assert rel <= max(10 * abs(seq - hi) / abs(hi), 1e-9)


def test_dot2_misaligned_and_ragged(gpu):
    ctx, torch = gpu
    rng = np.random.default_rng(3)
    for n in (1, 2, 5, 1001, 65537):
        x = rng.standard_normal(n + 1)
        y = rng.standard_normal(n + 1) * np.exp2(rng.integers(-20, 20, n + 1))
        xd, yd = dev(torch, x), dev(torch, y)
        # offset by one element: 8-byte aligned, not 16 -> scalar path
        out = red_ptr(ctx, "dot2", "f64", n, xd.data_ptr() + 8, yd.data_ptr() + 8)
        hi, _ = oracle.exact_dot(x[1:], y[1:])
        assert abs(out[0] - hi) <= 2 * ulp(hi) + oracle.bound_dot2(n, _abs_scale(x[1:], y[1:]) / abs(hi)) * abs(hi)
        # complex<double> at an 8-byte offset (two doubles per element)
        xc = (rng.standard_normal(2 * n + 1))
        yc = (rng.standard_normal(2 * n + 1))
        xcd, ycd = dev(torch, xc), dev(torch, yc)
        outc = red_ptr(ctx, "dot2", "c128", n, xcd.data_ptr() + 8, ycd.data_ptr() + 8)
        hc, _ = oracle.exact_dot(xc[1:].view(np.complex128), yc[1:].view(np.complex128))
        assert abs(complex(outc[0], outc[1]) - hc) <= 4 * ulp(abs(hc)) + 1e-12 * abs(hc)


def test_misaligned_element_pointer_rejected(gpu):
    ctx, torch = gpu
    from high_precision_blas1_b200 import _lib
    x = dev(torch, np.ones(16))
    out = np.zeros(4)
    st = _lib.lib.hpb_dot2_f64_host(ctx.h, 4, x.data_ptr() + 4, x.data_ptr(), out.ctypes.data)
    assert st == -1


@pytest.mark.parametrize("t", ["f64", "f32", "c128", "c64"])
def test_sum2_asum2_nrm2_against_exact(gpu, t):
    ctx, torch = gpu
    rng = np.random.default_rng(17)
    dt = {"f64": np.float64, "f32": np.float32, "c128": np.complex128, "c64": np.complex64}[t]
    cplx = t.startswith("c")
    for n in (0, 1, 7, 33, 4097, 300001):
        if cplx:
            x = (rng.standard_normal(n) + 1j * rng.standard_normal(n)) * np.exp2(rng.integers(-8, 8, n))
        else:
            x = rng.standard_normal(n) * np.exp2(rng.integers(-8, 8, n))
        x = x.astype(dt)
        xd = dev(torch, x)
        # Sum2
        s = red(ctx, "sum2", xd)
        shi, _ = oracle.exact_sum(x)
        got = complex(s[0], s[1]) if cplx else s[0]
        scale = float(np.sum(np.abs(x.view(np.float32 if t in ("f32", "c64") else np.float64).astype(np.float64))))
        assert abs(got - shi) <= oracle.bound_sum2(max(2 * n, 2), 1.0, EPS[t]) * scale + 1e-300, (t, n)
        # asum2 (complex: |re| + |im|)
        a = red(ctx, "asum2", xd)
        ahi, _ = oracle.exact_sum(x, absolute=True)
        assert abs(a[0] - ahi) <= 2 * ulp(ahi) + EPS[t] * ahi, (t, n)
        # nrm2 = sqrt(compensated sum of squares)
        r = red(ctx, "nrm2", xd)
        qhi, _ = oracle.exact_sumsq(x)
        assert abs(r[1] - qhi) <= 2 * ulp(qhi) + EPS[t] * qhi, (t, n)
        assert r[0] == pytest.approx(np.sqrt(qhi), rel=4 * EPS["f64"], abs=1e-300)


def test_sum2_golden_against_reference(gpu):
    ctx, torch = gpu
    for meta, d in load_golden("sum2_f64.npz"):
        x = d["x"]
        s = red(ctx, "sum2", dev(torch, x))
        a = red(ctx, "asum2", dev(torch, x))
        ex, exa = float(d["exact_sum"][0]), float(d["exact_asum"][0])
        scale = float(np.sum(np.abs(x)))
        n = max(meta["n"], 2)
        assert abs(s[0] - ex) <= oracle.bound_sum2(n, scale / abs(ex) if ex else 1e300) * abs(ex) + (
            0 if ex else 1e-300), meta
        # reference asum2 of the golden data (nonnegative terms): both faithful
        assert abs(a[0] - exa) <= 2 * ulp(exa), meta
        assert abs(a[0] - float(d["ref_asum2"])) <= 2 * ulp(exa), meta


@pytest.mark.parametrize("t", ["f64", "f32", "c128", "c64"])
def test_plain_reductions(gpu, t):
    ctx, torch = gpu
    rng = np.random.default_rng(23)
    dt = {"f64": np.float64, "f32": np.float32, "c128": np.complex128, "c64": np.complex64}[t]
    n = 100003
    x = rng.standard_normal(n * 2).view(np.complex128)[:n] if t.startswith("c") else rng.standard_normal(n)
    y = rng.standard_normal(n * 2).view(np.complex128)[:n] if t.startswith("c") else rng.standard_normal(n)
    x, y = x.astype(dt), y.astype(dt)
    xd, yd = dev(torch, x), dev(torch, y)
    o = red(ctx, "dot", xd, yd)
    got = complex(o[0], o[1]) if t.startswith("c") else o[0]
    hi, _ = oracle.exact_dot(x, y)
    tol = oracle.oro().oro_bound_dot_naive_real(float(n), 1.0, EPS[t]) * _abs_scale(x, y) * 4
    assert abs(got - hi) <= tol
    a = red(ctx, "asum", xd)
    ahi, _ = oracle.exact_sum(x, absolute=True)
    assert a[0] == pytest.approx(ahi, rel=n * EPS[t])
    q = red(ctx, "nrm2plain", xd)
    qhi, _ = oracle.exact_sumsq(x)
    assert q[1] == pytest.approx(qhi, rel=n * EPS[t])


def test_device_result_buffer_and_launch_count(gpu):
    """The async entry points write (hi, lo) into a device buffer."""
    ctx, torch = gpu
    from high_precision_blas1_b200 import _lib
    x = dev(torch, np.arange(1, 1001, dtype=np.float64))
    out = torch.zeros(4, dtype=torch.float64, device="cuda")
    before = _lib.lib.hpb_launch_count()
    ctx.check(_lib.lib.hpb_dot2_f64(ctx.h, 1000, x.data_ptr(), x.data_ptr(), out.data_ptr()))
    torch.cuda.synchronize()
    assert _lib.lib.hpb_launch_count() - before == 1  # one launch per Dot2
    assert out[0].item() == sum(i * i for i in range(1, 1001))


def test_inf_nan_propagate(gpu):
    ctx, torch = gpu
    x = np.ones(1000)
    x[517] = np.inf
    o = red(ctx, "dot2", dev(torch, x), dev(torch, np.ones(1000)))
    assert not np.isfinite(o[0])
    x[517] = np.nan
    o = red(ctx, "sum2", dev(torch, x))
    assert np.isnan(o[0])


@pytest.mark.parametrize("n", [1001, 65537, 1 << 20, (1 << 20) + 3])
def test_dot2_sum2_match_reference_gpu_kernels(gpu, n):
    """Against the reference's own GPU Ogita kernels (gpu_reduction_ogita,
    built for sm_100a into oracle/_ref) on the same device data: both within
    the compensated bound of the exact value, and within 2 ulp of each other
    where the condition number is <= 1e8 (n stays below the size at which
    the reference's in-place later passes race)."""
    rg = oracle.ref_gpu()
    if rg is None:
        pytest.skip("reference GPU reductions not built")
    ctx, torch = gpu
    rng = np.random.default_rng(n)
    cases = [(rng.standard_normal(n), rng.standard_normal(n))]
    if n >= 65537:
        cases.append(gendot(29, n, 1e16))
    for x, y in cases:
        xd, yd = dev(torch, x), dev(torch, y)
        ours = red(ctx, "dot2", xd, yd)
        theirs = np.zeros(2)
        assert rg.ref_gpu_dot2_f64(n, xd.data_ptr(), yd.data_ptr(), theirs.ctypes.data) == 0
        torch.cuda.synchronize()
        hi, _ = oracle.exact_dot(x, y)
        cond = oracle.condition_dot(x, y)
        bound = oracle.bound_dot2(n, cond) * abs(hi) + 2 * ulp(hi)
        assert abs(ours[0] - hi) <= bound and abs(theirs[0] - hi) <= bound
        if cond <= 1e8:
            assert abs(ours[0] - theirs[0]) <= 2 * ulp(theirs[0]), (ours[0], theirs[0])
    # Sum2
    x = rng.standard_normal(n) * np.exp2(rng.integers(-30, 30, n))
    xd = dev(torch, x)
    ours = red(ctx, "sum2", xd)
    theirs = np.zeros(1)
    assert rg.ref_gpu_sum2_f64(n, xd.data_ptr(), theirs.ctypes.data) == 0
    torch.cuda.synchronize()
    hi, _ = oracle.exact_sum(x)
    scale = float(np.sum(np.abs(x)))
    bound = oracle.bound_sum2(n, scale / abs(hi)) * abs(hi) + 2 * ulp(hi)
    assert abs(ours[0] - hi) <= bound and abs(theirs[0] - hi) <= bound
    if scale / abs(hi) <= 1e8:
        assert abs(ours[0] - theirs[0]) <= 2 * ulp(theirs[0])
