"""The device GenDot generator (hpb_gendot_f64_dev / _c128_dev, through the
C ABI) against its CPU restatement (oracle/gendot.c): the head pairs and the
tail's x values agree bit for bit; the tail's y values -- which divide out
the running dot D, a double-double that the device seeds from its Dot2 of
the head and the restatement from a sequential compensated sum -- agree to
a relative 1e-9; the achieved condition number (computed exactly) is that
of the host generator's scheme (within two orders of the requested one and
of the restatement's); the same seed gives the same vectors on every call;
the complex generator interleaves two real pairs so that Re conj(x).y
cancels."""
import ctypes as C

import numpy as np
import pytest

import oracle
from gpu_utils import host
from high_precision_blas1_b200 import _lib

pytestmark = pytest.mark.gpu


def gen_dev(ctx, torch, seed, n, cond):
    x = torch.empty(n, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    nfix = C.c_int64()
    ctx.check(_lib.lib.hpb_gendot_f64_dev(ctx.h, seed, n, cond, x.data_ptr(), y.data_ptr(), C.byref(nfix)),
              "hpb_gendot_f64_dev")
    torch.cuda.synchronize()
    return host(x), host(y), nfix.value


@pytest.mark.parametrize("n,cond", [(100000, 1e20), (40001, 1e8), (262144, 1e30), (1 << 21, 1e16), (7, 1e4), (1, 10.0)])
def test_matches_restatement(gpu, n, cond):
    ctx, torch = gpu
    x, y, nfix = gen_dev(ctx, torch, 11, n, cond)
    xr, yr, nfr = oracle.gendot_dev(11, n, cond)
    assert nfix == nfr
    head = n - nfix
    assert np.array_equal(x, xr) and np.array_equal(y[:head], yr[:head])
    # the tail entry j cancels D down to its target: a difference dD in the
    # double-double D moves x_j y_j by dD, |dD| <= ~n u^2 sum|x_i y_i|
    scale = np.abs(xr * yr).sum()
    assert np.all(np.abs(x[head:] * (y[head:] - yr[head:])) <= 1e-26 * scale)
    if n >= 1000:
        c_dev, c_ref = oracle.condition_dot(x, y), oracle.condition_dot(xr, yr)
        assert cond / 1e2 <= c_dev <= cond * 1e4, c_dev
        # beyond ~1e28 the double-double D's last bits (u^2 sum|xy|) reach the
        # final O(1) target, so the two generators' final dots -- and their
        # condition numbers -- part; both stay at least as ill-conditioned
        # as requested (checked above)
        if cond <= 1e28:
            assert c_ref / 1e2 <= c_dev <= c_ref * 1e2


def test_deterministic_and_seed_dependent(gpu):
    ctx, torch = gpu
    a = gen_dev(ctx, torch, 5, 300000, 1e24)
    b = gen_dev(ctx, torch, 5, 300000, 1e24)
    c = gen_dev(ctx, torch, 6, 300000, 1e24)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert not np.array_equal(a[0], c[0])


def test_dot2_bound_on_device_vectors(gpu):
    """The generated pair is a valid accuracy-sweep input: Dot2 of it meets
    the Ogita-Rump-Oishi bound against the exact dot."""
    ctx, torch = gpu
    from gpu_utils import red
    n = 1 << 20
    x = torch.empty(n, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    ctx.check(_lib.lib.hpb_gendot_f64_dev(ctx.h, 3, n, 1e28, x.data_ptr(), y.data_ptr(), None), "gendot")
    out = red(ctx, "dot2", x, y)
    xs, ys = host(x), host(y)
    ex = oracle.exact_dot(xs, ys)
    exact = ex[0] if isinstance(ex, tuple) else ex
    cond = oracle.condition_dot(xs, ys)
    err = abs(out[0] - exact) / abs(exact)
    assert err <= oracle.bound_dot2(n, cond)


def test_complex_layout(gpu):
    ctx, torch = gpu
    n = 65536
    x = torch.empty(2 * n, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    ctx.check(_lib.lib.hpb_gendot_c128_dev(ctx.h, 9, n, 1e18, x.data_ptr(), y.data_ptr()), "gendot_c128")
    torch.cuda.synchronize()
    xs, ys = host(x), host(y)
    a, b = gen_dev(ctx, torch, 9 ^ 0xA5A5, n, 1e18)[:2]
    c, d = gen_dev(ctx, torch, 9 ^ 0x5A5A, n, 1e18)[:2]
    assert np.array_equal(xs[0::2], a) and np.array_equal(xs[1::2], c)
    assert np.array_equal(ys[0::2], b) and np.array_equal(ys[1::2], d)


def test_errors(gpu):
    ctx, torch = gpu
    x = torch.empty(8, dtype=torch.float64, device="cuda")
    assert _lib.lib.hpb_gendot_f64_dev(ctx.h, 1, 8, 0.5, x.data_ptr(), x.data_ptr(), None) == -1
    assert _lib.lib.hpb_gendot_f64_dev(ctx.h, 1, -1, 10.0, x.data_ptr(), x.data_ptr(), None) == -1
    assert _lib.lib.hpb_gendot_f64_dev(ctx.h, 1, 0, 10.0, None, None, None) == 0
