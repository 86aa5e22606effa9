"""GPU parity of the sparse triangular solves and ILU(0) (hpb_csr_trsv_*,
hpb_csr_ilu0_*, through the C ABI) against the CPU restatement in
oracle/tri.c.  Every row is computed by the same sequence of roundings on
both sides, so the comparison is bit for bit (tolerance 0) for all four
element types; the restatement itself is checked against scipy's
triangular solver and against the defining property of ILU(0)
((L U)_ij = A_ij on A's pattern) in tests/test_tri_oracle.py.

Cases: the solver problems (2-D convection-diffusion, 3-D anisotropic
Poisson, complex Helmholtz), a random pattern whose rows hold more
dependencies than the kernel prefetches, row counts that leave a ragged
last tile, a single row, rows holding only a diagonal, in-place solves,
alpha != 1, and the error paths (unsorted columns, a missing diagonal,
a zero pivot)."""
import ctypes as C

import numpy as np
import pytest

import oracle
from gpu_utils import dev, host
from high_precision_blas1_b200 import _lib, problems

pytestmark = pytest.mark.gpu

DT = {"f32": np.float32, "f64": np.float64, "c64": np.complex64, "c128": np.complex128}
TILE = 8192


class Tri:
    def __init__(self, ctx, torch, A, upper):
        self.rp = dev(torch, A.row_ptr)
        self.ci = dev(torch, A.col_ind)
        self.h = C.c_void_p()
        st = _lib.lib.hpb_csr_tri_create(ctx.h, int(upper), A.n, A.nnz, self.rp.data_ptr(), self.ci.data_ptr(),
                                         C.byref(self.h))
        ctx.check(st, "hpb_csr_tri_create")

    def info(self):
        t, m, s, d = C.c_int32(), C.c_int32(), C.c_int64(), C.c_int()
        assert _lib.lib.hpb_csr_tri_info(self.h, C.byref(t), C.byref(m), C.byref(s), C.byref(d)) == 0
        return t.value, m.value, s.value, d.value

    def close(self):
        _lib.lib.hpb_csr_tri_destroy(self.h)


def trsv(ctx, torch, tri, t, val_d, b, unit, alpha=1.0, inplace=False):
    bd = dev(torch, b.astype(DT[t]))
    xd = bd if inplace else torch.zeros_like(bd)
    st = getattr(_lib.lib, f"hpb_csr_trsv_{t}")(ctx.h, tri.h, int(unit), val_d.data_ptr(), _lib.scalar(t, alpha),
                                               bd.data_ptr(), xd.data_ptr())
    ctx.check(st, "trsv")
    ctx.check(_lib.lib.hpb_csr_tri_check(ctx.h, tri.h), "tri_check")
    torch.cuda.synchronize()
    return host(xd)


def complexify(A, rng):
    return problems.CSR(A.n, A.row_ptr, A.col_ind, A.val + 1j * 0.3 * rng.standard_normal(A.nnz) * np.abs(A.val))


def banded_random(rng, n, width, density=0.7):
    """Rows with up to `width` entries on each side of a dominant diagonal."""
    rp, ci, va = [0], [], []
    for r in range(n):
        cols = [c for c in range(max(0, r - width), min(n, r + width + 1)) if c == r or rng.random() < density]
        ci.extend(cols)
        va.extend((2.0 * width + 1.0) if c == r else rng.standard_normal() for c in cols)
        rp.append(len(ci))
    return problems.CSR(n, np.array(rp, np.int32), np.array(ci, np.int32), np.array(va))


def row_scaled(A):
    """D^-1 A (D the stored diagonal; rows without one unscaled): the unit-
    and non-unit-diagonal solves of every test matrix then stay bounded."""
    rows = np.repeat(np.arange(A.n), np.diff(A.row_ptr))
    d = np.ones(A.n, dtype=A.val.dtype)
    on = A.col_ind == rows
    d[rows[on]] = A.val[on]
    return problems.CSR(A.n, A.row_ptr, A.col_ind, A.val / d[rows])


def typed(A, t, rng):
    """A in element type t, row-scaled (complex types get an imaginary part
    when A is real; real types take the real part of a complex A)."""
    if t in ("c64", "c128") and not np.iscomplexobj(A.val):
        A = complexify(A, rng)
    if t in ("f32", "f64") and np.iscomplexobj(A.val):
        A = problems.CSR(A.n, A.row_ptr, A.col_ind, A.val.real.copy())
    A = row_scaled(A)
    return A, A.val.astype(DT[t])


def problem(name, rng):
    if name == "convdiff64":
        return problems.convdiff2d(64)
    if name == "convdiff1024":
        return problems.convdiff2d(1024)
    if name == "poisson3d_32":
        return problems.poisson3d_aniso(32)
    if name == "helmholtz64":
        return problems.helmholtz2d(64)
    if name == "banded_ragged":  # 2.5 tiles, rows with up to 12 dependencies each side
        return banded_random(rng, 2 * TILE + 4099, 12)
    if name == "single_row":
        return problems.CSR(1, np.array([0, 1], np.int32), np.array([0], np.int32), np.array([3.0]))
    if name == "diag_only":
        n = TILE + 3
        return problems.CSR(n, np.arange(n + 1, dtype=np.int32), np.arange(n, dtype=np.int32), rng.random(n) + 1.0)
    raise KeyError(name)


CASES = ["convdiff64", "poisson3d_32", "helmholtz64", "banded_ragged", "single_row", "diag_only"]


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("t", ["f64", "f32", "c128", "c64"])
def test_trsv_bitwise(gpu, name, t):
    ctx, torch = gpu
    rng = np.random.default_rng(7)
    A, val = typed(problem(name, rng), t, rng)
    vd = dev(torch, val)
    b = rng.standard_normal(A.n) + (1j * rng.standard_normal(A.n) if t in ("c64", "c128") else 0)
    b = b.astype(DT[t])
    for upper in (False, True):
        tri = Tri(ctx, torch, A, upper)
        try:
            for unit in (True, False):
                for alpha in (1.0, -0.75):
                    got = trsv(ctx, torch, tri, t, vd, b, unit, alpha)
                    want = oracle.csr_trsv(A.row_ptr, A.col_ind, val, b, upper, unit, alpha)
                    assert np.array_equal(got, want), (name, t, upper, unit, alpha,
                                                       np.abs(got - want).max())
        finally:
            tri.close()


@pytest.mark.parametrize("t", ["f64", "c128", "f32"])
def test_trsv_in_place(gpu, t):
    ctx, torch = gpu
    rng = np.random.default_rng(3)
    A, val = typed(problems.convdiff2d(96), t, rng)
    vd = dev(torch, val)
    b = rng.standard_normal(A.n).astype(DT[t])
    for upper in (False, True):
        tri = Tri(ctx, torch, A, upper)
        got = trsv(ctx, torch, tri, t, vd, b, unit=not upper, inplace=True)
        tri.close()
        assert np.array_equal(got, oracle.csr_trsv(A.row_ptr, A.col_ind, val, b, upper, not upper))


@pytest.mark.parametrize("name", ["convdiff64", "poisson3d_32", "helmholtz64", "banded_ragged", "convdiff1024"])
@pytest.mark.parametrize("t", ["f64", "f32", "c128", "c64"])
def test_ilu0_bitwise_and_apply(gpu, name, t):
    ctx, torch = gpu
    if name == "convdiff1024" and t not in ("f64", "f32"):
        pytest.skip("one type pair at full size")
    rng = np.random.default_rng(11)
    A, val = typed(problem(name, rng), t, rng)
    lo = Tri(ctx, torch, A, False)
    up = Tri(ctx, torch, A, True)
    try:
        tiles, max_lv, _, has_diag = lo.info()
        assert tiles == (A.n + TILE - 1) // TILE and has_diag == 1 and max_lv >= 1
        lu = dev(torch, val)
        ctx.check(getattr(_lib.lib, f"hpb_csr_ilu0_{t}")(ctx.h, lo.h, lu.data_ptr()), "ilu0")
        torch.cuda.synchronize()
        want, zero_row = oracle.csr_ilu0(A.row_ptr, A.col_ind, val)
        assert zero_row == -1
        assert np.array_equal(host(lu), want), np.abs(host(lu) - want).max()
        # M^-1 r = U^-1 L^-1 r, as csr::preconditioner::apply does it
        r = (rng.standard_normal(A.n) + (1j * rng.standard_normal(A.n) if t in ("c64", "c128") else 0)).astype(DT[t])
        y = trsv(ctx, torch, lo, t, lu, r, unit=True)
        z = trsv(ctx, torch, up, t, lu, y, unit=False)
        y_o = oracle.csr_trsv(A.row_ptr, A.col_ind, want, r, False, True)
        z_o = oracle.csr_trsv(A.row_ptr, A.col_ind, want, y_o, True, False)
        assert np.array_equal(y, y_o) and np.array_equal(z, z_o)
    finally:
        lo.close()
        up.close()


def test_ilu0_is_exact_for_tridiagonal(gpu):
    """On a tridiagonal matrix ILU(0) is the exact LU: U^-1 L^-1 A x = x."""
    ctx, torch = gpu
    n = 3 * TILE + 17
    rng = np.random.default_rng(5)
    rp = [0]
    ci = []
    for r in range(n):
        ci.extend(c for c in (r - 1, r, r + 1) if 0 <= c < n)
        rp.append(len(ci))
    ci = np.array(ci, np.int32)
    rows = np.repeat(np.arange(n), np.diff(rp))
    val = np.where(ci == rows, 4.0, -1.0) + 0.1 * rng.standard_normal(len(ci))
    A = problems.CSR(n, np.array(rp, np.int32), ci, val)
    lo, up = Tri(ctx, torch, A, False), Tri(ctx, torch, A, True)
    lu = dev(torch, val)
    ctx.check(_lib.lib.hpb_csr_ilu0_f64(ctx.h, lo.h, lu.data_ptr()), "ilu0")
    x = rng.standard_normal(n)
    b = A.matvec(x)
    z = trsv(ctx, torch, up, "f64", lu, trsv(ctx, torch, lo, "f64", lu, b, unit=True), unit=False)
    lo.close()
    up.close()
    assert np.abs(z - x).max() < 1e-12


def test_errors(gpu):
    ctx, torch = gpu
    h = C.c_void_p()
    # unsorted columns in a row
    bad = problems.CSR(2, np.array([0, 2, 3], np.int32), np.array([1, 0, 1], np.int32), np.ones(3))
    rp, ci = dev(torch, bad.row_ptr), dev(torch, bad.col_ind)
    st = _lib.lib.hpb_csr_tri_create(ctx.h, 0, 2, 3, rp.data_ptr(), ci.data_ptr(), C.byref(h))
    assert st == -1 and h.value is None
    # column out of range
    oob = problems.CSR(2, np.array([0, 1, 2], np.int32), np.array([0, 5], np.int32), np.ones(2))
    rp, ci = dev(torch, oob.row_ptr), dev(torch, oob.col_ind)
    assert _lib.lib.hpb_csr_tri_create(ctx.h, 0, 2, 2, rp.data_ptr(), ci.data_ptr(), C.byref(h)) == -1
    # missing diagonal: unit solves work, non-unit and ILU(0) are refused
    nod = problems.CSR(2, np.array([0, 1, 2], np.int32), np.array([0, 0], np.int32), np.array([2.0, 1.0]))
    tri = Tri(ctx, torch, nod, False)
    assert tri.info()[3] == 0
    vd = dev(torch, nod.val)
    got = trsv(ctx, torch, tri, "f64", vd, np.array([1.0, 1.0]), unit=True)
    assert np.array_equal(got, np.array([1.0, 0.0]))
    bd, xd = dev(torch, np.ones(2)), dev(torch, np.zeros(2))
    assert _lib.lib.hpb_csr_trsv_f64(ctx.h, tri.h, 0, vd.data_ptr(), 1.0, bd.data_ptr(), xd.data_ptr()) == -1
    assert _lib.lib.hpb_csr_ilu0_f64(ctx.h, tri.h, vd.data_ptr()) == -1
    tri.close()
    # zero pivot: [[1, 1], [1, 1]] -> u_11 = 0
    zp = problems.CSR(2, np.array([0, 2, 4], np.int32), np.array([0, 1, 0, 1], np.int32), np.ones(4))
    tri = Tri(ctx, torch, zp, False)
    vd = dev(torch, zp.val)
    assert _lib.lib.hpb_csr_ilu0_f64(ctx.h, tri.h, vd.data_ptr()) == -5
    assert b"zero pivot in row 1" in _lib.lib.hpb_last_error(ctx.h)
    # the upper analysis cannot factor
    up = Tri(ctx, torch, zp, True)
    assert _lib.lib.hpb_csr_ilu0_f64(ctx.h, up.h, vd.data_ptr()) == -1
    up.close()
    tri.close()
    # empty pattern
    e = C.c_void_p()
    assert _lib.lib.hpb_csr_tri_create(ctx.h, 0, 0, 0, None, None, C.byref(e)) == 0
    assert _lib.lib.hpb_csr_tri_destroy(e) == 0


def sweeps(ctx, torch, tri, t, val_d, b, unit, k, alpha=1.0):
    bd = dev(torch, b.astype(DT[t]))
    xd = torch.zeros_like(bd)
    st = getattr(_lib.lib, f"hpb_csr_trsv_sweeps_{t}")(ctx.h, tri.h, int(unit), val_d.data_ptr(),
                                                       _lib.scalar(t, alpha), bd.data_ptr(), xd.data_ptr(), k)
    ctx.check(st, "trsv_sweeps")
    torch.cuda.synchronize()
    return host(xd)


@pytest.mark.parametrize("name", ["convdiff64", "poisson3d_32", "banded_ragged", "diag_only"])
@pytest.mark.parametrize("t", ["f64", "f32", "c128", "c64"])
def test_sweeps_bitwise(gpu, name, t):
    """Jacobi-sweep approximation of the triangular solves: bit for bit the
    CPU restatement for 0, 1 and 3 sweeps, both triangles, unit and not."""
    ctx, torch = gpu
    rng = np.random.default_rng(21)
    A, val = typed(problem(name, rng), t, rng)
    vd = dev(torch, val)
    b = (rng.standard_normal(A.n) + (1j * rng.standard_normal(A.n) if t.startswith("c") else 0)).astype(DT[t])
    for upper in (False, True):
        tri = Tri(ctx, torch, A, upper)
        try:
            for unit in (True, False):
                for k in (0, 1, 3):
                    got = sweeps(ctx, torch, tri, t, vd, b, unit, k, alpha=-0.5)
                    want = oracle.csr_trsv_sweeps(A.row_ptr, A.col_ind, val, b, upper, unit, k, alpha=-0.5)
                    assert np.array_equal(got, want), (name, t, upper, unit, k)
        finally:
            tri.close()


def test_sweeps_reach_the_exact_solve(gpu):
    """A triangle's Jacobi iteration is exact after as many sweeps as its
    longest dependency chain: then every row is formed from exact values in
    the same order as forward / backward substitution, bit for bit."""
    ctx, torch = gpu
    rng = np.random.default_rng(2)
    A, val = typed(problems.convdiff2d(8), "f64", rng)  # longest chain: 14 steps
    vd = dev(torch, val)
    b = rng.standard_normal(A.n)
    for upper in (False, True):
        tri = Tri(ctx, torch, A, upper)
        exact = trsv(ctx, torch, tri, "f64", vd, b, unit=not upper)
        assert not np.array_equal(sweeps(ctx, torch, tri, "f64", vd, b, not upper, 3), exact)
        assert np.array_equal(sweeps(ctx, torch, tri, "f64", vd, b, not upper, 15), exact)
        tri.close()


def random_long_range(rng, n, deps):
    """Each row depends on `deps` random earlier (lower) rows anywhere above
    it, plus a dominant diagonal and as many random later columns: most
    dependencies cross tiles, more of them than a tile's halo holds (so the
    solve's direct polling path runs too)."""
    rp, ci, va = [0], [], []
    for r in range(n):
        lo = rng.choice(r, size=min(deps, r), replace=False) if r else np.zeros(0, np.int64)
        hi = rng.choice(np.arange(r + 1, n), size=min(deps, n - r - 1), replace=False) if r + 1 < n else \
            np.zeros(0, np.int64)
        cols = np.sort(np.concatenate([lo, [r], hi]).astype(np.int64))
        ci.extend(cols.tolist())
        va.extend(float(2 * deps + 1) if c == r else rng.standard_normal() for c in cols)
        rp.append(len(ci))
    return problems.CSR(n, np.array(rp, np.int32), np.array(ci, np.int32), np.array(va))


@pytest.mark.parametrize("t", ["f64", "c128"])
def test_trsv_long_range_dependencies(gpu, t):
    ctx, torch = gpu
    rng = np.random.default_rng(31)
    A, val = typed(random_long_range(rng, 3 * TILE + 100, 3), t, rng)
    vd = dev(torch, val)
    b = (rng.standard_normal(A.n) + (1j * rng.standard_normal(A.n) if t.startswith("c") else 0)).astype(DT[t])
    for upper in (False, True):
        tri = Tri(ctx, torch, A, upper)
        try:
            for unit in (True, False):
                got = trsv(ctx, torch, tri, t, vd, b, unit)
                want = oracle.csr_trsv(A.row_ptr, A.col_ind, val, b, upper, unit)
                assert np.array_equal(got, want), (t, upper, unit)
        finally:
            tri.close()


def test_trsv_bounded_wait_runs_out(gpu):
    """The timeout path of the solve's bounded waits, without a fault: the
    testing hook withholds the global publish of the first tile's last row,
    so the second tile's rows that depend on it (row TILE + 127, through its
    grid neighbour one line below) wait until the 1 ms
    limit set on the analysis.  The launch ends, hpb_csr_tri_check reports
    HPB_ERROR_TIMEOUT once, the first tile's other rows are exact, and the
    next solve on the same analysis, hook off and default limit, is exact."""
    import time
    ctx, torch = gpu
    L = _lib.lib
    A = problems.convdiff2d(128)
    rng = np.random.default_rng(3)
    vd = dev(torch, A.val)
    b = rng.standard_normal(A.n)
    want = oracle.csr_trsv(A.row_ptr, A.col_ind, A.val, b, False, False, 1.0)
    tri = Tri(ctx, torch, A, False)
    try:
        assert tri.info()[0] == 2
        assert L.hpb_csr_tri_set_wait_limit(tri.h, 1_000_000) == 0
        assert L.hpb_csr_tri_test_withhold_row(tri.h, TILE - 1) == 0
        assert L.hpb_csr_tri_test_withhold_row(tri.h, A.n) != 0  # out of range refused
        bd = dev(torch, b)
        xd = torch.zeros_like(bd)
        t0 = time.perf_counter()
        ctx.check(L.hpb_csr_trsv_f64(ctx.h, tri.h, 0, vd.data_ptr(), 1.0, bd.data_ptr(), xd.data_ptr()), "trsv")
        assert L.hpb_csr_tri_check(ctx.h, tri.h) == -9  # HPB_ERROR_TIMEOUT
        assert time.perf_counter() - t0 < 2.0  # ended near the 1 ms limit, far below the 4 s default
        x = host(xd)
        assert np.array_equal(x[:TILE - 1], want[:TILE - 1])
        assert not np.isfinite(x[TILE - 1]) and not np.isfinite(x[TILE + 127])
        assert L.hpb_csr_tri_check(ctx.h, tri.h) == 0  # reported once
        assert L.hpb_csr_tri_test_withhold_row(tri.h, -1) == 0
        assert L.hpb_csr_tri_set_wait_limit(tri.h, 0) == 0
        got = trsv(ctx, torch, tri, "f64", vd, b, False)
        assert np.array_equal(got, want)
    finally:
        tri.close()
