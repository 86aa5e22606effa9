"""Host logic of the sharded reductions and the sharded SpMV
(high_precision_blas1_b200/sharded.py):
the contiguous partition, the rank-ordered merge of per-rank (hi, lo)
results (the library's host build, hpb_shard_merge_cpu, against the
oracle's plain-Python restatement, bit for bit), and the exchange itself
with 2 and 3 gloo ranks on CPU: every rank ends with the same bits, equal
to the oracle's merge of the ranks' results and within the Dot2 bound of
the exact dot product.  Each rank's local Dot2 here comes from the oracle
(no GPU in these tests); on a GPU it is hpb_dot2_* (tests/test_sharded_gpu.py).
The SpMV's halo plan (column renumbering, requests, send lists) is checked
by emulating the exchange in one process and with gloo ranks running the
all-to-all: the row blocks' products (scipy here, hpb_csr_spmv_* on a GPU)
equal the whole product bit for bit."""
import os
import sys
from pathlib import Path

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp  # noqa: F401  (spawned ranks)
from rank_utils import run_ranks

import scipy.sparse as sp

import oracle
from high_precision_blas1_b200 import problems, sharded

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    """A TCP port on 127.0.0.1 that nothing listens on right now."""
    import socket
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def two_sum(a, b):
    s = a + b
    bv = s - a
    av = s - bv
    return s, (b - bv) + (a - av)


def local_result(x, y):
    """(hi, lo) of the reference's sequential Dot2 of one slice."""
    out = np.zeros(3)
    oracle.oro().oro_dot2_seq_f64(x.shape[0], oracle._ptr(x), oracle._ptr(y), oracle._ptr(out))
    return np.array(two_sum(out[1], out[2]))


@pytest.mark.parametrize("n", [0, 1, 7, 64, 1000003])
@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_partition_covers_contiguously(n, world):
    parts = [sharded.partition(n, world, r) for r in range(world)]
    assert parts[0][0] == 0 and parts[-1][1] == n
    for (a, b), (c, _) in zip(parts, parts[1:]):
        assert b == c
    sizes = [b - a for a, b in parts]
    assert max(sizes) - min(sizes) <= 1 and sizes == sorted(sizes, reverse=True)


def test_partition_rejects_bad_arguments():
    for args in [(-1, 2, 0), (4, 0, 0), (4, 2, 2), (4, 2, -1)]:
        with pytest.raises(ValueError):
            sharded.partition(*args)


@pytest.mark.parametrize("is_complex", [False, True])
def test_merge_cpu_matches_oracle_bitwise(is_complex):
    rng = np.random.default_rng(5)
    comps = 2 if is_complex else 1
    for count in range(1, 10):
        for trial in range(20):
            hi = rng.standard_normal((count, comps)) * 10.0 ** rng.integers(-20, 20, (count, comps))
            err = rng.standard_normal((count, comps)) * 10.0 ** rng.integers(-20, 20, (count, comps))
            pairs = np.zeros((count, 2 * comps))
            for k in range(count):
                for q in range(comps):
                    pairs[k, q], pairs[k, comps + q] = two_sum(hi[k, q], err[k, q])
            got = sharded.merge_gathered_cpu(pairs, is_complex)
            want = oracle.shard_merge(pairs, is_complex)
            assert got.tobytes() == want.tobytes()
            if count == 1:  # one result merges to itself
                assert got.tobytes() == pairs[0].tobytes()


def test_merge_cpu_cancellation_keeps_the_error_terms():
    """hi terms that cancel exactly leave the lo terms: the merged value is
    their sum, which a plain sum of the his would lose."""
    pairs = np.array([[1.0e16, 1.0], [-1.0e16, 0.5]])
    got = sharded.merge_gathered_cpu(pairs, False)
    assert got[0] == 1.5 and got[1] == 0.0


def test_merge_cpu_rejects_bad_shapes():
    with pytest.raises(ValueError):
        sharded.merge_gathered_cpu(np.zeros(3), False)
    with pytest.raises(ValueError):
        sharded.merge_gathered_cpu(np.zeros(0), False)
    with pytest.raises(ValueError):
        sharded.merge_gathered_cpu(np.zeros(2), True)


def _worker(rank, world, port, n, cond, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        x, y, _ = oracle.gendot_dev(1234, n, cond)  # the same pair on every rank (seeded)
        lo, hi = sharded.partition(n, world, rank)
        local = torch.from_numpy(local_result(x[lo:hi].copy(), y[lo:hi].copy()))
        gathered = torch.zeros(2 * world, dtype=torch.float64)
        dist.all_gather_into_tensor(gathered, local)
        merged = sharded.merge_gathered_cpu(gathered.numpy(), False)
        q.put((rank, gathered.numpy().tobytes(), merged.tobytes()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_sharded_dot2(world):
    n, cond = 50_001, 1e12
    port = _free_port()
    out, codes = run_ranks(_worker, world, lambda r, q: (r, world, port, n, cond, q))
    assert codes == [0] * world
    gathered = {g for _, g, _ in out}
    merged = {m for _, _, m in out}
    assert len(gathered) == 1 and len(merged) == 1  # every rank holds the same bits
    x, y, _ = oracle.gendot_dev(1234, n, cond)
    parts = np.frombuffer(out[0][1], dtype=np.float64).reshape(world, 2)
    for r in range(world):
        lo, hi = sharded.partition(n, world, r)
        assert parts[r].tobytes() == local_result(x[lo:hi].copy(), y[lo:hi].copy()).tobytes()
    got = np.frombuffer(out[0][2], dtype=np.float64)
    assert got.tobytes() == oracle.shard_merge(parts, False).tobytes()
    ex_hi, ex_lo = oracle.exact_dot(x, y)
    exact = ex_hi + ex_lo
    c = oracle.condition_dot(x, y)
    assert abs(got[0] - exact) <= oracle.bound_dot2(n, c) * abs(exact) + 2.0 ** -53 * abs(exact)


# ------------------------------------------------------------ sharded SpMV


def _matrices():
    A = problems.convdiff2d(24)
    yield sp.csr_matrix((A.val, A.col_ind, A.row_ptr), shape=(A.n, A.n))
    R = sp.random(500, 500, density=0.02, random_state=9, format="csr") + sp.eye(500)
    R.sort_indices()
    yield R.tocsr()


def _rows(M, lo, hi):
    rp = M.indptr[lo:hi + 1].astype(np.int64)
    return rp - rp[0], M.indices[rp[0]:rp[-1]].copy(), M.data[rp[0]:rp[-1]].copy()


def _plans(M, world):
    n = M.shape[0]
    plans = []
    for r in range(world):
        lo, hi = sharded.partition(n, world, r)
        rp, ci, _ = _rows(M, lo, hi)
        plans.append(sharded.HaloPlan(rp, ci, n, world, r))
    for r, p in enumerate(plans):
        p.finish([plans[s].requests[r] for s in range(world)])
    return plans


def _emulated_product(M, plans, x):
    """Each rank's send buffer, the all-to-all done by hand, the local products."""
    world, n = len(plans), M.shape[0]
    send = [x[p.lo:p.hi][p.send_index] for p in plans]
    y = np.zeros(n)
    for r, p in enumerate(plans):
        segs = []
        for s, q in enumerate(plans):
            off = int(q.send_counts[:r].sum())
            segs.append(send[s][off:off + int(q.send_counts[r])])
        x_ext = np.concatenate([x[p.lo:p.hi]] + segs)
        assert x_ext.size == p.cols
        _, _, val = _rows(M, p.lo, p.hi)
        L = sp.csr_matrix((val, p.col_ind, p.row_ptr), shape=(p.rows, p.cols))
        y[p.lo:p.hi] = L @ x_ext
    return y


@pytest.mark.parametrize("world", [1, 2, 3, 4, 7])
def test_halo_plan_reproduces_the_product_bitwise(world):
    rng = np.random.default_rng(world)
    for M in _matrices():
        n = M.shape[0]
        plans = _plans(M, world)
        for r, p in enumerate(plans):
            assert p.recv_counts[r] == 0 and p.send_counts[r] == 0
            for s in range(world):  # what s asks of r is owned by r, and r sends exactly that
                assert np.all(sharded.owner_of(plans[s].requests[r], n, world) == r)
                assert p.send_counts[s] == plans[s].recv_counts[r]
            assert p.col_ind.size == 0 or (p.col_ind.min() >= 0 and p.col_ind.max() < p.cols)
        x = rng.standard_normal(n)
        assert _emulated_product(M, plans, x).tobytes() == (M @ x).tobytes()


def test_halo_plan_rejects_bad_input():
    with pytest.raises(ValueError):  # column out of range
        sharded.HaloPlan(np.array([0, 1]), np.array([5]), 4, 2, 0)
    with pytest.raises(ValueError):  # row_ptr does not hold this rank's 2 rows
        sharded.HaloPlan(np.array([0, 1, 2, 3]), np.array([0, 1, 2]), 4, 2, 0)
    p = sharded.HaloPlan(np.array([0, 1, 2]), np.array([0, 3]), 4, 2, 0)  # rank 0 owns 0, 1
    assert [r.tolist() for r in p.requests] == [[], [3]] and p.cols == 3
    with pytest.raises(ValueError):  # rank 1 asks rank 0 for index 3, which rank 1 owns
        p.finish([np.array([], np.int64), np.array([3])])
    with pytest.raises(ValueError):  # a rank asking itself
        p.finish([np.array([1]), np.array([], np.int64)])


def _spmv_worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        A = problems.convdiff2d(32)
        M = sp.csr_matrix((A.val, A.col_ind, A.row_ptr), shape=(A.n, A.n))
        lo, hi = sharded.partition(A.n, world, rank)
        rp, ci, val = _rows(M, lo, hi)
        plan = sharded.HaloPlan(rp, ci, A.n, world, rank).exchange_requests()
        x = np.random.default_rng(3).standard_normal(A.n)  # the same x on every rank (seeded)
        xl = torch.from_numpy(x[lo:hi].copy())
        send = xl[torch.from_numpy(plan.send_index.astype(np.int64))]
        halo = torch.zeros(plan.cols - plan.rows, dtype=torch.float64)
        dist.all_to_all_single(halo, send, output_split_sizes=plan.recv_counts.tolist(),
                               input_split_sizes=plan.send_counts.tolist())
        x_ext = np.concatenate([xl.numpy(), halo.numpy()])
        y = sp.csr_matrix((val, plan.col_ind, plan.row_ptr), shape=(plan.rows, plan.cols)) @ x_ext
        q.put((rank, lo, hi, y.tobytes()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_sharded_spmv(world):
    """The halo plan's request exchange and the per-product all-to-all over
    gloo ranks; the row blocks' products equal the whole product bit for bit."""
    port = _free_port()
    out, codes = run_ranks(_spmv_worker, world, lambda r, q: (r, world, port, q))
    assert codes == [0] * world
    A = problems.convdiff2d(32)
    M = sp.csr_matrix((A.val, A.col_ind, A.row_ptr), shape=(A.n, A.n))
    want = M @ np.random.default_rng(3).standard_normal(A.n)
    for rank, lo, hi, yb in out:
        assert np.frombuffer(yb, dtype=np.float64).tobytes() == want[lo:hi].tobytes()


# ------------------------------------------------------------ sharded solver
def local_result_c128(x, y):
    """(hi.re, hi.im, lo.re, lo.im) of the reference's sequential complex
    Dot2, sum conj(x_i) y_i, of one slice."""
    out = np.zeros(6)
    oracle.oro().oro_dot2_seq_c128(x.shape[0], oracle._ptr(x), oracle._ptr(y), oracle._ptr(out))
    hr, lr = two_sum(out[2], out[4])
    hi, li = two_sum(out[3], out[5])
    return np.array([hr, hi, lr, li])


class _HostOps:
    """The sharded solver's vector operations on host slices for these CPU
    tests: element-wise work in numpy, each rank's Dot2 from the oracle,
    the (hi, lo) results exchanged over gloo and merged with the library's
    host merge (one rank: no exchange)."""

    def __init__(self, n_local, world, dtype=np.float64):
        self.n, self.world, self.dtype = n_local, world, np.dtype(dtype)
        self.cplx = self.dtype == np.complex128

    def new(self):
        return np.zeros(self.n, dtype=self.dtype)

    def dot(self, x, y):
        local = torch.from_numpy(local_result_c128(x, y) if self.cplx else local_result(x, y))
        w = local.numel()
        if self.world == 1:
            merged = local.numpy()
        else:
            gathered = torch.zeros(w * self.world, dtype=torch.float64)
            dist.all_gather_into_tensor(gathered, local)
            merged = sharded.merge_gathered_cpu(gathered.numpy(), self.cplx)
        return complex(merged[0], merged[1]) if self.cplx else float(merged[0])

    def norm(self, x):
        return float(np.sqrt(self.dot(x, x).real))

    def axpby(self, a, x, b, y):
        y[:] = a * x + b * y

    def copy(self, x, y):
        y[:] = x

    def fill(self, y, v):
        y[:] = v


class _HostCSR:
    def __init__(self, plan, val):
        self.plan = plan
        self.M = sp.csr_matrix((val, plan.col_ind, plan.row_ptr), shape=(plan.rows, plan.cols))

    def apply(self, x, y):
        p = self.plan
        tdt = torch.complex128 if np.iscomplexobj(x) else torch.float64
        halo = torch.zeros(p.cols - p.rows, dtype=tdt)
        if p.world > 1:
            send = torch.from_numpy(x[p.send_index.astype(np.int64)].copy())
            dist.all_to_all_single(halo, send, output_split_sizes=p.recv_counts.tolist(),
                                   input_split_sizes=p.send_counts.tolist())
        y[:] = self.M @ np.concatenate([x, halo.numpy()])


def _system(method):
    if method == "bicgstabl_c128":
        A = problems.helmholtz2d(24, ppw=10.0, damping=0.5)
        return A, problems.rhs_uniform(A.n, 13, complex_=True)
    A = problems.convdiff2d(24)
    return A, problems.rhs_uniform(A.n, 11)


def _solve_rows(world, rank, method="bicgstabl"):
    A, b = _system(method)
    M = sp.csr_matrix((A.val, A.col_ind, A.row_ptr), shape=(A.n, A.n))
    lo, hi = sharded.partition(A.n, world, rank)
    rp, ci, val = _rows(M, lo, hi)
    plan = sharded.HaloPlan(rp, ci, A.n, world, rank)
    plan = plan.exchange_requests() if world > 1 else plan.finish([np.zeros(0)])
    x = np.zeros(hi - lo, dtype=b.dtype)
    ops, op = _HostOps(hi - lo, world, b.dtype), _HostCSR(plan, val)
    if method.startswith("bicgstabl"):
        ok, it, rel = sharded.bicgstabl(ops, op, b[lo:hi].copy(), x, L=2, rel_tol=1e-10, max_iters=2000)
    else:
        ok, it, rel = sharded.gmres(ops, op, b[lo:hi].copy(), x, m=20, rel_tol=1e-10, max_iters=2000,
                                    reorthogonalize=(method == "gmres_reorth"))
    return ok, it, rel, lo, hi, x


def _solver_worker(rank, world, port, method, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ok, it, rel, lo, hi, x = _solve_rows(world, rank, method)
        q.put((rank, ok, it, rel, lo, hi, x.tobytes(), str(x.dtype)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


METHODS = ["bicgstabl", "gmres", "gmres_reorth", "bicgstabl_c128"]


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_sharded_solvers(world, method):
    """BiCGStab(2) and GMRES(20) on row blocks of a 24 x 24
    convection-diffusion system, and complex BiCGStab(2) on a 24 x 24
    damped Helmholtz system (conj-linear inner products in the reference's
    argument order), across gloo ranks: every rank stops after
    the same iteration with the same residual ratio (the merged reductions
    are identical on every rank), the assembled solution meets the
    tolerance in a binary64 residual, and the iteration count is the
    one-rank solve's to within a cycle."""
    port = _free_port()
    out, codes = run_ranks(_solver_worker, world, lambda r, q: (r, world, port, method, q))
    assert codes == [0] * world
    out = sorted(out)
    assert all(o[1] for o in out)
    assert len({(o[2], o[3]) for o in out}) == 1
    A, b = _system(method)
    x = np.zeros(A.n, dtype=b.dtype)
    for _, _, _, _, lo, hi, xb, dt in out:
        x[lo:hi] = np.frombuffer(xb, dtype=dt)
    assert np.linalg.norm(b - A.matvec(x)) <= 1.5e-10 * np.linalg.norm(b)
    ok1, it1, _, _, _, x1 = _solve_rows(1, 0, method)
    assert ok1 and abs(out[0][2] - it1) <= (2 if method.startswith("bicgstabl") else 20)
    assert np.abs(x - x1).max() <= 1e-8 * np.abs(x1).max()
