"""GPU checks of the sharded reductions (high_precision_blas1_b200/sharded.py,
hpb_shard_merge):
  * the device merge gives the host merge's bits (hpb_shard_merge_cpu) and
    the oracle's restatement's;
  * slices of one vector reduced by hpb_dot2_f64 and merged on the device
    (the all-gather replaced by the slices' results side by side, one
    process, nothing waits on anything) equal the oracle's merge of those
    results and stay within the Dot2 bound of the exact dot product, for 2
    to 8 slices;
  * ShardedReductions on one rank -- without a process group, and over a
    one-rank NCCL group (the all-gather runs) -- returns the single-GPU
    reduction's bits (one result merges to itself);
  * ShardedCSR: 1-4 emulated ranks in one process (device gathers and
    row-block SpMVs, the all-to-all replaced by copies) and one rank over
    NCCL give the single-GPU SpMV's bits."""
import os

import numpy as np
import pytest

import oracle
from gpu_utils import dev, gendot, red
from high_precision_blas1_b200 import _lib, sharded

pytestmark = pytest.mark.gpu


def two_sum(a, b):
    s = a + b
    bv = s - a
    av = s - bv
    return s, (b - bv) + (a - av)


@pytest.mark.parametrize("is_complex", [False, True])
def test_device_merge_matches_host_merge(gpu, is_complex):
    ctx, torch = gpu
    rng = np.random.default_rng(11)
    comps = 2 if is_complex else 1
    for count in (1, 2, 3, 5, 8, 9, 64):
        pairs = np.zeros((count, 2 * comps))
        for k in range(count):
            for q in range(comps):
                a = rng.standard_normal() * 10.0 ** int(rng.integers(-30, 30))
                b = rng.standard_normal() * 10.0 ** int(rng.integers(-30, 30))
                pairs[k, q], pairs[k, comps + q] = two_sum(a, b)
        d_in = dev(torch, pairs.reshape(-1))
        d_out = torch.zeros(4, dtype=torch.float64, device="cuda")
        ctx.check(_lib.lib.hpb_shard_merge(ctx.h, count, int(is_complex), d_in.data_ptr(), d_out.data_ptr()))
        got = d_out[:2 * comps].cpu().numpy()
        assert got.tobytes() == sharded.merge_gathered_cpu(pairs, is_complex).tobytes()
        assert got.tobytes() == oracle.shard_merge(pairs, is_complex).tobytes()


def test_device_merge_rejects_bad_arguments(gpu):
    ctx, torch = gpu
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    invalid = -1  # HPB_ERROR_INVALID_VALUE
    assert _lib.lib.hpb_shard_merge(ctx.h, 0, 0, buf.data_ptr(), buf.data_ptr()) == invalid
    assert _lib.lib.hpb_shard_merge(ctx.h, 2, 0, None, buf.data_ptr()) == invalid
    assert _lib.lib.hpb_shard_merge(ctx.h, 2, 0, buf.data_ptr() + 4, buf.data_ptr()) == invalid
    assert _lib.lib.hpb_shard_merge_cpu(0, 0, None, None) == invalid


@pytest.mark.parametrize("world", [2, 3, 5, 8])
def test_slices_reduced_and_merged_on_device(gpu, world):
    ctx, torch = gpu
    n, cond = 1_000_003, 1e16
    x, y = gendot(77, n, cond)
    dx, dy = dev(torch, x), dev(torch, y)
    parts = torch.zeros(2 * world, dtype=torch.float64, device="cuda")
    for r in range(world):
        lo, hi = sharded.partition(n, world, r)
        ctx.check(_lib.lib.hpb_dot2_f64(ctx.h, hi - lo, dx.data_ptr() + 8 * lo, dy.data_ptr() + 8 * lo,
                                        parts.data_ptr() + 16 * r))
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    ctx.check(_lib.lib.hpb_shard_merge(ctx.h, world, 0, parts.data_ptr(), out.data_ptr()))
    hparts = parts.cpu().numpy()
    got = out.cpu().numpy()
    assert got.tobytes() == oracle.shard_merge(hparts, False).tobytes()
    ex_hi, ex_lo = oracle.exact_dot(x, y)
    exact = ex_hi + ex_lo
    c = oracle.condition_dot(x, y)
    assert abs(got[0] - exact) <= oracle.bound_dot2(n, c) * abs(exact) + 2.0 ** -53 * abs(exact)


TYPES = {"f32": (np.float32, "float32"), "f64": (np.float64, "float64"),
         "c64": (np.complex64, "complex64"), "c128": (np.complex128, "complex128")}


def _vectors(t, n, seed):
    rng = np.random.default_rng(seed)
    npt = TYPES[t][0]
    if np.issubdtype(npt, np.complexfloating):
        x = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(npt)
        y = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(npt)
    else:
        x = rng.standard_normal(n).astype(npt)
        y = rng.standard_normal(n).astype(npt)
    return x, y


def _check_one_rank(ctx, torch, S):
    for t in TYPES:
        x, y = _vectors(t, 300_007, 3)
        dx, dy = dev(torch, x), dev(torch, y)
        cplx = t in ("c64", "c128")
        w = 4 if cplx else 2
        want = red(ctx, "dot2", dx, dy)[:w]
        assert S.result("dot", dx, dy).tobytes() == want.tobytes()
        assert S.result("sum", dx).tobytes() == red(ctx, "sum2", dx)[:w].tobytes()
        assert S.result("asum", dx).tobytes() == red(ctx, "asum2", dx)[:2].tobytes()
        v = S.dot(dx, dy)
        assert (complex(want[0], want[1]) if cplx else want[0]) == v
        assert S.norm(dx) == float(np.sqrt(red(ctx, "dot2", dx, dx)[0]))


def test_one_rank_without_process_group(gpu):
    ctx, torch = gpu
    S = sharded.ShardedReductions(0)
    try:
        _check_one_rank(ctx, torch, S)
    finally:
        S.close()


def test_one_rank_nccl_group(gpu):
    ctx, torch = gpu
    import torch.distributed as dist
    port = 29900 + os.getpid() % 500
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            device_id=torch.device("cuda", 0))
    try:
        S = sharded.ShardedReductions(0)
        try:
            assert S.world == 1
            _check_one_rank(ctx, torch, S)
        finally:
            S.close()
    finally:
        torch.cuda.synchronize()
        dist.destroy_process_group()


# ------------------------------------------------------------ sharded SpMV
def _global_spmv(ctx, torch, A, x):
    d = [dev(torch, a) for a in (A.row_ptr, A.col_ind, A.val)]
    y = torch.zeros(A.n, dtype=torch.float64, device="cuda")
    ctx.check(_lib.lib.hpb_csr_spmv_f64(ctx.h, A.n, A.n, A.nnz, d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(),
                                        1.0, x.data_ptr(), 0.0, y.data_ptr()))
    return y.cpu().numpy()


def _rank_rows(A, lo, hi):
    rp = A.row_ptr[lo:hi + 1].astype(np.int64)
    return rp - rp[0], A.col_ind[rp[0]:rp[-1]].copy(), A.val[rp[0]:rp[-1]].copy()


@pytest.mark.parametrize("world", [1, 2, 3, 4])
def test_sharded_spmv_emulated_ranks(gpu, world):
    """Every rank's ShardedCSR in one process on one GPU: the device gathers
    of the send lists and the row-block SpMVs run through the library; only
    the all-to-all is replaced by copies between the ranks' buffers (nothing
    waits on anything).  The row blocks equal the whole SpMV bit for bit."""
    ctx, torch = gpu
    from high_precision_blas1_b200 import problems
    A = problems.convdiff2d(200)
    x = np.random.default_rng(8).standard_normal(A.n)
    want = _global_spmv(ctx, torch, A, dev(torch, x))
    plans, ops = [], []
    for r in range(world):
        lo, hi = sharded.partition(A.n, world, r)
        rp, ci, _ = _rank_rows(A, lo, hi)
        plans.append(sharded.HaloPlan(rp, ci, A.n, world, r))
    for r, p in enumerate(plans):
        p.finish([plans[s].requests[r] for s in range(world)])
    for r, p in enumerate(plans):
        rp, ci, val = _rank_rows(A, p.lo, p.hi)
        ops.append(sharded.ShardedCSR(0, rp, ci, val, A.n, plan=p))
    xs = [dev(torch, x[p.lo:p.hi]) for p in plans]
    ys = [torch.zeros(p.rows, dtype=torch.float64, device="cuda") for p in plans]
    try:
        for op, xl in zip(ops, xs):
            op.gather_send(xl)
        for r, (op, p) in enumerate(zip(ops, plans)):  # the all-to-all, by hand
            at = p.rows
            for s, q in enumerate(plans):
                off, cnt = int(q.send_counts[:r].sum()), int(q.send_counts[r])
                assert cnt == int(p.recv_counts[s])
                op.x_ext[at:at + cnt].copy_(ops[s].send_buf[off:off + cnt])
                at += cnt
            assert at == p.cols
        for op, xl, yl in zip(ops, xs, ys):
            op.local_spmv(xl, yl)
        got = np.concatenate([y.cpu().numpy() for y in ys])
        assert got.tobytes() == want.tobytes()
    finally:
        for op in ops:
            op.close()


def test_sharded_spmv_one_rank_nccl_group(gpu):
    ctx, torch = gpu
    import torch.distributed as dist
    from high_precision_blas1_b200 import problems
    A = problems.convdiff2d(128)
    x = np.random.default_rng(9).standard_normal(A.n)
    want = _global_spmv(ctx, torch, A, dev(torch, x))
    port = 29400 + os.getpid() % 500
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            device_id=torch.device("cuda", 0))
    try:
        op = sharded.ShardedCSR(0, A.row_ptr, A.col_ind, A.val, A.n)
        try:
            y = torch.zeros(A.n, dtype=torch.float64, device="cuda")
            op.apply(dev(torch, x), y)
            assert y.cpu().numpy().tobytes() == want.tobytes()
            assert op.plan.cols == A.n and int(op.plan.send_counts.sum()) == 0
        finally:
            op.close()
    finally:
        torch.cuda.synchronize()
        dist.destroy_process_group()


def test_sharded_bicgstabl_one_rank(gpu):
    """The sharded BiCGStab(4) driver on one rank (library kernels for the
    element-wise work, the reductions and the row-block SpMV): it meets the
    tolerance in a binary64 residual and takes the library's plain
    BiCGStab(4) iteration count to within a cycle (the same recurrences)."""
    ctx, torch = gpu
    import ctypes as C
    from high_precision_blas1_b200 import problems
    A = problems.convdiff2d(64)
    b = problems.rhs_uniform(A.n, 12)
    R = sharded.ShardedReductions(0)
    op = sharded.ShardedCSR(0, A.row_ptr, A.col_ind, A.val, A.n)
    try:
        x = torch.zeros(A.n, dtype=torch.float64, device="cuda")
        ok, it, rel = sharded.bicgstabl(sharded.ShardedVectorOps(R, A.n), op, dev(torch, b), x, L=4, rel_tol=1e-10,
                                        max_iters=4000)
        xs = x.cpu().numpy()
        assert ok and rel <= 1e-10
        assert np.linalg.norm(b - A.matvec(xs)) <= 1.5e-10 * np.linalg.norm(b)
        d = [dev(torch, a) for a in (A.row_ptr, A.col_ind, A.val, b, np.zeros(A.n))]
        p = _lib.solver_params("bicgstabl", basis=4, rel_tol=1e-10, max_iters=4000)
        rep = _lib.hpb_solver_report()
        st = _lib.lib.hpb_csr_solve_f64(C.byref(p), A.n, A.nnz, *[a.data_ptr() for a in d], C.byref(rep), None, 0)
        assert st == 0 and abs(rep.iters - it) <= 4, (rep.iters, it)
    finally:
        op.close()
        R.close()
