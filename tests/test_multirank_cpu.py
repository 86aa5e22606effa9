"""The multi-GPU path is replicas (one solve per rank, no data-path
collective); its host logic is tested here with two gloo ranks on CPU:
the job time is the maximum over ranks, every rank solves the same operator
with its own right-hand side, and the reference arm runs on rank 0 only."""
import io
import os
import sys
from contextlib import redirect_stdout
from pathlib import Path

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp  # noqa: F401  (spawned ranks)
from rank_utils import run_ranks

ROOT = Path(__file__).resolve().parent.parent


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ws, r, local = bench.dist_init(None)
        t = bench.max_over_ranks(torch, dist, 1.0 + 2.0 * rank, "cpu")
        A0, b0 = bench.solver_problem(0)
        A, b = bench.solver_problem(r)
        same_op = bool(np.array_equal(A.val, A0.val) and np.array_equal(A.col_ind, A0.col_ind))
        buf = io.StringIO()

        class Args:
            workload = "solver"
            steps = 1
            warmup = 1
        with redirect_stdout(buf):
            if r != 0:
                bench.run_reference(Args, ws, r)  # rank 0 would time the CPU reference; others return at once
        q.put((r, ws, t, same_op, bool(r == 0 or not np.array_equal(b, b0)), buf.getvalue()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_replica_logic():
    world = 2
    port = 29500 + (os.getpid() % 2000)
    out, codes = run_ranks(_worker, world, lambda r, q: (r, world, port, q))
    assert codes == [0] * world
    for r, ws, t, same_op, own_rhs, printed in out:
        assert ws == world
        assert t == pytest.approx(1.0 + 2.0 * (world - 1))  # the slowest rank's time, on every rank
        assert same_op and own_rhs
        assert printed == ""  # the reference arm prints on rank 0 only
