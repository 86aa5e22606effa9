"""Spawned gloo ranks for the CPU multi-process tests: start, collect one
queue message per rank, join; whatever happens, no rank outlives the test
(a rank blocked in a collective after another died is terminated)."""
import torch.multiprocessing as mp


def run_ranks(target, world: int, make_args, timeout: float = 300.0):
    """Run ``target(*make_args(rank, queue))`` in ``world`` spawned
    processes; returns (messages in arrival order, exit codes by rank)."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=target, args=make_args(r, q)) for r in range(world)]
    try:
        for p in procs:
            p.start()
        out = [q.get(timeout=timeout) for _ in range(world)]
        for p in procs:
            p.join(timeout=60)
        return out, [p.exitcode for p in procs]
    finally:
        for p in procs:
            if p.is_alive():
                p.terminate()
                p.join(5)
