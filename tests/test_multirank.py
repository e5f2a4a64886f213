"""The multi-process side of `bench.py --gpus N` on CPU: two gloo ranks (one process each, as under
torchrun) agree on the max-over-ranks time and the job-total counts that the replicas report, and
every rank other than 0 leaves the reference arm without work. No GPU."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import bench
    dist = bench.dist_setup(world)
    ms = 10.0 + 5.0 * rank                    # each replica's device time
    launches = 100 * (rank + 1)
    t = bench.dist_max(dist, ms)
    n = bench.dist_sum(dist, launches)
    dist.barrier()
    dist.destroy_process_group()

    class A:
        steps = 1
        gpus = world
    rc = bench.run_reference(A()) if rank != 0 else 0   # rank 0 would run the CPU oracle: skipped here
    out.put((rank, t, n, rc))


def test_two_gloo_ranks_reduce_time_and_counts():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [15.0, 15.0]        # the slowest replica's time, on every rank
    assert [r[2] for r in res] == [300.0, 300.0]      # launches summed over the job
    assert res[1][3] == 0                            # rank 1 leaves the reference arm at once
