"""World-size-2 tests of the bench's multi-rank path on CPU (gloo).

Every rank solves its own seeded replica, so the only cross-rank steps are
the timing reductions: the job's time is the maximum over ranks and its work
the sum, and the reference arm runs on rank 0 alone.
"""
import os
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, out):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    w, r, local = bench.dist_setup(world)
    assert (w, r, local) == (world, rank, rank)
    mx = bench.barrier_max([1.0 + rank, 10.0 - rank], w)
    sm = bench.barrier_sum([float(rank + 1)], w)
    bench.barrier(w)
    # the reference arm: ranks other than 0 return without work
    if rank != 0:
        sys.argv = ["bench.py", "--impl", "reference"]
        assert bench.run_reference(bench.parse_args()) is None
    import torch.distributed as dist
    dist.destroy_process_group()
    out.put((rank, mx, sm))


@pytest.mark.timeout(120)
def test_two_ranks_reduce_timing_over_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=100) for _ in procs)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    for rank, mx, sm in res:
        assert mx == [2.0, 10.0]     # max over ranks
        assert sm == [3.0]           # 1 + 2
