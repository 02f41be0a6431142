"""The N > 1 path of bench.py runs one independent replica box per rank
(the solvent timestep has no data exchange between replicas): the job's time
is the maximum over ranks and its rate sums the ranks' particles.  This runs
that host logic on two CPU ranks over gloo."""
import os
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local_ms = [12.5, 20.0][rank]  # the slower rank sets the job time
        t = bench.max_over_ranks(local_ms, world, device="cpu")
        rate = bench.job_rate(1000, world, 10, t / 1e3)
        out[rank] = (t, rate)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_replica_ranks_take_the_slowest_time():
    port = 29500 + os.getpid() % 1000
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
        assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
        res = dict(out)
    assert res[0] == res[1]
    t, rate = res[0]
    assert t == pytest.approx(20.0)
    assert rate == pytest.approx(1000 * 2 * 10 / 0.020)
