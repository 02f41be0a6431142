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


def _shard_rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, os.path.join(ROOT, "niamh-mpcd_b200"))
    from mpcd_b200 import workloads as W
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sides = W.ensemble_sides(512)
        work = [10 * int(L) ** 3 for L in sides]
        mine = W.shard_boxes(work, world, rank)
        # every rank learns every rank's boxes, as a collective would carry them
        got = [None] * world
        dist.all_gather_object(got, mine)
        out[rank] = got
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_ensemble_boxes_split_once_and_balanced_across_ranks(world):
    """bench.py --workload ensemble with N > 1 splits the one ensemble by
    box: every rank computes the same split, each box goes to exactly one
    rank, and the ranks' particle counts differ by at most one box."""
    sys.path.insert(0, os.path.join(ROOT, "niamh-mpcd_b200"))
    from mpcd_b200 import workloads as W
    port = 29600 + world + os.getpid() % 700
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_shard_rank, args=(r, world, port, out))
                 for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
        assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
        res = dict(out)
    views = [res[r] for r in range(world)]
    assert all(v == views[0] for v in views)  # the same split on every rank
    parts = views[0]
    flat = sorted(b for p in parts for b in p)
    assert flat == list(range(512))
    work = [10 * int(L) ** 3 for L in W.ensemble_sides(512)]
    loads = [sum(work[b] for b in p) for p in parts]
    assert max(loads) - min(loads) <= max(work)


def test_shard_boxes_edge_cases():
    sys.path.insert(0, os.path.join(ROOT, "niamh-mpcd_b200"))
    from mpcd_b200 import workloads as W
    assert W.shard_boxes([5, 1, 1], 1, 0) == [0, 1, 2]
    # more ranks than boxes: the surplus ranks get none
    assert [W.shard_boxes([3, 2], 3, r) for r in range(3)] == [[0], [1], []]
    # the largest box alone, the small ones together
    assert [W.shard_boxes([8, 1, 1, 1, 1], 2, r) for r in range(2)] == [[0], [1, 2, 3, 4]]
    with pytest.raises(ValueError):
        W.shard_boxes([1], 2, 2)
