"""Multi-rank ensemble host logic on CPU (gloo, world size 2).

Each rank takes its shard of the tissue batch (longest-processing-time
balance, no collective on the data path) and the timing reduction is a max
over ranks, as bench.py does under torchrun. The ranks check that the shards
partition the batch and agree on the reduced values.
"""
import os

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from epi_b200 import tissue as T
from epi_b200.ensemble import imbalance, shard_tissues


def _rank_main(rank, world, port, sizes, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    import torch
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        shards = shard_tissues(sizes, world)
        mine = shards[rank]
        # every rank computes the same partition without communicating
        gathered = [None] * world
        dist.all_gather_object(gathered, sorted(mine))
        # device time of this rank's shard (a stand-in proportional to its
        # particles) reduced by max, as bench.py reduces its CUDA-event time
        t = torch.tensor([float(sum(sizes[i] for i in mine))], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        out[rank] = (gathered, float(t.item()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_two_rank_shards_partition_the_batch(world):
    sizes = [t.n for t in T.config4(n_tissues=64)]
    port = 29500 + (os.getpid() % 1000)
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(world, port, sizes, out), nprocs=world, join=True)
        res = dict(out)
    g0, tmax0 = res[0]
    g1, tmax1 = res[1]
    assert g0 == g1
    flat = sorted(i for shard in g0 for i in shard)
    assert flat == list(range(len(sizes)))
    loads = [sum(sizes[i] for i in shard) for shard in g0]
    assert tmax0 == tmax1 == max(loads)
    assert imbalance(sizes, shard_tissues(sizes, world)) < 1.01


def _failing_rank_main(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    import torch
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=5))
    if rank == 1:
        # the failing rank: leaves between steps, before the timing reduction
        out[rank] = "left"
        os._exit(0)
    t = torch.tensor([1.0], dtype=torch.float64)
    try:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        out[rank] = "completed"
    except Exception as e:  # the bounded wait ends with an error, not a hang
        out[rank] = f"error: {type(e).__name__}"


def test_rank_that_leaves_is_detected_by_the_bounded_wait():
    """A rank that exits between steps: the surviving rank's next collective
    (the max-over-ranks timing reduction bench.py performs) ends with an
    error within the process group's timeout instead of waiting forever."""
    port = 29700 + (os.getpid() % 200)
    with mp.Manager() as m:
        out = m.dict()
        ctx = mp.get_context("spawn")
        procs = [ctx.Process(target=_failing_rank_main, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=60)
        alive = [p.is_alive() for p in procs]
        for p in procs:
            if p.is_alive():
                p.kill()
        res = dict(out)
    assert not any(alive), "a rank hung"
    assert res.get(1) == "left"
    assert str(res.get(0, "")).startswith("error"), res


def test_weak_scaling_job_per_rank():
    """bench.py's N-GPU ensemble job: N x 512 tissues of the same generator,
    balanced over the ranks, each rank generating only its own. The ranks'
    tissues partition the job, the first 512 tissues are the 1-GPU batch,
    and every rank holds about one GPU's worth (weak scaling)."""
    import bench
    world, per = 2, 64
    one, n_one, nt_one, _, _ = bench.rank_workload("ensemble", per, 1, 0)
    assert nt_one == per and n_one == sum(t.n for t in one)
    parts = [bench.rank_workload("ensemble", per, world, r) for r in range(world)]
    n_job = parts[0][1]
    assert all(p[1] == n_job and p[2] == world * per for p in parts)
    names = sorted(int(t.name[3:-1]) for p in parts for t in p[0])
    assert names == list(range(world * per))
    assert sum(t.n for p in parts for t in p[0]) == n_job
    loads = [sum(t.n for t in p[0]) for p in parts]
    assert max(loads) / (n_job / world) < 1.05
    by_name = {t.name: t for p in parts for t in p[0]}
    for t in one:
        assert np.array_equal(by_name[t.name].x, t.x)
    # a single tissue runs as one replica per rank
    mine, n_job1, nt1, _, _ = bench.rank_workload("c1", per, world, 1)
    assert len(mine) == 1 and nt1 == world and n_job1 == world * mine[0].n


def _gather_rank_main(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    from oracle import oracle as O
    from epi_b200.ensemble import gather_results, split_by_tissue
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        job = _gather_job()
        mine = shard_tissues([t.n for t in job], world)[rank]
        # this rank's shard stepped as one batch (the oracle stands in for the
        # rank's GPU context), its positions split back into tissues
        xs, ys, zs = [], [], []
        for i in mine:
            ora = O.OracleTissue(job[i])
            assert ora.step(5) == 0
            x, y, z = ora.positions()
            xs.append(x), ys.append(y), zs.append(z)
        cat = [np.concatenate(a) for a in (xs, ys, zs)]
        per = split_by_tissue(cat, [job[i].n for i in mine])
        res = gather_results(mine, per, dist)
        out[rank] = res
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _gather_job():
    return [T.config1(s) for s in range(3)] + [T.layered_tissue(16 + 8 * (s % 2), 2, s)
                                               for s in range(3)]


def test_two_rank_result_gather_is_in_job_order():
    """bench.py's multi-GPU job returns its results to rank 0: each rank's
    per-tissue positions (and adjoint gradients alike) assembled in job order
    equal the tissues run one batch on one device, tissue by tissue."""
    world = 2
    port = 29900 + (os.getpid() % 90)
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_gather_rank_main, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[1] is None
    got = res[0]
    job = _gather_job()
    assert len(got) == len(job)
    from oracle import oracle as O
    for t, r in zip(job, got):
        ora = O.OracleTissue(t)
        assert ora.step(5) == 0
        for a, b in zip(ora.positions(), r):
            assert np.array_equal(a, b)
