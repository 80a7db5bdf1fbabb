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
