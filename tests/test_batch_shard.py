"""Multi-GPU batches shard by garment with no collective on the data path: every rank drapes the garments that
``batch.shard`` gives it. Checked here on CPU: the split is a partition, deterministic and balanced, and two gloo
ranks that compute it independently agree on it (each rank gathers the others' lists)."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from drape_b200 import batch


def _sizes(count=64, seed=5):
    rng = np.random.default_rng(seed)
    return [int(round(x)) for x in np.exp(rng.uniform(np.log(2000), np.log(40000), count))]


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_shard_is_a_balanced_partition(world):
    sizes = _sizes()
    parts = batch.shard(sizes, world)
    assert len(parts) == world
    flat = sorted(g for p in parts for g in p)
    assert flat == list(range(len(sizes)))
    loads = [sum(sizes[g] for g in p) for p in parts]
    # Largest-first onto the least-loaded rank: the spread is at most one garment.
    assert max(loads) - min(loads) <= max(sizes)
    assert parts == batch.shard(sizes, world)


def test_shard_more_ranks_than_garments():
    parts = batch.shard([10, 20], 4)
    assert sorted(g for p in parts for g in p) == [0, 1]
    assert sum(1 for p in parts if not p) == 2


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = batch.shard(_sizes(), world)[rank]
        lists = [None] * world
        dist.all_gather_object(lists, mine)
        out[rank] = lists
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_split():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    expect = batch.shard(_sizes(), world)
    assert out[0] == out[1] == expect
