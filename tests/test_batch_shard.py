"""Multi-GPU batches shard by garment with no collective on the data path: every rank drapes the garments that
``batch.shard`` gives it. Checked here on CPU: the split is a partition, deterministic and balanced, two gloo ranks
that compute it independently agree on it (each rank gathers the others' lists), and two gloo ranks that each drape
their share (on the oracle, standing in for each rank's GPU) and gather the results on rank 0 reproduce the garments
draped in one process, position for position."""
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


def _garments():
    """Four small seeded tubes on their own bodies (uneven sizes), each its own scene."""
    from drape_b200 import scenes as S
    return [S.body_tube(7000 + k, n, field_n=32) for k, n in enumerate((300, 900, 500, 700))]


def _drape_share(indices, frames=20):
    """Each garment of `indices` on its own oracle solver: 10 frames Assembling, then Settling; final positions."""
    import oracle
    out = {}
    scenes = _garments()
    for g in indices:
        sc = scenes[g]
        o = oracle.OracleSolver()
        o.build(sc)
        gid = sc.garments[0].id
        o.set_phase(gid, 0)
        for f in range(frames):
            if f == 10:
                o.set_phase(gid, 1)
            o.step(1.0 / 60.0, 1, 2)
        out[g] = o.positions()
    return out


def _drape_rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sizes = [sc.garments[0].vertex_count for sc in _garments()]
        mine = batch.shard(sizes, world)[rank]
        results = _drape_share(mine)  # no data crosses between ranks while draping
        gathered = [None] * world if rank == 0 else None
        dist.gather_object(results, gathered, dst=0)
        if rank == 0:
            merged = {}
            for part in gathered:
                merged.update(part)
            out["merged"] = {k: v.tolist() for k, v in merged.items()}
            out["shares"] = batch.shard(sizes, world)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_drape_their_shares_and_gather(oracle_mod):
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    procs = [ctx.Process(target=_drape_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
        assert p.exitcode == 0
    merged = out["merged"]
    assert sorted(merged) == [0, 1, 2, 3]
    assert all(len(share) > 0 for share in out["shares"])
    alone = _drape_share(range(4))
    for g in range(4):
        assert np.array_equal(np.asarray(merged[g]), alone[g]), g
