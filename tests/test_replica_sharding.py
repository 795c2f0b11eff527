"""Replicas across ranks (asd_replicas): the split covers every replica once and balances spins,
and with two gloo ranks on CPU the rows come back to rank 0 in global order and the time is
the max over ranks.  No GPU is used."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import asd_replicas as R


def _batch_sizes(nrep=96, edges=(16, 24, 32, 48, 64), seed=4):
    """Spin counts of the uneven sc replica batch (same draw as asd_lattice.replica_batch)."""
    L = np.random.default_rng(seed).choice(np.asarray(edges), size=nrep)
    return [int(l) ** 3 for l in L]


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_shard_covers_each_replica_once_and_balances(world):
    sizes = _batch_sizes()
    parts = [R.shard(sizes, r, world) for r in range(world)]
    flat = sorted(g for p in parts for g in p)
    assert flat == list(range(len(sizes)))
    loads = [sum(sizes[g] for g in p) for p in parts]
    # greedy largest-first: no rank exceeds the mean by more than the largest replica
    assert max(loads) - sum(loads) / world <= max(sizes)
    assert parts == [R.shard(sizes, r, world) for r in range(world)]     # deterministic


def test_shard_rejects_bad_rank():
    with pytest.raises(ValueError):
        R.shard([1, 2], 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, sizes, out):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mine = R.shard(sizes, rank, world)
        rows = [{"g": g, "m": 1.0 / (1 + g), "rank": rank} for g in mine]
        got = R.gather_rows(rows, mine, dist, len(sizes))
        t = R.allmax(0.25 * (rank + 1), dist)
        if rank == 0:
            out.put((got, t))
        else:
            out.put(("other", got, t))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_gather_rows_in_global_order():
    sizes = _batch_sizes(nrep=23)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, sizes, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    root = [r for r in res if r[0] != "other"][0]
    other = [r for r in res if r[0] == "other"][0]
    rows, t = root
    assert [r["g"] for r in rows] == list(range(len(sizes)))
    assert all(r["m"] == 1.0 / (1 + r["g"]) for r in rows)
    assert {r["rank"] for r in rows} == {0, 1}
    for g, r in enumerate(rows):
        assert g in R.shard(sizes, r["rank"], 2)
    assert t == 0.5 and other[2] == 0.5            # max over ranks on both
    assert other[1] is None                         # rows only on rank 0
