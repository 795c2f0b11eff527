"""Independent replicas across GPUs: one process per GPU, each advancing its own share of the
replicas with no exchange during the run (the replicas of an M(T) sweep never interact).

* shard()      deterministic split of the replicas over ranks, balanced by spin count;
* gather_rows  per-replica result rows to rank 0, back in global replica order;
* allmax       the max over ranks of a time (every rank's work ends when the slowest does).

Each replica keeps the Philox stream of its global index, so its trajectory is the same
whatever rank runs it.  The collectives go through torch.distributed (NCCL between GPUs, gloo
on CPU); with no process group every helper is the single-process identity.
"""
from __future__ import annotations

from typing import List, Optional, Sequence


def shard(sizes: Sequence[int], rank: int, world: int) -> List[int]:
    """Global indices of the replicas that `rank` runs.  Largest first, each replica goes to the
    rank with the fewest spins so far (ties to the lower rank); the result is sorted."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must lie in [0, world)")
    load = [0] * world
    own: List[List[int]] = [[] for _ in range(world)]
    for r in sorted(range(len(sizes)), key=lambda k: (-int(sizes[k]), k)):
        q = min(range(world), key=lambda w: (load[w], w))
        own[q].append(r)
        load[q] += int(sizes[r])
    return sorted(own[rank])


def gather_rows(rows: Sequence[dict], mine: Sequence[int], dist=None, nrep: Optional[int] = None) -> Optional[list]:
    """Rows of this rank's replicas (in `mine` order) -> on rank 0 the rows of every replica in
    global order; None on the other ranks."""
    if dist is None:
        return list(rows)
    world = dist.get_world_size()
    objs = [None] * world
    dist.all_gather_object(objs, [(int(g), row) for g, row in zip(mine, rows)])
    if dist.get_rank() != 0:
        return None
    allrows = dict(pair for part in objs for pair in part)
    n = nrep if nrep is not None else len(allrows)
    if sorted(allrows) != list(range(n)):
        raise RuntimeError("replica rows missing or duplicated across ranks")
    return [allrows[g] for g in range(n)]


def allmax(v: float, dist=None) -> float:
    """Max of v over ranks (a CPU tensor: works with gloo; NCCL groups pass device tensors)."""
    if dist is None:
        return v
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(v)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
