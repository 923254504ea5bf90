"""Sharding independent evolutions over GPUs: one engine per GPU, one process per GPU.

A batch of evolutions (or a request stream) has no exchange step -- each evolution is its own
unit -- so it splits across ranks with no collective on the data path: rank r evolves the share
``assign`` gives it on its own device and engine, and the results come back to rank 0 by one
gather at the end. The share is size-balanced: evolutions in decreasing order of the engine's
device-byte estimate (hgx_estimate_device_bytes), each to the rank with the least estimated load
(longest-processing-time-first), so a few large evolutions do not land on one rank.

The process group is the caller's (``torch.distributed``, NCCL on GPUs, gloo on CPU); only
``gather_object`` crosses it.
"""
from __future__ import annotations

import heapq

from . import api


def assign(evolutions, world: int, estimate=None) -> list:
    """rank of each evolution: size-balanced by the byte estimate (ties to the lower rank)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    est = estimate or api.estimate_device_bytes
    sizes = [int(est(ev)) for ev in evolutions]
    order = sorted(range(len(evolutions)), key=lambda i: (-sizes[i], i))
    heap = [(0, r) for r in range(world)]
    owner = [0] * len(evolutions)
    for i in order:
        load, r = heapq.heappop(heap)
        owner[i] = r
        heapq.heappush(heap, (load + sizes[i], r))
    return owner


def local_share(evolutions, rank: int, world: int, estimate=None):
    """(indices, evolutions) this rank evolves, in input order."""
    owner = assign(evolutions, world, estimate)
    idx = [i for i, r in enumerate(owner) if r == rank]
    return idx, [evolutions[i] for i in idx]


def summary(res) -> dict:
    """What travels back to rank 0 per evolution: counts and the exact key multisets."""
    k = res.keys()
    return {"states": int(res.num_states), "events": int(res.num_events),
            "classes": int(res.num_classes), "causal": int(len(res.causal)),
            "branchial": int(len(res.branchial)), "truncated": bool(res.truncated),
            "keys": {n: v.tobytes() for n, v in k.items()}}


def evolve_sharded(engine, evolutions, dist=None, estimate=None, reduce=summary):
    """Evolve a batch split over the process group: each rank runs its share as one batch on
    its own engine; rank 0 returns reduce(result) per evolution in input order, other ranks
    return None. Without a process group (dist None or world 1) the whole batch runs here."""
    world = dist.get_world_size() if dist is not None else 1
    rank = dist.get_rank() if dist is not None else 0
    idx, mine = local_share(evolutions, rank, world, estimate)
    results = engine.evolve_batch(mine) if mine else []
    part = [(i, reduce(r)) for i, r in zip(idx, results)]
    if world == 1:
        return [p for _, p in sorted(part, key=lambda x: x[0])]
    gathered = [None] * world if rank == 0 else None
    dist.gather_object(part, gathered, dst=0)
    if rank != 0:
        return None
    out = [None] * len(evolutions)
    for chunk in gathered:
        for i, p in chunk:
            out[i] = p
    return out


def serve_sharded(make_server, arrivals, dist=None, estimate=None, **run_kw):
    """Serve a request stream split over the process group: each rank serves the requests
    ``assign`` gives it with its own Server (make_server() builds it on the rank's engine);
    rank 0 returns every request's (arrival, admitted, finished, events, states) in stream order,
    other ranks None."""
    world = dist.get_world_size() if dist is not None else 1
    rank = dist.get_rank() if dist is not None else 0
    evs = [ev for _, ev in arrivals]
    idx, _ = local_share(evs, rank, world, estimate)
    recs = make_server().run([arrivals[i] for i in idx], **run_kw) if idx else []
    part = [(i, (r.arrival, r.admitted, r.finished, int(r.result.num_events),
                 int(r.result.num_states))) for i, r in zip(idx, recs)]
    if world == 1:
        return [p for _, p in sorted(part, key=lambda x: x[0])]
    gathered = [None] * world if rank == 0 else None
    dist.gather_object(part, gathered, dst=0)
    if rank != 0:
        return None
    out = [None] * len(arrivals)
    for chunk in gathered:
        for i, p in chunk:
            out[i] = p
    return out
