"""Independent systems spread over ranks (one process per GPU).

A batch of independent solves shards with no data-path exchange: each rank
sets up and solves its own systems (as one tf_batch graph on its GPU), and
the only collective is the final gather of the per-system reports.

  assign(weights, world)      longest-processing-time-first: systems in
                              decreasing weight (ties by index) each go to
                              the rank with the least weight so far (ties to
                              the lowest rank); deterministic, so every rank
                              computes the same assignment without talking.
  gather_reports(local, owned, count, group)
                              all ranks' (index, report) pairs, reassembled
                              in global system order on every rank.
"""
from __future__ import annotations

from typing import Any, Sequence


def assign(weights: Sequence[int], world: int) -> list[list[int]]:
    """System indices per rank (each list ascending)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for k in sorted(range(len(weights)), key=lambda i: (-int(weights[i]), i)):
        if weights[k] < 0:
            raise ValueError("weights must be non-negative")
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(k)
        load[r] += int(weights[k])
    return [sorted(ks) for ks in out]


def imbalance(weights: Sequence[int], parts: list[list[int]]) -> float:
    """Largest rank load over the mean load (1.0 = perfect balance)."""
    loads = [sum(int(weights[k]) for k in ks) for ks in parts]
    mean = sum(loads) / len(loads)
    return max(loads) / mean if mean else 1.0


def gather_reports(local: Sequence[Any], owned: Sequence[int], count: int, group=None) -> list[Any]:
    """Every rank's reports in global system order (a list of `count`).

    local[i] is the report of system owned[i].  Uses one all_gather_object
    over the process group (any backend); with no initialised process group
    the local reports must already cover every system."""
    import torch.distributed as dist
    if len(local) != len(owned):
        raise ValueError("one report per owned system")
    pairs = list(zip(owned, local))
    if dist.is_available() and dist.is_initialized():
        everything: list = [None] * dist.get_world_size(group)
        dist.all_gather_object(everything, pairs, group=group)
        pairs = [p for part in everything for p in part]
    out: list[Any] = [None] * count
    seen = 0
    for k, rep in pairs:
        if not 0 <= k < count or out[k] is not None:
            raise ValueError(f"system {k} reported twice or out of range")
        out[k] = rep
        seen += 1
    if seen != count:
        raise ValueError(f"{count - seen} systems have no report")
    return out
