"""Multi-GPU: designs are independent, so a job of many designs is sharded
across ranks (one process per GPU) with no collective on the data path.

Every rank computes the same assignment (longest-processing-time-first on the
cell count, a deterministic greedy bin packing), solves its own designs on
its own GPU, and the per-design results (small dicts, no fields) are gathered
once at the end with ``all_gather_object``.  Within one design there is no
split: a single solve runs on one GPU (replicas only).
"""
from __future__ import annotations

from typing import Callable, List, Optional, Sequence

from .geometry import Design


def assign(designs: Sequence[Design], world: int) -> List[List[int]]:
    """Deterministic LPT assignment of design indices to ``world`` ranks,
    balancing total cells."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(designs)), key=lambda k: (-designs[k].M * designs[k].N, k))
    load = [0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for k in order:
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(k)
        load[r] += designs[k].M * designs[k].N
    for lst in out:
        lst.sort()
    return out


def run_sharded(designs: Sequence[Design], solve: Callable[[List[Design]], List[dict]], rank: int, world: int,
                group=None) -> List[Optional[dict]]:
    """Solve this rank's shard with ``solve`` and gather every rank's results
    into the original order (on every rank)."""
    mine = assign(designs, world)[rank]
    local = solve([designs[k] for k in mine]) if mine else []
    if len(local) != len(mine):
        raise RuntimeError("solve returned a result count different from its shard")
    pairs = list(zip(mine, local))
    if world > 1:
        import torch.distributed as dist
        gathered: List[list] = [None] * world  # type: ignore[list-item]
        dist.all_gather_object(gathered, pairs, group=group)
    else:
        gathered = [pairs]
    out: List[Optional[dict]] = [None] * len(designs)
    for part in gathered:
        for k, r in part:
            if out[k] is not None:
                raise RuntimeError(f"design {k} solved twice")
            out[k] = r
    return out
