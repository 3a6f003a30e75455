"""Batched solves of many designs of uneven size, and the project's autotuner.

A batch runs every design on one thread-block cluster (``cps_batch_solve``);
the two knobs are the cluster size (CTAs per design: more CTAs shorten one
design's phases, fewer CTAs let more designs run at once) and the number of
outer iterations a design runs per launch (its "visit": long visits amortise
the launch, short ones let the host retire converged designs and admit new
ones sooner).  :func:`autotune` times short visits of a sample of the actual
designs for each candidate cluster size and keeps the fastest in cell-updates
per second; results are cached per size bucket.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import cps
from .geometry import Design

CLUSTER_CANDIDATES = (2, 4, 8, 16)


def size_bucket(cells: float) -> int:
    """log2 bucket of a design's cell count (the autotuner's cache key)."""
    return int(round(math.log2(max(cells, 1.0))))


@dataclass
class TuneResult:
    cluster_ctas: int
    cell_updates_per_s: Dict[int, float] = field(default_factory=dict)


_CACHE: Dict[Tuple[int, int], TuneResult] = {}


def autotune(designs: Sequence[Design], precision: int = cps.CPS_FP64, device: int = 0, sample: int = 12,
             visit: int = 30, candidates: Sequence[int] = CLUSTER_CANDIDATES, use_cache: bool = True) -> TuneResult:
    """Pick the cluster size with the highest cell-updates/s on a sample of
    ``designs`` (``visit`` outer iterations each, from the zero state)."""
    cells = float(np.median([d.M * d.N for d in designs]))
    key = (size_bucket(cells), precision)
    if use_cache and key in _CACHE:
        return _CACHE[key]
    rng = np.random.default_rng(0)
    idx = rng.choice(len(designs), size=min(sample, len(designs)), replace=False)
    chosen = [designs[int(k)] for k in idx]
    solvers = [cps.Solver(d, precision=precision, device=device) for d in chosen]
    rates: Dict[int, float] = {}
    try:
        cps.batch_solve(solvers, 2, eps=0.0, cluster_ctas=candidates[0])  # warm-up (module load, first touch)
        for c in candidates:
            for s in solvers:
                s.reset_fields()
            res, ms = cps.batch_solve(solvers, visit, eps=0.0, cluster_ctas=c)
            work = sum(r["n_done"] * s.design.M * s.design.N for r, s in zip(res, solvers))
            rates[c] = work / (ms / 1e3) if ms > 0 else 0.0
    finally:
        for s in solvers:
            s.close()
    best = max(rates, key=rates.get)
    out = TuneResult(cluster_ctas=best, cell_updates_per_s=rates)
    _CACHE[key] = out
    return out


def solve_batch(designs: Sequence[Design], eps: float = 1e-6, max_outer: int = 200000,
                precision: int = cps.CPS_FP64, cluster_ctas: Optional[int] = None, visit: int = 0,
                device: int = 0) -> Tuple[List[dict], float]:
    """Solve all designs to ``eps``; returns (per-design results, device ms).

    ``visit`` > 0 splits the work into launches of at most ``visit`` outer
    iterations per design (converged designs leave the batch between
    launches); 0 runs everything in one launch."""
    if cluster_ctas is None:
        cluster_ctas = autotune(designs, precision, device).cluster_ctas
    solvers = [cps.Solver(d, precision=precision, device=device) for d in designs]
    total_ms = 0.0
    results: List[Optional[dict]] = [None] * len(designs)
    done_iters = [0] * len(designs)
    try:
        active = list(range(len(designs)))
        while active:
            budget = max_outer if visit <= 0 else visit
            budget = min(budget, max(max_outer - min(done_iters[k] for k in active), 1))
            res, ms = cps.batch_solve([solvers[k] for k in active], budget, eps=eps, cluster_ctas=cluster_ctas)
            total_ms += ms
            still = []
            for k, r in zip(active, res):
                done_iters[k] += r["n_done"]
                r = dict(r, outer_iterations=done_iters[k])
                results[k] = r
                if not r["converged"] and r["status"] == 0 and done_iters[k] < max_outer:
                    still.append(k)
            active = still
    finally:
        for s in solvers:
            s.close()
    return results, total_ms
