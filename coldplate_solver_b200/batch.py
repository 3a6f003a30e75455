"""Batched solves of many designs of uneven size, and the project's autotuner.

A batch places every design on a group of CTAs of a persistent launch
(``cps_batch_solve``): a group sized to the design (``tiles_per_cta``: each
CTA takes that many 8 x 32 tiles per phase, and the groups run in waves that
fill the device), a fixed group of K CTAs of one cooperative launch
(``group_ctas``), or one thread-block cluster with the hardware cluster
barrier (``cluster_ctas``).  The knobs are the placement (CTAs per design:
more CTAs shorten one design's phases, fewer CTAs let more designs run at
once, and the designs in flight share the 126 MB L2) and the number of outer
iterations a design runs per launch (its "visit": long visits amortise the
launch, short ones let the host retire converged designs and admit new ones
sooner), and the tile shape (8 x 32, 16 x 16 or 4 x 64 points per tile, one
library per shape: the halo a tile stages and the tiles a CTA walks).
:func:`autotune` times short visits of a sample of the actual designs for each
candidate placement, from the zero state and from a warm state, keeps the
fastest in cell-updates per second, times the other tile shapes with that
placement the same way, and then picks the visit length by solving the sample
to convergence once per candidate length; results are cached per size bucket.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import cps
from .geometry import Design

def mode_candidates(device: int = 0) -> List[dict]:
    """Placements the autotuner tries: groups sized to each design at 2, 4, 8
    and 16 tiles per CTA, fixed groups of 2x, 1x, 1/2x and 1/4x the SM count of
    CTAs, and thread-block clusters of 8 and 16 CTAs."""
    try:
        import torch
        sms = torch.cuda.get_device_properties(device).multi_processor_count
    except Exception:  # noqa: BLE001 - no torch/GPU: B200 count
        sms = 148
    groups = [2 * sms, sms, sms // 2, sms // 4]
    return ([{"tiles_per_cta": t} for t in (2, 4, 8, 16)] + [{"group_ctas": k} for k in groups if k >= 1] +
            [{"cluster_ctas": 8}, {"cluster_ctas": 16}])


def default_mode(device: int = 0) -> dict:
    """Placement used when none is given: groups of as many CTAs as the device
    has SMs (two designs in flight at two CTAs per SM), which measured fastest
    on the 16- and 64-design mixes; the autotuner picks per workload."""
    try:
        import torch
        return {"group_ctas": torch.cuda.get_device_properties(device).multi_processor_count}
    except Exception:  # noqa: BLE001 - no torch/GPU: B200 count
        return {"group_ctas": 148}


def mode_label(mode: dict) -> str:
    return ",".join(f"{k}={v}" for k, v in sorted(mode.items()))


def size_bucket(cells: float) -> int:
    """log2 bucket of a design's cell count (the autotuner's cache key)."""
    return int(round(math.log2(max(cells, 1.0))))


@dataclass
class TuneResult:
    mode: dict
    visit: int = 4096
    tile_j: int = 32
    cell_updates_per_s: Dict[str, float] = field(default_factory=dict)  # per placement, zero + warm states
    tile_cell_updates_per_s: Dict[int, float] = field(default_factory=dict)  # per tile width, chosen placement
    visit_ms: Dict[int, float] = field(default_factory=dict)  # device ms of the sample's converged solves per visit


_CACHE: Dict[Tuple[int, int, int], TuneResult] = {}


def _probe_rate(solvers, warm_fields, probe: int, mode: dict) -> float:
    """Cell-updates per second of ``probe`` outer iterations of the sample
    from the zero state and from its warm states, with placement ``mode``."""
    work, ms_total = 0.0, 0.0
    for start in ("zero", "warm"):
        for s, f in zip(solvers, warm_fields):
            s.reset_fields()
            if start == "warm":
                s.upload_fields(f["u"], f["v"], f["p"])
        res, ms = cps.batch_solve(solvers, probe, eps=0.0, **mode)
        work += sum(r["n_done"] * s.design.M * s.design.N for r, s in zip(res, solvers))
        ms_total += ms
    return work / (ms_total / 1e3) if ms_total > 0 else 0.0


def autotune(designs: Sequence[Design], precision: int = cps.CPS_FP64, device: int = 0, sample: int = 6,
             probe: int = 200, warm: int = 1500, visits: Sequence[int] = (512, 2048, 8192),
             candidates: Optional[Sequence[dict]] = None, tile_widths: Sequence[int] = cps.TILE_WIDTHS,
             eps: float = 1e-6, max_outer: int = 200000, use_cache: bool = True) -> TuneResult:
    """Pick the placement, the tile shape and the visit length for ``designs``.

    Placement: every candidate runs ``probe`` outer iterations of a sample of
    the designs twice, from the zero state (the early iterations, PCG at its
    cap) and from the state after ``warm`` iterations (the regime that most of
    a solve spends its iterations in); the placement with the most
    cell-updates per second over both wins.  Tile shape: with that placement
    every width of ``tile_widths`` is timed the same way (the 8 x 32 default
    included; a shape's warm states are its own, the same states to rounding).
    Visit: with that placement and shape the sample is solved to ``eps`` from
    the zero state once per candidate length, converged designs leaving
    between launches as in :class:`BatchRunner`; the length with the least
    device time wins.  Results are cached per size bucket, precision and
    sample size."""
    cells = float(np.median([d.M * d.N for d in designs]))
    key = (size_bucket(cells), precision, min(sample, len(designs)))
    if use_cache and key in _CACHE:
        return _CACHE[key]
    cands = list(candidates) if candidates is not None else mode_candidates(device)
    rng = np.random.default_rng(0)
    idx = rng.choice(len(designs), size=min(sample, len(designs)), replace=False)
    chosen = [designs[int(k)] for k in idx]
    rates: Dict[str, float] = {}
    tile_rates: Dict[int, float] = {}
    best, best_rate = cands[0], -1.0
    visit_ms: Dict[int, float] = {}

    def sample_at(tile_j: int):
        solvers = [cps.Solver(d, precision=precision, device=device, tile_j=tile_j) for d in chosen]
        warm_fields = []
        for s in solvers:
            s.reset_fields()
            s.solve(warm, eps=0.0)
            warm_fields.append(s.download())
        return solvers, warm_fields

    solvers, warm_fields = sample_at(32)
    try:
        cps.batch_solve(solvers, 2, eps=0.0, **cands[0])  # module load, first touch
        for mode in cands:
            try:
                rate = _probe_rate(solvers, warm_fields, probe, mode)
            except cps.CpsError:
                continue  # placement does not fit this device
            rates[mode_label(mode)] = rate
            if rate > best_rate:
                best, best_rate = mode, rate
    finally:
        for s in solvers:
            s.close()
    best_tile = 32
    if 32 in tile_widths:
        tile_rates[32] = best_rate
    else:
        best_rate = -1.0
    for tj in tile_widths:
        if tj == 32:
            continue
        solvers, warm_fields = sample_at(tj)
        try:
            cps.batch_solve(solvers, 2, eps=0.0, **best)
            rate = _probe_rate(solvers, warm_fields, probe, best)
        except cps.CpsError:
            continue
        finally:
            for s in solvers:
                s.close()
        tile_rates[tj] = rate
        if rate > best_rate:
            best_tile, best_rate = tj, rate
    for v in visits:
        with BatchRunner(chosen, precision=precision, device=device, mode=best, tile_j=best_tile) as br:
            _, ms, _ = br.run(eps=eps, max_outer=max_outer, visit=int(v))
        visit_ms[int(v)] = ms
    out = TuneResult(mode=dict(best), visit=min(visit_ms, key=visit_ms.get) if visit_ms else 4096,
                     tile_j=best_tile, cell_updates_per_s=rates, tile_cell_updates_per_s=tile_rates,
                     visit_ms=visit_ms)
    _CACHE[key] = out
    return out


class BatchRunner:
    """A set of designs kept resident on one GPU and solved together.

    ``run()`` resets every design to the zero state on the device and solves
    all of them to ``eps`` in launches of at most ``visit`` outer iterations
    per design; designs that converge leave the batch between launches.
    ``mode`` is the keyword of :func:`cps.batch_solve` that places designs:
    ``{"tiles_per_cta": R}`` (groups sized to each design, in waves),
    ``{"group_ctas": K}`` (groups of K CTAs of one cooperative launch) or
    ``{"cluster_ctas": C}`` (one thread-block cluster per design).
    ``tile_j``: the tile shape's width (all designs of a batch share it)."""

    def __init__(self, designs: Sequence[Design], precision: int = cps.CPS_MIXED, device: int = 0,
                 mode: Optional[dict] = None, tile_j: int = 32):
        self.designs = list(designs)
        self.tile_j = tile_j
        self.solvers = [cps.Solver(d, precision=precision, device=device, tile_j=tile_j) for d in self.designs]
        self.mode = dict(mode or default_mode(device))

    def close(self) -> None:
        for s in self.solvers:
            s.close()
        self.solvers = []

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def run(self, eps: float = 1e-6, max_outer: int = 200000, visit: int = 4096, reset: bool = True):
        """Returns (per-design results, device ms, launches).  Each result has
        the design's total outer_iterations and finished_ms, the device time
        from the start of the run to the end of the launch in which the design
        left the batch (converged, failed or out of budget)."""
        if reset:
            for s in self.solvers:
                s.reset_fields()
        n = len(self.solvers)
        done = [0] * n
        results: List[Optional[dict]] = [None] * n
        active = list(range(n))
        total_ms, launches = 0.0, 0
        while active:
            budget = min(visit, max(1, max_outer - min(done[k] for k in active)))
            res, ms = cps.batch_solve([self.solvers[k] for k in active], budget, eps=eps, **self.mode)
            total_ms += ms
            launches += 1
            still = []
            for k, r in zip(active, res):
                done[k] += r["n_done"]
                results[k] = dict(r, outer_iterations=done[k], finished_ms=total_ms)
                if not r["converged"] and r["status"] == 0 and done[k] < max_outer:
                    still.append(k)
            active = still
        return results, total_ms, launches


def solve_batch(designs: Sequence[Design], eps: float = 1e-6, max_outer: int = 200000,
                precision: int = cps.CPS_FP64, mode: Optional[dict] = None, visit: int = 4096,
                device: int = 0, tile_j: int = 32) -> Tuple[List[dict], float]:
    """Solve all designs to ``eps`` (placement ``mode``, or the autotuner's
    placement, tile shape and visit); returns (per-design results, device ms)."""
    if mode is None:
        tuned = autotune(designs, precision, device)
        mode, visit, tile_j = tuned.mode, tuned.visit, tuned.tile_j
    with BatchRunner(designs, precision, device, mode, tile_j=tile_j) as runner:
        res, ms, _ = runner.run(eps=eps, max_outer=max_outer, visit=visit, reset=False)
    return res, ms
