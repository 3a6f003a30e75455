"""Serving loop: continuous batching of SIMPLE solves on one GPU.

Requests (design candidates) arrive over time.  A request is admitted as soon
as its device footprint (``cps_footprint``) fits in the HBM budget and an
in-flight slot is free; admitted designs keep their fields resident until
they converge.  The GPU runs epochs: one ``cps_batch_solve`` launch advances
every in-flight design by at most ``visit`` outer iterations (each design on
its own group of CTAs of a cooperative launch, or its own thread-block
cluster; converged designs stop early).  Between epochs
the host retires converged designs (freeing their memory) and admits the
requests that arrived meanwhile, so new work overlaps with designs already on
the device.  A design's result does not depend on the mix it ran in: its
group computes exactly what it would compute alone.

Latency of a request = time from its arrival to the end of the epoch in which
it converged (queueing + admission + solve).
"""
from __future__ import annotations

import collections
import time
from dataclasses import dataclass, field
from typing import Deque, Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import batch, cps
from .geometry import Design


@dataclass
class Request:
    rid: int
    arrival: float
    design: Design
    admitted: float = float("nan")
    finished: float = float("nan")
    outer_iterations: int = 0
    converged: bool = False
    status: int = 0
    dp: float = float("nan")
    last: Tuple = ()
    fields: Optional[Dict[str, np.ndarray]] = None

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


@dataclass
class ServeStats:
    completed: int
    makespan_s: float
    solves_per_s: float
    latency_p50_s: float
    latency_p99_s: float
    max_inflight: int
    epochs: int
    device_ms: float
    peak_bytes: int
    requests: List[Request] = field(default_factory=list)


class Server:
    def __init__(self, budget_bytes: float = 120e9, visit: int = 300, cluster_ctas: Optional[int] = None,
                 precision: int = cps.CPS_MIXED, device: int = 0, max_inflight: int = 256, eps: float = 1e-6,
                 max_outer: int = 200000, keep_fields: bool = False, mode: Optional[dict] = None,
                 keep: Sequence[int] = ()):
        """``mode``: placement keyword of :func:`cps.batch_solve`
        (default: :func:`batch.default_mode`); ``cluster_ctas`` is shorthand
        for ``mode={"cluster_ctas": cluster_ctas}``.  ``keep_fields`` keeps
        every request's final fields (Request.fields), ``keep`` those of the
        requests with these indices in the stream."""
        self.budget = int(budget_bytes)
        self.visit = visit
        if mode is None:
            mode = {"cluster_ctas": cluster_ctas} if cluster_ctas else batch.default_mode(device)
        self.mode = dict(mode)
        self.precision = precision
        self.device = device
        self.max_inflight = max_inflight
        self.eps = eps
        self.max_outer = max_outer
        self.keep_fields = keep_fields
        self.keep = set(keep)

    def run(self, stream: Sequence[Tuple[float, Design]], real_time: bool = True) -> ServeStats:
        """Serve ``stream`` (arrival time in s, design).  With ``real_time``
        arrivals are released by the wall clock; otherwise all are available
        at t = 0 (a closed batch)."""
        reqs = [Request(k, float(t) if real_time else 0.0, d) for k, (t, d) in enumerate(stream)]
        pending: Deque[Request] = collections.deque(sorted(reqs, key=lambda r: r.arrival))
        inflight: List[Tuple[Request, cps.Solver, int]] = []
        used = peak = 0
        epochs = 0
        device_ms = 0.0
        max_seen = 0
        t0 = time.perf_counter()
        while pending or inflight:
            now = time.perf_counter() - t0
            # admission in arrival order (no overtaking), by footprint and slots
            while pending and pending[0].arrival <= now and len(inflight) < self.max_inflight:
                r = pending[0]
                fp = cps.footprint(r.design, self.precision)
                if used + fp > self.budget and inflight:
                    break
                pending.popleft()
                s = cps.Solver(r.design, precision=self.precision, device=self.device)
                r.admitted = time.perf_counter() - t0
                used += fp
                peak = max(peak, used)
                inflight.append((r, s, fp))
            max_seen = max(max_seen, len(inflight))
            if not inflight:
                if pending:
                    time.sleep(max(0.0, min(pending[0].arrival - (time.perf_counter() - t0), 0.05)))
                continue
            res, ms = cps.batch_solve([s for _, s, _ in inflight], self.visit, eps=self.eps, **self.mode)
            epochs += 1
            device_ms += ms
            end = time.perf_counter() - t0
            keep = []
            for (r, s, fp), o in zip(inflight, res):
                r.outer_iterations += o["n_done"]
                r.converged, r.status, r.last = o["converged"], o["status"], o["last"]
                if r.converged or r.status != 0 or r.outer_iterations >= self.max_outer:
                    r.finished = end
                    r.dp = s.full_dp()
                    if self.keep_fields or r.rid in self.keep:
                        r.fields = s.download()
                    s.close()
                    used -= fp
                else:
                    keep.append((r, s, fp))
            inflight = keep
        makespan = max((r.finished for r in reqs), default=0.0) - min((r.arrival for r in reqs), default=0.0)
        lat = np.array([r.latency for r in reqs]) if reqs else np.zeros(1)
        return ServeStats(completed=sum(r.converged for r in reqs), makespan_s=makespan,
                          solves_per_s=(sum(r.converged for r in reqs) / makespan) if makespan > 0 else 0.0,
                          latency_p50_s=float(np.percentile(lat, 50)), latency_p99_s=float(np.percentile(lat, 99)),
                          max_inflight=max_seen, epochs=epochs, device_ms=device_ms, peak_bytes=peak, requests=reqs)
