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

Order: a request is answered at the end of the epoch in which it converged,
so an epoch that advances every in-flight design makes a small request wait
for the visits of all the large ones.  With ``order="smallest"`` (default) an
epoch advances only the ``epoch_designs`` smallest in-flight designs (by cell
count: the outer iterations to converge grow with the design's size, so this
is shortest-job-first on an estimate of the work left), as many as keep every
group of CTAs busy; the others stay resident and wait.  ``"arrival"``
advances every in-flight design in every epoch.  Short visits (a few hundred
outer iterations) keep epochs short, so a converged design is answered soon
after it converges.

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


def concurrent_groups(mode: dict, device: int = 0) -> int:
    """Designs a placement advances at once: the resident CTAs (two per SM)
    over the CTAs per design (groups sized to a design: taken as 8)."""
    try:
        import torch
        sms = torch.cuda.get_device_properties(device).multi_processor_count
    except Exception:  # noqa: BLE001 - no torch/GPU: B200 count
        sms = 148
    ctas = mode.get("group_ctas") or mode.get("cluster_ctas") or 0
    return max(1, (2 * sms) // ctas) if ctas else 8


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
                 keep: Sequence[int] = (), order: str = "smallest", epoch_designs: int = 0):
        """``mode``: placement keyword of :func:`cps.batch_solve`
        (default: :func:`batch.default_mode`); ``cluster_ctas`` is shorthand
        for ``mode={"cluster_ctas": cluster_ctas}``.  ``keep_fields`` keeps
        every request's final fields (Request.fields), ``keep`` those of the
        requests with these indices in the stream.  ``order``: "smallest"
        (an epoch advances the ``epoch_designs`` smallest in-flight designs;
        0: twice the groups the placement runs at once) or "arrival" (every
        in-flight design, every epoch)."""
        if order not in ("smallest", "arrival"):
            raise ValueError(f"order must be 'smallest' or 'arrival', not {order!r}")
        self.order = order
        self.budget = int(budget_bytes)
        self.visit = visit
        if mode is None:
            mode = {"cluster_ctas": cluster_ctas} if cluster_ctas else batch.default_mode(device)
        self.mode = dict(mode)
        self.epoch_designs = int(epoch_designs) if epoch_designs > 0 else 2 * concurrent_groups(self.mode, device)
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
            if self.order == "smallest":
                inflight.sort(key=lambda e: (e[0].design.M * e[0].design.N, e[0].rid))
                run, waiting = inflight[:self.epoch_designs], inflight[self.epoch_designs:]
            else:
                run, waiting = inflight, []
            res, ms = cps.batch_solve([s for _, s, _ in run], self.visit, eps=self.eps, **self.mode)
            epochs += 1
            device_ms += ms
            end = time.perf_counter() - t0
            keep = list(waiting)
            for (r, s, fp), o in zip(run, res):
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
