#!/usr/bin/env python
"""Benchmark: converged SIMPLE solves per second on one B200 (and N GPUs).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload density|network|straight|mix|served|thermal] [--precision fp64|mixed]

A step is one converged solve (outer residual max(residU, residV,
residMassDof) <= 1e-6) of the workload's design(s), started from the zero
state.  The default workload is the largest single-design configuration: the
1000 x 500 density-field design (10 um, SOU, 2.5-D, RAMP Brinkman alpha).
``value`` is converged solves/s over all ranks with the inputs resident in
HBM (device time from CUDA events on the library's stream, L2 flushed between
steps); ``e2e`` is the same metric through the public C ABI with host
buffers: geometry and initial fields uploaded, the solve run, and u, v, p
downloaded, every step (wall clock).

``error_vs_fp64_oracle``: the solve's u, v, fluid-cell p and full dP against
the reference's own FP64 fixed point of the same design (committed fixture,
tests/golden/converged/), at the 1e-6 stop and again after the same solve is
continued to the fixture's residual (1e-10; 1e-12 for the density-field
designs), beside the reference's own 1e-6 stop state against its fixed point.  ``cpu_baseline``: the reference's own build on the
host cores, on a bounded sample of the solve (timed chunks from five states
along the trajectory), extrapolated with a per-iteration cost model linear in
the inner iteration counts.  With --precision mixed the line also carries the
plain FP64 path on the same design (``vs_plain_fp64_gpu``).

Multi-GPU (torchrun, one rank per GPU): every rank solves its own copy of the
workload (independent designs, no collective on the data path; weak scaling);
the timed region is bracketed by barriers and the max over ranks is taken.

--workload mix / served (one GPU): the many-design paths.  mix: the first
--designs designs of the seeded 64-design density-field mix (Nx log-uniform
in [256, 1024], Ny = Nx/2) solved together by the batched persistent kernel;
a step is the whole batch.  served: --requests Poisson arrivals (20/s) of
density-field designs (Nx in [128, 2048]) through the serving loop (HBM
admission, continuous batching, groups sized to each request, the 12 smallest
in-flight requests advanced per epoch of 512 outer iterations); latency is
wall clock from arrival to convergence.  Both lines carry the plain FP64 single-design path on the same
designs, one after another, as the comparison, and the relative dP
difference of every design against it.

--workload thermal: the 3-D conjugate-heat-transfer step on the
1000 x 500 x 9 crop of the density-field design's flow (--thermal-nx 500
for a quarter of it); a step is one thermal solve from T_inlet to a relative
residual of 1e-6; e2e uploads gamma, u, v and the heat flux and downloads the
temperature field every step.  Its CPU baseline is a scipy port of the same
algorithm (the reference's own thermal solve needs AMGCL, which is absent),
and --impl reference prints an unavailable line.

--impl reference times the reference solver's own CPU implementation
(oracle/_ref/ref_f64: its sources promoted to FP64, all host threads) on the
same workload: the whole solve to the 1e-6 stop, run in --steps chunks that
carry the state (u, v, p) from one chunk to the next; a solve that exceeds
--ref-time-cap seconds runs its remaining iterations (to the reference's
converged count) at the rate of its last chunk.  Both arms also report, under
cpu_baseline.as_shipped_fp32, the reference as shipped (FP32 throughout,
oracle/_ref/ref_f32) on the same design (the reference arm only when its FP64
solve took under two minutes); the FP64 build stays the reported value
because this library computes in FP64.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "converged solves/s (1e-6 outer residual)"
EPS = 1e-6
MAX_OUTER = 200000
L2_FLUSH_BYTES = 512 << 20  # > 126 MB L2


# The reference's own FP64 fixed point of each workload's design, from
# tests/golden/make_converged.py (committed fixtures).
ORACLE_FIXTURES = {"network": "network_500x250", "density": "density_1000x500"}
MIX_FIXTURES = {47: "mix47_258x129"}  # design index in the 64-design mix -> fixture
SERVED_FIXTURES = {14: "served14_137x68"}  # request index in the served stream -> fixture


def workload(name: str):
    from coldplate_solver_b200 import geometry as g
    if name == "network":
        d = g.channel_network()
        cfg = {"workload": "channel_network_500x250_sou_2.5d", "grid": "500x250", "dx_um": 20,
               "convection": "SOU", "two_point_five_d": True}
    elif name == "straight":
        d = g.straight_channel()
        cfg = {"workload": "straight_channel_200x100_fou", "grid": "200x100", "dx_um": 50, "convection": "FOU"}
    elif name == "density":
        d = g.density_field(Nx=1000)
        cfg = {"workload": "density_field_1000x500_sou_2.5d", "grid": "1000x500", "dx_um": 10, "convection": "SOU"}
    else:
        raise SystemExit(f"unknown workload {name}")
    cfg.update(uvAlpha=d.uvAlpha, pAlpha=d.pAlpha, eps=EPS)
    return d, cfg


# ---------------------------------------------------------------------------
# algorithmic bytes (per outer iteration, FP64: 8-byte elements)
# ---------------------------------------------------------------------------
def algorithmic_bytes(design, hist: np.ndarray, s: int = 8) -> float:
    """Minimal single-pass DRAM streams of one outer iteration:
    momentum set-up 6(nU+nV), Jacobi 6(Ku nU + Kv nV), mass residual 3 nP,
    PCG 12 Kp nP, correction 9 M N elements (s bytes each)."""
    nU, nV, nP, MN = design.nU, design.nV, design.nP, design.M * design.N
    ku, kv = hist[:, 6], hist[:, 7]
    kp = np.where(hist[:, 5] < design.maxPressureIter, hist[:, 5] + 1, design.maxPressureIter)
    per = 6 * (nU + nV) + 6 * (ku * nU + kv * nV) + 3 * nP + 12 * kp * nP + 9 * MN
    return float(s * per.sum())


# ---------------------------------------------------------------------------
# error against the FP64 oracle's fixed point
# ---------------------------------------------------------------------------
def oracle_fixture(name):
    """The committed fixed point of the reference's FP64 solve of a design
    (tests/golden/converged/<name>.npz), or None."""
    path = os.path.join(REPO, "tests", "golden", "converged", f"{name}.npz")
    return np.load(path) if name and os.path.exists(path) else None


def fluid_mask_p(design, fields=None) -> np.ndarray:
    """Fluid cells (gamma > 0.5) on p's index space; with a state, only those
    whose pressure it determines (geometry.pressure_determined_mask: cells
    enclosed by faces at the velocity clamp keep an arbitrary pressure)."""
    from coldplate_solver_b200 import geometry
    mask = np.zeros((design.M + 1, design.N + 1), dtype=bool)
    mask[1:design.M, 1:design.N] = design.gamma[:design.M - 1, :design.N - 1] > 0.5
    if fields is not None:
        mask &= geometry.pressure_determined_mask(design, fields["u"], fields["v"])
    return mask


def errors_vs_fixture(design, fields, dp: float, fx) -> dict:
    """Relative L2 of u, v and fluid-cell p and relative full dP against the
    fixture's fixed point (on the fixture's every stride-th row and column)."""
    st = int(fx["stride"])

    def rel(a, b):
        nb = float(np.linalg.norm(b))
        return float(np.linalg.norm(a - b)) / nb if nb > 0 else float(np.linalg.norm(a - b))
    mask = fluid_mask_p(design, fields)[::st, ::st]
    out = {k: rel(fields[k][::st, ::st], fx[k].astype(np.float64)) for k in ("u", "v")}
    out["p"] = rel(fields["p"][::st, ::st][mask], fx["p"].astype(np.float64)[mask])
    out["dP"] = abs(dp - float(fx["dp_full"])) / abs(float(fx["dp_full"]))
    return out


def oracle_error_block(solver, design, fx, fixture: str, eps_fixed: float = 1e-10, max_outer: int = 400000) -> dict:
    """error_vs_fp64_oracle of a solver left at its 1e-6 stop: its fields
    against the reference's FP64 fixed point; then the same state continued
    to the fixture's residual (1e-10; 1e-12 for the density-field designs)
    with the fixture's tight inner tolerances (those
    the fixture's second stage used; they do not enter the fixed point) and
    compared again; beside them the reference's own 1e-6 stop state against
    its fixed point."""
    from coldplate_solver_b200 import cps
    f = solver.download()
    at_stop = errors_vs_fixture(design, f, solver.full_dp(), fx)
    tight = json.loads(str(fx["tight"]))
    if "eps" in fx.files:
        eps_fixed = float(fx["eps"])  # the residual the fixture's second stage ran to
    with cps.Solver(design.replace(**tight), precision=solver.precision, device=solver.device) as s2:
        s2.upload_fields(f["u"], f["v"], f["p"])
        # in chunks; mixed precision stops at its own residual floor (~1e-10),
        # when a chunk no longer halves the best residual
        n, best = 0, np.inf
        while n < max_outer:
            h = s2.solve(min(20000, max_outer - n), eps=eps_fixed)
            n += len(h)
            r = float(np.min(np.maximum(np.maximum(h[:, 0], h[:, 1]), h[:, 3])))
            done = r <= eps_fixed or r > 0.5 * best
            best = min(best, r)
            if done:
                break
        at_fixed = errors_vs_fixture(design, s2.download(), s2.full_dp(), fx)
    return {"at_1e-6_stop": at_stop,
            "at_fixed_point": dict(at_fixed, residual_target=eps_fixed, residual_reached=best,
                                   outer_iterations_after_stop=int(n), inner_tolerances=tight),
            "reference_own_1e-6_stop": {"u": float(fx["stop_err_u"]), "v": float(fx["stop_err_v"]),
                                        "p": float(fx["stop_err_p"]), "dP": float(fx["stop_err_dp"])},
            "oracle": "the reference's own FP64 solve (its sources promoted to double): to its 1e-6 stop, then "
                      f"with tight inner tolerances to the {eps_fixed:g} residual; tests/golden/converged/{fixture}.npz",
            "note": "relative L2 on u, v and fluid-cell p (where the state determines p), relative full dP; a run "
                    "stopped at 1e-6 sits about as "
                    "far from the fixed point as the reference's own 1e-6 stop does (the residual wanders near "
                    "1e-6 with the default inner tolerances)"}


# ---------------------------------------------------------------------------
# clocks sampling
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(prefix="clocks_", suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        rows = []
        try:
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        except OSError:
            pass
        finally:
            try:
                os.unlink(self.path)
            except OSError:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [num(r[1]) for r in rows if num(r[1]) is not None]
        mx = [num(r[2]) for r in rows if num(r[2]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        loaded = [x for x in sm if mx and x > 0.5 * max(mx)] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------------------
# distributed plumbing
# ---------------------------------------------------------------------------
def dist_init(n_gpus: int):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    return rank, local, world


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, world: int, local: int) -> float:
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{local}")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------
# CPU baseline: the reference's own code (oracle/_ref/ref_f64), all host cores
# ---------------------------------------------------------------------------
def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def reference_solve(design, threads: int, est_iters: int, chunks: int, time_cap: float,
                    precision: str = "f64") -> dict:
    """The reference's own build (oracle/_ref/ref_f64: promoted to FP64, the
    default; ref_f32: as shipped) solving ``design`` from the zero state to
    the 1e-6 stop, in ``chunks`` calls that carry the state (u, v, p); its own
    timer around the calculateStep loop is summed.  A solve still running
    after ``time_cap`` seconds is extrapolated to ``est_iters`` outer
    iterations: the remaining ones at the rate of its last chunk (the
    latest, cheapest part of the trajectory it reached)."""
    from oracle import reference
    chunk = max(100, -(-int(1.3 * est_iters) // max(1, chunks)))
    state, total_s, done, n_chunks, converged, per_chunk_ms = None, 0.0, 0, 0, False, []
    last_rate = 0.0
    t0 = time.perf_counter()
    while not converged and done < MAX_OUTER and time.perf_counter() - t0 < time_cap:
        out = reference.run(design, chunk, precision=precision, eps=EPS, stop_on_conv=True, threads=threads,
                            init=state, timeout=time_cap + 600)
        total_s += float(out["elapsed"][0])
        per_chunk_ms.append(1e3 * float(out["elapsed"][0]))
        done += len(out["err"])
        last_rate = float(out["elapsed"][0]) / max(1, len(out["err"]))
        n_chunks += 1
        converged = bool(max(out["residU"][-1], out["residV"][-1], out["residMassDof"][-1]) <= EPS)
        state = {k: out[k] for k in ("u", "v", "p")}
    if converged:
        value = 1.0 / total_s
        sample = (f"the whole solve from the zero state to the 1e-6 stop ({done} outer iterations) in {n_chunks} "
                  f"chunks of <= {chunk} iterations carrying the state")
    else:
        est = total_s + max(0, est_iters - done) * last_rate
        value = 1.0 / est
        sample = (f"{done} outer iterations from the zero state (time cap {time_cap:.0f} s), the remaining "
                  f"{max(0, est_iters - done)} of the reference's {est_iters} to the 1e-6 stop at the rate of the "
                  f"last chunk ({1e3 * last_rate:.2f} ms per outer iteration)")
    return {"value": value, "sample": sample, "iters": done, "converged": converged, "chunks": n_chunks,
            "ms_per_chunk": float(np.mean(per_chunk_ms)), "ms_per_outer_iteration": 1e3 * total_s / max(1, done),
            "seconds": total_s}


def as_shipped_fp32(design, threads: int, est_iters: int, time_cap: float):
    """The reference as shipped (FP32 throughout, oracle/_ref/ref_f32) on the
    same workload, reported beside the FP64 figure: the FP64 build is the one
    this library's FP64 arithmetic is compared with; this one is what the
    reference's users run today.  None when the binary is absent."""
    from oracle import reference
    if not reference.available("f32"):
        return None
    r = reference_solve(design, threads, est_iters, 2, time_cap, precision="f32")
    return {"value": r["value"], "unit": "solves/s", "cores": threads, "outer_iterations": r["iters"],
            "converged": r["converged"], "ms_per_outer_iteration": r["ms_per_outer_iteration"], "sample": r["sample"]}


def cpu_baseline(design, hist: np.ndarray, starts, threads: int, chunk_s: float = 3.0, chunks: int = 2,
                 precision: str = "f64") -> dict:
    """The reference's own build (oracle/_ref/ref_f64; ref_f32 with
    precision "f32") on a bounded sample of the solve, extrapolated to the
    whole solve with a per-iteration cost model.

    Sample: from each state of ``starts`` (the zero state and states along
    this design's trajectory) the reference runs ``chunks`` consecutive chunks
    of about ``chunk_s`` seconds each (a 2-iteration probe sizes them),
    carrying its state; its own timer gives each chunk's time and its records
    the chunk's inner iteration counts.  Model: one outer iteration costs
    c0 + c1 (pIters + 1) + c2 (uSweeps + vSweeps), fitted by non-negative least
    squares over the chunks.  The whole solve's time is the model summed over
    ``hist``, the inner counts of the solve being timed (this library's FP64
    solve of the same design: the reference's arithmetic, so its counts are the
    reference's up to the order of the grid-wide sums)."""
    from scipy.optimize import nnls

    from oracle import reference
    if not reference.available(precision):
        return None
    rows, times, n_iters, t0 = [], [], 0, time.perf_counter()
    for st in starts:
        probe = reference.run(design, 2, precision=precision, threads=threads, init=st)
        per = max(float(probe["elapsed"][0]) / 2, 1e-5)
        n = int(max(2, min(20000, chunk_s / per)))
        state = st
        for _ in range(chunks):
            out = reference.run(design, n, precision=precision, threads=threads, init=state)
            k = len(out["err"])
            rows.append([k, float(np.sum(out["pIters"] + 1)), float(np.sum(out["uSweeps"] + out["vSweeps"]))])
            times.append(float(out["elapsed"][0]))
            n_iters += k
            state = {q: out[q] for q in ("u", "v", "p")}
    A, t = np.array(rows), np.array(times)
    coef, _ = nnls(A, t)
    fit = A @ coef
    T = float(coef[0] * len(hist) + coef[1] * np.sum(hist[:, 5] + 1) + coef[2] * np.sum(hist[:, 6] + hist[:, 7]))
    return {"value": 1.0 / T, "unit": "solves/s", "cores": threads, "kind": "reference",
            "precision": "f64 (the reference's sources promoted to double)" if precision == "f64"
            else "f32 (the reference as shipped)",
            "ms_per_outer_iteration": 1e3 * T / len(hist),
            "model_ms": {"per_outer_iteration": 1e3 * coef[0], "per_pcg_iteration": 1e3 * coef[1],
                         "per_jacobi_sweep": 1e3 * coef[2]},
            "model_fit_rel_rms": float(np.sqrt(np.mean(((fit - t) / t) ** 2))),
            "sample": (f"{n_iters} outer iterations of the reference in {len(times)} timed chunks of about "
                       f"{chunk_s:.0f} s from {len(starts)} states along this design's trajectory "
                       f"({time.perf_counter() - t0:.0f} s of wall time), extrapolated to the whole solve "
                       f"({len(hist)} outer iterations) with a per-iteration cost model linear in the inner "
                       f"iteration counts")}


def port_baseline(design, hist: np.ndarray, starts, chunk_s: float = 3.0) -> dict:
    """cpu_baseline's sample and cost model with the oracle's C restatement
    (one thread) in place of the reference's build, when that is absent."""
    from scipy.optimize import nnls

    from oracle import restatement as rs
    rows, times, n_iters = [], [], 0
    for st in starts:
        f = rs.new_fields(design)
        if st is not None:
            for k in ("u", "v", "p"):
                f[k][...] = st[k]
        t = time.perf_counter()
        rs.solve(design, f, 2, stop_on_conv=False)
        n = int(max(2, min(20000, chunk_s / max((time.perf_counter() - t) / 2, 1e-6))))
        t = time.perf_counter()
        hh = rs.solve(design, f, n, stop_on_conv=False)
        times.append(time.perf_counter() - t)
        rows.append([len(hh), float(np.sum(hh[:, 5] + 1)), float(np.sum(hh[:, 6] + hh[:, 7]))])
        n_iters += len(hh)
    coef, _ = nnls(np.array(rows), np.array(times))
    T = float(coef[0] * len(hist) + coef[1] * np.sum(hist[:, 5] + 1) + coef[2] * np.sum(hist[:, 6] + hist[:, 7]))
    return {"value": 1.0 / T, "unit": "solves/s", "cores": 1, "kind": "port",
            "ms_per_outer_iteration": 1e3 * T / len(hist),
            "sample": (f"{n_iters} outer iterations of the oracle's C restatement (one thread) from {len(starts)} "
                       f"states along this design's trajectory, extrapolated to the whole solve with a "
                       f"per-iteration cost model linear in the inner iteration counts")}


# ---------------------------------------------------------------------------
# arms
# ---------------------------------------------------------------------------
def run_b200(args) -> None:
    rank, local, world = dist_init(args.gpus)
    import torch

    from coldplate_solver_b200 import cps
    device = local
    torch.cuda.set_device(device)
    design, cfg = workload(args.workload)
    precision = cps.CPS_MIXED if args.precision == "mixed" else cps.CPS_FP64
    solver = cps.Solver(design, precision=precision, device=device)
    stream = torch.cuda.ExternalStream(solver.stream, device=device)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=device)

    start = None
    if args.start_outer > 0:
        # a late state of the solve: the state after start_outer outer iterations from zero
        solver.reset_fields()
        solver.solve(args.start_outer, eps=0.0)
        f = solver.download()
        start = tuple(np.ascontiguousarray(f[k]) for k in ("u", "v", "p"))

    def one_solve():
        if start is None:
            solver.reset_fields()
        else:
            solver.upload_fields(*start)
        return solver.solve(args.max_outer, eps=EPS)

    hist = None
    for _ in range(args.warmup):
        hist = one_solve()
    iters_per_solve = len(hist)
    converged = bool(max(hist[-1, 0], hist[-1, 1], hist[-1, 3]) <= EPS)

    # ---- device-resident timing ----
    barrier(world)
    torch.cuda.synchronize(device)
    solver.kernel_timing(reset=True)
    step_ms, alg_bytes, iters = [], 0.0, []
    with ClockSampler(device) as clocks:
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)  # evict the previous step's working set from L2
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            h = one_solve()
            with torch.cuda.stream(stream):
                e1.record(stream)
            e1.synchronize()
            step_ms.append(e0.elapsed_time(e1))
            alg_bytes += algorithmic_bytes(design, h)
            iters.append(len(h))
    torch.cuda.synchronize(device)
    barrier(world)
    kernel_ms, launches, outer_done = solver.kernel_timing(reset=True)
    total_s = max_over_ranks(sum(step_ms) / 1e3, world, local)
    value = world * args.steps / total_s

    # ---- end to end through the C ABI with host buffers ----
    M, N = design.M, design.N
    host_in = {k: torch.zeros(s, dtype=torch.float64).pin_memory().numpy()
               for k, s in (("u", (M + 1, N)), ("v", (M, N + 1)), ("p", (M + 1, N + 1)))}
    alpha = torch.from_numpy(design.alpha).pin_memory().numpy()
    gamma = torch.from_numpy(design.gamma).pin_memory().numpy()
    h2d = (alpha.nbytes + gamma.nbytes + sum(a.nbytes for a in host_in.values()))
    d2h = sum(a.nbytes for a in host_in.values()) + 8 * 8 * iters_per_solve
    e2e_steps = max(1, min(args.steps, 5))
    barrier(world)
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        solver.upload_geometry(alpha, gamma)
        solver.upload_fields(host_in["u"], host_in["v"], host_in["p"])
        solver.solve(args.max_outer, eps=EPS)
        solver.download()
    e2e_s = max_over_ranks(time.perf_counter() - t0, world, local)
    barrier(world)

    # ---- error against the FP64 oracle's fixed point (untimed) ----
    oracle_err = None
    fx = oracle_fixture(ORACLE_FIXTURES.get(args.workload))
    if fx is not None and args.max_outer >= MAX_OUTER and args.start_outer == 0:
        solver.reset_fields()
        solver.solve(args.max_outer, eps=EPS)
        oracle_err = oracle_error_block(solver, design, fx, ORACLE_FIXTURES[args.workload])

    # ---- the plain FP64 path on the same design, when this line is another precision ----
    plain = None
    if precision != cps.CPS_FP64:
        with cps.Solver(design, precision=cps.CPS_FP64, device=device) as sp:
            sp.reset_fields()
            sp.solve(args.max_outer, eps=EPS)  # warm-up
            ms_plain = []
            for _ in range(max(1, min(args.steps, 5))):
                sp.reset_fields()
                sp.kernel_timing(reset=True)
                hp = sp.solve(args.max_outer, eps=EPS)
                ms_plain.append(sp.kernel_timing(reset=True)[0])
            plain = {"value": 1e3 / float(np.mean(ms_plain)), "unit": "solves/s",
                     "outer_iterations_per_solve": int(len(hp)),
                     "speedup": value / (1e3 / float(np.mean(ms_plain)))}

    # ---- CPU baseline (rank 0, N = 1 only): a bounded sample of the reference ----
    cpu = None
    if world == 1 and rank == 0 and not args.no_cpu_baseline:
        starts = [None]
        for frac in (0.2, 0.4, 0.6, 0.8):
            solver.reset_fields()
            solver.solve(max(1, int(frac * iters_per_solve)), eps=0.0)
            f = solver.download()
            starts.append({k: f[k] for k in ("u", "v", "p")})
        cpu = cpu_baseline(design, h, starts, host_cores(), chunk_s=args.cpu_chunk_s)
        if cpu is not None:
            shipped = cpu_baseline(design, h, starts, host_cores(), chunk_s=args.cpu_chunk_s, chunks=1,
                                   precision="f32")
            if shipped is not None:
                shipped["note"] = ("the reference as shipped (FP32), extrapolated with this solve's FP64 inner "
                                   "counts; its own FP32 trajectory differs")
                cpu["as_shipped_fp32"] = shipped
        else:
            cpu = port_baseline(design, h, starts)

    solver.close()
    if rank != 0:
        return
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(REPO, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    kernel_s = kernel_ms / 1e3
    achieved = alg_bytes / kernel_s / 1e9 if kernel_s > 0 else None
    lat = sorted(step_ms)
    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * total_s / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if precision == cps.CPS_FP64 else "f32+f64",
        "data": "synthetic (seeded generator)", "impl": "b200",
        "config": dict(cfg, l2="flushed between steps (512 MiB write)", precision=args.precision,
                       outer_iterations_per_solve=iters_per_solve, converged=converged,
                       parallelism=f"replicas x{world}",
                       **({"start_outer": args.start_outer} if args.start_outer else {})),
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
        "cell_updates_per_s": world * design.M * design.N * sum(iters) / total_s,
        "e2e": {"value": world * e2e_steps / e2e_s, "unit": "solves/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None,
                     "traffic": MEASURED_TRAFFIC.get((args.workload, args.precision)),
                     "traffic_source": "ncu launch list of the full workload (dram bytes per launch)"
                     if (args.workload, args.precision) in MEASURED_TRAFFIC else None,
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs" if peaks else "fallback 6650 GB/s",
                     "kernel": "cps_grid_kernel", "kernel_ms_per_launch": kernel_ms / max(1, launches),
                     "algorithmic_bytes_per_launch": alg_bytes / max(1, launches)},
        "gpu_launches": int(launches),
        "clocks": clocks.summary(),
    }
    if oracle_err is not None:
        line["error_vs_fp64_oracle"] = oracle_err
    if plain is not None:
        line["vs_plain_fp64_gpu"] = plain
    if cpu is not None:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# thermal workload: the 3-D conjugate-heat-transfer solve downstream of the flow
# ---------------------------------------------------------------------------
THERMAL_METRIC = "converged thermal solves/s (relative residual 1e-6)"
# DRAM bytes (read + write) per launch of the thermal solve on the full
# 1000 x 500 x 9 workload (63 BiCGStab iterations), from a one-pass ncu launch
# list; profiles/cpt_solve_kernel_thermal_density_fp64.txt has the command.
THERMAL_TRAFFIC = 3.058e11


def thermal_bytes_per_iteration(n_levels_cells) -> float:
    """Minimal single-pass FP64 streams of one BiCGStab iteration of the
    thermal solve: two V-cycles (per level and cell, 2 + 2 damped-Jacobi
    sweeps, restriction and prolongation: 44 elements), the two matrix-vector
    products with their dots (10 elements each), s (3), the T/r update (8)
    and p (4) on the finest level."""
    n0 = n_levels_cells[0]
    return 8.0 * (2 * 44 * sum(n_levels_cells[:-1]) + (10 + 3 + 10 + 8 + 4) * n0)


def thermal_case(nx: int = 1000, setup_outer: int = 3000):
    """The thermal inputs of the nx x nx/2 density-field design: the flow
    after ``setup_outer`` outer iterations (untimed set-up), uniform base flux
    1e6 W/m^2, reference Params otherwise (H_t = the design's channel height)."""
    from coldplate_solver_b200 import cps, geometry as g, thermal as pt
    d = g.density_field(Nx=nx)
    with cps.Solver(d) as s:
        s.solve(setup_outer, eps=0.0)
        f = s.download()
    c = pt.ThermalCase.from_flow(d, f, q=1e6)
    cfg = {"workload": f"thermal_density_{c.Nx}x{c.Ny}x{c.Nz}", "grid": f"{c.Nx}x{c.Ny}x{c.Nz}", "dx_um": 10,
           "flow": f"density_field_{d.N}x{d.M} after {setup_outer} outer iterations", "q_w_m2": 1e6,
           "rtol": c.rtol, "k_interp": "RAMP qk=1"}
    return c, cfg


def run_thermal(args) -> None:
    rank, local, world = dist_init(args.gpus)
    import torch

    from coldplate_solver_b200 import thermal as pt
    device = local
    torch.cuda.set_device(device)
    case, cfg = thermal_case(args.thermal_nx)
    ts = pt.ThermalSolver(case, device=device)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=device)
    for _ in range(args.warmup):
        r = ts.solve()
    iters_per_solve = r["iterations"]
    levels_cells = []
    nx, ny = case.Nx, case.Ny
    while True:
        levels_cells.append(nx * ny * case.Nz)
        if nx == 1 and ny == 1:
            break
        nx, ny = (nx + 1) // 2, (ny + 1) // 2
    barrier(world)
    torch.cuda.synchronize(device)
    ts.timing(reset=True)
    step_ms, iters = [], []
    with ClockSampler(device) as clocks:
        for _ in range(args.steps):
            flush.fill_(1.0)
            torch.cuda.synchronize(device)
            before, _ = ts.timing()
            r = ts.solve()
            after, _ = ts.timing()
            step_ms.append(after - before)
            iters.append(r["iterations"])
    torch.cuda.synchronize(device)
    barrier(world)
    kernel_ms, n_levels = ts.timing(reset=True)
    total_s = max_over_ranks(sum(step_ms) / 1e3, world, local)
    value = world * args.steps / total_s
    alg_bytes = sum(iters) * thermal_bytes_per_iteration(levels_cells)
    # end to end through the C ABI: host inputs in, host temperature out
    pin = {k: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
           for k, a in (("gamma", case.gamma), ("u", case.u), ("v", case.v), ("q0", case.heat_flux()))}
    T_host = torch.zeros(case.Nz * case.Ny * case.Nx, dtype=torch.float64).pin_memory().numpy()
    h2d = sum(a.nbytes for a in pin.values())
    d2h = T_host.nbytes + 8 * 4
    e2e_steps = max(1, min(args.steps, 5))
    barrier(world)
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        ts.update(pin["gamma"], pin["u"], pin["v"], pin["q0"])
        ts.solve()
        T_host[:] = ts.temperature().ravel()
    e2e_s = max_over_ranks(time.perf_counter() - t0, world, local)
    barrier(world)
    cpu = None
    if world == 1 and rank == 0 and not args.no_cpu_baseline:
        from oracle import thermal as th
        p = th.ThermalParams(Nx=case.Nx, Ny=case.Ny, dx=case.dx, dy=case.dy, H_t=case.H_t, rtol=case.rtol)
        _, it_cpu, sec, done = th.mg_bicgstab_cpu(p, case.gamma, case.u, case.v, case.heat_flux(),
                                                   time_cap=args.cpu_time_cap)
        per_solve = sec if done else sec * max(1, iters_per_solve) / max(1, it_cpu)
        cpu = {"value": 1.0 / per_solve, "unit": "solves/s", "cores": 1, "kind": "port",
               "sample": (f"scipy port of this solve's algorithm (assembly, aggregation multigrid, BiCGStab), "
                          f"{it_cpu} iterations in {sec:.1f} s" + ("" if done else
                          f", extrapolated to the GPU's {iters_per_solve} iterations")),
               "note": "the reference's own thermal solve needs AMGCL, absent from the reference tree"}
    ts.close()
    if rank != 0:
        return
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(REPO, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    achieved = alg_bytes / (kernel_ms / 1e3) / 1e9 if kernel_ms > 0 else None
    line = {
        "metric": THERMAL_METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * total_s / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
        "impl": "b200",
        "config": dict(cfg, l2="flushed between steps (512 MiB write)", iterations_per_solve=iters_per_solve,
                       multigrid_levels=n_levels, parallelism=f"replicas x{world}"),
        "e2e": {"value": world * e2e_steps / e2e_s, "unit": "solves/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None,
                     "traffic": THERMAL_TRAFFIC if args.thermal_nx == 1000 else None,
                     "traffic_source": "ncu launch list of the full workload (dram bytes per launch, 63 iterations)"
                     if args.thermal_nx == 1000 else None,
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs" if peaks else "fallback 6650 GB/s",
                     "kernel": "cpt::solve_kernel", "kernel_ms_per_launch": kernel_ms / args.steps,
                     "algorithmic_bytes_per_launch": alg_bytes / args.steps},
        "gpu_launches": args.steps,
        "clocks": clocks.summary(),
    }
    if cpu is not None:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)


def run_reference(args) -> None:
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import reference
    if args.workload == "thermal":
        print(json.dumps({"impl": "reference", "unavailable": "the reference's thermal solve includes AMGCL, whose "
                          "headers are absent from the reference tree (ThermalSolver/amgcl is empty)"}), flush=True)
        return
    if args.workload == "served":
        print(json.dumps({"impl": "reference", "unavailable": "a served stream is a GPU serving loop; the "
                          "reference's CPU rate on the same designs is the mix arm's (--workload mix)"}))
        return
    if args.workload == "mix":
        run_reference_mix(args)
        return
    design, cfg = workload(args.workload)
    if not reference.available("f64"):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_f64 is not built (make -C oracle ref REF=<reference checkout>)"}))
        return
    threads = args.ref_threads or host_cores()
    for _ in range(args.warmup):
        reference.run(design, 10, precision="f64", threads=threads)
    r = reference_solve(design, threads, REFERENCE_ITERS.get(args.workload, 20000), args.steps, args.ref_time_cap)
    value, sample, done, chunks = r["value"], r["sample"], r["iters"], r["chunks"]
    # the as-shipped FP32 build beside it, when the FP64 solve was short enough to repeat
    shipped = (as_shipped_fp32(design, threads, REFERENCE_ITERS.get(args.workload, 20000), args.ref_time_cap)
               if r["seconds"] < 120.0 else None)
    print(json.dumps({
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": chunks,
        "warmup": args.warmup, "ms_per_step": r["ms_per_chunk"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
        "impl": "reference",
        "config": dict(cfg, outer_iterations_per_solve=done, converged=r["converged"],
                       ms_per_outer_iteration=r["ms_per_outer_iteration"]),
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": threads, "kind": "reference", "sample": sample,
                         "precision": "f64 (the reference's sources promoted to double)",
                         **({"as_shipped_fp32": shipped} if shipped is not None else {})},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def run_reference_mix(args) -> None:
    """The reference on the seeded subsample of the mix whose converged counts
    oracle/mix_counts.py recorded: each design solved from the zero state to
    its 1e-6 stop on all host cores, or, past --ref-design-cap seconds,
    extrapolated to its recorded count; solves/s = designs / summed time."""
    from coldplate_solver_b200 import geometry as g
    from oracle import reference
    path = os.path.join(REPO, "oracle", "mix_reference_counts.json")
    if not reference.available("f64") or not os.path.exists(path):
        print(json.dumps({"impl": "reference", "unavailable": "needs oracle/_ref/ref_f64 and "
                          "oracle/mix_reference_counts.json (python oracle/mix_counts.py)"}))
        return
    counts = json.load(open(path))
    mix = g.batch_mix(64)
    threads = host_cores()
    reference.run(mix[counts["designs"][0]["k"]], 10, precision="f64", threads=threads)  # warm-up
    rows, total = [], 0.0
    for row in counts["designs"]:
        r = reference_solve(mix[row["k"]], threads, row["iters"], 4, args.ref_design_cap)
        t = 1.0 / r["value"]
        total += t
        rows.append({"k": row["k"], "M": row["M"], "N": row["N"], "seconds": t, "converged": r["converged"],
                     "iters": r["iters"]})
    value = len(rows) / total
    sample = (f"{len(rows)} designs of the 64-design mix (seed {counts['subsample_seed']}), each solved to its own "
              f"1e-6 stop or extrapolated after {args.ref_design_cap:.0f} s to the count recorded by "
              f"oracle/mix_counts.py; solves/s = designs / summed time")
    print(json.dumps({
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": 1, "steps": len(rows),
        "warmup": 1, "ms_per_step": 1e3 * total / len(rows), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)", "impl": "reference",
        "config": {"workload": "density_mix_subsample_of_64_nx256-1024", "designs": rows, "eps": EPS},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


# ---------------------------------------------------------------------------
# many-design workloads: batched mix and served stream
# ---------------------------------------------------------------------------
def many_designs(args):
    from coldplate_solver_b200 import geometry as g
    if args.workload == "mix":
        designs = g.batch_mix(64)[: args.designs]
        cfg = {"workload": f"density_mix_{len(designs)}of64_nx256-1024", "designs": len(designs), "dx_um": 10,
               "convection": "SOU", "two_point_five_d": True, "nx_range": [256, 1024]}
        return designs, [0.0] * len(designs), cfg
    stream = g.served_stream(args.requests, rate=20.0)
    cfg = {"workload": f"served_stream_{args.requests}req_poisson20_nx128-2048", "requests": args.requests,
           "arrival_rate_per_s": 20.0, "nx_range": [128, 2048], "hbm_budget_gb": 120}
    return [d for _, d in stream], [t for t, _ in stream], cfg


def plain_fp64_sequential(designs, arrivals, device):
    """Every design alone on the single-design FP64 kernel, one after another
    (device time per solve); FIFO latencies for the given arrival times."""
    from coldplate_solver_b200 import cps
    rows = []
    for d in designs:
        with cps.Solver(d, precision=cps.CPS_FP64, device=device) as s:
            s.reset_fields()
            s.kernel_timing(reset=True)
            h = s.solve(MAX_OUTER, eps=EPS)
            ms, launches, it = s.kernel_timing(reset=True)
            rows.append({"ms": ms, "iters": int(it), "dp": s.full_dp(), "launches": launches,
                         "converged": bool(max(h[-1, 0], h[-1, 1], h[-1, 3]) <= EPS)})
    t, lat = 0.0, []
    for a, r in zip(arrivals, rows):
        t = max(t, a * 1e3) + r["ms"]
        lat.append(t - a * 1e3)
    return rows, lat


def run_many(args) -> None:
    import torch

    from coldplate_solver_b200 import batch, cps, serve
    rank, local, world = dist_init(args.gpus)
    device = local
    torch.cuda.set_device(device)
    designs, arrivals, cfg = many_designs(args)
    precision = cps.CPS_MIXED if args.precision == "mixed" else cps.CPS_FP64
    tuned = None
    tile_j = 32
    if args.visit is None:
        args.visit = 512 if args.workload == "served" else 4096
    if args.placement == "auto" and args.workload == "mix":
        # the project's autotuner: placement from zero- and warm-state probes,
        # visit length from converged solves of a sample (untimed)
        tuned = batch.autotune(designs, precision, device)
        mode, args.visit, tile_j = tuned.mode, tuned.visit, tuned.tile_j
    else:
        if args.placement == "auto" and args.workload == "served":
            # groups sized to each request (8 tiles per CTA): measured best for the
            # served stream among SM-count groups and sized groups, with either order
            mode = {"tiles_per_cta": 8}
        else:
            mode = (batch.default_mode(device) if args.placement in ("default", "auto")
                    else json.loads(args.placement))
    n = len(designs)
    clocks = None
    oracle_err = None
    if args.workload == "mix":
        # Designs shard across ranks (longest-processing-time assignment on the
        # cell count, no collective on the data path); each rank solves its
        # shard with the batched kernel and the per-design results are gathered
        # once at the end.
        from coldplate_solver_b200 import shard
        pos = {id(d): k for k, d in enumerate(designs)}  # a design's index, by identity (designs hold arrays)
        mine = [designs[k] for k in shard.assign(designs, world)[rank]]
        seq_mine, _ = plain_fp64_sequential(mine, [0.0] * len(mine), device)
        stats = {"ms_total": 0.0, "launches": 0, "wall": 0.0, "e2e_s": 0.0, "h2d": 0, "d2h": 0, "clocks": None}

        def solve_shard(ds):
            """This rank's designs: warm-up visits, the timed steps, the
            untimed error check against the oracle fixtures, then one e2e run
            from host memory to converged fields on the host."""
            idx = [pos[id(d)] for d in ds]
            with batch.BatchRunner(ds, precision=precision, device=device, mode=mode, tile_j=tile_j) as br:
                for _ in range(args.warmup):  # module load, first touch; short visits from the zero state
                    br.run(eps=EPS, max_outer=100, visit=100)
                with ClockSampler(device) as ck:
                    t0 = time.perf_counter()
                    for _ in range(args.steps):
                        res, ms, nl = br.run(eps=EPS, max_outer=MAX_OUTER, visit=args.visit)
                        stats["ms_total"] += ms
                        stats["launches"] += nl
                    stats["wall"] = time.perf_counter() - t0
                stats["clocks"] = ck
                out = []
                for k, r, s_ in zip(idx, res, br.solvers):
                    row = {"k": k, "iters": int(r["outer_iterations"]), "converged": bool(r["converged"]),
                           "finished_ms": float(r["finished_ms"]), "dp": s_.full_dp()}
                    fx = oracle_fixture(MIX_FIXTURES.get(k))
                    if fx is not None:
                        row["error_vs_fp64_oracle"] = oracle_error_block(s_, designs[k], fx, MIX_FIXTURES[k])
                    out.append(row)
            t1 = time.perf_counter()
            with batch.BatchRunner(ds, precision=precision, device=device, mode=mode, tile_j=tile_j) as br2:
                br2.run(eps=EPS, max_outer=MAX_OUTER, visit=args.visit, reset=False)
                fields = [s_.download() for s_ in br2.solvers]
            stats["e2e_s"] = time.perf_counter() - t1
            stats["h2d"] = sum(d.alpha.nbytes + d.gamma.nbytes for d in ds)
            stats["d2h"] = sum(sum(f[q].nbytes for q in ("u", "v", "p")) for f in fields)
            return out

        barrier(world)
        results = shard.run_sharded(designs, solve_shard, rank, world)
        clocks = stats["clocks"]
        step_s = max_over_ranks(stats["ms_total"] / 1e3 / args.steps, world, local)
        seq_s = max_over_ranks(sum(r["ms"] for r in seq_mine) / 1e3, world, local)
        e2e_s = max_over_ranks(stats["e2e_s"], world, local)
        launches = stats["launches"]
        seq = [None] * n
        gathered = [None] * world
        if world > 1:
            import torch.distributed as dist
            dist.all_gather_object(gathered, [(pos[id(d)], r) for d, r in zip(mine, seq_mine)])
        else:
            gathered = [[(pos[id(d)], r) for d, r in zip(mine, seq_mine)]]
        for part in gathered:
            for k, r in part:
                seq[k] = r
        seq_ms = 1e3 * seq_s
        seq_lat = [r["ms"] for r in seq]
        dps = [r["dp"] for r in results]
        iters = [r["iters"] for r in results]
        converged = sum(r["converged"] for r in results)
        lat = [r["finished_ms"] for r in results]
        value = n / step_s
        e2e = {"value": n / e2e_s, "unit": "solves/s", "h2d_bytes_per_step": stats["h2d"],
               "d2h_bytes_per_step": stats["d2h"]}
        timing = {"device_ms_per_step": 1e3 * step_s, "wall_s_per_step": stats["wall"] / args.steps}
        oracle_err = {str(r["k"]): r["error_vs_fp64_oracle"] for r in results if "error_vs_fp64_oracle" in r}
        cfg["parallelism"] = f"designs sharded x{world}"
    else:
        seq, seq_lat = plain_fp64_sequential(designs, arrivals, device)
        seq_ms = sum(r["ms"] for r in seq)
        srv = serve.Server(mode=mode, precision=precision, device=device, visit=args.visit, max_outer=MAX_OUTER,
                           keep=set(SERVED_FIXTURES), order="smallest", epoch_designs=args.epoch_designs)
        cfg["order"] = f"the {srv.epoch_designs} smallest in-flight requests advance in each epoch"
        warm = [(0.0, d) for d in designs[: min(4, n)]]
        for _ in range(args.warmup):
            serve.Server(mode=mode, precision=precision, device=device, visit=100, max_outer=100).run(
                warm, real_time=False)
        with ClockSampler(device) as clocks:
            st = srv.run(list(zip(arrivals, designs)), real_time=True)
        dps = [r.dp for r in st.requests]
        iters = [r.outer_iterations for r in st.requests]
        converged = st.completed
        lat = [1e3 * r.latency for r in st.requests]
        launches = st.epochs
        value = st.solves_per_s
        e2e = {"value": st.solves_per_s, "unit": "solves/s",
               "h2d_bytes_per_step": sum(d.alpha.nbytes + d.gamma.nbytes for d in designs),
               "d2h_bytes_per_step": 8 * n}
        timing = {"makespan_s": st.makespan_s, "device_ms": st.device_ms, "max_inflight": st.max_inflight,
                  "peak_bytes": st.peak_bytes}
    errs = [abs(a - r["dp"]) / abs(r["dp"]) for a, r in zip(dps, seq) if r["dp"] != 0]
    seq_value = n / (seq_ms / 1e3) if args.workload == "mix" else n / (max(seq_lat[k] + 1e3 * arrivals[k]
                                                                         for k in range(n)) / 1e3 - arrivals[0])
    if oracle_err is None and args.workload == "served":
        oracle_err = {}
        for k, name in SERVED_FIXTURES.items():
            fx = oracle_fixture(name)
            if k < n and fx is not None and st.requests[k].fields is not None:
                r = st.requests[k]
                oracle_err[str(k)] = {
                    "at_1e-6_stop": errors_vs_fixture(r.design, r.fields, r.dp, fx),
                    "reference_own_1e-6_stop": {"u": float(fx["stop_err_u"]), "v": float(fx["stop_err_v"]),
                                                "p": float(fx["stop_err_p"]), "dP": float(fx["stop_err_dp"])},
                    "oracle": f"tests/golden/converged/{name}.npz"}
    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "higher_is_better": True,
        "scaling": "strong" if args.workload == "mix" else "weak", "vs_baseline": None,
        "dtype": "f64" if precision == cps.CPS_FP64 else "f32+f64", "data": "synthetic (seeded generator)",
        "impl": "b200",
        "config": dict(cfg, precision=args.precision, placement=mode, visit=args.visit, eps=EPS,
                       tile=f"{256 // tile_j}x{tile_j}",
                       converged=f"{converged}/{n}", warmup="visits of 100 outer iterations per design",
                       l2="working set larger than L2 (all designs resident)"),
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
        "timing": timing,
        "outer_iterations": {"total": int(sum(iters)), "min": int(min(iters)), "max": int(max(iters))},
        "vs_plain_fp64_sequential": {
            "value": seq_value, "speedup": value / seq_value if seq_value > 0 else None,
            "device_ms": seq_ms, "latency_ms": {"p50": float(np.percentile(seq_lat, 50)),
                                                "p99": float(np.percentile(seq_lat, 99))},
            "outer_iterations_total": int(sum(r["iters"] for r in seq)),
            "converged": f"{sum(r['converged'] for r in seq)}/{n}"},
        "dp_rel_diff_vs_plain_fp64": {"max": float(max(errs)) if errs else None,
                                      "median": float(np.median(errs)) if errs else None,
                                      "note": "both stopped at the 1e-6 outer residual; see the parity tests "
                                              "for the 1e-10 comparison"},
        "e2e": e2e,
        "gpu_launches": int(launches),
        "clocks": clocks.summary() if clocks is not None else None,
    }
    if oracle_err:
        line["error_vs_fp64_oracle"] = oracle_err
    if tuned is not None:
        line["config"]["autotuned"] = {"placement": tuned.mode, "visit": tuned.visit,
                                       "tile": f"{256 // tuned.tile_j}x{tuned.tile_j}",
                                       "cell_updates_per_s": tuned.cell_updates_per_s,
                                       "tile_cell_updates_per_s": {f"{256 // k}x{k}": v for k, v in
                                                                   tuned.tile_cell_updates_per_s.items()},
                                       "visit_device_ms": {str(k): v for k, v in tuned.visit_ms.items()}}
    if rank == 0:
        print(json.dumps(line), flush=True)


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per launch of the
# single-design kernel, from the one-pass ncu launch list of the full default
# workload (`bench.py --steps 2 --warmup 3 --no-cpu-baseline`, 14 launches,
# FP64); profiles/cps_grid_kernel_network_500x250_fp64.txt has the command.
# Density 1000 x 500: two launches of the full workload (the first, early launch
# of a solve and the next, late one), 596.4 and 595.9 GB
# (profiles/cps_grid_kernel_density_1000x500_fp64.txt has the command).
MEASURED_TRAFFIC = {("network", "fp64"): 1.249e9, ("density", "fp64"): 5.962e11}

# Outer iterations of a converged FP64 solve of each workload (1e-6 outer
# residual): straight and network by the bit-exact FP64 oracle (the
# reference's own arithmetic, one thread), density by the reference's own
# FP64 build on 7 OpenMP threads: the first stage of its converged fixture
# (tests/golden/converged/density_1000x500.npz, n_stop; 435 s).
REFERENCE_ITERS = {"straight": 5564, "network": 9814, "density": 15420}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="density", choices=["straight", "network", "density", "mix", "served", "thermal"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--cpu-chunk-s", type=float, default=3.0,
                    help="CPU baseline: seconds per timed chunk of the reference (5 states x 2 chunks, FP64; "
                         "5 x 1 more for the as-shipped FP32 build)")
    ap.add_argument("--cpu-time-cap", type=float, default=90.0,
                    help="thermal CPU baseline: seconds after which the port's solve is extrapolated")
    ap.add_argument("--ref-threads", type=int, default=0,
                    help="reference arm: OpenMP threads of the reference (default: every host core)")
    ap.add_argument("--ref-time-cap", type=float, default=180.0,
                    help="reference arm: seconds after which an unfinished solve is extrapolated")
    ap.add_argument("--ref-design-cap", type=float, default=45.0,
                    help="reference arm, mix: seconds per design after which its solve is extrapolated")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--designs", type=int, default=64, help="mix: designs of the 64-design mix to solve")
    ap.add_argument("--requests", type=int, default=32, help="served: requests in the stream")
    ap.add_argument("--visit", type=int, default=None,
                    help="mix/served: outer iterations per design per launch (default: mix 4096 or the autotuner's; "
                         "served 512)")
    ap.add_argument("--placement", default="auto",
                    help='mix/served: "auto" (mix: the autotuner picks the placement, tile shape and visit length; '
                         'served: groups of 8 tiles per CTA), "default", or a JSON placement, e.g. '
                         '\'{"group_ctas": 148}\' or \'{"tiles_per_cta": 8}\'')
    ap.add_argument("--epoch-designs", type=int, default=12,
                    help="served: in-flight requests one epoch advances, smallest first")
    ap.add_argument("--thermal-nx", type=int, default=1000,
                    help="thermal: cells in x of the density-field design (y = x/2); 500 for small profiling captures")
    ap.add_argument("--start-outer", type=int, default=0,
                    help="straight/network/density: start every solve from the state after this many outer "
                         "iterations from zero (small profiling captures of the late phase)")
    ap.add_argument("--max-outer", type=int, default=MAX_OUTER,
                    help="cap on outer iterations per solve (small profiling captures; the line then says converged=false)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.workload in ("mix", "served"):
        run_many(args)
    elif args.workload == "thermal":
        run_thermal(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
