"""Generate the converged-state fixtures in tests/golden/converged/ from the
reference solver's own code (oracle/_ref/ref_f64: the reference's sources
promoted to double), run on all host cores.

For each design the reference solves from the zero state to its own 1e-6
stop (max(residU, residV, residMassDof) <= 1e-6) with the design's settings,
and then, carrying the state (u, v, p), on to the 1e-10 residual with tight
inner tolerances (TIGHT: PCG pTol 1e-10 with up to 1000 iterations, Jacobi
momentumTol 1e-10) -- for the density-field designs on to 1e-12 (``eps``
below), a margin: on the 500 x 250 design the state moves by less than 1e-8
between residual 1e-10 and 1e-12.  Where faces sit at the outer iteration's
velocity clamp (iterations.cpp:104) the pressure of the cells they enclose is
not determined by the fixed point; comparisons of p leave those cells out
(coldplate_solver_b200.geometry.pressure_determined_mask).  With the reference's default inner tolerances the
outer residual of these designs does not fall much below 1e-6: the PCG, held
to an absolute ||r|| < 1e-4, takes one step per outer iteration there, and the
residual wanders between ~3e-7 and ~4e-6 (the 1e-6 stop is one of its dips,
which is why the stop iteration moves with the order of the sums).  The
inner tolerances do not enter the fixed point of the iteration -- at a fixed
point the Jacobi and PCG corrections vanish, so it is the solution of the
discrete momentum and continuity equations -- and with tight ones the outer
residual falls geometrically; on the 137 x 68 served design the state at
residual 1e-8 is within 1.2e-8 relative of the state at the 1e-12 floor.
Stored per design:

  u, v, p        the fixed point (float32: its rounding, 6e-8 relative, is far
                 below the 1e-6 tolerance of the tests), every ``stride``-th
                 row and column (stride 2 for the 1000 x 500 design, 1 else)
  planes         the four sampled planes of the fixed point (x = 0, x = N hx,
                 core in, core out; flowArea, massFlux, avgStatic, avgDynamic,
                 avgTotal, valid), FP64
  dp_full        full inlet-outlet total-pressure drop of the fixed point
  n_stop, n_fixed            outer iterations to 1e-6 and then on to ``eps``
  eps            the residual the second stage ran to (1e-10, 1e-12 for the
                 density-field designs)
  stop_err_u/v/p, stop_err_dp  the reference's own 1e-6 stop state against
                 its fixed point (relative L2 on u, v and fluid-cell p where
                 the fixed point determines it,
                 relative dP): how far any run stopped at 1e-6 sits from the
                 fixed point
  tight          the inner tolerances of the second stage (JSON)
  generator, args            how to rebuild the design (geometry module)

Run from the repository root where the reference sources are available:
    make -C oracle ref REF=<reference checkout> && python tests/golden/make_converged.py [NAME ...]
The fixtures are committed; the tests read them without the reference.
``--save-state DIR`` also writes each design's full FP64 fixed point to
DIR/<name>_fp64.npz (not committed; a starting point for a deeper stage).
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from coldplate_solver_b200 import geometry as g  # noqa: E402
from oracle import reference  # noqa: E402

OUT = os.path.join(HERE, "converged")
EPS_STOP, EPS_FIXED = 1e-6, 1e-10
MAX_OUTER = 400000
TIGHT = {"pTol": 1e-10, "maxPressureIter": 1000, "momentumTol": 1e-10}


def design_of(generator: str, args: dict):
    """Rebuild a design from its generator name and arguments."""
    if generator == "channel_network":
        return g.channel_network(**args)
    if generator == "density_field":
        return g.density_field(**args)
    if generator == "batch_mix":
        return g.batch_mix(args["n"])[args["k"]]
    if generator == "served_stream":
        return g.served_stream(args["n"])[args["k"]][1]
    raise ValueError(generator)


# name -> (generator, arguments, stride, residual of the second stage)
CASES = {
    "network_500x250": ("channel_network", {}, 1, EPS_FIXED),
    "density_1000x500": ("density_field", {"Nx": 1000}, 2, 1e-12),
    "density_500x250": ("density_field", {"Nx": 500}, 1, 1e-12),
    "mix47_258x129": ("batch_mix", {"n": 64, "k": 47}, 1, EPS_FIXED),
    "served14_137x68": ("served_stream", {"n": 32, "k": 14}, 1, EPS_FIXED),
}


def fluid_mask_p(design, u=None, v=None) -> np.ndarray:
    """Cells whose density is fluid (gamma > 0.5), on p's index space; with a
    state (u, v), only those whose pressure it determines."""
    mask = np.zeros((design.M + 1, design.N + 1), dtype=bool)
    mask[1:design.M, 1:design.N] = design.gamma[:design.M - 1, :design.N - 1] > 0.5
    if u is not None:
        mask &= g.pressure_determined_mask(design, u, v)
    return mask


def rel(a, b) -> float:
    nb = float(np.linalg.norm(b))
    return float(np.linalg.norm(a - b)) / nb if nb > 0 else float(np.linalg.norm(a - b))


def full_dp(planes: np.ndarray) -> float:
    """avgTotal(x = 0) - avgTotal(x = N hx): the harness samples x = 0, N hx,
    core in, core out in that order."""
    return float(planes[0, 4] - planes[1, 4])


def make(name: str, threads: int, save_state: str = "") -> None:
    generator, args, stride, eps = CASES[name]
    d = design_of(generator, args)
    t0 = time.time()
    a = reference.run(d, MAX_OUTER, precision="f64", eps=EPS_STOP, stop_on_conv=True, threads=threads,
                      timeout=24 * 3600)
    n_stop = len(a["err"])
    print(f"{name}: 1e-6 stop after {n_stop} outer iterations ({time.time() - t0:.0f} s)", flush=True)
    stop = {k: a[k] for k in ("u", "v", "p")}
    b = reference.run(d.replace(**TIGHT), MAX_OUTER, precision="f64", eps=eps, stop_on_conv=True,
                      threads=threads, init=stop, timeout=24 * 3600)
    n_fixed = len(b["err"])
    last = max(b["residU"][-1], b["residV"][-1], b["residMassDof"][-1])
    if last > eps:
        raise RuntimeError(f"{name}: the reference did not reach {eps} in {MAX_OUTER} iterations ({last})")
    if save_state:
        os.makedirs(save_state, exist_ok=True)
        np.savez_compressed(os.path.join(save_state, name + "_fp64.npz"), u=b["u"], v=b["v"], p=b["p"],
                            residual=last, planes=b["planes"])
    mask = fluid_mask_p(d, b["u"], b["v"])
    dp_fixed, dp_stop = full_dp(b["planes"]), full_dp(a["planes"])
    s = stride
    os.makedirs(OUT, exist_ok=True)
    np.savez_compressed(
        os.path.join(OUT, name + ".npz"),
        u=b["u"][::s, ::s].astype(np.float32), v=b["v"][::s, ::s].astype(np.float32),
        p=b["p"][::s, ::s].astype(np.float32), stride=s, M=d.M, N=d.N,
        planes=b["planes"], dp_full=dp_fixed, dp_stop=dp_stop, n_stop=n_stop, n_fixed=n_fixed,
        stop_err_u=rel(a["u"], b["u"]), stop_err_v=rel(a["v"], b["v"]),
        stop_err_p=rel(a["p"][mask], b["p"][mask]), stop_err_dp=abs(dp_stop - dp_fixed) / abs(dp_fixed),
        residual_fixed=last, eps=eps, threads=threads, tight=json.dumps(TIGHT), generator=generator,
        args=json.dumps(args))
    print(f"{name}: {n_stop} + {n_fixed} outer iterations, dP {dp_fixed:.9g} Pa (at the 1e-6 stop {dp_stop:.9g}), "
          f"{time.time() - t0:.0f} s", flush=True)


def main(argv) -> None:
    """[--threads T] [--save-state DIR] [NAME ...]: OpenMP threads of the
    reference (default all host cores; give fewer when several designs are
    generated at once)."""
    threads = len(os.sched_getaffinity(0))
    save_state = ""
    while argv[:1] in (["--threads"], ["--save-state"]):
        if argv[0] == "--threads":
            threads = int(argv[1])
        else:
            save_state = argv[1]
        argv = argv[2:]
    for name in (argv or CASES):
        make(name, threads, save_state)


if __name__ == "__main__":
    main(sys.argv[1:])
