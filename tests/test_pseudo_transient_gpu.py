"""The pseudo-transient term and its CFL controllers on the GPU against the
oracle, which tests/test_pseudo_transient.py pins bit for bit to the
reference.  Tolerances as in test_parity_gpu.py: per-point values follow the
reference's operation order and only the grid-wide sums are grouped
differently.  The controllers run on the device after every outer iteration
from the grid-reduced residuals; their state is compared after the run.

Runs of several iterations are held to REL_RUN and kept to 8 iterations: the
pseudo-transient iteration on the straight channel amplifies a difference by
about 3x per outer iteration, most visibly in v, which is near zero there (the
FP64 oracle itself carries a 1e-14 perturbation of p to 1e-10 in v six
iterations later and to 8e-9 nine iterations later), so the sum-order
differences that every step adds outgrow 1e-10 within a few steps; one step
from a common state stays at REL_STEP."""
import ctypes

import numpy as np
import pytest

from coldplate_solver_b200 import cps, geometry
from oracle import restatement as rs

pytestmark = pytest.mark.gpu

REL_STEP = 1e-10
REL_RUN = 1e-8
FIELDS = ("u", "v", "p", "pStar", "uStar", "vStar", "dE", "dN")
DESIGNS = {
    "straight_fou": lambda: geometry.straight_channel(M=41, N=77, band=(10, 30)),
    "network_sou_2.5d": lambda: geometry.channel_network(M=64, N=131, h=20e-6, wmin=4, wmax=8, seed=7),
    "density": lambda: geometry.density_field(Nx=150, seed=2, sigma=4.0),
}
SETTINGS = {
    "ser_ls": dict(serMinIter=3),
    "ramp": dict(enableSER=False, cflRampStartRes=0.02, pseudoCFLInitial=0.2, cflRampSmooth=0.3),
    "ser_maxresid": dict(serMinIter=2, serUseMaxResid=True, enableLineSearch=False, serSmooth=0.8),
    "global_dt": dict(useLocalPseudoTime=False, timeStepMultiplier=0.002, serMinIter=4),
}


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / nb if nb > 0 else np.linalg.norm(a - b)


def pseudo_design(name, setting, mom=1):
    d = DESIGNS[name]().replace(enablePseudoTimeStepping=True, momentumSolverType=mom, **SETTINGS[setting])
    return d.replace(uvAlpha=0.5) if mom == 0 else d


def oracle_run(d, n):
    f = rs.new_fields(d)
    st = rs.pseudo_start(d)
    hist = []
    for it in range(n):
        diag = rs.step(d, f, pseudo_cfl=float(st[0]))
        st = rs.pseudo_update(d, st, diag, it)
        hist.append([diag[k] for k in rs.DIAG_NAMES])
    return f, np.array(hist), st


def check_against_oracle(d, h, f, state, n):
    fo, ho, sto = oracle_run(d, n)
    assert np.array_equal(h[:, 5], ho[:, 5]), (h[:, 5], ho[:, 5])
    for c in range(5):
        np.testing.assert_allclose(h[:, c], ho[:, c], rtol=1e-8, atol=1e-300)
    for k in FIELDS:
        assert rel(f[k], fo[k]) <= REL_RUN, (k, rel(f[k], fo[k]))
    np.testing.assert_allclose(state["pseudo_cfl"], sto[0], rtol=1e-8)
    np.testing.assert_allclose(state["ser_resid_prev"], sto[1], rtol=1e-6)
    assert state["ls_alpha"] == sto[2] and state["ls_backtracks"] == sto[3]


@pytest.mark.parametrize("mom", [1, 0])
@pytest.mark.parametrize("setting", sorted(SETTINGS))
@pytest.mark.parametrize("name", sorted(DESIGNS))
def test_pseudo_transient_solve_matches_the_oracle(name, setting, mom):
    d = pseudo_design(name, setting, mom)
    n = 8
    with cps.Solver(d) as s:
        h = s.solve(n, eps=0.0)
        f = s.download()
        st = s.pseudo_state()
    check_against_oracle(d, h, f, st, n)


@pytest.mark.parametrize("ctas", [3, 17])
def test_pseudo_transient_on_other_grids(ctas):
    d = pseudo_design("network_sou_2.5d", "ser_ls")
    n = 10
    with cps.Solver(d, grid_ctas=ctas) as s:
        h = s.solve(n, eps=0.0)
        f = s.download()
        st = s.pseudo_state()
    check_against_oracle(d, h, f, st, n)


def test_pseudo_transient_across_launches_and_steps():
    """The controllers' state and the iteration index carry from one call to
    the next: solve(4) + 3 x step + solve(5) equals one run of 12."""
    d = pseudo_design("density", "ser_ls")
    with cps.Solver(d) as s:
        hs = [s.solve(4, eps=0.0)]
        for _ in range(3):
            o = s.step()
            hs.append(np.array([[o[k] for k in ("residU", "residV", "residMass", "residMassDof", "err", "pIters",
                                                 "uSweeps", "vSweeps")]]))
        hs.append(s.solve(5, eps=0.0))
        f = s.download()
        st = s.pseudo_state()
    check_against_oracle(d, np.vstack(hs), f, st, 12)


def test_pseudo_transient_in_a_batch():
    """Designs with the term on (different settings) batched on CTA groups:
    each one equals its oracle run."""
    ds = [pseudo_design("straight_fou", "ser_ls"), pseudo_design("density", "ramp"),
          pseudo_design("network_sou_2.5d", "global_dt", mom=0)]
    n = 8
    solvers = [cps.Solver(d) for d in ds]
    try:
        res, _ = cps.batch_solve(solvers, n, eps=0.0, group_ctas=8)
        for d, s, r in zip(ds, solvers, res):
            assert r["n_done"] == n
            h = cps.get_history(s, n)
            check_against_oracle(d, h, s.download(), s.pseudo_state(), n)
    finally:
        for s in solvers:
            s.close()


def test_pseudo_state_api():
    d = pseudo_design("straight_fou", "ser_ls")
    with cps.Solver(d) as s:
        st = s.pseudo_state()
        assert st == {"pseudo_cfl": d.pseudo_cfl_start(), "ser_resid_prev": 0.0, "ls_alpha": 1.0, "ls_backtracks": 0}
        s.solve(8, eps=0.0)
        assert s.pseudo_state()["ser_resid_prev"] > 0.0
        s.set_pseudo_state(0.37, 1e-3, 0.5, 2)
        assert s.pseudo_state() == {"pseudo_cfl": 0.37, "ser_resid_prev": 1e-3, "ls_alpha": 0.5, "ls_backtracks": 2}
        s.reset_fields()  # a fresh solve: the controllers restart too
        assert s.pseudo_state()["pseudo_cfl"] == d.pseudo_cfl_start()
        p = cps.pseudo_from_design(d)
        p.time_step_multiplier = 0.0
        assert s.lib.cps_set_pseudo(s.ctx, ctypes.byref(p)) == cps.CPS_ERR_ARG
        p.time_step_multiplier = float("nan")
        assert s.lib.cps_set_pseudo(s.ctx, ctypes.byref(p)) == cps.CPS_ERR_ARG


def test_pseudo_step_with_a_given_cfl():
    """One step with the CFL number set from outside (the reference's own
    host controllers in the drop-in) equals the oracle's step at that CFL."""
    d = pseudo_design("network_sou_2.5d", "ser_ls")
    steady = d.replace(enablePseudoTimeStepping=False)
    fo = rs.new_fields(d)
    for _ in range(5):
        rs.step(steady, fo)
    with cps.Solver(d) as s:
        s.upload_fields(fo["u"], fo["v"], fo["p"])
        s.set_pseudo_state(1.7)
        s.step()
        f = s.download()
    rs.step(d, fo, pseudo_cfl=1.7)
    for k in FIELDS:
        assert rel(f[k], fo[k]) <= REL_STEP, (k, rel(f[k], fo[k]))


def test_pseudo_off_is_the_steady_path_bit_for_bit():
    d = DESIGNS["network_sou_2.5d"]()
    with cps.Solver(d) as a, cps.Solver(d.replace(enablePseudoTimeStepping=True)) as b:
        b.set_pseudo(d)  # enablePseudoTimeStepping = False switches it off again
        ha = a.solve(6, eps=0.0)
        hb = b.solve(6, eps=0.0)
        fa, fb = a.download(), b.download()
    assert np.array_equal(ha, hb)
    for k in FIELDS:
        assert np.array_equal(fa[k], fb[k]), k
