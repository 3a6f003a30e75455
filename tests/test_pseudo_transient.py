"""The pseudo-transient term and its CFL controllers (enablePseudoTimeStepping,
momentum_solver.cpp:231-241, iterations.cpp:189-217, time_control.cpp:43-166,
SIMPLE.cpp:321-327): the oracle's restatement against the reference's own
calculateStep and controllers (CPU), bit for bit in both precisions, for the
implicit and the explicit momentum path."""
import numpy as np
import pytest

from coldplate_solver_b200 import geometry
from oracle import reference
from oracle import restatement as rs

DESIGNS = {
    "straight_fou": lambda: geometry.straight_channel(M=20, N=40, band=(5, 15)),
    "network_sou_2.5d": lambda: geometry.channel_network(M=24, N=40, h=20e-6, wmin=3, wmax=6, seed=3),
    "density": lambda: geometry.density_field(Nx=48, seed=2, sigma=3.0),
}
# Controller settings: SER with its line search (the defaults), the residual
# ramp alone (SER off; a start residual at which the ramp's power law runs
# below its cap), SER on the step's error, and a global time step.  The line
# search never backtracks inside the outer loop: SER has just set
# serResidPrev to the residual it compares against.
SETTINGS = {
    "ser_ls": dict(serMinIter=3),
    "ramp": dict(enableSER=False, cflRampStartRes=0.02, pseudoCFLInitial=0.2, cflRampSmooth=0.3),
    "ser_maxresid": dict(serMinIter=2, serUseMaxResid=True, enableLineSearch=False, serSmooth=0.8),
    "global_dt": dict(useLocalPseudoTime=False, timeStepMultiplier=0.002, serMinIter=4),
}
FIELDS = ("u", "v", "p", "pStar", "uStar", "vStar", "dE", "dN")


def oracle_run(d, n, precision):
    """calculateStep followed by the controllers, n times, from the zero state;
    returns fields, the step diagnostics and the state after every step."""
    f = rs.new_fields(d, precision)
    st = rs.pseudo_start(d)
    hist, states = [], []
    for it in range(n):
        diag = rs.step(d, f, precision, pseudo_cfl=float(st[0]))
        st = rs.pseudo_update(d, st, diag, it, precision)
        hist.append([diag[k] for k in rs.DIAG_NAMES])
        states.append(st.copy())
    return f, np.array(hist), np.array(states)


@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("mom", [1, 0])
@pytest.mark.parametrize("setting", sorted(SETTINGS))
@pytest.mark.parametrize("name", sorted(DESIGNS))
def test_oracle_pseudo_transient_matches_the_reference(name, setting, mom, precision):
    if not reference.available(precision):
        pytest.skip(f"oracle/_ref/ref_{precision} not built")
    d = DESIGNS[name]().replace(enablePseudoTimeStepping=True, momentumSolverType=mom, **SETTINGS[setting])
    if mom == 0:
        d = d.replace(uvAlpha=0.5)
    n = 20
    ref = reference.run(d, n, precision=precision, stop_on_conv=False)
    f, h, st = oracle_run(d, n, precision)
    for k in FIELDS:
        assert np.array_equal(ref[k], f[k]), k
    np.testing.assert_array_equal(ref["pIters"], h[:, 5])
    for col, key in ((0, "residU"), (1, "residV"), (2, "residMass"), (4, "err")):
        np.testing.assert_array_equal(ref[key], h[:, col])
    np.testing.assert_array_equal(ref["pseudoCFL"], st[:, 0])
    np.testing.assert_array_equal(ref["pseudoState"].reshape(-1, 3), st[:, 1:])


def test_pseudo_transient_changes_the_step_and_the_cfl_moves():
    """The term is live: from the same state (three steady steps) the step
    differs from the steady one, and the controllers move the CFL number away
    from its start."""
    base = geometry.straight_channel(M=20, N=40, band=(5, 15))
    d = base.replace(enablePseudoTimeStepping=True, serMinIter=1)
    f0 = rs.new_fields(base)
    for _ in range(3):
        rs.step(base, f0)
    f1 = {k: a.copy() for k, a in f0.items()}
    rs.step(base, f0)
    rs.step(d, f1)
    assert not np.array_equal(f0["uStar"], f1["uStar"])
    _, _, st = oracle_run(d, 12, "f64")
    assert np.any(st[:, 0] != d.pseudo_cfl_start())


def test_oracle_solve_runs_the_controllers():
    """orc_solve's outer loop applies the controllers between steps, as the
    step-by-step loop above does."""
    d = geometry.straight_channel(M=20, N=40, band=(5, 15)).replace(enablePseudoTimeStepping=True, serMinIter=2)
    f_loop, h_loop, _ = oracle_run(d, 15, "f64")
    f = rs.new_fields(d)
    h = rs.solve(d, f, 15, stop_on_conv=False)
    for k in FIELDS:
        assert np.array_equal(f_loop[k], f[k]), k
    np.testing.assert_array_equal(h_loop, h)
