"""The inlet velocity ramp of cps_solve / cps_solve_monitored
(cps_set_inlet_ramp, SIMPLE.cpp:303-307) against the oracle's outer loop,
which tests/test_inlet_ramp.py pins to the reference's own loop.  Tolerances
as in test_parity_gpu.py and test_dp_gate_gpu.py."""
import numpy as np
import pytest

from coldplate_solver_b200 import cps, geometry
from oracle import restatement as rs

pytestmark = pytest.mark.gpu

FIELDS = ("u", "v", "p", "pStar", "uStar", "vStar", "dE", "dN")


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / nb if nb > 0 else np.linalg.norm(a - b)


@pytest.mark.parametrize("design", ["network", "density"])
def test_solve_with_ramp_matches_the_oracle(design):
    base = (geometry.channel_network(M=64, N=131, h=20e-6, wmin=4, wmax=8, seed=7) if design == "network"
            else geometry.density_field(Nx=150, seed=2, sigma=4.0))
    d = base.replace(enableInletRamp=True, rampSteps=5)
    n = 9
    fo = rs.new_fields(d)
    ho = rs.solve(d, fo, n, stop_on_conv=False)
    with cps.Solver(d) as s:
        h = s.solve(n, eps=0.0)
        f = s.download()
        # after the ramp the context's inlet velocity is the target again
        s.set_inlet_ramp(0)
        h_after = s.solve(1, eps=0.0)
    assert np.array_equal(h[:, 5], ho[:, 5])
    for c in range(5):
        np.testing.assert_allclose(h[:, c], ho[:, c], rtol=1e-8, atol=1e-300)
    for k in FIELDS:
        assert rel(f[k], fo[k]) <= 1e-10, (k, rel(f[k], fo[k]))
    o = rs.step(d, fo)  # the design's own inlet velocity
    np.testing.assert_allclose(h_after[0, :5], [o[k] for k in rs.DIAG_NAMES[:5]], rtol=1e-8, atol=1e-300)
    with cps.Solver(base) as plain:
        hp = plain.solve(n, eps=0.0)
    assert not np.array_equal(hp[:, 2], h[:, 2])  # the ramp changed the iteration


def test_ramp_with_the_pressure_drop_gate():
    """The monitored loop with the ramp over the gate's rampSteps, as the
    reference's runIterations runs them from one member."""
    d = geometry.straight_channel(M=20, N=40, band=(5, 15)).replace(enableInletRamp=True)
    xc = (0.25 * d.N * d.hx, 0.75 * d.N * d.hx)
    W, pct, ramp = 20, 0.5, 12
    f = rs.new_fields(d)
    dp_o, conv_o = rs.dp_gate_solve(d, f, 5000, W, pct, ramp, x_core=xc)
    assert conv_o
    with cps.Solver(d.replace(rampSteps=ramp)) as s:
        s.set_dp_monitor(gate=True, window=W, percent=pct, ramp_steps=ramp, x_core_in=xc[0], x_core_out=xc[1])
        hist, dp_g, conv_g = s.solve_monitored(5000, eps=0.0)
    assert conv_g
    assert abs(len(dp_g) - len(dp_o)) <= 1, (len(dp_g), len(dp_o))
    k = min(len(dp_g), len(dp_o))
    np.testing.assert_allclose(dp_g[:k], dp_o[:k], rtol=1e-9, atol=1e-9)


def test_ramp_restarts_with_reset_fields():
    d = geometry.channel_network(M=40, N=72, h=20e-6, wmin=4, wmax=8, seed=5).replace(enableInletRamp=True,
                                                                                     rampSteps=4)
    with cps.Solver(d) as s:
        h1 = s.solve(6, eps=0.0)
        s.reset_fields()
        h2 = s.solve(6, eps=0.0)
        assert s.lib.cps_set_inlet_ramp(s.ctx, -1) == cps.CPS_ERR_ARG
    assert np.array_equal(h1, h2)


def test_gate_with_ramp_and_pseudo_transient():
    """The monitored loop with the inlet ramp and the pseudo-transient term
    and its controllers all on, against the oracle's loop (which
    tests/test_inlet_ramp.py pins to the reference's runIterations).  The
    pseudo-transient iteration amplifies the sum-order differences of every
    step (measured: at most 1.1e-5 relative in the drops over the ~900
    iterations to the gate, the first iterations equal to 7 digits), so the
    drops are compared to 1e-4 and the stop iteration within two."""
    d = geometry.channel_network(M=24, N=40, h=20e-6, wmin=3, wmax=6, seed=3).replace(
        enableInletRamp=True, enablePseudoTimeStepping=True, serMinIter=5)
    xc = (0.25 * d.N * d.hx, 0.75 * d.N * d.hx)
    W, pct, ramp = 30, 0.2, 15
    f = rs.new_fields(d)
    dp_o, conv_o = rs.dp_gate_solve(d, f, 5000, W, pct, ramp, x_core=xc)
    assert conv_o
    with cps.Solver(d.replace(rampSteps=ramp)) as s:
        s.set_dp_monitor(gate=True, window=W, percent=pct, ramp_steps=ramp, x_core_in=xc[0], x_core_out=xc[1])
        hist, dp_g, conv_g = s.solve_monitored(5000, eps=0.0)
    assert conv_g
    assert abs(len(dp_g) - len(dp_o)) <= 2, (len(dp_g), len(dp_o))
    k = min(len(dp_g), len(dp_o))
    np.testing.assert_allclose(dp_g[:k], dp_o[:k], rtol=1e-4, atol=1e-9)
    np.testing.assert_allclose(dp_g[:30], dp_o[:30], rtol=1e-8, atol=1e-9)  # the ramp's iterations
