"""The outer loop's inlet velocity ramp (enableInletRamp, SIMPLE.cpp:303-307)
and, with it, the pseudo-transient controllers inside the reference's own
runIterations (CPU): the oracle's outer loop against the reference's loop,
bit for bit in the fields."""
import numpy as np
import pytest

from coldplate_solver_b200 import geometry
from oracle import reference
from oracle import restatement as rs

FIELDS = ("u", "v", "p", "pStar", "uStar", "vStar", "dE", "dN")


def test_ramp_values():
    d = geometry.straight_channel(M=20, N=40, band=(5, 15)).replace(enableInletRamp=True, rampSteps=8)
    U = d.inletVelocity
    got = [rs.inlet_velocity(d, it) for it in range(12)]
    assert got[:8] == [((it + 1) / 8) * U for it in range(8)]
    assert got[8:] == [U] * 4
    assert rs.inlet_velocity(d.replace(enableInletRamp=False), 0) == U
    assert rs.inlet_velocity(d.replace(rampSteps=0), 0) == U


@pytest.mark.skipif(not reference.available("f64"), reason="oracle/_ref/ref_f64 not built")
@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("mom", [1, 0])
def test_oracle_solve_with_ramp_matches_the_reference_steps(mom, precision):
    d = geometry.channel_network(M=24, N=40, h=20e-6, wmin=3, wmax=6, seed=3).replace(
        enableInletRamp=True, rampSteps=6, momentumSolverType=mom, uvAlpha=0.5 if mom == 0 else 0.7)
    n = 10
    ref = reference.run(d, n, precision=precision, stop_on_conv=False)
    f = rs.new_fields(d, precision)
    h = rs.solve(d, f, n, stop_on_conv=False, precision=precision)
    for k in FIELDS:
        assert np.array_equal(ref[k], f[k]), k
    np.testing.assert_array_equal(ref["residMass"], h[:, 2])


@pytest.mark.skipif(not reference.available("f64"), reason="oracle/_ref/ref_f64 not built")
@pytest.mark.parametrize("pseudo", [False, True])
def test_oracle_loop_matches_runIterations_with_ramp(pseudo):
    """The reference's own runIterations (its ramp, its controllers, its
    pressure-drop gate) against the oracle's loop: same stop iteration, same
    fields bit for bit."""
    d = geometry.straight_channel(M=20, N=40, band=(5, 15)).replace(enableInletRamp=True,
                                                                    enablePseudoTimeStepping=pseudo, serMinIter=4)
    xc = (0.25 * d.N * d.hx, 0.75 * d.N * d.hx)
    W, pct, ramp = 20, 0.5, 12
    ref = reference.run_iterations(d, 3000, W, pct, ramp, x_core=xc)
    f = rs.new_fields(d)
    dp, converged = rs.dp_gate_solve(d, f, 3000, W, pct, ramp, x_core=xc)
    assert converged and len(dp) < 3000
    assert len(ref["dpIter"]) == len(dp)
    np.testing.assert_allclose(ref["dp"], dp, rtol=1e-5, atol=1e-9)
    for k in ("u", "v", "p"):
        assert np.array_equal(ref[k], f[k]), k
