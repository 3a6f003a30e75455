"""The outer loop's pressure-drop gate (SIMPLE::runIterations,
SIMPLE.cpp:269-408): the oracle's restatement against the reference's own
loop run by the harness (CPU).  The reference logs the pressure drops with
six significant digits, so those are compared to 1e-5; the stop iteration
and the final fields must be identical."""
import numpy as np
import pytest

from coldplate_solver_b200 import geometry
from oracle import reference
from oracle import restatement as rs

CASES = {
    # name: (design, window, percent, ramp_steps, slope_gate, slope_window, slope_max_delta)
    "window": (lambda: geometry.straight_channel(M=20, N=40, band=(5, 15)), 20, 0.5, 10, False, 0, 0.0),
    "window+slope": (lambda: geometry.channel_network(M=24, N=40, h=20e-6, wmin=3, wmax=6, seed=3), 30, 0.2, 15,
                     True, 40, 5.0),
}


@pytest.mark.skipif(not reference.available("f64"), reason="oracle/_ref/ref_f64 not built")
@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_gate_matches_the_reference_loop(name):
    make, W, pct, ramp, sg, sw, smd = CASES[name]
    d = make()
    xc = (0.25 * d.N * d.hx, 0.75 * d.N * d.hx)
    ref = reference.run_iterations(d, 3000, W, pct, ramp, sg, sw, smd, x_core=xc)
    f = rs.new_fields(d)
    dp, converged = rs.dp_gate_solve(d, f, 3000, W, pct, ramp, sg, sw, smd, x_core=xc)
    assert converged and len(dp) < 3000
    assert len(ref["dpIter"]) == len(dp)
    assert np.array_equal(ref["dpIter"], np.arange(len(dp)))
    np.testing.assert_allclose(ref["dp"], dp, rtol=1e-5, atol=1e-9)
    for k in ("u", "v", "p"):
        assert np.array_equal(ref[k], f[k]), k
