"""Device-side pressure-drop monitor and gate (cps_set_dp_monitor,
cps_solve_monitored) against the oracle's restatement of the reference's
outer loop, which tests/test_dp_gate.py pins to the reference itself.

The device evaluates the same per-point arithmetic; only grid-wide sums are
grouped differently, so the pressure drops agree to 1e-9 relative over these
short runs and the gate stops on the same iteration (allowed to differ by
one, should a window statistic land within rounding of the threshold)."""
import ctypes

import numpy as np
import pytest

from coldplate_solver_b200 import cps, exportfiles, geometry
from oracle import reference
from oracle import restatement as rs

pytestmark = pytest.mark.gpu

CASES = {
    "window": (lambda: geometry.straight_channel(M=20, N=40, band=(5, 15)), 20, 0.5, 10, False, 0, 0.0),
    "window+slope": (lambda: geometry.channel_network(M=24, N=40, h=20e-6, wmin=3, wmax=6, seed=3), 30, 0.2, 15,
                     True, 40, 5.0),
    "network-band": (lambda: geometry.channel_network(M=64, N=130, h=20e-6, wmin=4, wmax=8, seed=3), 40, 0.5, 20,
                     False, 0, 0.0),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_device_gate_stops_where_the_reference_loop_stops(name):
    make, W, pct, ramp, sg, sw, smd = CASES[name]
    d = make()
    xc = (0.25 * d.N * d.hx, 0.75 * d.N * d.hx)
    f = rs.new_fields(d)
    dp_o, conv_o = rs.dp_gate_solve(d, f, 5000, W, pct, ramp, sg, sw, smd, x_core=xc)
    assert conv_o
    with cps.Solver(d) as s:
        s.set_dp_monitor(gate=True, window=W, percent=pct, slope_gate=sg, slope_window=sw, slope_max_delta=smd,
                         ramp_steps=ramp, x_core_in=xc[0], x_core_out=xc[1])
        hist, dp_g, conv_g = s.solve_monitored(5000, eps=0.0)
    assert conv_g
    assert abs(len(dp_g) - len(dp_o)) <= 1, (len(dp_g), len(dp_o))
    k = min(len(dp_g), len(dp_o))
    np.testing.assert_allclose(dp_g[:k], dp_o[:k], rtol=1e-9, atol=1e-9)
    assert len(hist) == len(dp_g)


def test_monitor_without_gate_logs_every_iteration_and_spans_launches():
    """The monitor alone changes nothing in the iteration; its log continues
    across launch chunks and a later cps_solve_monitored call."""
    d = geometry.straight_channel(M=20, N=40, band=(5, 15))
    xc = (0.25 * d.N * d.hx, 0.75 * d.N * d.hx)
    with cps.Solver(d) as plain:
        h0 = plain.solve(60, eps=0.0)
        f0 = plain.download()
    with cps.Solver(d) as s:
        s.set_dp_monitor(gate=False, window=5, percent=0.0, ramp_steps=0, x_core_in=xc[0], x_core_out=xc[1])
        h1, dp1, c1 = s.solve_monitored(25, eps=0.0)
        h2, dp2, c2 = s.solve_monitored(35, eps=0.0)
        f1 = s.download()
    assert not c1 and not c2 and len(dp1) == 25 and len(dp2) == 35
    assert np.array_equal(np.vstack([h1, h2]), h0)
    for k in ("u", "v", "p"):
        assert np.array_equal(f0[k], f1[k]), k
    fo = rs.new_fields(d)
    for it in range(60):
        rs.step(d, fo)
        if it in (0, 24, 25, 59):
            dp_ref = [rs.sample_plane(d, fo, x)[4] for x in (xc[0], xc[1], 0.0, d.N * d.hx)]
            row = (dp1 if it < 25 else dp2)[it if it < 25 else it - 25]
            np.testing.assert_allclose(row[0], dp_ref[0] - dp_ref[1], rtol=1e-9)
            np.testing.assert_allclose(row[1], dp_ref[2] - dp_ref[3], rtol=1e-9)


def test_monitor_arguments_are_checked():
    d = geometry.straight_channel(M=10, N=12, band=(3, 7))
    with cps.Solver(d) as s:
        with pytest.raises(cps.CpsError) as e:
            s.solve_monitored(5)
        assert e.value.status == cps.CPS_ERR_ARG
        with pytest.raises(cps.CpsError) as e:
            s.set_dp_monitor(window=0)
        assert e.value.status == cps.CPS_ERR_ARG
        with pytest.raises(cps.CpsError) as e:
            s.set_dp_monitor(window=100000)
        assert e.value.status == cps.CPS_ERR_ARG
        s.set_dp_monitor(window=5, ramp_steps=0)
        s.set_dp_monitor(enabled=False)
        with pytest.raises(cps.CpsError):
            s.solve_monitored(5)


@pytest.mark.skipif(not reference.available("f64"), reason="oracle/_ref/ref_f64 not built")
def test_device_logs_match_the_reference_logs(tmp_path):
    """residuals.txt and pressure_drop_history.txt from the device's monitored
    solve (cps_save_logs) against the ones the reference's own runIterations
    writes: the same rows, numbers equal to the six digits both print."""
    d = geometry.straight_channel(M=20, N=40, band=(5, 15))
    xc = (0.25 * d.N * d.hx, 0.75 * d.N * d.hx)
    ref = reference.run_iterations(d, 3000, 20, 0.5, 10, x_core=xc)
    with cps.Solver(d) as s:
        s.set_dp_monitor(gate=True, window=20, percent=0.5, ramp_steps=10, x_core_in=xc[0], x_core_out=xc[1])
        hist, dp, conv = s.solve_monitored(3000, eps=0.0)
    assert conv
    exportfiles.save_logs(str(tmp_path), hist, dp=dp)
    for name, cols in (("residuals.txt", 7), ("pressure_drop_history.txt", 5)):
        mine = (tmp_path / name).read_text().splitlines()
        theirs = ref["logs"][name].decode().splitlines()
        assert mine[0] == theirs[0]
        assert abs(len(mine) - len(theirs)) <= 1
        k = min(len(mine), len(theirs))
        a = np.array([[float(x) for x in ln.split()] for ln in mine[1:k]]).reshape(-1, cols)
        b = np.array([[float(x) for x in ln.split()] for ln in theirs[1:k]]).reshape(-1, cols)
        np.testing.assert_allclose(a, b, rtol=2e-5, atol=1e-12)
