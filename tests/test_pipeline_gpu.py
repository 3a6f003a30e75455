"""One pass of the design loop (flow, thermal crop, thermal solve, metrics)
on the GPU equals the same steps called one by one.  (The energy balance is
not asserted: at this channel's low Peclet number much of the heat leaves by
conduction through the fixed-temperature inlet face, which the reference's
balance, counting the outlet only, reports as imbalance.)"""
import numpy as np
import pytest

from coldplate_solver_b200 import cps, geometry, pipeline
from coldplate_solver_b200 import thermal as pt

pytestmark = pytest.mark.gpu


def test_design_loop_pass_equals_its_steps():
    d = geometry.straight_channel(M=24, N=48, band=(6, 18))
    out = pipeline.solve_design(d, q=2e5, eps=1e-6, max_outer=20000, N_in_buffer=4, N_out_buffer=4)
    assert out["flow_converged"] and out["thermal"]["converged"]
    with cps.Solver(d) as s:
        h = s.solve(20000, eps=1e-6)
        f = s.download()
    assert np.array_equal(h, out["flow_history"])
    c = pt.ThermalCase.from_flow(d, f, q=2e5, N_in_buffer=4, N_out_buffer=4)
    assert (c.Nx, c.Ny) == (40, 24)
    with pt.ThermalSolver(c) as ts:
        ts.solve()
        T = ts.temperature()
    assert np.array_equal(T, out["T"])
    e = out["energy"]
    assert e["Q_in"] == pytest.approx(2e5 * c.Nx * c.Ny * c.dx * c.dy)
    assert out["metrics"]["T_avg_base"] > c.T_inlet and out["metrics"] == pt.metrics(c, T)


def test_design_loop_pass_leaves_the_reference_files(tmp_path):
    """export_dir: saveAll's files, runIterations' two logs and the thermal
    program's four outputs; the monitor that fills the logs leaves the flow
    history unchanged."""
    import os
    d = geometry.straight_channel(M=24, N=48, band=(6, 18))
    plain = pipeline.solve_design(d, q=2e5, eps=1e-6, max_outer=20000, N_in_buffer=4, N_out_buffer=4)
    out = pipeline.solve_design(d, q=2e5, eps=1e-6, max_outer=20000, N_in_buffer=4, N_out_buffer=4,
                                export_dir=str(tmp_path))
    assert np.array_equal(out["flow_history"], plain["flow_history"])
    assert np.array_equal(out["T"], plain["T"])
    names = set(os.listdir(tmp_path))
    for n in ("u.txt", "v.txt", "p.txt", "u_thermal.txt", "v_thermal.txt", "fluid_results.vtk", "residuals.txt",
              "pressure_drop_history.txt", "thermal_results_3d.vtk", "thermal_metrics.txt", "k_thermal.txt",
              "thermal_gradient_3d.vtk"):
        assert n in names, n
    rows = (tmp_path / "pressure_drop_history.txt").read_text().splitlines()[1:]
    assert len(rows) == len(out["flow_history"]) == len(out["dp_log"])
    last = [float(x) for x in rows[-1].split()]
    np.testing.assert_allclose(last[1:], out["dp_log"][-1], rtol=1e-5)
    assert abs(out["dp_log"][-1][1] - out["dp"]) <= 1e-5 * abs(out["dp"])  # full total drop = full_dp
