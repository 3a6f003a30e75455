"""The thermal step's outputs (cps_thermal_compute_metrics, cps_thermal_save;
host code) against the reference's own thermal output module
(ThermalSolver/thermal_output.cpp compiled under oracle/thermal_out_harness.cpp):
the metrics equal bit for bit and thermal_metrics.txt, k_thermal.txt and
thermal_gradient_3d.vtk are byte-identical.  thermal_results_3d.vtk is
written by a member of the reference's solver class (save_vtk), which is run
through oracle/thermal_asm_harness.cpp (the class compiled with its AMGCL solve
cut out): byte-identical too."""
import os

import numpy as np
import pytest

from coldplate_solver_b200 import thermal as pt
from oracle import reference


def field(Nx=23, Ny=11, seed=0):
    rng = np.random.default_rng(seed)
    gamma = (rng.random((Ny, Nx)) > 0.5).astype(float)
    gamma[rng.random((Ny, Nx)) > 0.8] = 0.42
    T = 30.0 + 20.0 * rng.random((9, Ny, Nx))
    u = rng.normal(0.1, 0.05, (Ny, Nx)) * gamma
    v = rng.normal(0.0, 0.02, (Ny, Nx)) * gamma
    return gamma, T, u, v


@pytest.mark.skipif(not os.access(os.path.join(reference.REF_DIR, "thermal_out"), os.X_OK),
                    reason="oracle/_ref/thermal_out not built")
@pytest.mark.parametrize("seed,qk,dx", [(0, 1.0, 1e-5), (1, 10.0, 2.3e-5)])
def test_outputs_equal_the_reference_module(tmp_path, seed, qk, dx):
    gamma, T, u, v = field(seed=seed)
    ref = reference.run_thermal_outputs(T, gamma, dx, dx, H_t=5e-4, qk=qk)
    m = ref["metrics"]
    # the reference's Params::dx() = (Nx dx) / Nx is what the library is given
    case = pt.ThermalCase(gamma=gamma, u=u, v=v, dx=m["dx"], dy=m["dy"], H_t=5e-4, qk=qk)
    got = pt.metrics(case, T)
    for k, val in got.items():
        assert val == m[k], (k, val, m[k])
    pt.save(str(tmp_path), case, T)
    for name in ("thermal_metrics.txt", "k_thermal.txt", "thermal_gradient_3d.vtk"):
        assert (tmp_path / name).read_bytes() == ref["files"][name], name
    lines = (tmp_path / "thermal_results_3d.vtk").read_text().splitlines()
    Ny, Nx = gamma.shape
    n = 9 * Ny * Nx
    assert lines[:4] == ["# vtk DataFile Version 3.0", "Thermal3D", "ASCII", "DATASET RECTILINEAR_GRID"]
    assert lines[4] == f"DIMENSIONS {Nx + 1} {Ny + 1} 10"
    assert f"CELL_DATA {n}" in lines
    for tag in ("SCALARS Temperature double 1", "SCALARS Region int 1", "SCALARS Density double 1",
                "SCALARS ThermalConductivity double 1", "VECTORS Velocity double"):
        assert tag in lines, tag
    start = lines.index("SCALARS Temperature double 1") + 2
    np.testing.assert_allclose([float(x) for x in lines[start:start + n]], T.ravel(), rtol=1e-5)


def test_from_export_reads_the_reference_inputs(tmp_path):
    gamma, T, u, v = field(Nx=7, Ny=5, seed=2)
    (tmp_path / "thermal_params.txt").write_text("5 7 2.5e-05 2.5e-05 750000 0.0004\n")
    (tmp_path / "geometry_thermal.txt").write_text(
        "\n".join(" ".join(repr(float(1.0 - g)) for g in row) for row in gamma) + "\n")
    (tmp_path / "u_thermal.txt").write_text("\n".join("\t".join(repr(float(x)) for x in row) for row in u) + "\n")
    (tmp_path / "v_thermal.txt").write_text("\n".join("\t".join(repr(float(x)) for x in row) for row in v) + "\n")
    c = pt.ThermalCase.from_export(str(tmp_path), qk=3.0)
    assert (c.Nx, c.Ny) == (7, 5) and c.q == 750000 and c.H_t == 0.0004 and c.qk == 3.0
    assert c.dx == (7 * 2.5e-05) / 7 and c.dy == (5 * 2.5e-05) / 5
    np.testing.assert_array_equal(c.gamma, 1.0 - (1.0 - gamma))
    np.testing.assert_array_equal(c.u, u)
    np.testing.assert_array_equal(c.v, v)


@pytest.mark.skipif(not os.access(os.path.join(reference.REF_DIR, "thermal_asm"), os.X_OK),
                    reason="oracle/_ref/thermal_asm not built")
@pytest.mark.parametrize("seed,Ht", [(0, 5e-4), (3, 4e-3)])
def test_results_vtk_equals_the_reference_writer(tmp_path, seed, Ht):
    gamma, T, u, v = field(seed=seed)
    Ny, Nx = gamma.shape
    dx = 1.7e-5
    ref = reference.run_thermal_assembly(Nx, Ny, dx, dx, gamma, u, v, np.zeros((Ny, Nx)), H_t=Ht, T=T)
    ddx, ddy = (float(x) for x in ref["dxdy"])
    case = pt.ThermalCase(gamma=gamma, u=u, v=v, dx=ddx, dy=ddy, H_t=Ht)
    pt.save(str(tmp_path), case, T)
    assert (tmp_path / "thermal_results_3d.vtk").read_bytes() == ref["vtk"]


def test_from_flow_crop_and_cell_sizes():
    """from_flow: the thermal crop between the buffers, saveAll's cell-centred
    velocities, and the thermal program's cell sizes (Nx dx)/Nx."""
    from coldplate_solver_b200 import geometry
    d = geometry.straight_channel(M=12, N=30, h=2.3e-5, band=(3, 9))
    rng = np.random.default_rng(4)
    f = {"u": rng.normal(size=(d.M + 1, d.N)), "v": rng.normal(size=(d.M, d.N + 1))}
    c = pt.ThermalCase.from_flow(d, f, q=1e5, N_in_buffer=3, N_out_buffer=5)
    assert (c.Nx, c.Ny) == (22, 12)
    assert c.dx == (22 * d.hx) / 22 and c.dy == (12 * d.hy) / 12
    np.testing.assert_array_equal(c.u, (0.5 * (f["u"][:-1, :] + f["u"][1:, :]))[:, 3:25])
    np.testing.assert_array_equal(c.v, (0.5 * (f["v"][:, :-1] + f["v"][:, 1:]))[:, 3:25])
    np.testing.assert_array_equal(c.gamma, d.gamma[:, 3:25])


def _printed_balance(text: str) -> dict:
    import re
    out = {}
    for key, name in (("T_base", "T_base"), ("T_fin", "T_fin"), ("T_fluid", "T_fluid")):
        a, b = re.search(rf"{key}:\s*\[([^,]+), ([^\]]+)\]", text).groups()
        out[f"{name}_min"], out[f"{name}_max"] = a.strip(), b.strip()
    for key, name in (("Q_in", "Q_in"), ("T_out", "T_out"), ("Q_out", "Q_out"), ("Imbalance", "imbalance")):
        out[name] = re.search(rf"{key}\s*=\s*(\S+?)(?:%|\s)", text).group(1)
    return out


@pytest.mark.skipif(not os.access(os.path.join(reference.REF_DIR, "thermal_asm"), os.X_OK),
                    reason="oracle/_ref/thermal_asm not built")
@pytest.mark.parametrize("seed,Ht,nz", [(0, 5e-4, (2, 7)), (5, 3e-3, (3, 5)), (9, 8e-4, (1, 1))])
def test_energy_balance_equals_the_reference_print(seed, Ht, nz):
    """thermal.energy_balance against the ranges and energy balance the
    reference's own solve prints (two decimals) for the same field."""
    gamma, T, u, v = field(seed=seed)
    Ny, Nx = gamma.shape
    T = T[:1].repeat(nz[0] + nz[1], axis=0) + np.random.default_rng(seed).random((nz[0] + nz[1], Ny, Nx))
    q0 = np.random.default_rng(seed + 1).uniform(1e9, 3e9, (Ny, Nx))
    ref = reference.run_thermal_assembly(Nx, Ny, 2e-5, 2e-5, gamma, u, v, q0, nz_solid=nz[0], nz_fluid=nz[1],
                                         H_t=Ht, T=T)
    printed = _printed_balance(ref["stdout"])
    dxy = [float(x) for x in ref["dxdy"]]
    case = pt.ThermalCase(gamma=gamma, u=u, v=v, dx=dxy[0], dy=dxy[1], q0=q0, H_t=Ht, nz_solid=nz[0],
                          nz_fluid=nz[1])
    mine = pt.energy_balance(case, T)
    for k, text in printed.items():
        assert f"{mine[k]:.2f}" == text, (k, mine[k], text)


def test_energy_balance_equals_the_oracle_loops():
    """thermal.energy_balance (vectorised, sums in the reference's order) and
    the oracle's per-cell loops give the same bits."""
    from oracle import thermal as th
    gamma, T, u, v = field(Nx=31, Ny=17, seed=3)
    q0 = np.random.default_rng(2).uniform(1e5, 1e6, gamma.shape)
    case = pt.ThermalCase(gamma=gamma, u=u, v=v, dx=2e-5, dy=2e-5, q0=q0, H_t=5e-4)
    p = th.ThermalParams(Nx=case.Nx, Ny=case.Ny, dx=case.dx, dy=case.dy, H_t=case.H_t)
    mine, ora = pt.energy_balance(case, T), th.energy_balance(p, gamma, u, q0, T)
    for k in ("T_base_min", "T_base_max", "T_fluid_min", "T_fluid_max", "T_fin_min", "T_fin_max", "Q_in", "T_out",
              "Q_out", "imbalance"):
        assert mine[k] == ora[k], (k, mine[k], ora[k])
