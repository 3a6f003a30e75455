"""The reference's own thermal program (ThermalSolver/thermal_solver.cpp: its
main, ThermalSolver3D and the output module) built with the two-line drop-in
of coldplate_solver_b200/host/b200_thermal_dropin.h in place of its AMGCL
solve (oracle/_ref/thermal_dropin, linked to libcps.so): run on exported
files, it writes the same four files, byte for byte, as this library's own
thermal path (thermal.ThermalCase.from_export, ThermalSolver, thermal.save)
on the same files."""
import os
import subprocess

import numpy as np
import pytest

from coldplate_solver_b200 import thermal as pt

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(REPO, "oracle", "_ref", "thermal_dropin")
OUTPUTS = ("thermal_results_3d.vtk", "thermal_metrics.txt", "k_thermal.txt", "thermal_gradient_3d.vtk")


def write_export(d, Nx, Ny, seed, dx=2.5e-5, q=7.5e5, Ht=4e-4):
    rng = np.random.default_rng(seed)
    solid = (rng.random((Ny, Nx)) > 0.6).astype(float)
    solid[rng.random((Ny, Nx)) > 0.9] = 0.5
    solid[:, 0] = 0.0
    u = np.abs(rng.normal(0.2, 0.1, (Ny, Nx))) * (1.0 - solid)
    v = rng.normal(0.0, 0.03, (Ny, Nx)) * (1.0 - solid)
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, "thermal_params.txt"), "w") as f:
        f.write(f"{Ny} {Nx} {dx!r} {dx!r} {q!r} {Ht!r}\n")
    for name, a, sep in (("geometry_thermal.txt", solid, " "), ("u_thermal.txt", u, "\t"), ("v_thermal.txt", v, "\t")):
        with open(os.path.join(d, name), "w") as f:
            f.write("\n".join(sep.join(repr(float(x)) for x in row) for row in a) + "\n")


@pytest.mark.skipif(not os.access(BIN, os.X_OK), reason="oracle/_ref/thermal_dropin not built")
@pytest.mark.parametrize("shape,seed,qk,mode", [((40, 24), 0, 1.0, 1), ((33, 17), 1, 3.0, 2), ((48, 20), 2, 1.0, 0)])
def test_reference_program_through_the_dropin(tmp_path, shape, seed, qk, mode):
    Nx, Ny = shape
    ref_dir, own_dir = str(tmp_path / "ref"), str(tmp_path / "own")
    write_export(ref_dir, Nx, Ny, seed)
    write_export(own_dir, Nx, Ny, seed)
    proc = subprocess.run([BIN, ref_dir, repr(qk), str(mode)], capture_output=True, text=True, timeout=300)
    assert proc.returncode == 0, proc.stdout[-2000:] + proc.stderr[-2000:]
    case = pt.ThermalCase.from_export(own_dir, qk=qk, k_interp_mode=mode)
    with pt.ThermalSolver(case) as s:
        res = s.solve()
        T = s.temperature()
    assert res["converged"]
    pt.save(own_dir, case, T)
    for name in OUTPUTS:
        with open(os.path.join(ref_dir, name), "rb") as a, open(os.path.join(own_dir, name), "rb") as b:
            assert a.read() == b.read(), name
