"""The thermal oracle (CPU): the vectorised restatement of the reference's
3-D CHT assembly (thermal_solver.cpp:420-517) equals the per-cell
restatement in the reference's own loop structure bit for bit, and the
direct solution keeps the reference's energy balance."""
import os

import numpy as np
import pytest

from oracle import reference
from oracle import thermal as th


def case(Nx=13, Ny=9, seed=0, mode=1, qk=3.0, Ht=4e-4):
    rng = np.random.default_rng(seed)
    gamma = (rng.random((Ny, Nx)) > 0.4).astype(float)
    gamma[rng.random((Ny, Nx)) > 0.8] = rng.random() * 0.9 + 0.05  # buffer cells
    gamma[:, 0] = 1.0
    u = rng.normal(0.2, 0.15, (Ny, Nx)) * gamma
    v = rng.normal(0.0, 0.05, (Ny, Nx)) * gamma
    q0 = rng.uniform(5e5, 1.5e6, (Ny, Nx))
    p = th.ThermalParams(Nx=Nx, Ny=Ny, dx=20e-6, dy=20e-6, H_t=Ht, k_interp_mode=mode, qk=qk)
    return p, gamma, u, v, q0


@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("seed", [0, 1])
def test_vectorised_assembly_equals_the_loops(mode, seed):
    p, gamma, u, v, q0 = case(seed=seed, mode=mode)
    a, b = th.assemble(p, gamma, u, v, q0)
    c, d = th.assemble_loops(p, gamma, u, v, q0)
    for k in th.PLANES:
        assert np.array_equal(a[k], c[k]), k
    assert np.array_equal(b, d)


def test_direct_solution_satisfies_the_system_and_balances_energy():
    """A channel with inflow at x = 0 and outflow at x = L: the heat put in
    through the base leaves with the fluid (the reference prints this
    imbalance; with its upwind scheme and walls it is small)."""
    Nx, Ny = 40, 12
    gamma = np.zeros((Ny, Nx))
    gamma[3:9, :] = 1.0
    u = np.where(gamma > 0, 0.3, 0.0)
    v = np.zeros((Ny, Nx))
    q0 = np.full((Ny, Nx), 1e5)
    p = th.ThermalParams(Nx=Nx, Ny=Ny, dx=50e-6, dy=50e-6, H_t=5e-4)
    planes, b = th.assemble(p, gamma, u, v, q0)
    T = th.solve_direct(p, gamma, u, v, q0)
    assert th.relative_residual(p, planes, b, T) < 1e-12
    e = th.energy_balance(p, gamma, u, q0, T)
    assert abs(e["imbalance"]) < 1.0, e
    assert e["T_base_max"] > e["T_out"] > p.T_inlet


def test_cpu_port_reaches_the_stop_rule():
    """The CPU port timed as the thermal benchmark's CPU baseline solves the
    same system to the same stop rule."""
    p, gamma, u, v, q0 = case(Nx=40, Ny=24, seed=3)
    u = np.abs(u)
    T, it, sec, done = th.mg_bicgstab_cpu(p, gamma, u, v, q0)
    planes, b = th.assemble(p, gamma, u, v, q0)
    assert done and it < 200
    assert th.relative_residual(p, planes, b, T) <= p.rtol * 1.0001
    Td = th.solve_direct(p, gamma, u, v, q0)
    assert np.linalg.norm(T - Td) / np.linalg.norm(Td - p.T_inlet) < 1e-3


@pytest.mark.skipif(not os.access(os.path.join(reference.REF_DIR, "thermal_asm"), os.X_OK),
                    reason="oracle/_ref/thermal_asm not built")
@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("shape", [(13, 9), (31, 17)])
def test_assembly_equals_the_reference_assembly(shape, mode):
    """The oracle's assembly against the reference's own ThermalSolver3D::solve
    assembly (run with its AMGCL solve cut out): every CSR entry and the
    right-hand side, bit for bit."""
    Nx, Ny = shape
    p, gamma, u, v, q0 = case(Nx=Nx, Ny=Ny, seed=Nx + mode, mode=mode)
    ref = reference.run_thermal_assembly(Nx, Ny, p.dx, p.dy, gamma, u, v, q0, H_t=p.H_t, qk=p.qk,
                                         k_interp_mode=mode)
    p.dx, p.dy = float(ref["dxdy"][0]), float(ref["dxdy"][1])  # Params::dx() = (Nx dx) / Nx
    planes, b = th.assemble(p, gamma, u, v, q0)
    A = th.to_csr(p, planes)
    A.sort_indices()
    assert np.array_equal(A.indptr, ref["row_ptr"]) and np.array_equal(A.indices, ref["col_idx"])
    assert np.array_equal(A.data, ref["values"])
    assert np.array_equal(b.ravel(), ref["b"])


GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
ASM_FIXTURES = sorted(f for f in os.listdir(GOLDEN) if f.startswith("thermal_asm_"))


def test_assembly_fixtures_exist():
    assert len(ASM_FIXTURES) >= 4


@pytest.mark.parametrize("name", ASM_FIXTURES)
def test_assembly_equals_the_reference_fixture(name):
    """The committed output of the reference's own assembly (no reference
    needed at test time) against the oracle's, bit for bit."""
    p, x, A_ref, b_ref = th.load_assembly_fixture(os.path.join(GOLDEN, name))
    planes, b = th.assemble(p, x["gamma"], x["u"], x["v"], x["q0"])
    A = th.to_csr(p, planes)
    A.sort_indices()
    assert th.same_csr(A, A_ref)
    assert np.array_equal(b.ravel().view(np.uint64), b_ref.view(np.uint64))


@pytest.mark.skipif(not os.access(os.path.join(reference.REF_DIR, "thermal_asm"), os.X_OK),
                    reason="oracle/_ref/thermal_asm not built")
@pytest.mark.parametrize("shape,nz,mode", [((1, 7), (2, 7), 1), ((9, 1), (2, 7), 2), ((5, 3), (1, 3), 0),
                                           ((2, 2), (3, 1), 1), ((17, 12), (1, 1), 2), ((1, 1), (1, 1), 1)])
def test_edge_grid_assembly_equals_the_reference(shape, nz, mode):
    """One column, one row, single layers, a single cell: the oracle's
    assembly against the reference's own, bit for bit."""
    Nx, Ny = shape
    p, gamma, u, v, q0 = case(Nx=Nx, Ny=Ny, seed=7 + Nx, mode=mode)
    p.nz_solid, p.nz_fluid = nz
    ref = reference.run_thermal_assembly(Nx, Ny, p.dx, p.dy, gamma, u, v, q0, nz_solid=nz[0], nz_fluid=nz[1],
                                         H_t=p.H_t, qk=p.qk, k_interp_mode=mode)
    p.dx, p.dy = float(ref["dxdy"][0]), float(ref["dxdy"][1])
    planes, b = th.assemble(p, gamma, u, v, q0)
    A = th.to_csr(p, planes)
    A.sort_indices()
    assert np.array_equal(A.indptr, ref["row_ptr"]) and np.array_equal(A.indices, ref["col_idx"])
    assert np.array_equal(A.data, ref["values"])
    assert np.array_equal(b.ravel(), ref["b"])
