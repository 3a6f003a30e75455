"""The thermal oracle (CPU): the vectorised restatement of the reference's
3-D CHT assembly (thermal_solver.cpp:420-517) equals the per-cell
restatement in the reference's own loop structure bit for bit, and the
direct solution keeps the reference's energy balance."""
import numpy as np
import pytest

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
