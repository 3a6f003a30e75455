"""The 3-D conjugate-heat-transfer solve on the GPU (cps_thermal_*) against
the thermal oracle (oracle/thermal.py) and the reference's own assembly: the
device-assembled system equals the committed CSR matrix and right-hand side
of the reference's ThermalSolver3D::solve (tests/golden/thermal_asm_*) and the
oracle's restatement of it bit for bit, and the device solution satisfies the
reference's stop rule on that system and agrees with its exact (direct)
solution (the reference's AMGCL solve itself cannot be built)."""
import os

import numpy as np
import pytest

from coldplate_solver_b200 import cps, geometry
from coldplate_solver_b200 import thermal as pt
from oracle import restatement as rs
from oracle import thermal as th

pytestmark = pytest.mark.gpu


def random_case(Nx, Ny, seed, mode=1, qk=3.0, q0=True):
    rng = np.random.default_rng(seed)
    gamma = (rng.random((Ny, Nx)) > 0.4).astype(float)
    gamma[rng.random((Ny, Nx)) > 0.85] = 0.37
    gamma[:, 0] = 1.0
    u = np.abs(rng.normal(0.2, 0.15, (Ny, Nx))) * gamma
    v = rng.normal(0.0, 0.05, (Ny, Nx)) * gamma
    q = rng.uniform(5e5, 1.5e6, (Ny, Nx)) if q0 else None
    return pt.ThermalCase(gamma=gamma, u=u, v=v, dx=20e-6, dy=20e-6, q=8e5, q0=q, H_t=4e-4, k_interp_mode=mode,
                          qk=qk)


def oracle_params(c: pt.ThermalCase) -> th.ThermalParams:
    return th.ThermalParams(Nx=c.Nx, Ny=c.Ny, dx=c.dx, dy=c.dy, nz_solid=c.nz_solid, nz_fluid=c.nz_fluid,
                            H_b=c.H_b, H_t=c.H_t, k_s=c.k_s, k_f=c.k_f, rho=c.rho, Cp=c.Cp, T_inlet=c.T_inlet,
                            rtol=c.rtol, maxiter=c.maxiter, k_interp_mode=c.k_interp_mode, qk=c.qk)


def flow_case(M=64, N=131, outer=300, q=1e6):
    d = geometry.channel_network(M=M, N=N, h=20e-6, wmin=4, wmax=8, seed=7)
    with cps.Solver(d) as s:
        s.solve(outer, eps=0.0)
        f = s.download()
    return pt.ThermalCase.from_flow(d, f, q=q)


@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("shape", [(13, 9), (37, 23)])
def test_device_system_equals_the_oracle_assembly(shape, mode):
    c = random_case(*shape, seed=shape[0] + mode, mode=mode, q0=mode != 0)
    with pt.ThermalSolver(c) as s:
        planes, b = s.system()
    po, bo = th.assemble(oracle_params(c), c.gamma, c.u, c.v, c.heat_flux())
    for k in th.PLANES:
        assert np.array_equal(planes[k], po[k]), k
    assert np.array_equal(b, bo)


GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("name", sorted(f for f in os.listdir(GOLDEN) if f.startswith("thermal_asm_")))
def test_device_system_equals_the_reference_assembly(name):
    p, x, A_ref, b_ref = th.load_assembly_fixture(os.path.join(GOLDEN, name))
    c = pt.ThermalCase(gamma=x["gamma"], u=x["u"], v=x["v"], dx=p.dx, dy=p.dy, q0=x["q0"], nz_solid=p.nz_solid,
                       nz_fluid=p.nz_fluid, H_b=p.H_b, H_t=p.H_t, k_s=p.k_s, k_f=p.k_f, rho=p.rho, Cp=p.Cp,
                       T_inlet=p.T_inlet, k_interp_mode=p.k_interp_mode, qk=p.qk)
    with pt.ThermalSolver(c) as s:
        planes, b = s.system()
    A = th.to_csr(p, planes)
    A.sort_indices()
    assert th.same_csr(A, A_ref)
    assert np.array_equal(np.asarray(b).ravel().view(np.uint64), b_ref.view(np.uint64))


@pytest.mark.parametrize("shape", [(13, 9), (37, 23), (64, 40)])
def test_solution_matches_the_direct_solve(shape):
    c = random_case(*shape, seed=5)
    c.rtol = 1e-10
    c.maxiter = 2000
    p = oracle_params(c)
    with pt.ThermalSolver(c) as s:
        r = s.solve()
        T = s.temperature()
    assert r["converged"] and r["true_rel_residual"] <= 1e-9, r
    Td = th.solve_direct(p, c.gamma, c.u, c.v, c.heat_flux())
    err = np.linalg.norm(T - Td) / np.linalg.norm(Td - c.T_inlet)
    assert err <= 1e-5, err


def test_flow_driven_case_meets_the_reference_stop_rule():
    """Velocities from a flow solve of a channel network: the default stop rule
    (relative residual 1e-6 from T = T_inlet), checked on the oracle's
    system, in a modest number of preconditioned iterations; two solves agree
    bit for bit; the energy balance equals the oracle's statement of it."""
    c = flow_case()
    p = oracle_params(c)
    with pt.ThermalSolver(c) as s:
        r = s.solve()
        T = s.temperature()
        r2 = s.solve()
        T2 = s.temperature()
        ms, levels = s.timing()
    assert r["converged"] and r["iterations"] < 300 and r["true_rel_residual"] <= 1.0001e-6, r
    assert np.array_equal(T, T2) and r == r2
    planes, b = th.assemble(p, c.gamma, c.u, c.v, c.heat_flux())
    assert th.relative_residual(p, planes, b, T) <= 1.0001e-6
    Td = th.solve_direct(p, c.gamma, c.u, c.v, c.heat_flux())
    assert np.linalg.norm(T - Td) / np.linalg.norm(Td - c.T_inlet) <= 1e-3
    e_dev = pt.energy_balance(c, T)
    e_ora = th.energy_balance(p, c.gamma, c.u, c.heat_flux(), T)
    for k in ("T_base_max", "T_fluid_max", "T_fin_max", "Q_in", "Q_out", "T_out"):
        assert abs(e_dev[k] - e_ora[k]) <= 1e-9 * max(1.0, abs(e_ora[k])), k
    assert levels == 9 and ms > 0


def test_update_equals_a_fresh_solver():
    a = random_case(37, 23, seed=1)
    b = random_case(37, 23, seed=2)
    with pt.ThermalSolver(a) as s:
        s.solve()
        s.update(gamma=b.gamma, u=b.u, v=b.v, q0=b.q0)
        s.solve()
        T1 = s.temperature()
        pl1, b1 = s.system()
    with pt.ThermalSolver(b) as s:
        s.solve()
        T2 = s.temperature()
        pl2, b2 = s.system()
    assert np.array_equal(T1, T2) and np.array_equal(b1, b2)


def test_arguments_are_validated():
    import ctypes
    lib = cps.load_library()
    d = cps.CpsThermalDesc()
    lib.cps_thermal_defaults(ctypes.byref(d))
    h = cps._P()
    assert lib.cps_thermal_create(ctypes.byref(d), ctypes.byref(h)) == cps.CPS_ERR_ARG  # Nx = 0
    d.Nx, d.Ny, d.dx, d.dy = 4, 4, 1e-5, 1e-5
    assert lib.cps_thermal_create(ctypes.byref(d), ctypes.byref(h)) == cps.CPS_ERR_ARG  # no inputs
    g = np.ones((4, 4))
    d.gamma = d.u = d.v = g.ctypes.data
    d.k_interp_mode = 3
    assert lib.cps_thermal_create(ctypes.byref(d), ctypes.byref(h)) == cps.CPS_ERR_ARG


@pytest.mark.parametrize("shape,nz", [((1, 7), (2, 7)), ((9, 1), (2, 7)), ((5, 3), (1, 3)), ((2, 2), (3, 1)),
                                      ((17, 12), (1, 1))])
def test_edge_grids_match_the_oracle(shape, nz):
    """Degenerate and small grids (one column, one row, single layers): the
    hierarchy still ends in one column, the system equals the oracle's and
    the solution its direct solve."""
    c = random_case(*shape, seed=11)
    c.nz_solid, c.nz_fluid = nz
    c.rtol = 1e-10
    p = oracle_params(c)
    with pt.ThermalSolver(c) as s:
        planes, b = s.system()
        r = s.solve()
        T = s.temperature()
    po, bo = th.assemble(p, c.gamma, c.u, c.v, c.heat_flux())
    for k in th.PLANES:
        assert np.array_equal(planes[k], po[k]), k
    assert np.array_equal(b, bo)
    Td = th.solve_direct(p, c.gamma, c.u, c.v, c.heat_flux())
    assert r["converged"], r
    assert np.linalg.norm(T - Td) / max(np.linalg.norm(Td - c.T_inlet), 1e-300) <= 1e-5


def test_warm_start_from_a_previous_solution():
    """cps_thermal_solve_from: from the converged field nothing is left to do;
    after a 5 % change of the heat flux, a start from the previous field
    needs fewer iterations than the start from T_inlet and reaches the same
    solution (to the stop rule's accuracy)."""
    c = flow_case()
    with pt.ThermalSolver(c) as s:
        s.solve()
        T1 = s.temperature()
        r0 = s.solve_from()
        assert r0["iterations"] == 0 and r0["converged"] and r0["true_rel_residual"] <= 1e-6
        s.update(q0=c.heat_flux() * 1.05)
        cold = s.solve()
        T_cold = s.temperature()
        warm = s.solve_from(T1)
        T_warm = s.temperature()
    assert cold["converged"] and warm["converged"] and warm["true_rel_residual"] <= 1.0001e-6
    assert warm["iterations"] < cold["iterations"], (warm, cold)
    assert np.linalg.norm(T_warm - T_cold) / np.linalg.norm(T_cold - c.T_inlet) <= 1e-3
