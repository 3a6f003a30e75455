"""The explicit momentum path (momentumSolverType = 0) on the GPU against the
oracle, which tests/test_explicit_momentum.py pins bit for bit to the
reference.  The tolerances are those of test_parity_gpu.py: per-point values
follow the reference's operation order, only the grid-wide sums (PCG dots)
are grouped differently; the explicit update has no Jacobi sweeps (both
sweep counts read 0 here, where the reference has no count at all)."""
import numpy as np
import pytest

from coldplate_solver_b200 import cps, geometry
from oracle import restatement as rs

pytestmark = pytest.mark.gpu

REL_STEP = 1e-10
REL_MIXED_STEP = 1e-3
FIELDS = ("u", "v", "p", "pStar", "uStar", "vStar", "dE", "dN")
DESIGNS = {
    "straight_fou": lambda: geometry.straight_channel(M=41, N=77, band=(10, 30)),
    "network_sou_2.5d": lambda: geometry.channel_network(M=64, N=131, h=20e-6, wmin=4, wmax=8, seed=7),
    "density": lambda: geometry.density_field(Nx=150, seed=2, sigma=4.0),
}


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / nb if nb > 0 else np.linalg.norm(a - b)


def explicit(name):
    return DESIGNS[name]().replace(momentumSolverType=0, uvAlpha=0.5, pAlpha=0.2)


@pytest.mark.parametrize("ctas", [0, 3])
@pytest.mark.parametrize("name", sorted(DESIGNS))
def test_explicit_steps_match_the_oracle(name, ctas):
    d = explicit(name)
    n = 6
    with cps.Solver(d, grid_ctas=ctas) as s:
        h = s.solve(n, eps=0.0)
        f = s.download()
    fo = rs.new_fields(d)
    ho = rs.solve(d, fo, n, stop_on_conv=False)
    assert np.array_equal(h[:, 5], ho[:, 5]), (h[:, 5], ho[:, 5])
    assert not h[:, 6:].any()
    for c in range(4):
        np.testing.assert_allclose(h[:, c], ho[:, c], rtol=1e-8, atol=1e-300)
    for k in FIELDS:
        assert rel(f[k], fo[k]) <= REL_STEP, (k, rel(f[k], fo[k]))


def test_explicit_path_mixed_precision_tracks_fp64():
    d = explicit("network_sou_2.5d")
    with cps.Solver(d, precision=cps.CPS_MIXED) as s:
        s.solve(4, eps=0.0)
        fm = s.download()
    fo = rs.new_fields(d)
    rs.solve(d, fo, 4, stop_on_conv=False)
    for k in ("u", "v", "uStar", "vStar", "dE", "dN"):
        assert rel(fm[k], fo[k]) <= REL_MIXED_STEP, (k, rel(fm[k], fo[k]))


def test_explicit_flag_is_validated():
    d = explicit("straight_fou")
    desc, keep = cps.make_desc(d)
    desc.momentum_explicit = 2
    import ctypes
    ctx = ctypes.c_void_p()
    lib = cps.load_library()
    assert lib.cps_create(ctypes.byref(desc), ctypes.byref(ctx)) == cps.CPS_ERR_ARG
