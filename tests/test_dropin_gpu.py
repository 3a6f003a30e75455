"""The drop-in inside the reference's own driver: the FP64 reference built
with the two-line calculateStep patch (pressureSolverType = 5 routes each
outer iteration through libcps.so) against the unpatched FP64 reference.
Same tolerances as the direct C-ABI parity tests."""
import numpy as np
import pytest

from conftest import load_golden
from coldplate_solver_b200 import geometry

pytestmark = pytest.mark.gpu

FIELDS = ("u", "v", "p", "pStar", "uStar", "vStar", "dE", "dN")


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / nb if nb > 0 else np.linalg.norm(a - b)


@pytest.mark.parametrize("case", ["network_30x48_sou25d", "density_20x40_random_state", "straight_full"])
def test_reference_driver_with_b200_branch(case):
    from oracle import reference
    if not (reference.available("dropin") and reference.available("f64")):
        pytest.skip("reference binaries not built in this checkout")
    if case == "straight_full":
        d, init, n = geometry.straight_channel(), None, 40
    else:
        d, init, z = load_golden(case)
        n = int(z["n_outer"])
    a = reference.run(d, n, precision="dropin", init=init)
    b = reference.run(d, n, precision="f64", init=init)
    # calculateStep's signature carries the PCG count only (iterations.cpp:82); the
    # Jacobi sweep counts are not observable through it on the B200 branch.
    assert np.array_equal(a["pIters"], b["pIters"])
    for k in ("residU", "residV", "residMass", "residMassDof", "err"):
        np.testing.assert_allclose(a[k], b[k], rtol=1e-8, atol=1e-300)
    for k in FIELDS:
        assert rel(a[k], b[k]) <= 1e-10, (k, rel(a[k], b[k]))
    np.testing.assert_allclose(a["planes"], b["planes"], rtol=1e-10, atol=1e-300)


@pytest.mark.parametrize("mom", [1, 0])
def test_reference_driver_with_pseudo_transient(mom):
    """The pseudo-transient term through the drop-in: the reference's own CFL
    controllers run on the host after every step and hand the CFL number to
    the next B200 step."""
    from oracle import reference
    if not (reference.available("dropin") and reference.available("f64")):
        pytest.skip("reference binaries not built in this checkout")
    d = geometry.channel_network(M=40, N=72, h=20e-6, wmin=4, wmax=8, seed=5).replace(
        enablePseudoTimeStepping=True, serMinIter=3, momentumSolverType=mom, uvAlpha=0.5 if mom == 0 else 0.7)
    n = 15
    a = reference.run(d, n, precision="dropin")
    b = reference.run(d, n, precision="f64")
    assert np.array_equal(a["pIters"], b["pIters"])
    for k in ("residU", "residV", "residMass", "err"):
        np.testing.assert_allclose(a[k], b[k], rtol=1e-8, atol=1e-300)
    np.testing.assert_allclose(a["pseudoCFL"], b["pseudoCFL"], rtol=1e-9)
    for k in FIELDS:
        assert rel(a[k], b[k]) <= 1e-10, (k, rel(a[k], b[k]))


def test_design_loop_in_one_process():
    """Two designs of one grid through the reference's own driver in one
    process (harness mode 4): object A runs design A and is destroyed, a new
    object B in the same storage runs design B, then B is edited in place back
    to design A from the zero state.  Each phase through the drop-in equals the
    same phase of the unpatched FP64 reference: the new object is told from
    the old one at the same address, and the in-place edit reaches the GPU."""
    from oracle import reference
    if not (reference.available("dropin") and reference.available("f64")):
        pytest.skip("reference binaries not built in this checkout")
    da = geometry.channel_network(M=40, N=72, h=20e-6, wmin=4, wmax=8, seed=5)
    db = geometry.channel_network(M=40, N=72, h=20e-6, wmin=4, wmax=8, seed=11)
    assert not np.array_equal(da.gamma, db.gamma)
    n = 20
    a = reference.run_design_loop(da, db, n, precision="dropin")
    b = reference.run_design_loop(da, db, n, precision="f64")
    for k in (1, 2, 3):
        assert np.array_equal(a[f"pIters{k}"], b[f"pIters{k}"]), k
        np.testing.assert_allclose(a[f"err{k}"], b[f"err{k}"], rtol=1e-8, atol=1e-300)
        for f in ("u", "v", "p"):
            assert rel(a[f"{f}{k}"], b[f"{f}{k}"]) <= 1e-10, (k, f, rel(a[f"{f}{k}"], b[f"{f}{k}"]))
    # phase 3 is design A from the zero state again; phase 2 is another design
    assert rel(a["u3"], a["u1"]) <= 1e-10
    assert rel(a["u2"], a["u1"]) > 1e-3


def test_mixed_precision_through_the_registry():
    """pressureSolverType = 6 selects the mixed-precision path (FP32 inner
    solves inside the FP64 defect correction): after 10 outer iterations it
    stays within the mixed path's per-step tolerance (1e-3 relative) of the
    FP64 reference."""
    from oracle import reference
    if not (reference.available("dropin") and reference.available("f64")):
        pytest.skip("reference binaries not built in this checkout")
    d = geometry.channel_network(M=40, N=72, h=20e-6, wmin=4, wmax=8, seed=5)
    a = reference.run(d, 10, precision="dropin", solver_type=6)
    b = reference.run(d, 10, precision="f64")
    for k in ("u", "v", "p"):
        assert rel(a[k], b[k]) <= 1e-3, (k, rel(a[k], b[k]))
    c = reference.run(d, 10, precision="dropin", solver_type=5)
    assert rel(a["u"], c["u"]) > 0.0  # the registry value reached the library
