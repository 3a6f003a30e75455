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
