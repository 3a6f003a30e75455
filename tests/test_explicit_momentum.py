"""The explicit momentum path (momentumSolverType = 0, iterations.cpp:176-441,
pseudo-transient off): the oracle's restatement against the reference's own
calculateStep (CPU), bit for bit in both precisions."""
import numpy as np
import pytest

from coldplate_solver_b200 import geometry
from oracle import reference
from oracle import restatement as rs

DESIGNS = {
    "straight_fou": lambda: geometry.straight_channel(M=20, N=40, band=(5, 15)),
    "network_sou_2.5d": lambda: geometry.channel_network(M=24, N=40, h=20e-6, wmin=3, wmax=6, seed=3),
    "density": lambda: geometry.density_field(Nx=48, seed=2, sigma=3.0),
}
FIELDS = ("u", "v", "p", "pStar", "uStar", "vStar", "dE", "dN")


@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("name", sorted(DESIGNS))
def test_oracle_explicit_path_matches_the_reference(name, precision):
    if not reference.available(precision):
        pytest.skip(f"oracle/_ref/ref_{precision} not built")
    d = DESIGNS[name]().replace(momentumSolverType=0, uvAlpha=0.5, pAlpha=0.2)
    n = 25
    ref = reference.run(d, n, precision=precision, stop_on_conv=False)
    f = rs.new_fields(d, precision)
    h = rs.solve(d, f, n, stop_on_conv=False, precision=precision)
    assert len(h) == n
    for k in FIELDS:
        assert np.array_equal(ref[k], f[k]), k
    np.testing.assert_array_equal(ref["pIters"], h[:, 5])
    for col, key in ((0, "residU"), (1, "residV"), (2, "residMass")):
        np.testing.assert_array_equal(ref[key], h[:, col])
