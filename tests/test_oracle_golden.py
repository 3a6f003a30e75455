"""The oracle's C restatement is pinned to the reference solver's own outputs.

Golden fixtures (tests/golden/*.npz) were produced by the reference's code
built from its sources (tests/golden/make_golden.py) with sequential
reductions; the restatement must reproduce them bit for bit in FP64 (the
reference promoted to double) and FP32 (as shipped): every field, the
residual history, the inner iteration counts and the sampled planes.
"""
import numpy as np
import pytest

from conftest import golden_history, golden_names, load_golden
from coldplate_solver_b200 import geometry

FIELDS = ("u", "v", "p", "pStar", "uStar", "vStar", "dE", "dN")


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("name", golden_names())
def test_restatement_matches_reference_bit_exact(oracle_lib, name, prec):
    rs = oracle_lib
    d, init, z = load_golden(name)
    f = rs.new_fields(d, prec)
    if init is not None:
        for k in ("u", "v", "p"):
            f[k][...] = init[k]
    hist = rs.solve(d, f, int(z["n_outer"]), stop_on_conv=False, precision=prec)
    ref = golden_history(z, prec)
    assert hist.shape == ref.shape
    assert np.array_equal(hist, ref), np.abs(hist - ref).max(axis=0)
    for k in FIELDS:
        assert np.array_equal(f[k].astype(np.float64), z[f"{prec}_{k}"]), k
    xs = [0.0, d.N * d.hx, 0.01, 0.05]
    planes = np.stack([rs.sample_plane(d, f, x, prec) for x in xs])
    assert np.array_equal(planes, z[f"{prec}_planes"])


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_alpha_build_matches_reference(oracle_lib, prec):
    z = np.load(__import__("conftest").GOLDEN + "/alpha_ramp_17x23.npz")
    amax = 0.00089 / 1e-14 if prec == "f64" else float(np.float32(0.00089) / np.float32(1e-14))
    a, g = oracle_lib.build_alpha(z["gamma_in"], amax, 1.0, prec)
    assert np.array_equal(a.astype(np.float64), z[f"{prec}_alpha"])
    assert np.array_equal(g.astype(np.float64), z[f"{prec}_gamma"])


def test_package_alpha_builder_matches_reference():
    z = np.load(__import__("conftest").GOLDEN + "/alpha_ramp_17x23.npz")
    a, g = geometry.alpha_ramp_reference(z["gamma_in"])
    assert np.array_equal(a, z["f64_alpha"])
    assert np.array_equal(g, z["f64_gamma"])


def test_restatement_step_equals_solve(oracle_lib):
    rs = oracle_lib
    d, _, _ = load_golden("network_30x48_sou25d")
    f1, f2 = rs.new_fields(d), rs.new_fields(d)
    h = rs.solve(d, f1, 4, stop_on_conv=False)
    for k in range(4):
        diag = rs.step(d, f2)
        assert list(diag.values()) == list(h[k])
    for k in FIELDS:
        assert np.array_equal(f1[k], f2[k])


def test_restatement_phases(oracle_lib):
    """stop_after=1/2 leave the later fields untouched (used to localise GPU differences)."""
    rs = oracle_lib
    d, _, _ = load_golden("straight_11x13")
    f = rs.new_fields(d)
    rs.step(d, f)
    u_before = f["u"].copy()
    rs.step(d, f, stop_after=1)
    assert np.array_equal(f["u"], u_before)
    assert np.abs(f["uStar"]).max() > 0


def test_convergence_rule_stops_early(oracle_lib):
    rs = oracle_lib
    d = geometry.straight_channel(M=12, N=20, band=(3, 9))
    f = rs.new_fields(d)
    h = rs.solve(d, f, 5000, eps=1e-6)
    conv = np.maximum(np.maximum(h[:, 0], h[:, 1]), h[:, 3])
    assert len(h) < 5000 and conv[-1] <= 1e-6 and (conv[:-1] > 1e-6).all()
