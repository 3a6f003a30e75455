"""The boundary's file formats against the reference's own readers and
saveAll (run by the oracle harness on the same files and values; CPU).
Readers must return exactly what the reference reads; every file saveAll
writes must be byte-identical."""
import os
import tempfile

import numpy as np
import pytest

from coldplate_solver_b200 import exportfiles as ef
from oracle import reference

pytestmark = pytest.mark.skipif(not reference.available("f64"), reason="oracle/_ref/ref_f64 not built")


def case_texts(M=7, N=11, seed=0, short=False, extra=""):
    rng = np.random.default_rng(seed)
    ct = np.where(rng.random((M, N)) < 0.3, 1.0, 0.0)
    ct[rng.random((M, N)) < 0.2] = 0.25  # a few continuous (buffer) values
    rows = [" ".join(f"{x:g}" for x in row) for row in ct]
    geo = "\n".join(rows) + "\n"
    if short:
        geo = "\n".join(rows[: M // 2]) + "\n"
    params = f"{M} {N} 2e-05 2.5e-05 0.15 2 3{extra}\n"
    return {"fluid_params.txt": params, "geometry_fluid.txt": geo}


def write(d, texts):
    for k, v in texts.items():
        with open(os.path.join(d, k), "w") as f:
            f.write(v)


@pytest.mark.parametrize("extra,short", [("", False), (" 0.0005", False), (" 0.0005 997 1e-6", True)])
def test_case_readers_match_the_reference(extra, short):
    texts = case_texts(short=short, extra=extra)
    ref = reference.run_io(texts)
    with tempfile.TemporaryDirectory() as d:
        write(d, texts)
        p = ef.read_case_params(os.path.join(d, "fluid_params.txt"))
        ct, gm, n = ef.read_geometry(os.path.join(d, "geometry_fluid.txt"), p.M, p.N)
    assert (p.M, p.N, p.N_in_buffer, p.N_out_buffer) == (ref["M"], ref["N"], ref["N_in_buffer"], ref["N_out_buffer"])
    assert (p.hx, p.hy, p.U_in) == (ref["hx"], ref["hy"], ref["U_in"])
    if extra:
        assert p.Ht == ref["Ht"]
    else:
        assert p.Ht is None
    assert np.array_equal(ct, ref["cellType"]) and np.array_equal(gm, ref["gammaLoaded"])
    assert n == (p.M // 2 * p.N if short else p.M * p.N)


def test_missing_geometry_means_all_fluid():
    texts = case_texts()
    ref = reference.run_io({"fluid_params.txt": texts["fluid_params.txt"]})
    with tempfile.TemporaryDirectory() as d:
        ct, gm, n = ef.read_geometry(os.path.join(d, "missing.txt"), ref["M"], ref["N"])
    assert n == 0 and np.array_equal(gm, ref["gammaLoaded"]) and np.all(gm == 1.0)


def test_restart_reader_matches_the_reference():
    texts = case_texts()
    M, N = 7, 11
    rng = np.random.default_rng(1)
    mats = {"u": rng.normal(size=(M + 1, N)), "v": rng.normal(size=(M, N + 1)), "p": rng.normal(size=(M + 1, N + 1))}
    rtexts = {f"{k}.txt": "\n".join(" ".join(repr(float(x)) for x in row) for row in m) + "\n" for k, m in mats.items()}
    rtexts["v.txt"] = rtexts["v.txt"][: len(rtexts["v.txt"]) // 2]  # incomplete: falls back to zeros
    ref = reference.run_io(texts, restart=rtexts)
    with tempfile.TemporaryDirectory() as d:
        write(d, rtexts)
        f, n = ef.read_restart(d, M, N)
    assert n == 2
    for k in ("u", "v", "p"):
        assert np.array_equal(f[k], ref[k]), k
    assert np.array_equal(f["u"], mats["u"]) and not f["v"].any()


def test_save_all_is_byte_identical_to_the_reference():
    texts = case_texts(M=9, N=13, extra=" 0.0005")
    M, N = 9, 13
    rng = np.random.default_rng(2)
    fields = {"u": rng.normal(size=(M + 1, N)) * 0.1, "v": rng.normal(size=(M, N + 1)) * 0.01,
              "p": rng.normal(size=(M + 1, N + 1)) * 300.0}
    ref = reference.run_io(texts, save=fields)
    assert "fluid_results.vtk" in ref["written"] and "u_thermal.txt" in ref["written"]
    with tempfile.TemporaryDirectory() as d:
        ef.save_all(d, M, N, ref["hx"], ref["hy"], fields, ref["gamma"], ref["alpha"], cellType=ref["cellType"],
                    N_in_buffer=ref["N_in_buffer"], N_out_buffer=ref["N_out_buffer"])
        mine = {name: open(os.path.join(d, name)).read() for name in sorted(os.listdir(d))}
    assert sorted(mine) == sorted(ref["written"])
    for name, text in ref["written"].items():
        assert mine[name] == text, name


def test_design_from_export_builds_what_the_reference_constructor_builds():
    texts = case_texts(M=9, N=13, extra=" 0.0005")
    ref = reference.run_io(texts)
    with tempfile.TemporaryDirectory() as d:
        write(d, texts)
        design, ct = ef.design_from_export(d)
    assert (design.M, design.N, design.hx, design.hy, design.inletVelocity, design.Ht_channel) == (
        ref["M"], ref["N"], ref["hx"], ref["hy"], ref["U_in"], ref["Ht"])
    assert np.array_equal(design.gamma, ref["gamma"]) and np.array_equal(design.alpha, ref["alpha"])
    assert np.array_equal(ct, ref["cellType"])
