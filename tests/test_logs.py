"""runIterations' two logs (initLogFiles / writeIterationLogs,
output.cpp:268-313) written by cps_save_logs (host code), against the files
the reference's own runIterations writes (harness mode 2): fed the values the
reference logged, the writer reproduces both files byte for byte."""
import numpy as np
import pytest

from coldplate_solver_b200 import exportfiles, geometry
from oracle import reference


def parse(text: bytes, cols: int) -> np.ndarray:
    lines = text.decode().splitlines()[1:]
    return np.array([[float(x) for x in ln.split()] for ln in lines]).reshape(-1, cols)


@pytest.mark.skipif(not reference.available("f64"), reason="oracle/_ref/ref_f64 not built")
@pytest.mark.parametrize("pseudo", [False, True])
def test_logs_equal_the_reference_files(tmp_path, pseudo):
    d = geometry.straight_channel(M=20, N=40, band=(5, 15))
    if pseudo:
        d = d.replace(enablePseudoTimeStepping=True, enableSER=True, serMinIter=3)
    xc = (0.25 * d.N * d.hx, 0.75 * d.N * d.hx)
    ref = reference.run_iterations(d, 3000, 20, 0.5, 10, x_core=xc)
    res = parse(ref["logs"]["residuals.txt"], 7)       # iter, mass, U, V, core, full, CFL
    dph = parse(ref["logs"]["pressure_drop_history.txt"], 5)
    n = res.shape[0]
    assert n > 20 and dph.shape[0] == n
    assert np.array_equal(res[:, 0], np.arange(n)) and np.array_equal(dph[:, 0], np.arange(n))
    hist = np.zeros((n, 8))
    hist[:, 0], hist[:, 1], hist[:, 2] = res[:, 2], res[:, 3], res[:, 1]
    exportfiles.save_logs(str(tmp_path), hist, dp=dph[:, 1:], cfl=res[:, 6])
    for name in ("residuals.txt", "pressure_drop_history.txt"):
        assert (tmp_path / name).read_bytes() == ref["logs"][name], name
    if not pseudo:  # the CFL column is the constant pseudoCFL default
        assert np.all(res[:, 6] == 0.1)
        exportfiles.save_logs(str(tmp_path / "c"), hist, dp=dph[:, 1:])
        assert (tmp_path / "c" / "residuals.txt").read_bytes() == ref["logs"]["residuals.txt"]


def test_logs_edge_cases(tmp_path):
    """No rows: the two headers only; no pressure drops: logged as 0; bad arguments are refused."""
    from coldplate_solver_b200 import cps
    exportfiles.save_logs(str(tmp_path / "empty"), np.zeros((0, 8)))
    assert (tmp_path / "empty" / "residuals.txt").read_text() == (
        "Iter MassResid UResid VResid Core_dP_AfterInletBuffer(Pa) Full_dP_FullSystem(Pa) CFL\n")
    assert (tmp_path / "empty" / "pressure_drop_history.txt").read_text() == (
        "Iter Core_Total(Pa) Full_Total(Pa) Core_Static(Pa) Full_Static(Pa)\n")
    h = np.zeros((2, 8))
    h[:, 0], h[:, 1], h[:, 2] = [1e-3, 2e-4], [5e-4, 1.5e-5], [0.25, 1.0 / 3.0]
    exportfiles.save_logs(str(tmp_path / "nodp"), h, iter0=7, cfl0=0.5)
    assert (tmp_path / "nodp" / "residuals.txt").read_text().splitlines()[1:] == [
        "7 0.25 0.001 0.0005 0 0 0.5", "8 0.333333 0.0002 1.5e-05 0 0 0.5"]
    assert (tmp_path / "nodp" / "pressure_drop_history.txt").read_text().splitlines()[1:] == ["7 0 0 0 0", "8 0 0 0 0"]
    lib = cps.load_library()
    assert lib.cps_save_logs(None, 0, 0, None, None, None, 0.0) == cps.CPS_ERR_ARG
    assert lib.cps_save_logs(str(tmp_path).encode(), 3, 0, None, None, None, 0.0) == cps.CPS_ERR_ARG
