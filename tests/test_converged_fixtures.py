"""The converged-state fixtures (tests/golden/converged/, written by
tests/golden/make_converged.py from the reference's own FP64 solve) and the
reference harness's design-loop mode, checked on the CPU.

* Every fixture rebuilds its design from the generator it names, with the
  grid it records, and its full dP is the difference of its own sampled
  planes.
* The small fixtures are fixed points of the oracle's C restatement: started
  from the fixture's state (rounded to float32, which perturbs the stiff
  Brinkman rows of the momentum equations to a residual of a few 1e-6) with
  the fixture's tight inner tolerances, the restated iteration stays there:
  its residual only decays, and its state moves by less than the 1e-6
  relative the GPU tests allow.
* Harness mode 4 (a design loop in one process) of the unpatched FP64
  reference equals separate runs of each design bit for bit, so the GPU test
  that runs the same mode through the drop-in compares like with like.
"""
import json
import os

import numpy as np
import pytest

from coldplate_solver_b200 import geometry

HERE = os.path.dirname(os.path.abspath(__file__))
CONVERGED = os.path.join(HERE, "golden", "converged")
NAMES = sorted(f[:-4] for f in os.listdir(CONVERGED) if f.endswith(".npz")) if os.path.isdir(CONVERGED) else []


def design_of(z):
    gen, args = str(z["generator"]), json.loads(str(z["args"]))
    if gen == "channel_network":
        return geometry.channel_network(**args)
    if gen == "density_field":
        return geometry.density_field(**args)
    if gen == "batch_mix":
        return geometry.batch_mix(args["n"])[args["k"]]
    if gen == "served_stream":
        return geometry.served_stream(args["n"])[args["k"]][1]
    raise ValueError(gen)


@pytest.mark.parametrize("name", NAMES)
def test_fixture_rebuilds_its_design(name):
    z = np.load(os.path.join(CONVERGED, name + ".npz"))
    d = design_of(z)
    st = int(z["stride"])
    assert (int(z["M"]), int(z["N"])) == (d.M, d.N)
    assert z["u"].shape == np.zeros((d.M + 1, d.N))[::st, ::st].shape
    assert z["p"].shape == np.zeros((d.M + 1, d.N + 1))[::st, ::st].shape
    # planes: x = 0, x = N hx, core in, core out; full dP = avgTotal(x = 0) - avgTotal(x = N hx)
    assert float(z["dp_full"]) == pytest.approx(float(z["planes"][0, 4] - z["planes"][1, 4]), rel=1e-15)
    assert float(z["residual_fixed"]) <= 1e-10
    tight = json.loads(str(z["tight"]))
    assert tight["pTol"] <= 1e-10 and tight["momentumTol"] <= 1e-10
    # the reference's own 1e-6 stop sits measurably away from its fixed point
    assert 0.0 < float(z["stop_err_u"]) < 0.1


@pytest.mark.parametrize("name", [n for n in NAMES if n.startswith(("served", "mix"))])
def test_small_fixture_is_a_fixed_point_of_the_restatement(name, oracle_lib):
    rs = oracle_lib
    z = np.load(os.path.join(CONVERGED, name + ".npz"))
    d = design_of(z).replace(**json.loads(str(z["tight"])))
    assert int(z["stride"]) == 1
    f = rs.new_fields(d)
    for k in ("u", "v", "p"):
        f[k][...] = z[k].astype(np.float64)
    start = {k: f[k].copy() for k in ("u", "v", "p")}
    h = rs.solve(d, f, 20, stop_on_conv=False)
    resid = np.maximum(np.maximum(h[:, 0], h[:, 1]), h[:, 3])
    assert resid.max() <= 1e-5 and resid[-1] < resid[0], resid
    for k in ("u", "v", "p"):
        rel = np.linalg.norm(f[k] - start[k]) / np.linalg.norm(start[k])
        assert rel <= 1e-6, (k, rel)


def test_design_loop_mode_equals_separate_runs():
    from oracle import reference
    if not reference.available("f64"):
        pytest.skip("oracle/_ref/ref_f64 not built")
    da = geometry.channel_network(M=24, N=40, h=20e-6, wmin=3, wmax=6, seed=5)
    db = geometry.channel_network(M=24, N=40, h=20e-6, wmin=3, wmax=6, seed=11)
    loop = reference.run_design_loop(da, db, 8, precision="f64")
    ra = reference.run(da, 8, precision="f64")
    rb = reference.run(db, 8, precision="f64")
    for k in ("u", "v", "p"):
        assert np.array_equal(loop[f"{k}1"], ra[k])
        assert np.array_equal(loop[f"{k}2"], rb[k])
        assert np.array_equal(loop[f"{k}3"], ra[k])
    assert np.array_equal(loop["pIters1"], ra["pIters"]) and np.array_equal(loop["pIters2"], rb["pIters"])


def test_bench_lines_have_their_fixtures():
    """Every workload whose bench line states its error against the
    reference's FP64 fixed point has that fixture committed, for the very
    design the bench solves (the single designs by workload name, mix design
    47 and served request 14 by index)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(os.path.dirname(HERE), "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    for workload, name in bench.ORACLE_FIXTURES.items():
        z = np.load(os.path.join(CONVERGED, name + ".npz"))
        d, _ = bench.workload(workload)
        dz = design_of(z)
        assert (d.M, d.N) == (dz.M, dz.N) == (int(z["M"]), int(z["N"])), workload
        assert np.array_equal(d.alpha, dz.alpha) and np.array_equal(d.gamma, dz.gamma), workload
    # the reference arm extrapolates the 1000 x 500 solve to the reference's own stop count
    z = np.load(os.path.join(CONVERGED, bench.ORACLE_FIXTURES["density"] + ".npz"))
    assert bench.REFERENCE_ITERS["density"] == int(z["n_stop"])
    mix = geometry.batch_mix(64)
    for k, name in bench.MIX_FIXTURES.items():
        dz = design_of(np.load(os.path.join(CONVERGED, name + ".npz")))
        assert np.array_equal(mix[k].alpha, dz.alpha), name
    stream = geometry.served_stream(32)
    for k, name in bench.SERVED_FIXTURES.items():
        dz = design_of(np.load(os.path.join(CONVERGED, name + ".npz")))
        assert np.array_equal(stream[k][1].alpha, dz.alpha), name
