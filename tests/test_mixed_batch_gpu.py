"""Mixed-precision (FP32 inner solves in FP64 defect correction) and batched
(one thread-block cluster per design) paths, against the oracle and the plain
FP64 path.

Tolerances: a mixed-precision outer iteration applies FP32 corrections to FP64
fields.  Its inner solves are inexact by design (Jacobi RMS 1e-5, PCG
||r|| < 1e-4) and test their stop rules on FP32-stored values, so they stop
at slightly different iterates than the FP64 ones (a Jacobi sweep earlier or
later, a PCG residual at the tolerance instead of below it); from an
identical state the fields therefore agree with the FP64 step only to the
inner tolerances: REL_MIXED_STEP = 1e-3 relative L2 (observed 4e-5 to 1.5e-4
on stiff Brinkman fields).  At
convergence both sit on the same FP64 fixed point (REL_FIELD = 1e-6,
REL_DP = 1e-5, as for the FP64 path).  A
batched design differs from the same design solved alone on the whole grid
only in the grouping of the grid-wide sums: REL_STEP = 1e-10 and identical
inner iteration counts.
"""
import numpy as np
import pytest

from coldplate_solver_b200 import cps, geometry

pytestmark = pytest.mark.gpu

REL_MIXED_STEP = 1e-3
REL_STEP = 1e-10
REL_FIELD = 1e-6
REL_DP = 1e-5
FIELDS = ("u", "v", "p", "pStar", "uStar", "vStar", "dE", "dN")


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / nb if nb > 0 else np.linalg.norm(a - b)


def fluid_p(design, p):
    mask = np.zeros_like(p, dtype=bool)
    mask[1:design.M, 1:design.N] = design.gamma[:design.M - 1, :design.N - 1] > 0.5
    return p[mask]


def random_state(d, seed):
    rng = np.random.default_rng(seed)
    return {"u": rng.normal(0, 0.05, (d.M + 1, d.N)), "v": rng.normal(0, 0.02, (d.M, d.N + 1)),
            "p": rng.normal(0, 5.0, (d.M + 1, d.N + 1))}


@pytest.mark.parametrize("which", ["straight", "network", "density"])
def test_mixed_steps_close_to_oracle(which):
    from oracle import restatement as rs
    d = {"straight": geometry.straight_channel(M=40, N=70, band=(10, 30)),
         "network": geometry.channel_network(M=60, N=120, h=20e-6, wmin=4, wmax=8, seed=2),
         "density": geometry.density_field(Nx=128, seed=5, sigma=4.0)}[which]
    init = random_state(d, 1)
    with cps.Solver(d, precision=cps.CPS_MIXED) as s:
        s.upload_fields(init["u"], init["v"], init["p"])
        h = s.solve(1, eps=0.0)
        f = s.download()
    fr = rs.new_fields(d)
    for k in ("u", "v", "p"):
        fr[k][...] = init[k]
    hr = rs.solve(d, fr, 1, stop_on_conv=False)
    # sweep 1's residual is the FP64 defect, so the first U/V stop decisions match
    for k in ("u", "v", "uStar", "vStar", "dE", "dN"):
        assert rel(f[k], fr[k]) <= REL_MIXED_STEP, (k, rel(f[k], fr[k]))
    assert rel(fluid_p(d, f["p"]), fluid_p(d, fr["p"])) <= REL_MIXED_STEP
    np.testing.assert_allclose(h[0, :4], hr[0, :4], rtol=1e-4)


def test_mixed_converges_to_fp64_fixed_point():
    d = geometry.straight_channel()
    with cps.Solver(d) as a, cps.Solver(d, precision=cps.CPS_MIXED) as b:
        ha = a.solve(20000, eps=1e-6)
        hb = b.solve(20000, eps=1e-6)
        assert abs(len(hb) - len(ha)) <= 0.3 * len(ha), (len(ha), len(hb))
        a.solve(100000, eps=1e-10)
        b.solve(100000, eps=1e-10)
        fa, fb = a.download(), b.download()
        dpa, dpb = a.full_dp(), b.full_dp()
    for k in ("u", "v"):
        assert rel(fb[k], fa[k]) <= REL_FIELD, (k, rel(fb[k], fa[k]))
    assert rel(fluid_p(d, fb["p"]), fluid_p(d, fa["p"])) <= REL_FIELD
    assert abs(dpb - dpa) <= REL_DP * abs(dpa), (dpa, dpb)


def uneven_designs():
    return [geometry.straight_channel(M=30, N=50, band=(8, 20)),
            geometry.channel_network(M=64, N=130, h=20e-6, wmin=4, wmax=8, seed=3),
            geometry.density_field(Nx=96, seed=1, sigma=3.0),
            geometry.density_field(Nx=150, seed=2, sigma=4.0, twoFiveD=False),
            geometry.straight_channel(M=9, N=11, band=(2, 6)),
            geometry.channel_network(M=40, N=90, h=20e-6, wmin=3, wmax=6, seed=9)]


@pytest.mark.parametrize("mode,size", [("cluster", 1), ("cluster", 4), ("cluster", 8), ("cluster", 16),
                                       ("group", 3), ("group", 37), ("group", 74), ("wave", 1), ("wave", 4)])
def test_batch_matches_solo_solves(mode, size):
    designs = uneven_designs()
    n = 7
    solo = []
    for d in designs:
        with cps.Solver(d) as s:
            h = s.solve(n, eps=0.0)
            solo.append((h, s.download()))
    solvers = [cps.Solver(d) for d in designs]
    try:
        if mode == "cluster":
            res, ms = cps.batch_solve(solvers, n, eps=0.0, cluster_ctas=size)
        elif mode == "group":
            res, ms = cps.batch_solve(solvers, n, eps=0.0, group_ctas=size)
        else:
            res, ms = cps.batch_solve(solvers, n, eps=0.0, tiles_per_cta=size)
        assert ms > 0
        for k, s in enumerate(solvers):
            assert res[k]["n_done"] == n and res[k]["status"] == 0
            hb = cps.get_history(s, n)
            hs, fs = solo[k]
            assert np.array_equal(hb[:, 5:], hs[:, 5:]), (k, hb[:, 5:], hs[:, 5:])
            np.testing.assert_allclose(hb[:, :5], hs[:, :5], rtol=1e-8, atol=1e-300)
            fb = s.download()
            for f in FIELDS:
                assert rel(fb[f], fs[f]) <= REL_STEP, (k, f, rel(fb[f], fs[f]))
    finally:
        for s in solvers:
            s.close()


@pytest.mark.parametrize("kw", [{"cluster_ctas": 8}, {"group_ctas": 37}, {"tiles_per_cta": 2}])
def test_batch_result_is_the_same_alone_and_in_the_mix(kw):
    designs = uneven_designs()
    target = 2
    with cps.Solver(designs[target]) as alone:
        cps.batch_solve([alone], 9, eps=0.0, **kw)
        fa = alone.download()
    solvers = [cps.Solver(d) for d in designs]
    try:
        cps.batch_solve(solvers, 9, eps=0.0, **kw)
        fm = solvers[target].download()
    finally:
        for s in solvers:
            s.close()
    for f in FIELDS:
        assert np.array_equal(fa[f], fm[f]), f


def tiles(d):
    return ((d.M - 1 + 7) // 8) * ((d.N - 1 + 31) // 32)


@pytest.mark.parametrize("tpc", [1, 3, 8])
@pytest.mark.parametrize("precision", [cps.CPS_FP64, cps.CPS_MIXED])
def test_wave_batch_is_bitwise_the_solo_solve_on_as_many_ctas(tpc, precision):
    """A design's group in a wave has ceil(tiles / tiles_per_cta) CTAs and then
    computes exactly what the single-design kernel computes on that many CTAs."""
    designs = uneven_designs() + [geometry.density_field(Nx=300, seed=4)]
    n = 6
    solo = []
    for d in designs:
        k = -(-tiles(d) // tpc)
        with cps.Solver(d, precision=precision, grid_ctas=k) as s:
            solo.append((s.solve(n, eps=0.0), s.download()))
    solvers = [cps.Solver(d, precision=precision) for d in designs]
    try:
        res, _ = cps.batch_solve(solvers, n, eps=0.0, tiles_per_cta=tpc)
        for k, s in enumerate(solvers):
            assert res[k]["n_done"] == n and res[k]["status"] == 0
            hs, fs = solo[k]
            assert np.array_equal(cps.get_history(s, n), hs), k
            fb = s.download()
            for f in FIELDS:
                assert np.array_equal(fb[f], fs[f]), (k, f)
    finally:
        for s in solvers:
            s.close()


def test_batch_stops_each_design_at_convergence():
    designs = [geometry.straight_channel(M=20, N=40, band=(5, 15)),
               geometry.straight_channel(M=16, N=24, band=(4, 12)),
               geometry.straight_channel(M=30, N=60, band=(8, 22))]
    solo_iters = []
    for d in designs:
        with cps.Solver(d) as s:
            solo_iters.append(len(s.solve(4000, eps=1e-6)))
    solvers = [cps.Solver(d) for d in designs]
    try:
        res, _ = cps.batch_solve(solvers, 4000, eps=1e-6, cluster_ctas=4)
    finally:
        for s in solvers:
            s.close()
    for k, r in enumerate(res):
        assert r["converged"], r
        assert abs(r["n_done"] - solo_iters[k]) <= max(3, solo_iters[k] // 5), (r["n_done"], solo_iters[k])


@pytest.mark.parametrize("kw", [{"cluster_ctas": 8}, {"group_ctas": 16}, {"tiles_per_cta": 4}])
def test_batch_mixed_precision_runs(kw):
    designs = uneven_designs()[:4]
    solvers = [cps.Solver(d, precision=cps.CPS_MIXED) for d in designs]
    try:
        res, _ = cps.batch_solve(solvers, 5, eps=0.0, **kw)
        for s, r in zip(solvers, res):
            assert r["n_done"] == 5 and r["status"] == 0
            assert np.isfinite(s.download()["u"]).all()
    finally:
        for s in solvers:
            s.close()


def test_batch_rejects_mixed_precisions():
    d = geometry.straight_channel(M=10, N=12, band=(3, 7))
    a, b = cps.Solver(d), cps.Solver(d, precision=cps.CPS_MIXED)
    try:
        with pytest.raises(cps.CpsError) as e:
            cps.batch_solve([a, b], 2)
        assert e.value.status == cps.CPS_ERR_ARG
    finally:
        a.close()
        b.close()


@pytest.mark.parametrize("which", ["straight", "network"])
def test_single_reduction_pcg_fp64_tracks_the_reference_pcg(which):
    """The single-reduction recurrences produce the reference PCG's iterates in
    exact arithmetic; in FP64 one outer iteration from an identical state stays
    within 1e-8 of the oracle (only rounding of the carried vectors differs)."""
    from oracle import restatement as rs
    d = {"straight": geometry.straight_channel(M=40, N=70, band=(10, 30)),
         "network": geometry.channel_network(M=60, N=120, h=20e-6, wmin=4, wmax=8, seed=2)}[which]
    init = random_state(d, 5)
    with cps.Solver(d, pcg_variant=cps.CPS_PCG_SINGLE_REDUCTION) as s:
        s.upload_fields(init["u"], init["v"], init["p"])
        h = s.solve(1, eps=0.0)
        f = s.download()
    fr = rs.new_fields(d)
    for k in ("u", "v", "p"):
        fr[k][...] = init[k]
    hr = rs.solve(d, fr, 1, stop_on_conv=False)
    assert h[0, 5] == hr[0, 5]
    for k in FIELDS:
        assert rel(f[k], fr[k]) <= 1e-8, (k, rel(f[k], fr[k]))


def test_single_reduction_pcg_converges_to_the_same_fixed_point():
    d = geometry.straight_channel()
    with cps.Solver(d) as a, cps.Solver(d, pcg_variant=cps.CPS_PCG_SINGLE_REDUCTION) as b:
        a.solve(100000, eps=1e-10)
        b.solve(100000, eps=1e-10)
        fa, fb = a.download(), b.download()
        dpa, dpb = a.full_dp(), b.full_dp()
    for k in ("u", "v"):
        assert rel(fb[k], fa[k]) <= REL_FIELD, (k, rel(fb[k], fa[k]))
    assert abs(dpb - dpa) <= REL_DP * abs(dpa)
