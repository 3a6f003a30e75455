"""Serving loop: continuous batching with HBM-footprint admission.

The key property: each request's result is the same alone and in the mix.
Within one placement a design's group of CTAs (a thread-block cluster, or a
group sized to the design) computes exactly what it would compute alone, so
the comparison is exact (bit for bit) on the fields and the iteration count;
across precisions and placements the tolerances of the other tests apply."""
import numpy as np
import pytest

from coldplate_solver_b200 import batch, cps, geometry, serve

pytestmark = pytest.mark.gpu


def small_stream(n=6, seed=3):
    rng = np.random.default_rng(seed)
    out = []
    t = 0.0
    for k in range(n):
        t += float(rng.exponential(0.02))
        nx = int(rng.integers(40, 120))
        if k % 2:
            d = geometry.density_field(Nx=nx, seed=k, sigma=3.0, U=float(rng.uniform(0.05, 0.3)))
        else:
            d = geometry.straight_channel(M=nx // 2, N=nx, band=(nx // 8, nx // 3))
        out.append((t, d))
    return out


@pytest.mark.parametrize("mode", [{"cluster_ctas": 4}, {"tiles_per_cta": 2}])
@pytest.mark.parametrize("precision", [cps.CPS_FP64, cps.CPS_MIXED])
def test_each_result_is_the_same_alone_and_in_the_mix(precision, mode):
    stream = small_stream()
    srv = serve.Server(visit=40, mode=mode, precision=precision, keep_fields=True, max_outer=30000)
    stats = srv.run(stream, real_time=True)
    assert stats.completed == len(stream), [(r.converged, r.outer_iterations) for r in stats.requests]
    assert stats.max_inflight >= 2  # requests overlapped on the device
    for r in stats.requests:
        alone = serve.Server(visit=40, mode=mode, precision=precision, keep_fields=True, max_outer=30000)
        s1 = alone.run([(0.0, r.design)], real_time=False)
        a = s1.requests[0]
        assert a.outer_iterations == r.outer_iterations
        for k in ("u", "v", "p"):
            assert np.array_equal(a.fields[k], r.fields[k]), (r.rid, k)
        assert a.dp == r.dp


def test_smallest_first_order_gives_the_arrival_order_results():
    """The in-flight order changes only which epoch a design finishes in,
    never what it computes."""
    stream = small_stream(5, seed=5)
    a = serve.Server(visit=40, keep_fields=True, max_outer=30000, order="arrival").run(stream, real_time=False)
    b = serve.Server(visit=40, keep_fields=True, max_outer=30000, order="smallest").run(stream, real_time=False)
    for ra, rb in zip(a.requests, b.requests):
        assert ra.outer_iterations == rb.outer_iterations and ra.dp == rb.dp
        for k in ("u", "v", "p"):
            assert np.array_equal(ra.fields[k], rb.fields[k]), (ra.rid, k)


def test_admission_respects_the_memory_budget():
    stream = small_stream(5, seed=7)
    fps = [cps.footprint(d, cps.CPS_MIXED) for _, d in stream]
    budget = sorted(fps)[-1] + sorted(fps)[-2]  # at most two of the largest at once
    srv = serve.Server(budget_bytes=budget, visit=60, cluster_ctas=4, max_outer=30000)
    stats = srv.run(stream, real_time=False)
    assert stats.completed == len(stream)
    assert stats.peak_bytes <= budget
    assert stats.max_inflight <= 5


def test_latency_statistics():
    stream = small_stream(8, seed=11)
    stats = serve.Server(visit=50, max_outer=30000).run(stream, real_time=True)
    lat = [r.latency for r in stats.requests]
    assert all(x > 0 for x in lat)
    assert stats.latency_p99_s >= stats.latency_p50_s > 0
    assert stats.solves_per_s > 0


def test_autotuner_picks_a_candidate_and_batch_solves():
    designs = [geometry.density_field(Nx=nx, seed=nx, sigma=3.0) for nx in (48, 64, 80, 96)]
    t = batch.autotune(designs, sample=4, probe=10, warm=50, visits=(100, 400), use_cache=False)
    assert t.mode in batch.mode_candidates() and all(v > 0 for v in t.cell_updates_per_s.values())
    res, ms = batch.solve_batch(designs, eps=1e-6, max_outer=40000, mode=t.mode, visit=500)
    assert all(r["converged"] for r in res) and ms > 0
