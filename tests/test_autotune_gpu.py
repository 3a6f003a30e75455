"""The autotuner over the batched solve's knobs (batch.autotune): the
placement (groups sized to each design, fixed CTA groups, thread-block
clusters), timed from the zero state and from a warm state, and the visit
length (outer iterations per design per launch), timed on converged solves of
the sample, and the tile shape (8 x 32, 16 x 16, 4 x 64: one library each).
On a sample of the 64-design mix it returns one of its candidates with the
measured rates and times, and a batch run with the choice converges every
design.  Every tile shape reaches the same converged state to within the
solve's own stop tolerance."""
import numpy as np
import pytest

from coldplate_solver_b200 import batch, cps, geometry

pytestmark = pytest.mark.gpu


def test_autotune_picks_placement_and_visit_on_a_mix_sample():
    mix = geometry.batch_mix(64)
    small = sorted(range(64), key=lambda k: mix[k].M * mix[k].N)[:6]
    designs = [mix[k] for k in small]
    cands = [{"group_ctas": 148}, {"group_ctas": 37}, {"tiles_per_cta": 4}]
    visits = (256, 2048)
    t = batch.autotune(designs, precision=cps.CPS_FP64, sample=4, probe=60, warm=300, visits=visits,
                       candidates=cands, max_outer=60000, use_cache=False)
    assert t.mode in cands
    assert t.visit in visits
    assert set(t.cell_updates_per_s) == {batch.mode_label(m) for m in cands}
    assert all(v > 0 for v in t.cell_updates_per_s.values())
    assert set(t.visit_ms) == set(visits) and all(v > 0 for v in t.visit_ms.values())
    assert t.tile_j in cps.TILE_WIDTHS and set(t.tile_cell_updates_per_s) == set(cps.TILE_WIDTHS)
    assert all(v > 0 for v in t.tile_cell_updates_per_s.values())
    res, ms = batch.solve_batch(designs[:2], eps=1e-6, max_outer=60000, mode=t.mode, visit=t.visit,
                                tile_j=t.tile_j)
    assert all(r["converged"] for r in res) and ms > 0


@pytest.mark.parametrize("tile_j", [16, 64])
def test_tile_shapes_give_the_default_shape_result(tile_j):
    """Each library reports its shape; 10 outer iterations of a 2.5-D density
    design agree with the 8 x 32 build to rounding (the shape regroups the
    grid-wide sums only), and both converge to the same tight fixed point."""
    assert cps.tile_shape(cps.load_library(cps.lib_path(tile_j))) == (256 // tile_j, tile_j)
    d = geometry.density_field(Nx=150, seed=4, sigma=3.0)
    out = {}
    for tj in (32, tile_j):
        with cps.Solver(d, tile_j=tj) as s:
            h = s.solve(10, eps=0.0)
            out[tj] = (h, s.download())
    (ha, fa), (hb, fb) = out[32], out[tile_j]
    assert np.array_equal(ha[:, 5:], hb[:, 5:])  # inner iteration counts
    for k in ("u", "v", "p"):
        assert np.linalg.norm(fa[k] - fb[k]) <= 1e-9 * np.linalg.norm(fa[k]), k
    tight = d.replace(pTol=1e-10, maxPressureIter=1000, momentumTol=1e-10)
    fixed = {}
    for tj in (32, tile_j):
        with cps.Solver(tight, tile_j=tj) as s:
            h = s.solve(100000, eps=1e-10)
            assert max(h[-1, 0], h[-1, 1], h[-1, 3]) <= 1e-10
            fixed[tj] = s.download()
    for k in ("u", "v", "p"):
        assert np.linalg.norm(fixed[32][k] - fixed[tile_j][k]) <= 1e-8 * np.linalg.norm(fixed[32][k]), k
