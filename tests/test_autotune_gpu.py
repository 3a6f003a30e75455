"""The autotuner over the batched solve's knobs (batch.autotune): the
placement (groups sized to each design, fixed CTA groups, thread-block
clusters), timed from the zero state and from a warm state, and the visit
length (outer iterations per design per launch), timed on converged solves of
the sample.  On a sample of the 64-design mix it returns one of its
candidates with the measured rates and times, and a batch run with the
choice converges every design."""
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
    res, ms = batch.solve_batch(designs[:2], eps=1e-6, max_outer=60000, mode=t.mode, visit=t.visit)
    assert all(r["converged"] for r in res) and ms > 0
