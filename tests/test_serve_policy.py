"""The serving loop's scheduling rule, checked on the CPU (no GPU calls):
which designs an epoch advances under the "smallest" order."""
import pytest

from coldplate_solver_b200 import serve


def test_concurrent_groups_follow_the_placement():
    # two resident CTAs per SM on 148 SMs
    assert serve.concurrent_groups({"group_ctas": 148}) == 2
    assert serve.concurrent_groups({"group_ctas": 74}) == 4
    assert serve.concurrent_groups({"cluster_ctas": 8}) == 37
    assert serve.concurrent_groups({"tiles_per_cta": 4}) == 8


def test_epoch_designs_default_and_override():
    assert serve.Server().epoch_designs == 4  # default placement: SM-count groups
    assert serve.Server(mode={"group_ctas": 148}).epoch_designs == 4
    assert serve.Server(mode={"group_ctas": 148}, epoch_designs=3).epoch_designs == 3


def test_unknown_order_is_refused():
    with pytest.raises(ValueError):
        serve.Server(mode={"group_ctas": 148}, order="random")
