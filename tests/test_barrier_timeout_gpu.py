"""Failure detection of the persistent kernels without a GPU fault: the grid
barrier every persistent kernel synchronises with (an arrival counter polled
by one thread per CTA) has a time limit.  cps_barrier_selftest makes its wait
run out on purpose -- the barrier expects one CTA more than the launch has, a
count nothing will reach -- and the host reads the timeout status the kernel
records; the device stays usable for the next solve."""
import ctypes

import numpy as np
import pytest

from coldplate_solver_b200 import cps, geometry

pytestmark = pytest.mark.gpu

LIMIT_MS = 2000.0  # the barrier's %globaltimer limit


@pytest.mark.parametrize("ctas", [1, 8, 148])
def test_barrier_wait_ends_with_a_timeout_status(ctas):
    lib = cps.load_library()
    ms = ctypes.c_double()
    st = lib.cps_barrier_selftest(0, ctas, ctypes.byref(ms))
    assert st == cps.CPS_ERR_TIMEOUT, (st, lib.cps_last_error(None))
    assert b"timed out" in lib.cps_last_error(None)
    assert LIMIT_MS * 0.95 <= ms.value < LIMIT_MS * 5, ms.value


def test_device_usable_after_a_timeout():
    lib = cps.load_library()
    assert lib.cps_barrier_selftest(0, 4, None) == cps.CPS_ERR_TIMEOUT
    d = geometry.straight_channel(M=12, N=20, band=(3, 9))
    with cps.Solver(d) as s:
        hist = s.solve(30, eps=0.0)
    assert hist.shape == (30, 8) and np.all(np.isfinite(hist))
