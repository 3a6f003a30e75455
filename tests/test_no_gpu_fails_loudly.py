"""Without a CUDA device the product path fails loudly: every compute entry
point returns CPS_ERR_CUDA (raised as CpsError in Python) with CUDA's message,
and nothing falls back to a CPU path.  Runs only where no GPU is visible."""
import numpy as np
import pytest

from coldplate_solver_b200 import cps, geometry
from coldplate_solver_b200 import thermal as pt


def _gpu_visible() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


pytestmark = pytest.mark.skipif(_gpu_visible(), reason="a GPU is visible")


def test_flow_solver_raises_without_a_gpu():
    d = geometry.straight_channel(M=10, N=12, band=(3, 7))
    with pytest.raises(cps.CpsError) as e:
        cps.Solver(d)
    assert e.value.status == cps.CPS_ERR_CUDA


def test_thermal_solver_raises_without_a_gpu():
    g = np.ones((4, 6))
    c = pt.ThermalCase(gamma=g, u=0.1 * g, v=0 * g, dx=1e-5, dy=1e-5, q=1e5)
    with pytest.raises(cps.CpsError) as e:
        pt.ThermalSolver(c)
    assert e.value.status == cps.CPS_ERR_CUDA


def test_barrier_selftest_reports_cuda_error_without_a_gpu():
    lib = cps.load_library()
    assert lib.cps_barrier_selftest(0, 4, None) == cps.CPS_ERR_CUDA
    assert lib.cps_last_error(None)
