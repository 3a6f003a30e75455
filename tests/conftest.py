import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

GOLDEN = os.path.join(REPO, "tests", "golden")

from coldplate_solver_b200.geometry import Design  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libcps.so")
    config.addinivalue_line("markers", "slow: long-running")


def golden_names():
    return sorted(f[:-4] for f in os.listdir(GOLDEN)
                  if f.endswith(".npz") and not f.startswith(("alpha", "thermal_asm_")))


def load_golden(name):
    """Returns (design, init_fields_or_None, npz) for a golden fixture."""
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    kw = {}
    for k in ("M", "N", "convectionScheme", "maxPressureIter", "maxMomentumIter"):
        kw[k] = int(z[k])
    for k in ("enableTwoPointFiveD", "enableConvectionScaling"):
        kw[k] = bool(z[k])
    for k in ("hx", "hy", "inletVelocity", "Ht_channel", "twoPointFiveDSinkMultiplier", "uvAlpha", "pAlpha", "rho",
              "eta", "pTol", "momentumTol"):
        kw[k] = float(z[k])
    d = Design(gamma=z["gamma"], alpha=z["alpha"], name=name, **kw)
    init = None
    if "u0" in z.files:
        init = {"u": z["u0"], "v": z["v0"], "p": z["p0"]}
    return d, init, z


def golden_history(z, prec):
    return np.stack([z[f"{prec}_{k}"].astype(np.float64) for k in
                     ("residU", "residV", "residMass", "residMassDof", "err", "pIters", "uSweeps", "vSweeps")], 1)


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import restatement
    restatement.lib()
    return restatement
