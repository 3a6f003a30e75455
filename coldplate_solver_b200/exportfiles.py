"""The reference's files at the boundary, through libcps's C++ readers and
writer (include/cps.h): the case a geometry export leaves in ExportFiles
(fluid_params.txt, geometry_fluid.txt; SIMPLE.cpp:31-47, 517-584), the
restart matrices u/v/p.txt (SIMPLE.cpp:203-232), saveAll's output
(output.cpp:73-266) and the outer loop's logs (output.cpp:268-313).  Host
code only; no GPU is needed."""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass
from typing import Dict, Optional

import numpy as np

from . import cps


@dataclass
class CaseParams:
    M: int
    N: int
    hx: float
    hy: float
    U_in: float
    N_in_buffer: int
    N_out_buffer: int
    Ht: Optional[float]


def _lib():
    return cps.load_library()


def _check(st: int) -> None:
    if st != cps.CPS_OK:
        raise cps.CpsError(st, _lib().cps_io_last_error().decode())


def read_case_params(path: str) -> CaseParams:
    """fluid_params.txt as SIMPLE::loadParameters reads it."""
    p = cps.CpsCaseParams()
    _check(_lib().cps_read_case_params(path.encode(), ctypes.byref(p)))
    return CaseParams(p.M, p.N, p.hx, p.hy, p.U_in, p.N_in_buffer, p.N_out_buffer, p.Ht if p.has_Ht else None)


def read_geometry(path: str, M: int, N: int):
    """geometry_fluid.txt: returns (cellType, gamma = 1 - cellType, values read)."""
    ct, gm = np.zeros((M, N)), np.zeros((M, N))
    n = ctypes.c_int(0)
    _check(_lib().cps_read_geometry(path.encode(), M, N, cps._dptr(ct), cps._dptr(gm), ctypes.byref(n)))
    return ct, gm, n.value


def read_restart(directory: str, M: int, N: int):
    """dir/{u,v,p}.txt: returns ({"u", "v", "p"}, number of complete files)."""
    f = {"u": np.zeros((M + 1, N)), "v": np.zeros((M, N + 1)), "p": np.zeros((M + 1, N + 1))}
    n = ctypes.c_int(0)
    _check(_lib().cps_read_restart(directory.encode(), M, N, cps._dptr(f["u"]), cps._dptr(f["v"]),
                                   cps._dptr(f["p"]), ctypes.byref(n)))
    return f, n.value


def save_all(directory: str, M: int, N: int, hx: float, hy: float, fields: Dict[str, np.ndarray],
             gamma: np.ndarray, alpha: np.ndarray, cellType: Optional[np.ndarray] = None, N_in_buffer: int = 0,
             N_out_buffer: int = 0) -> None:
    """SIMPLE::saveAll into ``directory`` (row-major arrays of the reference's shapes)."""
    os.makedirs(directory, exist_ok=True)
    arrs = {k: np.ascontiguousarray(fields[k], dtype=np.float64) for k in ("u", "v", "p")}
    g = np.ascontiguousarray(gamma, dtype=np.float64)
    a = np.ascontiguousarray(alpha, dtype=np.float64)
    c = None if cellType is None else np.ascontiguousarray(cellType, dtype=np.float64)
    _check(_lib().cps_save_all(directory.encode(), M, N, hx, hy, N_in_buffer, N_out_buffer, cps._dptr(arrs["u"]),
                               cps._dptr(arrs["v"]), cps._dptr(arrs["p"]), cps._dptr(c), cps._dptr(g), cps._dptr(a),
                               cps.CPS_ROW_MAJOR))


# cps_step_out (include/cps.h) as a NumPy record
_STEP_OUT = np.dtype([("residU", "f8"), ("residV", "f8"), ("residMass", "f8"), ("residMassDof", "f8"), ("err", "f8"),
                      ("pIters", "i4"), ("uSweeps", "i4"), ("vSweeps", "i4")], align=True)
assert _STEP_OUT.itemsize == ctypes.sizeof(cps.CpsStepOut)


def save_logs(directory: str, hist: np.ndarray, dp: Optional[np.ndarray] = None, cfl: Optional[np.ndarray] = None,
              cfl0: float = 0.1, iter0: int = 0) -> None:
    """runIterations' residuals.txt and pressure_drop_history.txt
    (output.cpp:268-313) into ``directory``: ``hist`` is a solve's (n, 8)
    history (residU, residV, residMass, ...), ``dp`` the (n, 4) drops of
    cps_solve_monitored (core total, full total, core static, full static;
    None logs 0), ``cfl`` the per-iteration CFL numbers (None: ``cfl0``, the
    reference's pseudoCFL default, on every row)."""
    os.makedirs(directory, exist_ok=True)
    h = np.asarray(hist, dtype=np.float64).reshape(-1, 8)
    n = h.shape[0]
    rows = np.zeros(max(1, n), dtype=_STEP_OUT)  # cps_step_out[n]; only the three residuals are logged
    rows["residU"][:n], rows["residV"][:n], rows["residMass"][:n] = h[:, 0], h[:, 1], h[:, 2]
    d = None if dp is None else np.ascontiguousarray(np.asarray(dp, dtype=np.float64).reshape(n, 4))
    c = None if cfl is None else np.ascontiguousarray(np.asarray(cfl, dtype=np.float64).reshape(n))
    _check(_lib().cps_save_logs(directory.encode(), n, iter0, rows.ctypes.data_as(ctypes.POINTER(cps.CpsStepOut)),
                                cps._dptr(d), cps._dptr(c), cfl0))


def design_from_export(directory: str, **overrides):
    """A Design from an ExportFiles directory as the reference's constructor
    builds it (SIMPLE.cpp:18-29): grid and inlet velocity from
    fluid_params.txt, gamma = 1 - cellType from geometry_fluid.txt, alpha by
    buildAlphaFromDensity (SIMPLE.cpp:589-630, wall rows forced); the other
    SIMPLE.h settings are the Design defaults unless given in ``overrides``.
    With the 2.5-D model on and no Ht in the file, Ht falls back to hy
    (SIMPLE.cpp:52-57).  Returns (design, cellType)."""
    from . import geometry
    p = read_case_params(os.path.join(directory, "fluid_params.txt"))
    ct, gamma, _ = read_geometry(os.path.join(directory, "geometry_fluid.txt"), p.M, p.N)
    alpha, gamma = geometry.alpha_ramp_reference(gamma)
    kw = dict(M=p.M, N=p.N, hx=p.hx, hy=p.hy, inletVelocity=p.U_in, gamma=gamma, alpha=alpha,
              Ht_channel=p.Ht if p.Ht is not None else 0.0, name=os.path.basename(os.path.normpath(directory)))
    kw.update(overrides)
    d = geometry.Design(**kw)
    if d.enableTwoPointFiveD and not d.Ht_channel > 0.0:
        d = d.replace(Ht_channel=p.hy)
    return d, ct
