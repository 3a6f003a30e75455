"""One pass of the cold-plate design loop on the GPU: the flow solve to its
stop, the thermal crop of the result, the 3-D conjugate-heat-transfer solve
and the numbers the reference reports for a design (pressure drop,
temperature statistics, energy balance).  The reference runs these as two
programs that exchange text files (SIMPLE's saveAll, then ThermalSolver's
main, thermal_solver.cpp:706-763); here the fields stay on the GPU between the
flow solve and the thermal assembly except for one download of u and v.
"""
from __future__ import annotations

from typing import Dict, Optional, Tuple

import numpy as np

from . import cps, exportfiles, thermal
from .geometry import Design

PSEUDO_CFL_DEFAULT = 0.1  # SIMPLE.h:263, the CFL column of residuals.txt while pseudo-time stepping is off


def solve_design(design: Design, q: float, eps: float = 1e-6, max_outer: int = 200000,
                 N_in_buffer: int = 0, N_out_buffer: int = 0, precision: int = cps.CPS_FP64,
                 thermal_params: Optional[Dict] = None, export_dir: Optional[str] = None,
                 x_core: Optional[Tuple[float, float]] = None) -> Dict[str, object]:
    """Flow to ``eps`` (or ``max_outer`` outer iterations), then the thermal
    solve with base heat flux ``q`` [W/m^2] on the crop between the inlet and
    outlet buffers.  Returns the flow history (n, 8), the full pressure drop,
    the flow fields, the temperature field (Nz, Ny, Nx), the thermal solve's
    result, ThermalMetrics and the energy balance.

    With ``export_dir`` the pass also leaves there the files the reference's
    two programs write: saveAll's (output.cpp:73-266), runIterations' two logs
    (output.cpp:268-313) and the thermal program's four outputs.  The flow then
    runs with the pressure-drop monitor on (its gate off, which leaves the
    iteration unchanged) so that every row carries its drops, the core planes
    at ``x_core`` (default: the buffer boundaries, N_in_buffer hx and
    (N - N_out_buffer) hx); the logs' CFL column is pseudoCFL's default, which
    is what the reference logs while pseudo-time stepping is off (with it on,
    the column is not recorded here)."""
    dp_log = None
    with cps.Solver(design, precision=precision) as s:
        if export_dir is None:
            hist = s.solve(max_outer, eps=eps)
        else:
            xc = x_core if x_core is not None else (N_in_buffer * design.hx, (design.N - N_out_buffer) * design.hx)
            s.set_dp_monitor(gate=False, window=1, percent=0.0, ramp_steps=0, x_core_in=xc[0], x_core_out=xc[1])
            hist, dp_log, _ = s.solve_monitored(max_outer, eps=eps)
        dp = s.full_dp()
        fields = s.download()
    case = thermal.ThermalCase.from_flow(design, fields, q=q, N_in_buffer=N_in_buffer, N_out_buffer=N_out_buffer,
                                         **(thermal_params or {}))
    with thermal.ThermalSolver(case) as ts:
        res = ts.solve()
        T = ts.temperature()
    if export_dir is not None:
        exportfiles.save_all(export_dir, design.M, design.N, design.hx, design.hy, fields, design.gamma, design.alpha,
                             N_in_buffer=N_in_buffer, N_out_buffer=N_out_buffer)
        exportfiles.save_logs(export_dir, hist, dp=dp_log, cfl0=PSEUDO_CFL_DEFAULT)
        thermal.save(export_dir, case, T)
    return {"flow_history": hist, "flow_converged": bool(len(hist) and max(hist[-1, 0], hist[-1, 1], hist[-1, 3]) <= eps),
            "dp": dp, "fields": fields, "thermal_case": case, "T": T, "thermal": res, "dp_log": dp_log,
            "metrics": thermal.metrics(case, T), "energy": thermal.energy_balance(case, T)}
