"""One pass of the cold-plate design loop on the GPU: the flow solve to its
stop, the thermal crop of the result, the 3-D conjugate-heat-transfer solve
and the numbers the reference reports for a design (pressure drop,
temperature statistics, energy balance).  The reference runs these as two
programs that exchange text files (SIMPLE's saveAll, then ThermalSolver's
main, thermal_solver.cpp:706-763); here the fields stay on the GPU between the
flow solve and the thermal assembly except for one download of u and v.
"""
from __future__ import annotations

from typing import Dict, Optional

import numpy as np

from . import cps, thermal
from .geometry import Design


def solve_design(design: Design, q: float, eps: float = 1e-6, max_outer: int = 200000,
                 N_in_buffer: int = 0, N_out_buffer: int = 0, precision: int = cps.CPS_FP64,
                 thermal_params: Optional[Dict] = None) -> Dict[str, object]:
    """Flow to ``eps`` (or ``max_outer`` outer iterations), then the thermal
    solve with base heat flux ``q`` [W/m^2] on the crop between the inlet and
    outlet buffers.  Returns the flow history (n, 8), the full pressure drop,
    the flow fields, the temperature field (Nz, Ny, Nx), the thermal solve's
    result, ThermalMetrics and the energy balance."""
    with cps.Solver(design, precision=precision) as s:
        hist = s.solve(max_outer, eps=eps)
        dp = s.full_dp()
        fields = s.download()
    case = thermal.ThermalCase.from_flow(design, fields, q=q, N_in_buffer=N_in_buffer, N_out_buffer=N_out_buffer,
                                         **(thermal_params or {}))
    with thermal.ThermalSolver(case) as ts:
        res = ts.solve()
        T = ts.temperature()
    return {"flow_history": hist, "flow_converged": bool(len(hist) and max(hist[-1, 0], hist[-1, 1], hist[-1, 3]) <= eps),
            "dp": dp, "fields": fields, "thermal_case": case, "T": T, "thermal": res,
            "metrics": thermal.metrics(case, T), "energy": thermal.energy_balance(case, T)}
