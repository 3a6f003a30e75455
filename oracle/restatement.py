"""ctypes binding of the oracle's C restatement, oracle/liboracle.so (TEST
INFRASTRUCTURE ONLY).

``precision="f64"`` is the reference promoted to double (the parity reference),
``"f32"`` the reference as shipped.  Fields are row-major numpy arrays in the
reference's index space: u/uStar/dE (M+1, N), v/vStar/dN (M, N+1), p/pStar
(M+1, N+1).
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from typing import Dict, Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

FIELD_NAMES = ("u", "v", "p", "pStar", "uStar", "vStar", "dE", "dN")
DIAG_NAMES = ("residU", "residV", "residMass", "residMassDof", "err", "pIters", "uSweeps", "vSweeps")


def build() -> str:
    """Compile liboracle.so with the recipe in oracle/Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE, "restatement"], check=True)
    return _LIB_PATH


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
    return _lib


def field_shapes(M: int, N: int) -> Dict[str, tuple]:
    return {"u": (M + 1, N), "v": (M, N + 1), "p": (M + 1, N + 1), "pStar": (M + 1, N + 1),
            "uStar": (M + 1, N), "vStar": (M, N + 1), "dE": (M + 1, N), "dN": (M, N + 1)}


def new_fields(design, precision: str = "f64") -> Dict[str, np.ndarray]:
    """All fields zero, as SIMPLE::initializeMemory leaves them (SIMPLE.cpp:184-197)."""
    dt = np.float64 if precision == "f64" else np.float32
    return {k: np.zeros(s, dtype=dt) for k, s in field_shapes(design.M, design.N).items()}


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _check(fields: Dict[str, np.ndarray], design, dt) -> None:
    for k, s in field_shapes(design.M, design.N).items():
        a = fields[k]
        if a.shape != s or a.dtype != dt or not a.flags.c_contiguous:
            raise ValueError(f"field {k}: expected {s} {dt} C-contiguous, got {a.shape} {a.dtype}")


def step(design, fields: Dict[str, np.ndarray], precision: str = "f64", stop_after: int = 3,
         pseudo_cfl: Optional[float] = None, inlet_velocity: Optional[float] = None) -> Dict[str, float]:
    """One outer iteration in place (iterations.cpp:82-526); ``pseudo_cfl``:
    the CFL number of the pseudo-transient term (default: the first step's);
    ``inlet_velocity``: this step's inlet velocity (default: the design's)."""
    dt = np.float64 if precision == "f64" else np.float32
    _check(fields, design, dt)
    alpha = np.ascontiguousarray(design.alpha, dtype=dt)
    gamma = np.ascontiguousarray(design.gamma, dtype=dt)
    diag = np.zeros(8, dtype=np.float64)
    fn = lib().orc64_step if precision == "f64" else lib().orc32_step
    dp = design.real_params(pseudo_cfl)
    if inlet_velocity is not None:
        dp[6] = inlet_velocity
    rc = fn(_ptr(design.int_params()), _ptr(dp), ctypes.c_int(stop_after),
            *[_ptr(fields[k]) for k in FIELD_NAMES], _ptr(alpha), _ptr(gamma), _ptr(diag))
    if rc != 0:
        raise RuntimeError(f"oracle step failed ({rc})")
    return dict(zip(DIAG_NAMES, diag.tolist()))


def solve(design, fields: Dict[str, np.ndarray], max_outer: int, eps: float = 1e-6, stop_on_conv: bool = True,
          precision: str = "f64") -> np.ndarray:
    """Outer iterations until max(residU, residV, residMassDof) <= eps (or
    ``max_outer``); returns the (steps, 8) diagnostic history."""
    dt = np.float64 if precision == "f64" else np.float32
    _check(fields, design, dt)
    alpha = np.ascontiguousarray(design.alpha, dtype=dt)
    gamma = np.ascontiguousarray(design.gamma, dtype=dt)
    hist = np.zeros((max_outer, 8), dtype=np.float64)
    fn = lib().orc64_solve if precision == "f64" else lib().orc32_solve
    n = fn(_ptr(design.int_params()), _ptr(design.real_params()), ctypes.c_int(max_outer), ctypes.c_double(eps),
           ctypes.c_int(int(stop_on_conv)), *[_ptr(fields[k]) for k in FIELD_NAMES], _ptr(alpha), _ptr(gamma),
           _ptr(hist))
    if n < 0:
        raise RuntimeError("oracle solve failed")
    return hist[:n]


def inlet_velocity(design, iteration: int, precision: str = "f64", ramp_steps: Optional[int] = None) -> float:
    """The inlet velocity of outer iteration ``iteration`` (SIMPLE.cpp:303-307):
    the ramp (iter + 1) / rampSteps of inletVelocity while it runs
    (``ramp_steps`` overrides ``design.rampSteps``)."""
    ip = design.int_params()
    if ramp_steps is not None:
        ip[17] = ramp_steps
    fn = lib().orc64_inlet_velocity if precision == "f64" else lib().orc32_inlet_velocity
    fn.restype = ctypes.c_double
    return fn(_ptr(ip), _ptr(design.real_params()), ctypes.c_int(iteration))


def pseudo_start(design) -> np.ndarray:
    """The CFL controllers' state before the first step: pseudoCFL,
    serResidPrev, lsCurrentAlpha, lsBacktrackCount (SIMPLE.cpp:78-82,
    SIMPLE.h:255-313)."""
    return np.array([design.pseudo_cfl_start(), 0.0, 1.0, 0.0], dtype=np.float64)


def pseudo_update(design, state: np.ndarray, diag: Dict[str, float], iteration: int,
                  precision: str = "f64") -> np.ndarray:
    """The outer loop's CFL controllers after the step with index
    ``iteration`` (SIMPLE.cpp:321-327, time_control.cpp:43-166); returns the
    new state."""
    st = np.array(state, dtype=np.float64, copy=True)
    resid = diag["err"] if design.serUseMaxResid else diag["residMass"]
    fn = lib().orc64_pseudo_update if precision == "f64" else lib().orc32_pseudo_update
    fn(_ptr(design.int_params()), _ptr(design.real_params(float(st[0]))), _ptr(st), ctypes.c_double(resid),
       ctypes.c_int(iteration))
    return st


def sample_plane(design, fields: Dict[str, np.ndarray], x: float, precision: str = "f64") -> np.ndarray:
    """postprocessing.cpp:97-230; returns flowArea, massFlux, avgStatic,
    avgDynamic, avgTotal, valid."""
    dt = np.float64 if precision == "f64" else np.float32
    out = np.zeros(6, dtype=np.float64)
    gamma = np.ascontiguousarray(design.gamma, dtype=dt)
    fn = lib().orc64_sample_plane if precision == "f64" else lib().orc32_sample_plane
    fn(ctypes.c_int(design.M), ctypes.c_int(design.N), ctypes.c_double(design.hx), ctypes.c_double(design.hy),
       ctypes.c_double(design.rho), ctypes.c_double(x), _ptr(np.ascontiguousarray(fields["u"], dtype=dt)),
       _ptr(np.ascontiguousarray(fields["v"], dtype=dt)), _ptr(np.ascontiguousarray(fields["p"], dtype=dt)),
       _ptr(gamma), _ptr(out))
    return out


def full_dp(design, fields: Dict[str, np.ndarray], precision: str = "f64") -> float:
    """Full inlet-outlet total-pressure drop (SIMPLE.cpp:256-257, 349)."""
    a = sample_plane(design, fields, 0.0, precision)
    b = sample_plane(design, fields, design.N * design.hx, precision)
    return float(a[4] - b[4])


def build_alpha(gamma: np.ndarray, alpha_max: float, q: float, precision: str = "f64"):
    """SIMPLE.cpp:589-630; returns (alpha, gamma_after_wall_forcing)."""
    dt = np.float64 if precision == "f64" else np.float32
    g = np.array(gamma, dtype=dt, copy=True, order="C")
    a = np.zeros_like(g)
    fn = lib().orc64_build_alpha if precision == "f64" else lib().orc32_build_alpha
    fn(ctypes.c_int(g.shape[0]), ctypes.c_int(g.shape[1]), ctypes.c_double(alpha_max), ctypes.c_double(q),
       _ptr(g), _ptr(a))
    return a, g


def dp_gate_solve(design, fields: Dict[str, np.ndarray], max_outer: int, window: int, percent: float,
                  ramp_steps: int, slope_gate: bool = False, slope_window: int = 0, slope_max_delta: float = 0.0,
                  x_core=(0.01, 0.05), precision: str = "f64"):
    """The outer loop of SIMPLE::runIterations (SIMPLE.cpp:269-408) with the
    residual test off: the inlet ramp (over ``ramp_steps`` with
    ``design.enableInletRamp``), one outer iteration, the CFL controllers (with
    ``design.enablePseudoTimeStepping``), the four planes (core inlet and
    outlet, x = 0, x = N hx), the four pressure drops, then the pressure-drop
    window and slope gate, until the gate passes or ``max_outer``.  Returns
    (dp (n, 4): core total, full total, core static, full static; converged)."""
    xs = (x_core[0], x_core[1], 0.0, design.N * design.hx)
    hist = [0.0] * window      # dpHistory, slot k
    idx, filled = 0, False
    slope_buf = []             # (iter, value), oldest first
    rows = []
    st = pseudo_start(design)
    for it in range(max_outer):
        diag = step(design, fields, precision, stop_after=3, pseudo_cfl=float(st[0]),
                    inlet_velocity=inlet_velocity(design, it, precision, ramp_steps))
        st = pseudo_update(design, st, diag, it, precision)
        m = [sample_plane(design, fields, x, precision) for x in xs]
        core, full = m[0][4] - m[1][4], m[2][4] - m[3][4]
        rows.append((core, full, m[0][2] - m[1][2], m[2][2] - m[3][2]))
        if slope_gate and slope_window > 0:
            slope_buf.append((it, core))
            if len(slope_buf) > slope_window:
                slope_buf.pop(0)
        if it >= ramp_steps:
            hist[idx] = core
            idx = (idx + 1) % window
            if idx == 0:
                filled = True
            if filled:
                s = 0.0
                for k in range(window):
                    s += hist[k]
                mean = s / float(window)
                var = 0.0
                for k in range(window):
                    dd = hist[k] - mean
                    var += dd * dd
                std = math.sqrt(var / float(window))
                denom = max(abs(mean), 1.0)
                std_pct = (std / denom) * 100.0
                latest = hist[(idx - 1 + window) % window]
                delta_pct = (abs(latest - mean) / denom) * 100.0
                ok = True
                if slope_gate and slope_window > 0 and len(slope_buf) >= slope_window:
                    x0 = float(slope_buf[0][0])
                    sx = sy = sxx = sxy = 0.0
                    n = float(len(slope_buf))
                    for (xi, yi) in slope_buf:
                        x = float(xi) - x0
                        sx += x
                        sy += yi
                        sxx += x * x
                        sxy += x * yi
                    den = n * sxx - sx * sx
                    slope = 0.0 if abs(den) < 1e-12 else (n * sxy - sx * sy) / den
                    ok = abs(slope) <= slope_max_delta / float(slope_window)
                if std_pct < percent and delta_pct < percent and ok:
                    return np.array(rows), True
    return np.array(rows), False
