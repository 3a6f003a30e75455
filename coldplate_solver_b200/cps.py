"""ctypes binding of libcps.so (the C ABI declared in include/cps.h).

The product path: every call goes to the CUDA library.  There is no CPU
fallback -- if libcps.so is missing or cannot initialise a GPU, the calls
raise.
"""
from __future__ import annotations

import ctypes
import os
from typing import Dict, Optional

import numpy as np

from .geometry import Design

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libcps.so")
TILE_WIDTHS = (32, 16, 64)  # the tile shapes built: 8 x 32 (libcps.so), 16 x 16, 4 x 64


def lib_path(tile_j: int = 32) -> str:
    """The library whose kernels evaluate tiles of ``tile_j`` columns
    (256 / tile_j rows)."""
    if tile_j not in TILE_WIDTHS:
        raise ValueError(f"tile width {tile_j} is not built (have {TILE_WIDTHS})")
    return LIB_PATH if tile_j == 32 else os.path.join(_PKG, f"libcps_t{tile_j}.so")

CPS_OK = 0
CPS_ERR_ARG, CPS_ERR_OOM, CPS_ERR_CUDA, CPS_ERR_TIMEOUT, CPS_ERR_DIVERGED, CPS_ERR_STATE = -1, -2, -3, -4, -5, -6
CPS_ROW_MAJOR, CPS_COL_MAJOR = 0, 1
CPS_FP64, CPS_MIXED = 0, 1
CPS_PCG_REFERENCE, CPS_PCG_SINGLE_REDUCTION = 0, 1

_STATUS_NAMES = {0: "OK", -1: "CPS_ERR_ARG", -2: "CPS_ERR_OOM", -3: "CPS_ERR_CUDA", -4: "CPS_ERR_TIMEOUT",
                 -5: "CPS_ERR_DIVERGED", -6: "CPS_ERR_STATE"}


class CpsError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{_STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class CpsDesc(ctypes.Structure):
    _fields_ = [
        ("M", ctypes.c_int), ("N", ctypes.c_int),
        ("hx", ctypes.c_double), ("hy", ctypes.c_double),
        ("rho", ctypes.c_double), ("eta", ctypes.c_double),
        ("uvAlpha", ctypes.c_double), ("pAlpha", ctypes.c_double),
        ("pTol", ctypes.c_double), ("maxPressureIter", ctypes.c_int),
        ("momentumTol", ctypes.c_double), ("maxMomentumIter", ctypes.c_int),
        ("convectionScheme", ctypes.c_int), ("enableTwoPointFiveD", ctypes.c_int),
        ("enableConvectionScaling", ctypes.c_int),
        ("Ht_channel", ctypes.c_double), ("twoPointFiveDSinkMultiplier", ctypes.c_double),
        ("precision", ctypes.c_int),
        ("alpha", ctypes.POINTER(ctypes.c_double)), ("gamma", ctypes.POINTER(ctypes.c_double)),
        ("layout", ctypes.c_int), ("device", ctypes.c_int), ("grid_ctas", ctypes.c_int),
        ("pcg_variant", ctypes.c_int),
        ("momentum_explicit", ctypes.c_int),
    ]


class CpsStepIn(ctypes.Structure):
    _fields_ = [("inletVelocity", ctypes.c_double)]


class CpsStepOut(ctypes.Structure):
    _fields_ = [("residU", ctypes.c_double), ("residV", ctypes.c_double), ("residMass", ctypes.c_double),
                ("residMassDof", ctypes.c_double), ("err", ctypes.c_double), ("pIters", ctypes.c_int),
                ("uSweeps", ctypes.c_int), ("vSweeps", ctypes.c_int)]


class CpsPlane(ctypes.Structure):
    _fields_ = [("flowArea", ctypes.c_double), ("massFlux", ctypes.c_double), ("avgStatic", ctypes.c_double),
                ("avgDynamic", ctypes.c_double), ("avgTotal", ctypes.c_double), ("valid", ctypes.c_int)]


class CpsBatchOpts(ctypes.Structure):
    _fields_ = [("cluster_ctas", ctypes.c_int), ("max_clusters", ctypes.c_int), ("max_outer", ctypes.c_int),
                ("eps", ctypes.c_double), ("order_by_size", ctypes.c_int), ("group_ctas", ctypes.c_int),
                ("tiles_per_cta", ctypes.c_int)]


class CpsDpMonitor(ctypes.Structure):
    _fields_ = [("gate", ctypes.c_int), ("window", ctypes.c_int), ("percent", ctypes.c_double),
                ("slope_gate", ctypes.c_int), ("slope_window", ctypes.c_int), ("slope_max_delta", ctypes.c_double),
                ("ramp_steps", ctypes.c_int), ("x_core_in", ctypes.c_double), ("x_core_out", ctypes.c_double)]


class CpsCaseParams(ctypes.Structure):
    _fields_ = [("M", ctypes.c_int), ("N", ctypes.c_int), ("hx", ctypes.c_double), ("hy", ctypes.c_double),
                ("U_in", ctypes.c_double), ("N_in_buffer", ctypes.c_int), ("N_out_buffer", ctypes.c_int),
                ("Ht", ctypes.c_double), ("has_Ht", ctypes.c_int)]


class CpsPseudo(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int) for k in ("enable", "use_local", "enable_ser", "enable_line_search",
                                             "enable_cfl_ramp", "ser_use_max_resid", "ser_min_iter",
                                             "ls_max_tries")] + \
               [(k, ctypes.c_double) for k in ("target_velocity", "time_step_multiplier", "min_pseudo_speed",
                                                "pseudo_cfl", "cfl_initial", "cfl_max", "cfl_ramp_start_res",
                                                "cfl_ramp_exponent", "cfl_ramp_smooth", "ser_cfl_min", "ser_cfl_max",
                                                "ser_smooth", "ser_max_increase", "ser_max_decrease",
                                                "ls_alpha_min", "ls_alpha_reduce", "ls_resid_increase_tol", "time_step")]


class CpsPseudoState(ctypes.Structure):
    _fields_ = [("pseudo_cfl", ctypes.c_double), ("ser_resid_prev", ctypes.c_double), ("ls_alpha", ctypes.c_double),
                ("ls_backtracks", ctypes.c_int), ("pad", ctypes.c_int)]


def pseudo_from_design(design: Design) -> CpsPseudo:
    """The cps_pseudo block of a design's pseudo-transient settings
    (reference member names, SIMPLE.h:255-313)."""
    d = design
    return CpsPseudo(enable=int(d.enablePseudoTimeStepping), use_local=int(d.useLocalPseudoTime),
                     enable_ser=int(d.enableSER), enable_line_search=int(d.enableLineSearch),
                     enable_cfl_ramp=int(d.enableCflRamp), ser_use_max_resid=int(d.serUseMaxResid),
                     ser_min_iter=d.serMinIter, ls_max_tries=d.lsMaxTries, target_velocity=d.inletVelocity,
                     time_step_multiplier=d.timeStepMultiplier, min_pseudo_speed=d.minPseudoSpeed,
                     pseudo_cfl=d.pseudoCFL, cfl_initial=d.pseudoCFLInitial, cfl_max=d.pseudoCFLMax,
                     cfl_ramp_start_res=d.cflRampStartRes, cfl_ramp_exponent=d.cflRampExponent,
                     cfl_ramp_smooth=d.cflRampSmooth, ser_cfl_min=d.serCFLMin, ser_cfl_max=d.serCFLMax,
                     ser_smooth=d.serSmooth, ser_max_increase=d.serMaxIncrease, ser_max_decrease=d.serMaxDecrease,
                     ls_alpha_min=d.lsAlphaMin, ls_alpha_reduce=d.lsAlphaReduce,
                     ls_resid_increase_tol=d.lsResidIncreaseTol)


class CpsThermalDesc(ctypes.Structure):
    _fields_ = [("Nx", ctypes.c_int), ("Ny", ctypes.c_int), ("nz_solid", ctypes.c_int), ("nz_fluid", ctypes.c_int),
                ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("H_b", ctypes.c_double), ("H_t", ctypes.c_double),
                ("k_s", ctypes.c_double), ("k_f", ctypes.c_double), ("rho", ctypes.c_double), ("Cp", ctypes.c_double),
                ("T_inlet", ctypes.c_double), ("rtol", ctypes.c_double), ("maxiter", ctypes.c_int),
                ("k_interp_mode", ctypes.c_int), ("qk", ctypes.c_double), ("gamma", ctypes.c_void_p),
                ("u", ctypes.c_void_p), ("v", ctypes.c_void_p), ("q0", ctypes.c_void_p), ("q", ctypes.c_double),
                ("device", ctypes.c_int), ("mg_sweeps", ctypes.c_int), ("mg_omega", ctypes.c_double),
                ("mg_overcorrect", ctypes.c_double)]


class CpsThermalResult(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("converged", ctypes.c_int), ("rel_residual", ctypes.c_double),
                ("true_rel_residual", ctypes.c_double)]


class CpsThermalMetrics(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in (
        "T_avg_base", "T_avg_fluid", "T_avg_solid", "T_avg_global", "T_std_base", "T_std_fluid", "T_std_global",
        "T_range_base", "T_range_fluid", "T_range_global", "T_uniformity_base", "T_uniformity_global",
        "grad_max", "grad_avg", "grad_max_base", "grad_avg_base")] + \
        [(k, ctypes.c_int) for k in ("grad_max_i", "grad_max_j", "grad_max_k", "pad")]


class CpsBatchResult(ctypes.Structure):
    _fields_ = [("n_done", ctypes.c_int), ("converged", ctypes.c_int), ("status", ctypes.c_int),
                ("last", CpsStepOut)]


# Every symbol include/cps.h declares, with its ctypes signature.
_P = ctypes.c_void_p
_D = ctypes.POINTER(ctypes.c_double)
SIGNATURES = {
    "cps_create": (ctypes.c_int, [ctypes.POINTER(CpsDesc), ctypes.POINTER(_P)]),
    "cps_destroy": (None, [_P]),
    "cps_upload_fields": (ctypes.c_int, [_P, _D, _D, _D, ctypes.c_int]),
    "cps_step": (ctypes.c_int, [_P, ctypes.POINTER(CpsStepIn), ctypes.POINTER(CpsStepOut)]),
    "cps_solve": (ctypes.c_int, [_P, ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.POINTER(CpsStepOut),
                                 ctypes.POINTER(ctypes.c_int)]),
    "cps_sample_plane": (ctypes.c_int, [_P, ctypes.c_double, ctypes.POINTER(CpsPlane)]),
    "cps_download_fields": (ctypes.c_int, [_P, _D, _D, _D, _D, _D, _D, _D, _D, ctypes.c_int]),
    "cps_footprint": (ctypes.c_int, [ctypes.POINTER(CpsDesc), ctypes.POINTER(ctypes.c_ulonglong)]),
    "cps_upload_geometry": (ctypes.c_int, [_P, _D, _D, ctypes.c_int]),
    "cps_reset_fields": (ctypes.c_int, [_P]),
    "cps_get_stream": (ctypes.c_int, [_P, ctypes.POINTER(_P)]),
    "cps_kernel_timing": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_longlong),
                                         ctypes.POINTER(ctypes.c_longlong), ctypes.c_int]),
    "cps_batch_solve": (ctypes.c_int, [ctypes.POINTER(_P), ctypes.c_int, _D, ctypes.POINTER(CpsBatchOpts),
                                       ctypes.POINTER(CpsBatchResult), _D]),
    "cps_get_history": (ctypes.c_int, [_P, ctypes.c_int, ctypes.POINTER(CpsStepOut)]),
    "cps_solve_noalloc": (ctypes.c_int, [ctypes.POINTER(CpsDesc), ctypes.c_int, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P,
                                         ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.POINTER(CpsStepOut),
                                         ctypes.POINTER(ctypes.c_int), _P]),
    "cps_set_dp_monitor": (ctypes.c_int, [_P, ctypes.POINTER(CpsDpMonitor)]),
    "cps_solve_monitored": (ctypes.c_int, [_P, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                           ctypes.POINTER(CpsStepOut), _D, ctypes.POINTER(ctypes.c_int),
                                           ctypes.POINTER(ctypes.c_int)]),
    "cps_set_inlet_ramp": (ctypes.c_int, [_P, ctypes.c_int]),
    "cps_pseudo_defaults": (ctypes.c_int, [ctypes.POINTER(CpsPseudo), ctypes.c_double]),
    "cps_set_pseudo": (ctypes.c_int, [_P, ctypes.POINTER(CpsPseudo)]),
    "cps_get_pseudo_state": (ctypes.c_int, [_P, ctypes.POINTER(CpsPseudoState)]),
    "cps_set_pseudo_state": (ctypes.c_int, [_P, ctypes.POINTER(CpsPseudoState)]),
    "cps_read_case_params": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(CpsCaseParams)]),
    "cps_read_geometry": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, _D, _D,
                                         ctypes.POINTER(ctypes.c_int)]),
    "cps_read_restart": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, _D, _D, _D,
                                        ctypes.POINTER(ctypes.c_int)]),
    "cps_save_all": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                    ctypes.c_int, ctypes.c_int, _D, _D, _D, _D, _D, _D, ctypes.c_int]),
    "cps_io_last_error": (ctypes.c_char_p, []),
    "cps_thermal_defaults": (ctypes.c_int, [ctypes.POINTER(CpsThermalDesc)]),
    "cps_thermal_create": (ctypes.c_int, [ctypes.POINTER(CpsThermalDesc), ctypes.POINTER(_P)]),
    "cps_thermal_update": (ctypes.c_int, [_P, _D, _D, _D, _D]),
    "cps_thermal_solve": (ctypes.c_int, [_P, ctypes.POINTER(CpsThermalResult)]),
    "cps_thermal_solve_from": (ctypes.c_int, [_P, _D, ctypes.POINTER(CpsThermalResult)]),
    "cps_thermal_download": (ctypes.c_int, [_P, _D]),
    "cps_thermal_system": (ctypes.c_int, [_P, _D, _D]),
    "cps_thermal_timing": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int),
                                          ctypes.c_int]),
    "cps_thermal_compute_metrics": (ctypes.c_int, [ctypes.POINTER(CpsThermalDesc), _D, _D,
                                                   ctypes.POINTER(CpsThermalMetrics)]),
    "cps_thermal_save": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(CpsThermalDesc), _D, _D, _D, _D]),
    "cps_thermal_destroy": (None, [_P]),
    "cps_thermal_last_error": (ctypes.c_char_p, [_P]),
    "cps_last_error": (ctypes.c_char_p, [_P]),
    "cps_barrier_selftest": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]),
    "cps_save_logs": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(CpsStepOut), _P, _P,
                                     ctypes.c_double]),
    "cps_version": (ctypes.c_char_p, []),
    "cps_tile_shape": (ctypes.c_int, [ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
}

_libs: Dict[str, ctypes.CDLL] = {}


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load libcps.so (or a tile-shape variant) once and bind every exported
    entry point (raises if missing)."""
    if path in _libs:
        return _libs[path]
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is not built; run `python -c 'import __graft_entry__ as g; g.build()'`")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _libs[path] = lib
    return lib


def tile_shape(lib: Optional[ctypes.CDLL] = None) -> tuple:
    """(rows, columns) of the tiles a library's kernels evaluate."""
    lib = lib or load_library()
    r, c = ctypes.c_int(0), ctypes.c_int(0)
    st = lib.cps_tile_shape(ctypes.byref(r), ctypes.byref(c))
    if st != CPS_OK:
        raise CpsError(st, lib.cps_last_error(None).decode())
    return r.value, c.value


def _dptr(a: Optional[np.ndarray]):
    if a is None:
        return None
    return a.ctypes.data_as(_D)


def field_shapes(M: int, N: int) -> Dict[str, tuple]:
    return {"u": (M + 1, N), "v": (M, N + 1), "p": (M + 1, N + 1), "pStar": (M + 1, N + 1),
            "uStar": (M + 1, N), "vStar": (M, N + 1), "dE": (M + 1, N), "dN": (M, N + 1)}


def make_desc(design: Design, precision: int = CPS_FP64, device: int = 0, grid_ctas: int = 0,
              pcg_variant: int = CPS_PCG_REFERENCE):
    """Build a CpsDesc; returns (desc, keepalive) -- keep the arrays alive."""
    alpha = np.ascontiguousarray(design.alpha, dtype=np.float64)
    gamma = np.ascontiguousarray(design.gamma, dtype=np.float64)
    d = CpsDesc(M=design.M, N=design.N, hx=design.hx, hy=design.hy, rho=design.rho, eta=design.eta,
                uvAlpha=design.uvAlpha, pAlpha=design.pAlpha, pTol=design.pTol,
                maxPressureIter=design.maxPressureIter, momentumTol=design.momentumTol,
                maxMomentumIter=design.maxMomentumIter, convectionScheme=design.convectionScheme,
                enableTwoPointFiveD=int(design.enableTwoPointFiveD),
                enableConvectionScaling=int(design.enableConvectionScaling), Ht_channel=design.Ht_channel,
                twoPointFiveDSinkMultiplier=design.twoPointFiveDSinkMultiplier, precision=precision,
                alpha=_dptr(alpha), gamma=_dptr(gamma), layout=CPS_ROW_MAJOR, device=device, grid_ctas=grid_ctas,
                pcg_variant=pcg_variant, momentum_explicit=int(design.momentumSolverType == 0))
    return d, (alpha, gamma)


def footprint(design: Design, precision: int = CPS_FP64) -> int:
    lib = load_library()
    d, keep = make_desc(design, precision)
    out = ctypes.c_ulonglong(0)
    st = lib.cps_footprint(ctypes.byref(d), ctypes.byref(out))
    if st != CPS_OK:
        raise CpsError(st, lib.cps_last_error(None).decode())
    return int(out.value)


class Solver:
    """One resident design on the GPU (a cps_ctx).

    Mirrors the reference's per-design state: ``step()`` is one
    ``SIMPLE::calculateStep`` (iterations.cpp:82-526), ``solve()`` the
    residual-stopped part of ``runIterations`` (SIMPLE.cpp:299-318),
    ``sample_plane()`` ``samplePlaneAtX`` (postprocessing.cpp:97-230).
    """

    def __init__(self, design: Design, precision: int = CPS_FP64, device: int = 0, grid_ctas: int = 0,
                 pcg_variant: int = CPS_PCG_REFERENCE, tile_j: int = 32):
        """``tile_j``: tile columns of the kernels (a library per shape, see
        :data:`TILE_WIDTHS`); designs solved in one batch share it."""
        self.lib = load_library(lib_path(tile_j))
        self.tile_j = tile_j
        self.design = design
        self.precision, self.device = precision, device
        desc, keep = make_desc(design, precision, device, grid_ctas, pcg_variant)
        ctx = _P()
        st = self.lib.cps_create(ctypes.byref(desc), ctypes.byref(ctx))
        if st != CPS_OK:
            raise CpsError(st, self.lib.cps_last_error(None).decode())
        self.ctx = ctx
        self.inletVelocity = design.inletVelocity
        if design.enablePseudoTimeStepping:
            self.set_pseudo(design)
        if design.enableInletRamp and design.rampSteps > 0:
            self.set_inlet_ramp(design.rampSteps)

    def _check(self, st: int) -> None:
        if st != CPS_OK:
            raise CpsError(st, self.lib.cps_last_error(self.ctx).decode())

    def close(self) -> None:
        if getattr(self, "ctx", None):
            self.lib.cps_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def upload_fields(self, u=None, v=None, p=None) -> None:
        M, N = self.design.M, self.design.N
        arrs = []
        for a, s in ((u, (M + 1, N)), (v, (M, N + 1)), (p, (M + 1, N + 1))):
            if a is None:
                arrs.append(None)
            else:
                a = np.ascontiguousarray(a, dtype=np.float64)
                if a.shape != s:
                    raise ValueError(f"expected shape {s}, got {a.shape}")
                arrs.append(a)
        self._check(self.lib.cps_upload_fields(self.ctx, *[_dptr(a) for a in arrs], CPS_ROW_MAJOR))

    def upload_geometry(self, alpha: np.ndarray, gamma: np.ndarray) -> None:
        M, N = self.design.M, self.design.N
        a = np.ascontiguousarray(alpha, dtype=np.float64)
        g = np.ascontiguousarray(gamma, dtype=np.float64)
        if a.shape != (M, N) or g.shape != (M, N):
            raise ValueError("alpha and gamma must be (M, N)")
        self._check(self.lib.cps_upload_geometry(self.ctx, _dptr(a), _dptr(g), CPS_ROW_MAJOR))

    def reset_fields(self) -> None:
        self._check(self.lib.cps_reset_fields(self.ctx))

    @property
    def stream(self) -> int:
        s = _P()
        self._check(self.lib.cps_get_stream(self.ctx, ctypes.byref(s)))
        return int(s.value or 0)

    def kernel_timing(self, reset: bool = False):
        """(kernel_ms, launches, outer_iterations) since the last reset."""
        ms, n, it = ctypes.c_double(), ctypes.c_longlong(), ctypes.c_longlong()
        self._check(self.lib.cps_kernel_timing(self.ctx, ctypes.byref(ms), ctypes.byref(n), ctypes.byref(it),
                                               int(reset)))
        return ms.value, n.value, it.value

    def step(self, inletVelocity: Optional[float] = None) -> Dict[str, float]:
        out = CpsStepOut()
        sin = CpsStepIn(self.inletVelocity if inletVelocity is None else inletVelocity)
        self._check(self.lib.cps_step(self.ctx, ctypes.byref(sin), ctypes.byref(out)))
        return {k: getattr(out, k) for k, _ in CpsStepOut._fields_}

    def solve(self, max_outer: int, eps: float = 1e-6, inletVelocity: Optional[float] = None) -> np.ndarray:
        """Returns the (n, 8) history: residU, residV, residMass, residMassDof,
        err, pIters, uSweeps, vSweeps."""
        hist = (CpsStepOut * max(1, max_outer))()
        nd = ctypes.c_int(0)
        uin = self.inletVelocity if inletVelocity is None else inletVelocity
        self._check(self.lib.cps_solve(self.ctx, uin, max_outer, eps, hist, ctypes.byref(nd)))
        out = np.zeros((nd.value, 8))
        for k in range(nd.value):
            h = hist[k]
            out[k] = (h.residU, h.residV, h.residMass, h.residMassDof, h.err, h.pIters, h.uSweeps, h.vSweeps)
        return out

    def set_pseudo(self, design: Optional[Design] = None) -> None:
        """cps_set_pseudo with the pseudo-transient settings of ``design``
        (default: this solver's); ``enablePseudoTimeStepping = False``
        switches the term off.  Resets the CFL controllers' state."""
        p = pseudo_from_design(self.design if design is None else design)
        self._check(self.lib.cps_set_pseudo(self.ctx, ctypes.byref(p)))

    def set_inlet_ramp(self, ramp_steps: int) -> None:
        """cps_set_inlet_ramp: solve() and solve_monitored() ramp the inlet
        velocity over the first ``ramp_steps`` outer iterations (0: off)."""
        self._check(self.lib.cps_set_inlet_ramp(self.ctx, int(ramp_steps)))

    def pseudo_state(self) -> Dict[str, float]:
        """The CFL controllers' state: pseudo_cfl, ser_resid_prev, ls_alpha,
        ls_backtracks."""
        st = CpsPseudoState()
        self._check(self.lib.cps_get_pseudo_state(self.ctx, ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in CpsPseudoState._fields_ if k != "pad"}

    def set_pseudo_state(self, pseudo_cfl: float, ser_resid_prev: float = 0.0, ls_alpha: float = 1.0,
                         ls_backtracks: int = 0) -> None:
        st = CpsPseudoState(pseudo_cfl=pseudo_cfl, ser_resid_prev=ser_resid_prev, ls_alpha=ls_alpha,
                            ls_backtracks=ls_backtracks)
        self._check(self.lib.cps_set_pseudo_state(self.ctx, ctypes.byref(st)))

    def set_dp_monitor(self, gate: bool = True, window: int = 500, percent: float = 1.0, slope_gate: bool = False,
                       slope_window: int = 1000, slope_max_delta: float = 10.0, ramp_steps: int = 1000,
                       x_core_in: float = 0.01, x_core_out: float = 0.05, enabled: bool = True) -> None:
        """Attach the pressure-drop monitor/gate (cps_set_dp_monitor); the
        defaults are the reference's (SIMPLE.h:88-89, 98-103, 346)."""
        if not enabled:
            self._check(self.lib.cps_set_dp_monitor(self.ctx, None))
            return
        m = CpsDpMonitor(gate=int(gate), window=window, percent=percent, slope_gate=int(slope_gate),
                         slope_window=slope_window, slope_max_delta=slope_max_delta, ramp_steps=ramp_steps,
                         x_core_in=x_core_in, x_core_out=x_core_out)
        self._check(self.lib.cps_set_dp_monitor(self.ctx, ctypes.byref(m)))

    def solve_monitored(self, max_outer: int, eps: float = 1e-6, inletVelocity: Optional[float] = None):
        """cps_solve_monitored: returns (history (n, 8), pressure drops (n, 4):
        core total, full total, core static, full static, dp_converged)."""
        hist = (CpsStepOut * max(1, max_outer))()
        dp = np.zeros((max(1, max_outer), 4))
        nd, conv = ctypes.c_int(0), ctypes.c_int(0)
        uin = self.inletVelocity if inletVelocity is None else inletVelocity
        self._check(self.lib.cps_solve_monitored(self.ctx, uin, max_outer, eps, hist, _dptr(dp), ctypes.byref(nd),
                                                 ctypes.byref(conv)))
        out = np.zeros((nd.value, 8))
        for k in range(nd.value):
            h = hist[k]
            out[k] = (h.residU, h.residV, h.residMass, h.residMassDof, h.err, h.pIters, h.uSweeps, h.vSweeps)
        return out, dp[: nd.value].copy(), bool(conv.value)

    def sample_plane(self, x: float) -> np.ndarray:
        pl = CpsPlane()
        self._check(self.lib.cps_sample_plane(self.ctx, x, ctypes.byref(pl)))
        return np.array([pl.flowArea, pl.massFlux, pl.avgStatic, pl.avgDynamic, pl.avgTotal, float(pl.valid)])

    def full_dp(self) -> float:
        """Full inlet-outlet total-pressure drop (SIMPLE.cpp:256-257, 349)."""
        a = self.sample_plane(0.0)
        b = self.sample_plane(self.design.N * self.design.hx)
        return float(a[4] - b[4])

    def download(self) -> Dict[str, np.ndarray]:
        shapes = field_shapes(self.design.M, self.design.N)
        out = {k: np.zeros(s) for k, s in shapes.items()}
        self._check(self.lib.cps_download_fields(self.ctx, *[_dptr(out[k]) for k in
                                                            ("u", "v", "p", "pStar", "uStar", "vStar", "dE", "dN")],
                                                 CPS_ROW_MAJOR))
        return out


def history_to_array(hist, n: int) -> np.ndarray:
    out = np.zeros((n, 8))
    for k in range(n):
        h = hist[k]
        out[k] = (h.residU, h.residV, h.residMass, h.residMassDof, h.err, h.pIters, h.uSweeps, h.vSweeps)
    return out


def batch_solve(solvers, max_outer: int, eps: float = 1e-6, cluster_ctas: int = 8, max_clusters: int = 0,
                order_by_size: bool = True, inlet_velocities=None, group_ctas: int = 0, tiles_per_cta: int = 0):
    """Advance many resident designs together (cps_batch_solve): on
    thread-block clusters of ``cluster_ctas``, on groups of ``group_ctas`` CTAs,
    or (``tiles_per_cta`` > 0) on groups sized to each design, in waves.
    Returns (results, kernel_ms); results[k] is a dict with n_done, converged,
    status and the last step's diagnostics."""
    if not solvers:
        return [], 0.0
    lib = solvers[0].lib
    if any(s.lib is not lib for s in solvers):
        raise ValueError("the designs of one batch must share one tile shape (one library)")
    n = len(solvers)
    ctxs = (_P * n)(*[s.ctx for s in solvers])
    uin = np.ascontiguousarray([s.inletVelocity if inlet_velocities is None else inlet_velocities[k]
                                for k, s in enumerate(solvers)], dtype=np.float64)
    opts = CpsBatchOpts(cluster_ctas=cluster_ctas, max_clusters=max_clusters, max_outer=max_outer, eps=eps,
                        order_by_size=int(order_by_size), group_ctas=group_ctas, tiles_per_cta=tiles_per_cta)
    res = (CpsBatchResult * n)()
    ms = ctypes.c_double(0.0)
    st = lib.cps_batch_solve(ctxs, n, _dptr(uin), ctypes.byref(opts), res, ctypes.byref(ms))
    if st not in (CPS_OK, CPS_ERR_DIVERGED, CPS_ERR_TIMEOUT):
        raise CpsError(st, lib.cps_last_error(None).decode())
    out = []
    for k in range(n):
        r = res[k]
        last = r.last
        out.append({"n_done": r.n_done, "converged": bool(r.converged), "status": r.status,
                    "last": (last.residU, last.residV, last.residMass, last.residMassDof, last.err, last.pIters,
                             last.uSweeps, last.vSweeps)})
    return out, ms.value


def get_history(solver: "Solver", n: int) -> np.ndarray:
    """The first n (<= 4096) diagnostics of the solver's last launch chunk or batch visit."""
    hist = (CpsStepOut * max(1, n))()
    solver._check(solver.lib.cps_get_history(solver.ctx, n, hist))
    return history_to_array(hist, n)
