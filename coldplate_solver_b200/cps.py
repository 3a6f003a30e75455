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

CPS_OK = 0
CPS_ERR_ARG, CPS_ERR_OOM, CPS_ERR_CUDA, CPS_ERR_TIMEOUT, CPS_ERR_DIVERGED, CPS_ERR_STATE = -1, -2, -3, -4, -5, -6
CPS_ROW_MAJOR, CPS_COL_MAJOR = 0, 1
CPS_FP64, CPS_MIXED = 0, 1

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
    "cps_last_error": (ctypes.c_char_p, [_P]),
    "cps_version": (ctypes.c_char_p, []),
}

_lib: Optional[ctypes.CDLL] = None


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load libcps.so and bind every exported entry point (raises if missing)."""
    global _lib
    if _lib is not None and path == LIB_PATH:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is not built; run `python -c 'import __graft_entry__ as g; g.build()'`")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path == LIB_PATH:
        _lib = lib
    return lib


def _dptr(a: Optional[np.ndarray]):
    if a is None:
        return None
    return a.ctypes.data_as(_D)


def field_shapes(M: int, N: int) -> Dict[str, tuple]:
    return {"u": (M + 1, N), "v": (M, N + 1), "p": (M + 1, N + 1), "pStar": (M + 1, N + 1),
            "uStar": (M + 1, N), "vStar": (M, N + 1), "dE": (M + 1, N), "dN": (M, N + 1)}


def make_desc(design: Design, precision: int = CPS_FP64, device: int = 0, grid_ctas: int = 0):
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
                alpha=_dptr(alpha), gamma=_dptr(gamma), layout=CPS_ROW_MAJOR, device=device, grid_ctas=grid_ctas)
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

    def __init__(self, design: Design, precision: int = CPS_FP64, device: int = 0, grid_ctas: int = 0):
        self.lib = load_library()
        self.design = design
        desc, keep = make_desc(design, precision, device, grid_ctas)
        ctx = _P()
        st = self.lib.cps_create(ctypes.byref(desc), ctypes.byref(ctx))
        if st != CPS_OK:
            raise CpsError(st, self.lib.cps_last_error(None).decode())
        self.ctx = ctx
        self.inletVelocity = design.inletVelocity

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
