"""The 3-D conjugate-heat-transfer step downstream of the flow solve, on the
GPU (include/cps_thermal.h): the system of ThermalSolver3D::solve
(ThermalSolver/thermal_solver.cpp:420-560) assembled on the device and solved
by multigrid-preconditioned BiCGStab.

A ``ThermalCase`` carries the reference's Params (thermal_solver.cpp:147-193)
and the 2-D inputs its main() loads (:706-760): gamma (1 = fluid), the
cell-centred velocities of the thermal crop and the base heat flux.
``ThermalCase.from_export`` reads the files the reference reads;
``ThermalCase.from_flow`` builds the same inputs from a flow result in memory
(the crop saveAll writes as u_thermal.txt / v_thermal.txt, output.cpp:146-171).
"""
from __future__ import annotations

import ctypes
import dataclasses
import os
from typing import Dict, Optional

import numpy as np

from . import cps


@dataclasses.dataclass
class ThermalCase:
    gamma: np.ndarray           # (Ny, Nx), 1 = fluid
    u: np.ndarray               # (Ny, Nx) cell-centred x velocity [m/s]
    v: np.ndarray               # (Ny, Nx) cell-centred y velocity [m/s]
    dx: float
    dy: float
    q: float = 0.0              # uniform base heat flux [W/m^2] (thermal_params.txt)
    q0: Optional[np.ndarray] = None  # (Ny, Nx) base heat flux, overrides q
    nz_solid: int = 2
    nz_fluid: int = 7
    H_b: float = 0.0005
    H_t: float = 0.004
    k_s: float = 400.0
    k_f: float = 0.6
    rho: float = 998.0
    Cp: float = 4180.0
    T_inlet: float = 30.0
    rtol: float = 1e-6
    maxiter: int = 1000
    k_interp_mode: int = 1
    qk: float = 1.0

    def __post_init__(self) -> None:
        self.gamma = np.ascontiguousarray(self.gamma, dtype=np.float64)
        self.u = np.ascontiguousarray(self.u, dtype=np.float64)
        self.v = np.ascontiguousarray(self.v, dtype=np.float64)
        if self.q0 is not None:
            self.q0 = np.ascontiguousarray(self.q0, dtype=np.float64)
        if self.gamma.ndim != 2 or self.u.shape != self.gamma.shape or self.v.shape != self.gamma.shape:
            raise ValueError("gamma, u and v must have the same (Ny, Nx) shape")
        if self.q0 is not None and self.q0.shape != self.gamma.shape:
            raise ValueError("q0 must have the (Ny, Nx) shape of gamma")

    @property
    def Ny(self) -> int:
        return self.gamma.shape[0]

    @property
    def Nx(self) -> int:
        return self.gamma.shape[1]

    @property
    def Nz(self) -> int:
        return self.nz_solid + self.nz_fluid

    def heat_flux(self) -> np.ndarray:
        return self.q0 if self.q0 is not None else np.full(self.gamma.shape, float(self.q))

    @staticmethod
    def from_export(directory: str, qk: float = 1.0, k_interp_mode: int = 1) -> "ThermalCase":
        """The inputs the reference's main() reads (thermal_solver.cpp:706-760):
        thermal_params.txt (M N dx dy qf Ht), geometry_thermal.txt (0 = fluid,
        1 = solid, inverted here to gamma), u_thermal.txt, v_thermal.txt
        (missing velocity files leave zero velocity)."""
        with open(os.path.join(directory, "thermal_params.txt")) as f:
            tok = f.read().split()
        _M, _N, dx, dy, qf, Ht = int(tok[0]), int(tok[1]), float(tok[2]), float(tok[3]), float(tok[4]), float(tok[5])

        def read_2d(path):
            rows = []
            if not os.path.exists(path):
                return None
            with open(path) as f:
                for line in f:
                    if not line.strip() or line.startswith("#"):
                        continue
                    rows.append([float(x) for x in line.split()])
            return rows

        geo = read_2d(os.path.join(directory, "geometry_thermal.txt"))
        if not geo:
            raise FileNotFoundError("could not load geometry_thermal.txt")
        Ny, Nx = len(geo), len(geo[0])
        gamma = np.array([[1.0 - x for x in row[:Nx]] for row in geo])
        u = np.zeros((Ny, Nx))
        v = np.zeros((Ny, Nx))
        uu = read_2d(os.path.join(directory, "u_thermal.txt"))
        vv = read_2d(os.path.join(directory, "v_thermal.txt"))
        if uu:
            for j in range(min(Ny, len(uu))):
                for i in range(min(Nx, len(uu[j]))):
                    u[j, i] = uu[j][i]
                    v[j, i] = vv[j][i]
        # Params::dx() = Lx / Nx with Lx = cols * dx (thermal_solver.cpp:188, 723)
        return ThermalCase(gamma=gamma, u=u, v=v, dx=(Nx * dx) / Nx, dy=(Ny * dy) / Ny, q=qf, H_t=Ht, qk=qk,
                           k_interp_mode=k_interp_mode)

    @staticmethod
    def from_flow(design, fields: Dict[str, np.ndarray], q: float, N_in_buffer: int = 0, N_out_buffer: int = 0,
                  **params) -> "ThermalCase":
        """The thermal inputs of a flow result: the cell-centred velocities
        of saveAll's thermal crop (output.cpp:87-103, 146-171) and the crop of
        the design's gamma; H_t = the design's channel height when it has one.
        The cell sizes are the thermal program's own, Params::dx() = (Nx dx)/Nx
        (thermal_solver.cpp:723, 184), as it computes them from dx."""
        U, V = fields["u"], fields["v"]
        uC = 0.5 * (U[:-1, :] + U[1:, :])
        vC = 0.5 * (V[:, :-1] + V[:, 1:])
        lo, hi = N_in_buffer, design.N - N_out_buffer
        if "H_t" not in params and design.Ht_channel > 0:
            params["H_t"] = design.Ht_channel
        nx, ny = hi - lo, design.M
        return ThermalCase(gamma=design.gamma[:, lo:hi], u=uC[:, lo:hi], v=vC[:, lo:hi], dx=(nx * design.hx) / nx,
                           dy=(ny * design.hy) / ny, q=q, **params)


def _desc(case: ThermalCase) -> "cps.CpsThermalDesc":
    lib = cps.load_library()
    d = cps.CpsThermalDesc()
    lib.cps_thermal_defaults(ctypes.byref(d))
    for k in ("nz_solid", "nz_fluid", "dx", "dy", "H_b", "H_t", "k_s", "k_f", "rho", "Cp", "T_inlet", "rtol",
              "maxiter", "k_interp_mode", "qk", "q"):
        setattr(d, k, getattr(case, k))
    d.Nx, d.Ny = case.Nx, case.Ny
    return d


def metrics(case: ThermalCase, T: np.ndarray) -> Dict[str, float]:
    """compute_thermal_metrics (thermal_output.cpp:135-320) of a temperature
    field (Nz, Ny, Nx): volume-weighted averages, deviations, ranges,
    uniformity and gradient statistics (cps_thermal_compute_metrics)."""
    lib = cps.load_library()
    T = np.ascontiguousarray(T, dtype=np.float64)
    if T.shape != (case.Nz, case.Ny, case.Nx):
        raise ValueError("T must be (Nz, Ny, Nx)")
    m = cps.CpsThermalMetrics()
    d = _desc(case)
    st = lib.cps_thermal_compute_metrics(ctypes.byref(d), cps._dptr(T), cps._dptr(case.gamma), ctypes.byref(m))
    if st != cps.CPS_OK:
        raise cps.CpsError(st, "cps_thermal_compute_metrics: bad arguments")
    return {k: getattr(m, k) for k, _ in cps.CpsThermalMetrics._fields_ if k != "pad"}


def save(directory: str, case: ThermalCase, T: np.ndarray) -> None:
    """The files the reference's thermal main writes (thermal_results_3d.vtk,
    thermal_metrics.txt, k_thermal.txt, thermal_gradient_3d.vtk;
    cps_thermal_save)."""
    lib = cps.load_library()
    T = np.ascontiguousarray(T, dtype=np.float64)
    if T.shape != (case.Nz, case.Ny, case.Nx):
        raise ValueError("T must be (Nz, Ny, Nx)")
    d = _desc(case)
    st = lib.cps_thermal_save(directory.encode(), ctypes.byref(d), cps._dptr(T), cps._dptr(case.gamma),
                              cps._dptr(case.u), cps._dptr(case.v))
    if st != cps.CPS_OK:
        raise cps.CpsError(st, f"cps_thermal_save: could not write to {directory}")


class ThermalSolver:
    """One thermal case resident on the GPU (a cps_thermal handle)."""

    def __init__(self, case: ThermalCase, device: int = 0, mg_sweeps: int = 0, mg_omega: float = 0.0,
                 mg_overcorrect: float = 0.0):
        self.lib = cps.load_library()
        self.case = case
        d = _desc(case)
        d.device = device
        d.mg_sweeps, d.mg_omega, d.mg_overcorrect = mg_sweeps, mg_omega, mg_overcorrect
        d.gamma, d.u, d.v = case.gamma.ctypes.data, case.u.ctypes.data, case.v.ctypes.data
        d.q0 = case.q0.ctypes.data if case.q0 is not None else None
        h = cps._P()
        st = self.lib.cps_thermal_create(ctypes.byref(d), ctypes.byref(h))
        if st != cps.CPS_OK:
            raise cps.CpsError(st, self.lib.cps_thermal_last_error(None).decode())
        self.h = h

    def _check(self, st: int) -> None:
        if st != cps.CPS_OK:
            raise cps.CpsError(st, self.lib.cps_thermal_last_error(self.h).decode())

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.cps_thermal_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def solve(self) -> Dict[str, float]:
        r = cps.CpsThermalResult()
        self._check(self.lib.cps_thermal_solve(self.h, ctypes.byref(r)))
        return {"iterations": r.iterations, "converged": bool(r.converged), "rel_residual": r.rel_residual,
                "true_rel_residual": r.true_rel_residual}

    def solve_from(self, T0: Optional[np.ndarray] = None) -> Dict[str, float]:
        """The solve from T0 (Nz, Ny, Nx), or from the last result when None
        (cps_thermal_solve_from: a warm start for design loops)."""
        r = cps.CpsThermalResult()
        T = None if T0 is None else np.ascontiguousarray(T0, dtype=np.float64)
        if T is not None and T.shape != (self.case.Nz, self.case.Ny, self.case.Nx):
            raise ValueError("T0 must be (Nz, Ny, Nx)")
        self._check(self.lib.cps_thermal_solve_from(self.h, cps._dptr(T), ctypes.byref(r)))
        return {"iterations": r.iterations, "converged": bool(r.converged), "rel_residual": r.rel_residual,
                "true_rel_residual": r.true_rel_residual}

    def update(self, gamma=None, u=None, v=None, q0=None) -> None:
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (gamma, u, v, q0)]
        for a in arrs:
            if a is not None and a.shape != self.case.gamma.shape:
                raise ValueError("inputs must be (Ny, Nx)")
        self._check(self.lib.cps_thermal_update(self.h, *[cps._dptr(a) for a in arrs]))

    def temperature(self) -> np.ndarray:
        c = self.case
        T = np.zeros((c.Nz, c.Ny, c.Nx))
        self._check(self.lib.cps_thermal_download(self.h, cps._dptr(T)))
        return T

    def system(self):
        """(planes dict W/E/S/N/B/T/diag, b), each (Nz, Ny, Nx)."""
        c = self.case
        n = c.Nz * c.Ny * c.Nx
        planes = np.zeros(7 * n)
        b = np.zeros(n)
        self._check(self.lib.cps_thermal_system(self.h, cps._dptr(planes), cps._dptr(b)))
        names = ("cW", "cE", "cS", "cN", "cB", "cT", "diag")
        return ({k: planes[p * n:(p + 1) * n].reshape(c.Nz, c.Ny, c.Nx) for p, k in enumerate(names)},
                b.reshape(c.Nz, c.Ny, c.Nx))

    def timing(self, reset: bool = False):
        ms, lv = ctypes.c_double(), ctypes.c_int()
        self._check(self.lib.cps_thermal_timing(self.h, ctypes.byref(ms), ctypes.byref(lv), int(reset)))
        return ms.value, lv.value


def energy_balance(case: ThermalCase, T: np.ndarray) -> Dict[str, float]:
    """The temperature ranges and energy balance the reference prints after
    its solve (thermal_solver.cpp:567-619)."""
    nzs, Nz = case.nz_solid, case.Nz
    fluid = np.zeros(T.shape, dtype=bool)
    fluid[nzs:] = case.gamma > 0.01
    fin = np.ones(T.shape, dtype=bool)
    fin[:nzs] = False
    fin &= ~fluid
    out = {"T_base_min": float(T[:nzs].min()), "T_base_max": float(T[:nzs].max()),
           "T_fluid_min": float(T[fluid].min()) if fluid.any() else 1e30,
           "T_fluid_max": float(T[fluid].max()) if fluid.any() else -1e30,
           "T_fin_min": float(T[fin].min()) if fin.any() else 1e30,
           "T_fin_max": float(T[fin].max()) if fin.any() else -1e30}
    # The sums run in the reference's order, one term after another (cumsum),
    # so that they round as its loops do.
    terms = (case.heat_flux() * case.dx * case.dy).ravel()
    Q_in = float(np.cumsum(terms)[-1]) if terms.size else 0.0
    dz_f = case.H_t / case.nz_fluid
    flows, heats = [], []
    for k in range(nzs, Nz):
        z = (k - nzs + 0.5) * dz_f / case.H_t
        po = 4.0 * z * (1 - z)
        uu = case.u[:, -1] * po
        m = (case.gamma[:, -1] > 0.01) & (uu > 0)
        mflow = case.rho * uu[m] * (case.dy * dz_f)
        flows.append(mflow)
        heats.append(mflow * T[k, m, -1])
    flows, heats = np.concatenate(flows), np.concatenate(heats)
    mdot = float(np.cumsum(flows)[-1]) if flows.size else 0.0
    mdotT = float(np.cumsum(heats)[-1]) if heats.size else 0.0
    T_out = mdotT / mdot if mdot > 0 else case.T_inlet
    Q_out = mdot * case.Cp * (T_out - case.T_inlet)
    out.update(Q_in=Q_in, T_out=T_out, Q_out=Q_out, imbalance=100 * (Q_in - Q_out) / (Q_in + 1e-30))
    return out
