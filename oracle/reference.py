"""Runner for the reference solver's own code, compiled from its sources by
oracle/Makefile into oracle/_ref/ref_f32 and oracle/_ref/ref_f64 (TEST
INFRASTRUCTURE ONLY).

Each call runs the harness in a scratch directory (the reference's
constructor reads ExportFiles/ from the working directory) and returns its
records: the per-iteration residual history, the inner iteration counts, the
final fields (row-major, reference index space) and four sampled planes.
"""
from __future__ import annotations

import os
import subprocess
import tempfile
from typing import Dict, Optional

import numpy as np

from . import casefile

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(_HERE, "_ref")


def binary(precision: str) -> str:
    """"f64": the reference promoted to FP64; "f32": as shipped; "dropin": the
    FP64 reference with the B200 drop-in patched into calculateStep (selected
    by pressureSolverType = 5), linked to libcps.so."""
    return os.path.join(REF_DIR, {"f64": "ref_f64", "f32": "ref_f32", "dropin": "ref_dropin"}[precision])


def available(precision: str = "f64") -> bool:
    return os.access(binary(precision), os.X_OK)


def case_records(design, max_outer: int, eps: float = 1e-6, stop_on_conv: bool = False, threads: int = 1,
                 init: Optional[Dict[str, np.ndarray]] = None, mode: int = 0, x_core=(0.01, 0.05)) -> dict:
    rec = {
        "M": [design.M], "N": [design.N], "mode": [mode], "threads": [threads],
        "hx": [design.hx], "hy": [design.hy], "U_in": [design.inletVelocity], "Ht": [design.Ht_channel],
        "rho": [design.rho], "eta": [design.eta], "kmin": [1e-14], "q": [1.0], "conv": [design.convectionScheme], "twoFiveD": [int(design.enableTwoPointFiveD)],
        "convScale": [int(design.enableConvectionScaling)], "sinkMult": [design.twoPointFiveDSinkMultiplier],
        "uvAlpha": [design.uvAlpha], "pAlpha": [design.pAlpha], "pTol": [design.pTol],
        "maxPIter": [design.maxPressureIter], "momTol": [design.momentumTol],
        "maxMomIter": [design.maxMomentumIter], "momType": [int(design.momentumSolverType)],
        "maxOuter": [max_outer], "stopOnConv": [int(stop_on_conv)],
        "eps": [eps], "xCoreIn": [x_core[0]], "xCoreOut": [x_core[1]],
        "alpha": design.alpha, "gamma": design.gamma,
    }
    if init is not None:
        rec["u0"], rec["v0"], rec["p0"] = init["u"], init["v"], init["p"]
    if design.enableInletRamp:
        rec["inletRamp"], rec["rampSteps"] = [1], [int(design.rampSteps)]
    if design.enablePseudoTimeStepping:
        ip, dp = design.int_params(), design.real_params(design.pseudoCFL)
        rec["pseudoI"] = [int(x) for x in ip[8:16]]
        rec["pseudoD"] = [float(x) for x in dp[11:28]]
    return rec


def run(design, max_outer: int, precision: str = "f64", eps: float = 1e-6, stop_on_conv: bool = False,
        threads: int = 1, init: Optional[Dict[str, np.ndarray]] = None, timeout: float = 3600,
        solver_type: int = 5) -> Dict[str, np.ndarray]:
    """Run the reference's calculateStep loop on ``design``; fields come back
    reshaped to the reference's shapes.  With precision "dropin" the steps
    run through the B200 drop-in (pressureSolverType = ``solver_type``: 5
    FP64, 6 mixed precision)."""
    if not available(precision):
        raise FileNotFoundError(f"{binary(precision)} not built (make -C oracle ref REF=<reference checkout>)")
    with tempfile.TemporaryDirectory(prefix="cps_ref_") as tmp:
        cpath, opath = os.path.join(tmp, "case.bin"), os.path.join(tmp, "out.bin")
        rec = case_records(design, max_outer, eps, stop_on_conv, threads, init)
        if precision == "dropin":
            rec["solverType"] = [int(solver_type)]
        casefile.write_records(cpath, rec)
        env = dict(os.environ, OMP_NUM_THREADS=str(threads))
        proc = subprocess.run([binary(precision), cpath, opath], cwd=tmp, env=env, stdout=subprocess.DEVNULL,
                              stderr=subprocess.PIPE, timeout=timeout)
        if proc.returncode != 0:
            raise RuntimeError(f"reference harness failed: {proc.stderr.decode()[-2000:]}")
        out = casefile.read_records(opath)
    M, N = design.M, design.N
    shapes = {"u": (M + 1, N), "v": (M, N + 1), "p": (M + 1, N + 1), "pStar": (M + 1, N + 1),
              "uStar": (M + 1, N), "vStar": (M, N + 1), "dE": (M + 1, N), "dN": (M, N + 1)}
    for k, s in shapes.items():
        out[k] = out[k].reshape(s)
    out["planes"] = out["planes"].reshape(4, 6)
    return out


def run_design_loop(design_a, design_b, n: int, precision: str = "f64", threads: int = 1,
                    solver_type: int = 5, timeout: float = 3600) -> Dict[str, np.ndarray]:
    """Harness mode 4, a design loop in one process: a SIMPLE object runs ``n``
    steps of ``design_a`` from the zero state and is destroyed; a new object,
    constructed in the same storage, runs ``n`` steps of ``design_b``; then its
    alpha and gamma are set to ``design_a``'s and u, v, p to zero in place, and
    it runs ``n`` steps again.  The two designs share the grid and solver
    settings of ``design_a``.  Returns errK, pItersK, uK, vK, pK for the phases
    K = 1, 2, 3.  With precision "dropin" the steps run through the B200
    drop-in (pressureSolverType = ``solver_type``: 5 FP64, 6 mixed)."""
    if not available(precision):
        raise FileNotFoundError(f"{binary(precision)} not built (make -C oracle ref REF=<reference checkout>)")
    if (design_a.M, design_a.N) != (design_b.M, design_b.N):
        raise ValueError("the two designs must share the grid")
    with tempfile.TemporaryDirectory(prefix="cps_ref_") as tmp:
        cpath, opath = os.path.join(tmp, "case.bin"), os.path.join(tmp, "out.bin")
        rec = case_records(design_a, n, 0.0, False, threads, None, mode=4)
        rec["alpha2"], rec["gamma2"] = design_b.alpha, design_b.gamma
        if precision == "dropin":
            rec["solverType"] = [int(solver_type)]
        casefile.write_records(cpath, rec)
        env = dict(os.environ, OMP_NUM_THREADS=str(threads))
        proc = subprocess.run([binary(precision), cpath, opath], cwd=tmp, env=env, stdout=subprocess.DEVNULL,
                              stderr=subprocess.PIPE, timeout=timeout)
        if proc.returncode != 0:
            raise RuntimeError(f"reference harness failed: {proc.stderr.decode()[-2000:]}")
        out = casefile.read_records(opath)
    M, N = design_a.M, design_a.N
    for k in (1, 2, 3):
        out[f"u{k}"] = out[f"u{k}"].reshape(M + 1, N)
        out[f"v{k}"] = out[f"v{k}"].reshape(M, N + 1)
        out[f"p{k}"] = out[f"p{k}"].reshape(M + 1, N + 1)
    return out


def run_iterations(design, max_iterations: int, window: int, percent: float, ramp_steps: int,
                   slope_gate: bool = False, slope_window: int = 0, slope_max_delta: float = 0.0,
                   x_core=(0.01, 0.05), precision: str = "f64", threads: int = 1,
                   timeout: float = 3600) -> Dict[str, np.ndarray]:
    """The reference's own SIMPLE::runIterations (SIMPLE.cpp:237-449) with its
    pressure-drop gate on and the residual test off (epsilon = 0); with
    ``design.enableInletRamp`` its inlet ramp runs over ``ramp_steps`` (the
    one member rampSteps serves both), with ``design.enablePseudoTimeStepping``
    its CFL controllers run after every step.  Returns its
    per-iteration pressure-drop log (``dpIter``; ``dp`` (n, 4): core total,
    full total, core static, full static, as pressure_drop_history.txt prints
    them, 6 significant digits), the final fields and ``logs``: the texts of
    the residuals.txt and pressure_drop_history.txt it wrote."""
    if not available(precision):
        raise FileNotFoundError(f"{binary(precision)} not built (make -C oracle ref REF=<reference checkout>)")
    with tempfile.TemporaryDirectory(prefix="cps_ref_") as tmp:
        cpath, opath = os.path.join(tmp, "case.bin"), os.path.join(tmp, "out.bin")
        rec = case_records(design, max_iterations, 0.0, False, threads, None, mode=2, x_core=x_core)
        rec.update({"dpWindow": [int(window)], "dpPercent": [float(percent)], "dpSlopeGate": [int(slope_gate)],
                    "dpSlopeWindow": [int(slope_window)], "dpSlopeMaxDelta": [float(slope_max_delta)],
                    "rampSteps": [int(ramp_steps)], "inletRamp": [int(design.enableInletRamp)]})
        casefile.write_records(cpath, rec)
        env = dict(os.environ, OMP_NUM_THREADS=str(threads))
        proc = subprocess.run([binary(precision), cpath, opath], cwd=tmp, env=env, stdout=subprocess.DEVNULL,
                              stderr=subprocess.PIPE, timeout=timeout)
        if proc.returncode != 0:
            raise RuntimeError(f"reference harness failed: {proc.stderr.decode()[-2000:]}")
        out = casefile.read_records(opath)
        out["logs"] = {}
        for name in ("residuals.txt", "pressure_drop_history.txt"):
            with open(os.path.join(tmp, "ExportFiles", name), "rb") as f:
                out["logs"][name] = f.read()
    M, N = design.M, design.N
    for k, s in {"u": (M + 1, N), "v": (M, N + 1), "p": (M + 1, N + 1)}.items():
        out[k] = out[k].reshape(s)
    out["dp"] = out["dp"].reshape(-1, 4)
    return out


def run_io(files: Dict[str, str], restart: Optional[Dict[str, str]] = None,
           save: Optional[Dict[str, np.ndarray]] = None, precision: str = "f64", timeout: float = 600) -> dict:
    """The reference's own file handling (harness mode 3): ``files``
    (ExportFiles/fluid_params.txt, geometry_fluid.txt as text) are read by its
    constructor; ``restart`` ({u,v,p}.txt texts) by its restart loader; with
    ``save`` (u, v, p arrays) its saveAll writes ExportFiles.  Returns what it
    read (M, N, buffers, hx, hy, U_in, Ht, cellType, gamma after the wall rows
    of buildAlphaFromDensity, gammaLoaded = as loadDensityField leaves it,
    alpha, u, v, p)
    and ``written``: every file left in ExportFiles, as text."""
    if not available(precision):
        raise FileNotFoundError(f"{binary(precision)} not built (make -C oracle ref REF=<reference checkout>)")
    with tempfile.TemporaryDirectory(prefix="cps_ref_io_") as tmp:
        os.makedirs(os.path.join(tmp, "ExportFiles"))
        for name, text in files.items():
            with open(os.path.join(tmp, "ExportFiles", name), "w") as f:
                f.write(text)
        rec = {"M": [0], "N": [0], "mode": [3], "threads": [1]}
        if restart is not None:
            os.makedirs(os.path.join(tmp, "restart"))
            for name, text in restart.items():
                with open(os.path.join(tmp, "restart", name), "w") as f:
                    f.write(text)
            rec["restart"] = [1]
        if save is not None:
            rec["save"] = [1]
            rec["u0"], rec["v0"], rec["p0"] = save["u"], save["v"], save["p"]
        cpath, opath = os.path.join(tmp, "case.bin"), os.path.join(tmp, "out.bin")
        casefile.write_records(cpath, rec)
        proc = subprocess.run([binary(precision), cpath, opath], cwd=tmp, stdout=subprocess.DEVNULL,
                              stderr=subprocess.PIPE, timeout=timeout, env=dict(os.environ, OMP_NUM_THREADS="1"))
        if proc.returncode != 0:
            raise RuntimeError(f"reference harness failed: {proc.stderr.decode()[-2000:]}")
        out = casefile.read_records(opath)
        written = {}
        for name in sorted(os.listdir(os.path.join(tmp, "ExportFiles"))):
            if name not in files:
                with open(os.path.join(tmp, "ExportFiles", name)) as f:
                    written[name] = f.read()
    M, N, nin, nout = (int(x) for x in out["MN"])
    hx, hy, uin, ht = (float(x) for x in out["params"])
    res = {"M": M, "N": N, "N_in_buffer": nin, "N_out_buffer": nout, "hx": hx, "hy": hy, "U_in": uin, "Ht": ht,
           "written": written}
    for k, shape in {"cellType": (M, N), "gamma": (M, N), "gammaLoaded": (M, N), "alpha": (M, N),
                     "u": (M + 1, N), "v": (M, N + 1), "p": (M + 1, N + 1)}.items():
        res[k] = out[k].reshape(shape)
    return res


def build_alpha(gamma: np.ndarray, kmin: float = 1e-14, q: float = 1.0, precision: str = "f64", eta: float = 0.00089):
    """The reference's own buildAlphaFromDensity (SIMPLE.cpp:589-630) on
    ``gamma`` with alpha_max = eta / kmin (SIMPLE.cpp:65-66); returns (alpha, gamma)."""
    M, N = gamma.shape
    with tempfile.TemporaryDirectory(prefix="cps_ref_") as tmp:
        cpath, opath = os.path.join(tmp, "case.bin"), os.path.join(tmp, "out.bin")
        casefile.write_records(cpath, {"M": [M], "N": [N], "mode": [1], "threads": [1], "hx": [1e-5], "hy": [1e-5],
                                       "U_in": [0.1], "Ht": [0.0], "rho": [997.0], "eta": [eta],
                                       "kmin": [kmin], "q": [q], "gamma": gamma})
        proc = subprocess.run([binary(precision), cpath, opath], cwd=tmp, stdout=subprocess.DEVNULL,
                              stderr=subprocess.PIPE, timeout=600)
        if proc.returncode != 0:
            raise RuntimeError(proc.stderr.decode()[-2000:])
        out = casefile.read_records(opath)
    return out["alpha"].reshape(M, N), out["gamma"].reshape(M, N)


def run_thermal_outputs(T: np.ndarray, gamma: np.ndarray, dx: float, dy: float, nz_solid: int = 2,
                        nz_fluid: int = 7, H_b: float = 0.0005, H_t: float = 0.004, k_s: float = 400.0,
                        k_f: float = 0.6, qk: float = 1.0, timeout: float = 600) -> Dict[str, object]:
    """The reference's thermal output module (ThermalSolver/thermal_output.cpp,
    harness oracle/thermal_out_harness.cpp) on a temperature field T
    (Nz, Ny, Nx) and gamma (Ny, Nx): returns its metrics (with its
    Params::dx(), dy()) and the bytes of the files it writes."""
    path = os.path.join(REF_DIR, "thermal_out")
    if not os.access(path, os.X_OK):
        raise FileNotFoundError(f"{path} not built (make -C oracle ref REF=<reference checkout>)")
    Ny, Nx = gamma.shape
    with tempfile.TemporaryDirectory(prefix="cps_thout_") as tmp:
        cpath, opath = os.path.join(tmp, "case.bin"), os.path.join(tmp, "out.bin")
        outdir = os.path.join(tmp, "out")
        os.mkdir(outdir)
        casefile.write_records(cpath, {"ints": np.array([Nx, Ny, nz_solid, nz_fluid], dtype=np.int32),
                                       "reals": [dx, dy, H_b, H_t, k_s, k_f, qk],
                                       "T": np.ascontiguousarray(T, dtype=np.float64).ravel(),
                                       "gamma": np.ascontiguousarray(gamma, dtype=np.float64).ravel()})
        proc = subprocess.run([path, cpath, opath, outdir], cwd=tmp, stdout=subprocess.DEVNULL,
                              stderr=subprocess.PIPE, timeout=timeout)
        if proc.returncode != 0:
            raise RuntimeError(f"thermal_out failed: {proc.stderr.decode()[-2000:]}")
        vals = casefile.read_records(opath)["metrics"]
        files = {}
        for name in os.listdir(outdir):
            with open(os.path.join(outdir, name), "rb") as f:
                files[name] = f.read()
    keys = ("T_avg_base", "T_avg_fluid", "T_avg_solid", "T_avg_global", "T_std_base", "T_std_fluid", "T_std_global",
            "T_range_base", "T_range_fluid", "T_range_global", "T_uniformity_base", "T_uniformity_global",
            "grad_max", "grad_avg", "grad_max_base", "grad_avg_base", "grad_max_i", "grad_max_j", "grad_max_k",
            "dx", "dy")
    return {"metrics": dict(zip(keys, vals.tolist())), "files": files}


def run_thermal_assembly(Nx: int, Ny: int, dx: float, dy: float, gamma: np.ndarray, u: np.ndarray, v: np.ndarray,
                         q0: np.ndarray, nz_solid: int = 2, nz_fluid: int = 7, H_b: float = 0.0005,
                         H_t: float = 0.004, k_s: float = 400.0, k_f: float = 0.6, rho: float = 998.0,
                         Cp: float = 4180.0, T_inlet: float = 30.0, qk: float = 1.0, k_interp_mode: int = 1,
                         T: Optional[np.ndarray] = None, timeout: float = 600) -> Dict[str, object]:
    """The matrix (CSR) and right-hand side the reference's own
    ThermalSolver3D::solve assembles (harness oracle/thermal_asm_harness.cpp),
    with the reference's Params::dx() = (Nx dx) / Nx.  Given a temperature
    field T (Nz, Ny, Nx), the stand-in solve hands it back as the solution,
    and the result also has the bytes of the thermal_results_3d.vtk the
    reference's save_vtk writes for it ("vtk") and the text its solve printed
    ("stdout": the temperature ranges and the energy balance)."""
    path = os.path.join(REF_DIR, "thermal_asm")
    if not os.access(path, os.X_OK):
        raise FileNotFoundError(f"{path} not built (make -C oracle ref REF=<reference checkout>)")
    with tempfile.TemporaryDirectory(prefix="cps_thasm_") as tmp:
        cpath, opath = os.path.join(tmp, "case.bin"), os.path.join(tmp, "out.bin")
        casefile.write_records(cpath, {
            "ints": np.array([Nx, Ny, nz_solid, nz_fluid, k_interp_mode], dtype=np.int32),
            "reals": [dx, dy, H_b, H_t, k_s, k_f, rho, Cp, T_inlet, qk],
            "gamma": np.ascontiguousarray(gamma, dtype=np.float64).ravel(),
            "u": np.ascontiguousarray(u, dtype=np.float64).ravel(),
            "v": np.ascontiguousarray(v, dtype=np.float64).ravel(),
            "q0": np.ascontiguousarray(q0, dtype=np.float64).ravel(),
            **({} if T is None else {"T": np.ascontiguousarray(T, dtype=np.float64).ravel()})})
        env = dict(os.environ, OMP_NUM_THREADS="1")
        proc = subprocess.run([path, cpath, opath], cwd=tmp, env=env, stdout=subprocess.PIPE,
                              stderr=subprocess.PIPE, timeout=timeout)
        if proc.returncode != 0:
            raise RuntimeError(f"thermal_asm failed: {proc.stderr.decode()[-2000:]}")
        out: Dict[str, object] = dict(casefile.read_records(opath))
        out["stdout"] = proc.stdout.decode(errors="replace")
        if T is not None:
            with open(os.path.join(tmp, "thermal_results_3d.vtk"), "rb") as f:
                out["vtk"] = f.read()
        return out
