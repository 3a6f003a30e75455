"""libcps.so loads, exports every entry point include/*.h declares, its structs
have the layout the ctypes binding assumes, and its host-only functions
(defaults, thermal metrics and files) behave.  No GPU calls."""
import ctypes
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import REPO
from coldplate_solver_b200 import cps

HEADERS = [os.path.join(REPO, "include", f) for f in os.listdir(os.path.join(REPO, "include")) if f.endswith(".h")]


def declared_functions():
    names = []
    for h in HEADERS:
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(cps_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = cps.load_library()
    names = declared_functions()
    assert len(names) >= 10
    for n in names:
        assert hasattr(lib, n), n
        assert n in cps.SIGNATURES, f"{n} has no ctypes signature"
    out = subprocess.run(["nm", "-D", "--defined-only", cps.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (cps_\w+)", out))
    assert set(names) <= exported


def test_struct_layout_matches_c():
    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "cps.h"
#include "cps_thermal.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu\n", sizeof(cps_desc), offsetof(cps_desc, precision), offsetof(cps_desc, alpha),
         offsetof(cps_desc, grid_ctas), sizeof(cps_step_out), offsetof(cps_step_out, vSweeps), sizeof(cps_plane));
  printf("%zu %zu %zu %zu %zu\n", sizeof(cps_batch_opts), offsetof(cps_batch_opts, tiles_per_cta),
         sizeof(cps_dp_monitor), offsetof(cps_dp_monitor, ramp_steps), offsetof(cps_dp_monitor, x_core_out));
  printf("%zu %zu %zu\n", sizeof(cps_case_params), offsetof(cps_case_params, N_in_buffer),
         offsetof(cps_case_params, has_Ht));
  printf("%zu %zu %zu %zu %zu %zu\n", sizeof(cps_thermal_desc), offsetof(cps_thermal_desc, gamma),
         offsetof(cps_thermal_desc, mg_overcorrect), sizeof(cps_thermal_result), sizeof(cps_thermal_metrics),
         offsetof(cps_thermal_metrics, grad_max_k));
  printf("%zu %zu %zu %zu %zu\n", sizeof(cps_pseudo), offsetof(cps_pseudo, target_velocity),
         offsetof(cps_pseudo, ls_resid_increase_tol), sizeof(cps_pseudo_state), offsetof(cps_pseudo_state, ls_backtracks));
  return 0;
}'''
    with tempfile.TemporaryDirectory() as t:
        c, exe = os.path.join(t, "l.c"), os.path.join(t, "l")
        open(c, "w").write(src)
        subprocess.run(["/usr/bin/gcc", "-I", os.path.join(REPO, "include"), c, "-o", exe], check=True)
        vals = list(map(int, subprocess.run([exe], capture_output=True, text=True).stdout.split()))
    py = [ctypes.sizeof(cps.CpsDesc), cps.CpsDesc.precision.offset, cps.CpsDesc.alpha.offset,
          cps.CpsDesc.grid_ctas.offset, ctypes.sizeof(cps.CpsStepOut), cps.CpsStepOut.vSweeps.offset,
          ctypes.sizeof(cps.CpsPlane), ctypes.sizeof(cps.CpsBatchOpts), cps.CpsBatchOpts.tiles_per_cta.offset,
          ctypes.sizeof(cps.CpsDpMonitor), cps.CpsDpMonitor.ramp_steps.offset, cps.CpsDpMonitor.x_core_out.offset,
          ctypes.sizeof(cps.CpsCaseParams), cps.CpsCaseParams.N_in_buffer.offset, cps.CpsCaseParams.has_Ht.offset,
          ctypes.sizeof(cps.CpsThermalDesc), cps.CpsThermalDesc.gamma.offset, cps.CpsThermalDesc.mg_overcorrect.offset,
          ctypes.sizeof(cps.CpsThermalResult), ctypes.sizeof(cps.CpsThermalMetrics),
          cps.CpsThermalMetrics.grad_max_k.offset,
          ctypes.sizeof(cps.CpsPseudo), cps.CpsPseudo.target_velocity.offset,
          cps.CpsPseudo.ls_resid_increase_tol.offset, ctypes.sizeof(cps.CpsPseudoState),
          cps.CpsPseudoState.ls_backtracks.offset]
    assert vals == py


def test_argument_validation_without_gpu():
    lib = cps.load_library()
    from coldplate_solver_b200 import geometry
    d = geometry.straight_channel(M=10, N=12, band=(3, 7))
    desc, keep = cps.make_desc(d)
    out = ctypes.c_ulonglong()
    assert lib.cps_footprint(ctypes.byref(desc), ctypes.byref(out)) == cps.CPS_OK
    assert out.value > 33 * 11 * 32 * 8
    bad, keep2 = cps.make_desc(d)
    bad.M = 2
    assert lib.cps_footprint(ctypes.byref(bad), ctypes.byref(out)) == cps.CPS_ERR_ARG
    assert b"too small" in lib.cps_last_error(None)
    bad.M, bad.hx = 10, -1.0
    assert lib.cps_footprint(ctypes.byref(bad), ctypes.byref(out)) == cps.CPS_ERR_ARG
    assert lib.cps_create(None, None) == cps.CPS_ERR_ARG
    assert lib.cps_step(None, None, None) == cps.CPS_ERR_ARG
    assert lib.cps_barrier_selftest(0, 0, None) == cps.CPS_ERR_ARG
    assert lib.cps_barrier_selftest(0, 1025, None) == cps.CPS_ERR_ARG
    assert b"1..1024" in lib.cps_last_error(None)
    assert lib.cps_version().startswith(b"cps")


def test_host_defaults_match_the_reference_members():
    """cps_pseudo_defaults and cps_thermal_defaults (host code) give the
    reference's member defaults, the same the Python dataclasses carry."""
    from coldplate_solver_b200 import geometry, thermal
    from oracle import thermal as th
    lib = cps.load_library()
    p = cps.CpsPseudo()
    assert lib.cps_pseudo_defaults(ctypes.byref(p), 0.25) == cps.CPS_OK
    d = geometry.straight_channel(M=10, N=12, band=(3, 7)).replace(inletVelocity=0.25)
    ref = cps.pseudo_from_design(d)
    for name, _ in cps.CpsPseudo._fields_:
        if name in ("enable", "time_step"):
            continue
        assert getattr(p, name) == getattr(ref, name), name
    assert p.enable == 0 and p.time_step == 0.0
    t = cps.CpsThermalDesc()
    assert lib.cps_thermal_defaults(ctypes.byref(t)) == cps.CPS_OK
    tp = th.ThermalParams(Nx=1, Ny=1, dx=1.0, dy=1.0)
    tc = thermal.ThermalCase(gamma=np.ones((1, 1)), u=np.zeros((1, 1)), v=np.zeros((1, 1)), dx=1.0, dy=1.0)
    for name in ("nz_solid", "nz_fluid", "H_b", "H_t", "k_s", "k_f", "rho", "Cp", "T_inlet", "rtol", "maxiter",
                 "k_interp_mode", "qk"):
        assert getattr(t, name) == getattr(tp, name) == getattr(tc, name), name


def test_thermal_host_functions_validate(tmp_path):
    lib = cps.load_library()
    d = cps.CpsThermalDesc()
    lib.cps_thermal_defaults(ctypes.byref(d))
    m = cps.CpsThermalMetrics()
    T = np.zeros(9)
    g = np.ones(1)
    assert lib.cps_thermal_compute_metrics(ctypes.byref(d), cps._dptr(T), cps._dptr(g), ctypes.byref(m)) == cps.CPS_ERR_ARG
    d.Nx, d.Ny, d.dx, d.dy = 1, 1, 1e-5, 1e-5
    assert lib.cps_thermal_compute_metrics(ctypes.byref(d), cps._dptr(T), cps._dptr(g), ctypes.byref(m)) == cps.CPS_OK
    assert lib.cps_thermal_save(str(tmp_path / "missing" / "dir").encode(), ctypes.byref(d), cps._dptr(T), cps._dptr(g),
                                cps._dptr(g), cps._dptr(g)) == cps.CPS_ERR_ARG
