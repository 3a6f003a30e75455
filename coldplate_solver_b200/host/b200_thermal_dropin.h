// Drop-in for the thermal step's linear solve: ThermalSolver3D::solve
// (ThermalSolver/thermal_solver.cpp:420-562) assembles the 7-point CHT system
// and hands it to AMGCL (IDR(s) + smoothed aggregation, :532-550).  The patched
// build replaces that block with
//
//   auto t2 = chrono::high_resolution_clock::now();
//   auto [iters, res] = b200ThermalSolve(p, gamma, u_xy, v_xy, q0, T);
//
// which assembles the same system on the GPU from the same members (Params p,
// the 2-D gamma / u_xy / v_xy / q0 and the temperature vector T) and solves it
// to p.rtol (BiCGStab with structured aggregation multigrid), leaving the
// solution in T and returning {iterations, relative residual} as the AMGCL
// call does.  Everything after the block (the 3-D velocity field, the energy
// balance, the output files) is unchanged.  Errors of the C ABI are thrown as
// std::runtime_error with the library's message.
#pragma once

#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "cps_thermal.h"

template <class Params>
std::pair<int, double> b200ThermalSolve(const Params& p, const std::vector<double>& gamma,
                                        const std::vector<double>& u_xy, const std::vector<double>& v_xy,
                                        const std::vector<double>& q0, std::vector<double>& T) {
  cps_thermal_desc td;
  cps_thermal_defaults(&td);
  td.Nx = p.Nx;
  td.Ny = p.Ny;
  td.dx = p.dx();
  td.dy = p.dy();
  td.nz_solid = p.nz_solid;
  td.nz_fluid = p.nz_fluid;
  td.H_b = p.H_b;
  td.H_t = p.H_t;
  td.k_s = p.k_s;
  td.k_f = p.k_f;
  td.rho = p.rho;
  td.Cp = p.Cp;
  td.T_inlet = p.T_inlet;
  td.rtol = p.rtol;
  td.maxiter = p.maxiter;
  td.k_interp_mode = p.k_interp_mode;
  td.qk = p.qk;
  const size_t n2 = (size_t)p.Nx * p.Ny;
  if (gamma.size() != n2 || u_xy.size() != n2 || v_xy.size() != n2 || q0.size() != n2)
    throw std::runtime_error("b200ThermalSolve: gamma, u_xy, v_xy and q0 need Nx * Ny entries");
  td.gamma = gamma.data();
  td.u = u_xy.data();
  td.v = v_xy.data();
  td.q0 = q0.data();
  T.resize(n2 * (size_t)(p.nz_solid + p.nz_fluid));
  cps_thermal* th = nullptr;
  cps_thermal_result r{};
  if (cps_thermal_create(&td, &th) != CPS_OK) throw std::runtime_error(cps_thermal_last_error(nullptr));
  if (cps_thermal_solve(th, &r) != CPS_OK || cps_thermal_download(th, T.data()) != CPS_OK) {
    const std::string msg = cps_thermal_last_error(th);
    cps_thermal_destroy(th);
    throw std::runtime_error(msg);
  }
  cps_thermal_destroy(th);
  return {r.iterations, r.rel_residual};
}
