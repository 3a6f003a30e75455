/*
 * cps_thermal.h -- C ABI of the B200 3-D conjugate-heat-transfer solve
 * (libcps.so), the step downstream of the flow solve.
 *
 * Replaces ThermalSolver3D::solve (ThermalSolver/thermal_solver.cpp:420-560):
 * the same finite-volume system (7-point stencil on Nx x Ny x Nz cells,
 * nz_solid base-plate layers under nz_fluid channel layers, upwind advection
 * with the parabolic z-profile of the 2-D velocity, RAMP/harmonic/linear
 * conductivity of gamma, fixed inlet temperature, base heat flux), assembled
 * on the device and solved there by BiCGStab preconditioned with a
 * structured aggregation multigrid V-cycle, where the reference builds a CSR
 * matrix on the host and hands it to AMGCL (smoothed-aggregation AMG +
 * IDR(s), :533-545).  Stop rule: ||b - A T||_2 <= rtol ||b||_2 from
 * T = T_inlet, as the reference's solver call (:548).
 *
 * Index space: T[k][j][i], P = k*Nx*Ny + j*Nx + i (thermal_solver.cpp:241);
 * 2-D inputs are Ny x Nx row-major (row j = y), gamma = 1 fluid, 0 solid
 * (:740-746: the reference inverts geometry_thermal.txt to this convention).
 */
#ifndef CPS_THERMAL_H
#define CPS_THERMAL_H

#include "cps.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int Nx, Ny;              /* cells in x (columns) and y (rows) */
  int nz_solid, nz_fluid;  /* Params::nz_solid, nz_fluid (thermal_solver.cpp:150-151) */
  double dx, dy;           /* Params::dx(), dy() = Lx/Nx, Ly/Ny [m] */
  double H_b, H_t;         /* base plate thickness, channel height [m] */
  double k_s, k_f;         /* solid and fluid conductivity [W/m-K] */
  double rho, Cp;          /* fluid density [kg/m^3], heat capacity [J/kg-K] */
  double T_inlet;          /* inlet temperature [C] */
  double rtol;             /* relative residual of the stop rule */
  int maxiter;             /* Krylov iterations at most */
  int k_interp_mode;       /* 0 linear, 1 RAMP, 2 harmonic (thermal_solver.cpp:283-312) */
  double qk;               /* RAMP parameter */
  const double* gamma;     /* host Ny x Nx, 1 = fluid */
  const double* u;         /* host Ny x Nx cell-centred x velocity (u_thermal.txt) [m/s] */
  const double* v;         /* host Ny x Nx cell-centred y velocity (v_thermal.txt) [m/s] */
  const double* q0;        /* host Ny x Nx base heat flux [W/m^2], or NULL for q everywhere */
  double q;                /* uniform base heat flux when q0 == NULL (thermal_params.txt) */
  int device;              /* CUDA device ordinal */
  int mg_sweeps;           /* damped-Jacobi sweeps before and after each coarse correction (0: 2) */
  double mg_omega;         /* Jacobi damping (0: 0.8) */
  double mg_overcorrect;   /* scale of the coarse correction (0: 1.7) */
} cps_thermal_desc;

typedef struct cps_thermal cps_thermal;

typedef struct {
  int iterations;           /* BiCGStab iterations run */
  int converged;            /* the stop rule was met */
  double rel_residual;      /* ||r||/||b|| of the recurrence at the stop */
  double true_rel_residual; /* ||b - A T||/||b|| recomputed from T */
} cps_thermal_result;

/* The reference's defaults (Params, thermal_solver.cpp:147-193). */
cps_status cps_thermal_defaults(cps_thermal_desc* d);

/* Allocate the device state, upload the inputs and assemble the system and
 * the multigrid hierarchy. */
cps_status cps_thermal_create(const cps_thermal_desc* d, cps_thermal** out);

/* New gamma / u / v / q0 (any may be NULL to keep) for the same grid:
 * reassembles the system and the hierarchy. */
cps_status cps_thermal_update(cps_thermal* t, const double* gamma, const double* u, const double* v,
                              const double* q0);

/* Solve from T = T_inlet (thermal_solver.cpp:425); *res may be NULL. */
cps_status cps_thermal_solve(cps_thermal* t, cps_thermal_result* res);

/* The same solve from a given temperature field (Nz x Ny x Nx; NULL: the
 * handle's current one, i.e. the last solve's result): a warm start for a
 * design loop whose successive designs differ little.  No counterpart in the
 * reference, which starts every solve from T_inlet. */
cps_status cps_thermal_solve_from(cps_thermal* t, const double* T0, cps_thermal_result* res);

/* Temperature, Nz x Ny x Nx doubles. */
cps_status cps_thermal_download(cps_thermal* t, double* T);

/* The assembled system: planes = 7 x (Nz*Ny*Nx) doubles in the order W, E,
 * S, N, B (k-1), T (k+1), diagonal (each off-diagonal the merged CSR entry of
 * SparseMatrix::from_coo, 0 where the reference has none); b = Nz*Ny*Nx
 * doubles.  Either may be NULL. */
cps_status cps_thermal_system(cps_thermal* t, double* planes, double* b);

/* Device time of the solve launches since the last reset, CUDA events on the
 * launching stream; *levels = multigrid levels. */
cps_status cps_thermal_timing(cps_thermal* t, double* kernel_ms, int* levels, int reset);

/* The statistics ThermalMetrics holds (thermal_output.cpp:14-42, computed as
 * compute_thermal_metrics does, :135-320: volume-weighted over the base plate
 * k < nz_solid, the fluid gamma > 0.01 and the solid fins above the base). */
typedef struct {
  double T_avg_base, T_avg_fluid, T_avg_solid, T_avg_global;
  double T_std_base, T_std_fluid, T_std_global;
  double T_range_base, T_range_fluid, T_range_global;
  double T_uniformity_base, T_uniformity_global;
  double grad_max, grad_avg, grad_max_base, grad_avg_base;
  int grad_max_i, grad_max_j, grad_max_k, pad;
} cps_thermal_metrics;

/* Host code, no GPU.  d supplies the grid (Nx, Ny, nz_solid, nz_fluid, dx,
 * dy, H_b, H_t); T is Nz x Ny x Nx, gamma Ny x Nx (1 = fluid). */
cps_status cps_thermal_compute_metrics(const cps_thermal_desc* d, const double* T, const double* gamma,
                                       cps_thermal_metrics* out);

/* The files the reference's thermal main writes after its solve
 * (thermal_solver.cpp:750-763) into directory dir, with the reference's
 * number formats: thermal_results_3d.vtk (ThermalSolver3D::save_vtk, :622-662;
 * needs u and v, Ny x Nx, and d's conductivity settings), thermal_metrics.txt
 * (save_thermal_metrics, thermal_output.cpp:326-371), k_thermal.txt
 * (save_k_field, :530-568) and thermal_gradient_3d.vtk
 * (compute_gradient_field + save_gradient_vtk, :411-524). */
cps_status cps_thermal_save(const char* dir, const cps_thermal_desc* d, const double* T, const double* gamma,
                            const double* u, const double* v);

void cps_thermal_destroy(cps_thermal* t);
const char* cps_thermal_last_error(const cps_thermal* t);

#ifdef __cplusplus
}
#endif

#endif /* CPS_THERMAL_H */
