// The thermal step's outputs at the boundary (host code of libcps.so): the
// statistics and files the reference's thermal main produces after its solve
// (ThermalSolver/thermal_solver.cpp:622-662, 750-763; thermal_output.cpp).
// Sums run in the reference's loop order and numbers are printed with its
// stream formats, so the values and the files match the reference's own for
// the same temperature field.
#include <algorithm>
#include <cmath>
#include <fstream>
#include <iomanip>
#include <string>
#include <vector>

#include "../../include/cps_thermal.h"

namespace {

struct Grid {
  int Nx, Ny, Nz, nzs;
  double dx, dy;
  std::vector<double> dz;
};

bool make_grid(const cps_thermal_desc* d, Grid& g) {
  if (!d || d->Nx < 1 || d->Ny < 1 || d->nz_solid < 1 || d->nz_fluid < 1 || !(d->dx > 0) || !(d->dy > 0)) return false;
  g.Nx = d->Nx;
  g.Ny = d->Ny;
  g.nzs = d->nz_solid;
  g.Nz = d->nz_solid + d->nz_fluid;
  g.dx = d->dx;
  g.dy = d->dy;
  g.dz.assign(g.Nz, 0.0);
  for (int k = 0; k < d->nz_solid; ++k) g.dz[k] = d->H_b / d->nz_solid;  // thermal_solver.cpp:237-239
  for (int k = 0; k < d->nz_fluid; ++k) g.dz[d->nz_solid + k] = d->H_t / d->nz_fluid;
  return true;
}

// compute_gradient_components (thermal_output.cpp:64-105): central
// differences inside, one-sided at the faces, the mean spacing in z.
void gradient(const Grid& g, const double* T, int i, int j, int k, double& gx, double& gy, double& gz) {
  const int Nx = g.Nx, Ny = g.Ny, Nz = g.Nz;
  const int P = k * Nx * Ny + j * Nx + i;
  if (i == 0) gx = (T[P + 1] - T[P]) / g.dx;
  else if (i == Nx - 1) gx = (T[P] - T[P - 1]) / g.dx;
  else gx = (T[P + 1] - T[P - 1]) / (2.0 * g.dx);
  if (j == 0) gy = (T[P + Nx] - T[P]) / g.dy;
  else if (j == Ny - 1) gy = (T[P] - T[P - Nx]) / g.dy;
  else gy = (T[P + Nx] - T[P - Nx]) / (2.0 * g.dy);
  const int top = P + Nx * Ny, bot = P - Nx * Ny;
  if (k == 0) gz = (T[top] - T[P]) / g.dz[0];
  else if (k == Nz - 1) gz = (T[P] - T[bot]) / g.dz[Nz - 1];
  else {
    const double dz_avg = 0.5 * (g.dz[k - 1] + g.dz[k]);
    gz = (T[top] - T[bot]) / (2.0 * dz_avg);
  }
}

void metrics(const Grid& g, const double* T, const double* gamma, cps_thermal_metrics& m) {
  m = cps_thermal_metrics{};
  const int Nx = g.Nx, Ny = g.Ny, Nz = g.Nz;
  double sTb = 0, sVb = 0, sTf = 0, sVf = 0, sTs = 0, sVs = 0, sTg = 0, sVg = 0;
  double minb = 1e30, maxb = -1e30, minf = 1e30, maxf = -1e30, ming = 1e30, maxg = -1e30;
  // volume-weighted sums and ranges (thermal_output.cpp:146-202)
  for (int k = 0; k < Nz; ++k) {
    const double V = g.dx * g.dy * g.dz[k];
    for (int j = 0; j < Ny; ++j)
      for (int i = 0; i < Nx; ++i) {
        const double t = T[k * Nx * Ny + j * Nx + i], TV = t * V;
        sTg += TV;
        sVg += V;
        ming = std::min(ming, t);
        maxg = std::max(maxg, t);
        if (k < g.nzs) {
          sTb += TV;
          sVb += V;
          minb = std::min(minb, t);
          maxb = std::max(maxb, t);
        } else if (gamma[j * Nx + i] > 0.01) {
          sTf += TV;
          sVf += V;
          minf = std::min(minf, t);
          maxf = std::max(maxf, t);
        } else {
          sTs += TV;
          sVs += V;
        }
      }
  }
  m.T_avg_base = sVb > 0 ? sTb / sVb : 0.0;
  m.T_avg_fluid = sVf > 0 ? sTf / sVf : 0.0;
  m.T_avg_solid = sVs > 0 ? sTs / sVs : 0.0;
  m.T_avg_global = sVg > 0 ? sTg / sVg : 0.0;
  m.T_range_base = sVb > 0 ? maxb - minb : 0.0;
  m.T_range_fluid = sVf > 0 ? maxf - minf : 0.0;
  m.T_range_global = sVg > 0 ? maxg - ming : 0.0;
  // volume-weighted variances (:207-245)
  double vb = 0, vf = 0, vg = 0;
  for (int k = 0; k < Nz; ++k) {
    const double V = g.dx * g.dy * g.dz[k];
    for (int j = 0; j < Ny; ++j)
      for (int i = 0; i < Nx; ++i) {
        const double t = T[k * Nx * Ny + j * Nx + i];
        const double dg = t - m.T_avg_global;
        vg += V * dg * dg;
        if (k < g.nzs) {
          const double db = t - m.T_avg_base;
          vb += V * db * db;
        } else if (gamma[j * Nx + i] > 0.01) {
          const double df = t - m.T_avg_fluid;
          vf += V * df * df;
        }
      }
  }
  m.T_std_base = std::sqrt(sVb > 0 ? vb / sVb : 0.0);
  m.T_std_fluid = std::sqrt(sVf > 0 ? vf / sVf : 0.0);
  m.T_std_global = std::sqrt(sVg > 0 ? vg / sVg : 0.0);
  auto uniformity = [](double sd, double avg) {
    if (avg <= 0.0) return 0.0;
    return std::max(0.0, std::min(1.0, 1.0 - (sd / avg)));
  };
  m.T_uniformity_base = uniformity(m.T_std_base, m.T_avg_base);
  m.T_uniformity_global = uniformity(m.T_std_global, m.T_avg_global);
  // gradient statistics (:262-307)
  m.grad_max = -1e30;
  m.grad_max_base = -1e30;
  double sgg = 0, sgb = 0;
  for (int k = 0; k < Nz; ++k) {
    const double V = g.dx * g.dy * g.dz[k];
    for (int j = 0; j < Ny; ++j)
      for (int i = 0; i < Nx; ++i) {
        double gx, gy, gz;
        gradient(g, T, i, j, k, gx, gy, gz);
        const double mag = std::sqrt(gx * gx + gy * gy + gz * gz);
        sgg += mag * V;
        if (mag > m.grad_max) {
          m.grad_max = mag;
          m.grad_max_i = i;
          m.grad_max_j = j;
          m.grad_max_k = k;
        }
        if (k < g.nzs) {
          sgb += mag * V;
          if (mag > m.grad_max_base) m.grad_max_base = mag;
        }
      }
  }
  m.grad_avg = sVg > 0 ? sgg / sVg : 0.0;
  m.grad_avg_base = sVb > 0 ? sgb / sVb : 0.0;
}

// kval (thermal_solver.cpp:283-312)
double kval(const cps_thermal_desc* d, const double* gamma, int i, int j, int k) {
  if (k < d->nz_solid) return d->k_s;
  double g = std::max(0.0, std::min(1.0, gamma[j * d->Nx + i]));
  if (d->k_interp_mode == 1) return d->k_f + (d->k_s - d->k_f) * (1.0 - g) / (1.0 + d->qk * g);
  if (d->k_interp_mode == 2) return d->k_s * d->k_f / ((1.0 - g) * d->k_f + g * d->k_s + 1e-30);
  return d->k_s * (1.0 - g) + d->k_f * g;
}

void coordinates(std::ofstream& f, const Grid& g) {
  f << "X_COORDINATES " << g.Nx + 1 << " double\n";
  for (int i = 0; i <= g.Nx; ++i) f << i * g.dx << " ";
  f << "\n";
  f << "Y_COORDINATES " << g.Ny + 1 << " double\n";
  for (int j = 0; j <= g.Ny; ++j) f << j * g.dy << " ";
  f << "\n";
  f << "Z_COORDINATES " << g.Nz + 1 << " double\n";
  double z = 0;
  for (int k = 0; k <= g.Nz; ++k) {
    f << z << " ";
    if (k < g.Nz) z += g.dz[k];
  }
  f << "\n";
}

}  // namespace

extern "C" {

cps_status cps_thermal_compute_metrics(const cps_thermal_desc* d, const double* T, const double* gamma,
                                       cps_thermal_metrics* out) {
  Grid g;
  if (!make_grid(d, g) || !T || !gamma || !out) return CPS_ERR_ARG;
  metrics(g, T, gamma, *out);
  return CPS_OK;
}

cps_status cps_thermal_save(const char* dir, const cps_thermal_desc* d, const double* T, const double* gamma,
                            const double* u, const double* v) {
  Grid g;
  if (!dir || !make_grid(d, g) || !T || !gamma || !u || !v) return CPS_ERR_ARG;
  const std::string base(dir);
  const int Nx = g.Nx, Ny = g.Ny, Nz = g.Nz;
  auto region = [&](int i, int j, int k) { return k < g.nzs ? 0 : (gamma[j * Nx + i] > 0.01 ? 1 : 0); };
  {
    // ThermalSolver3D::save_vtk (thermal_solver.cpp:622-662) with the velocity
    // field of :550-564 (the 2-D velocity times the z profile in the fluid)
    std::ofstream f(base + "/thermal_results_3d.vtk");
    if (!f) return CPS_ERR_ARG;
    f << "# vtk DataFile Version 3.0\nThermal3D\nASCII\nDATASET RECTILINEAR_GRID\n";
    f << "DIMENSIONS " << Nx + 1 << " " << Ny + 1 << " " << Nz + 1 << "\n";
    coordinates(f, g);
    f << "CELL_DATA " << Nx * Ny * Nz << "\n";
    f << "SCALARS Temperature double 1\nLOOKUP_TABLE default\n";
    for (int k = 0; k < Nz; ++k)
      for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i) f << T[k * Nx * Ny + j * Nx + i] << "\n";
    f << "SCALARS Region int 1\nLOOKUP_TABLE default\n";
    for (int k = 0; k < Nz; ++k)
      for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i) f << region(i, j, k) << "\n";
    f << "SCALARS Density double 1\nLOOKUP_TABLE default\n";
    for (int k = 0; k < Nz; ++k)
      for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i) {
          if (k < g.nzs) f << "0\n";
          else f << gamma[j * Nx + i] << "\n";
        }
    f << "SCALARS ThermalConductivity double 1\nLOOKUP_TABLE default\n";
    for (int k = 0; k < Nz; ++k)
      for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i) f << kval(d, gamma, i, j, k) << "\n";
    f << "VECTORS Velocity double\n";
    for (int k = 0; k < Nz; ++k) {
      double po = 0;
      if (k >= g.nzs) {  // pois (thermal_solver.cpp:336-340)
        const double zz = (k - g.nzs + 0.5) * (d->H_t / d->nz_fluid) / d->H_t;
        po = 4.0 * zz * (1 - zz);
      }
      for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i) {
          double U = 0, V = 0;
          if (region(i, j, k) == 1) {
            U = u[j * Nx + i] * po;
            V = v[j * Nx + i] * po;
          }
          f << U << " " << V << " " << 0.0 << "\n";
        }
    }
    if (!f) return CPS_ERR_ARG;
  }
  {
    // save_thermal_metrics (thermal_output.cpp:326-371)
    cps_thermal_metrics m;
    metrics(g, T, gamma, m);
    std::ofstream f(base + "/thermal_metrics.txt");
    if (!f) return CPS_ERR_ARG;
    f << std::fixed << std::setprecision(4);
    f << "# Thermal Metrics - Volume-Weighted Statistics" << std::endl;
    f << "# All temperatures in [C]" << std::endl;
    f << "#" << std::endl;
    f << "# Average Temperatures" << std::endl;
    f << "T_avg_base    " << m.T_avg_base << std::endl;
    f << "T_avg_fluid   " << m.T_avg_fluid << std::endl;
    f << "T_avg_solid   " << m.T_avg_solid << std::endl;
    f << "T_avg_global  " << m.T_avg_global << std::endl;
    f << "#" << std::endl;
    f << "# Standard Deviations" << std::endl;
    f << "T_std_base    " << m.T_std_base << std::endl;
    f << "T_std_fluid   " << m.T_std_fluid << std::endl;
    f << "T_std_global  " << m.T_std_global << std::endl;
    f << "#" << std::endl;
    f << "# Temperature Ranges (max - min)" << std::endl;
    f << "T_range_base  " << m.T_range_base << std::endl;
    f << "T_range_fluid " << m.T_range_fluid << std::endl;
    f << "T_range_global" << m.T_range_global << std::endl;
    f << "#" << std::endl;
    f << "# Uniformity Indices (1 = uniform, 0 = non-uniform)" << std::endl;
    f << "T_uniformity_base   " << m.T_uniformity_base << std::endl;
    f << "T_uniformity_global " << m.T_uniformity_global << std::endl;
    f << "#" << std::endl;
    f << "# Thermal Gradients [C/m]" << std::endl;
    f << "grad_max          " << m.grad_max << std::endl;
    f << "grad_avg          " << m.grad_avg << std::endl;
    f << "grad_max_base     " << m.grad_max_base << std::endl;
    f << "grad_avg_base     " << m.grad_avg_base << std::endl;
    f << "grad_max_loc      " << m.grad_max_i << " " << m.grad_max_j << " " << m.grad_max_k << std::endl;
    if (!f) return CPS_ERR_ARG;
  }
  {
    // save_k_field (thermal_output.cpp:530-568): the RAMP conductivity of the channel region
    std::ofstream f(base + "/k_thermal.txt");
    if (!f) return CPS_ERR_ARG;
    f << std::fixed << std::setprecision(6);
    for (int j = 0; j < Ny; ++j) {
      for (int i = 0; i < Nx; ++i) {
        const double gg = std::max(0.0, std::min(1.0, gamma[j * Nx + i]));
        const double num = 1.0 - gg, den = 1.0 + d->qk * gg;
        f << d->k_f + (d->k_s - d->k_f) * num / den;
        if (i < Nx - 1) f << "\t";
      }
      f << "\n";
    }
    if (!f) return CPS_ERR_ARG;
  }
  {
    // compute_gradient_field + save_gradient_vtk (thermal_output.cpp:411-524)
    std::ofstream f(base + "/thermal_gradient_3d.vtk");
    if (!f) return CPS_ERR_ARG;
    f << "# vtk DataFile Version 3.0\n";
    f << "Thermal Gradient Field\n";
    f << "ASCII\n";
    f << "DATASET RECTILINEAR_GRID\n";
    f << "DIMENSIONS " << Nx + 1 << " " << Ny + 1 << " " << Nz + 1 << "\n";
    coordinates(f, g);
    f << "CELL_DATA " << Nx * Ny * Nz << "\n";
    std::vector<double> mag((size_t)Nx * Ny * Nz);
    f << "VECTORS TemperatureGradient double\n";
    for (int k = 0; k < Nz; ++k)
      for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i) {
          double gx, gy, gz;
          gradient(g, T, i, j, k, gx, gy, gz);
          mag[(size_t)k * Nx * Ny + j * Nx + i] = std::sqrt(gx * gx + gy * gy + gz * gz);
          f << gx << " " << gy << " " << gz << "\n";
        }
    f << "SCALARS GradientMagnitude double 1\n";
    f << "LOOKUP_TABLE default\n";
    for (size_t P = 0; P < mag.size(); ++P) f << mag[P] << "\n";
    if (!f) return CPS_ERR_ARG;
  }
  return CPS_OK;
}

}  // extern "C"
