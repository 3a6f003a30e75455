// Runs the reference's thermal output module (ThermalSolver/thermal_output.cpp,
// compiled where it lies; TEST INFRASTRUCTURE ONLY) on a given temperature
// field: compute_thermal_metrics, save_thermal_metrics, save_k_field,
// compute_gradient_field + save_gradient_vtk.  The module expects the Params
// type of thermal_solver.cpp, which cannot be compiled here (it needs AMGCL);
// the stand-in below carries the members the module reads, with the same
// meaning (dx() = Lx / Nx as in the reference's main, thermal_solver.cpp:723).
//
//   thermal_out case.bin out.bin outdir
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

using namespace std;

struct Params {
  int Nx = 0, Ny = 0, nz_solid = 2, nz_fluid = 7;
  double Lx = 0, Ly = 0, H_b = 0.0005, H_t = 0.004;
  double k_s = 400.0, k_f = 0.6, qk = 1.0;
  int k_interp_mode = 1;
  double dx() const { return Lx / Nx; }
  double dy() const { return Ly / Ny; }
  double dz_s() const { return H_b / nz_solid; }
  double dz_f() const { return H_t / nz_fluid; }
  int Nz() const { return nz_solid + nz_fluid; }
};

#include "ThermalSolver/thermal_output.cpp"

namespace {

struct Rec {
  std::vector<double> d;
  std::vector<int32_t> i;
};

std::map<std::string, Rec> read_records(const char* path) {
  std::map<std::string, Rec> out;
  FILE* f = std::fopen(path, "rb");
  if (!f) throw std::runtime_error("cannot open case file");
  char name[17] = {0};
  while (std::fread(name, 1, 16, f) == 16) {
    char t;
    int64_t n;
    if (std::fread(&t, 1, 1, f) != 1 || std::fread(&n, 8, 1, f) != 1) break;
    Rec& r = out[std::string(name, strnlen(name, 16))];
    if (t == 'd') {
      r.d.resize(n);
      if (std::fread(r.d.data(), 8, n, f) != (size_t)n) throw std::runtime_error("short record");
    } else {
      r.i.resize(n);
      if (std::fread(r.i.data(), 4, n, f) != (size_t)n) throw std::runtime_error("short record");
    }
    std::memset(name, 0, sizeof name);
  }
  std::fclose(f);
  return out;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 4) {
    std::fprintf(stderr, "usage: %s case.bin out.bin outdir\n", argv[0]);
    return 2;
  }
  try {
    auto rec = read_records(argv[1]);
    const std::vector<int32_t>& ip = rec.at("ints").i;      // Nx Ny nz_solid nz_fluid
    const std::vector<double>& dp = rec.at("reals").d;      // dx dy H_b H_t k_s k_f qk
    Params p;
    p.Nx = ip[0];
    p.Ny = ip[1];
    p.nz_solid = ip[2];
    p.nz_fluid = ip[3];
    p.Lx = p.Nx * dp[0];  // main: p.Lx = cols * dx (thermal_solver.cpp:723)
    p.Ly = p.Ny * dp[1];
    p.H_b = dp[2];
    p.H_t = dp[3];
    p.k_s = dp[4];
    p.k_f = dp[5];
    p.qk = dp[6];
    std::vector<double> dz(p.Nz());  // ThermalSolver3D constructor (thermal_solver.cpp:237-239)
    for (int k = 0; k < p.nz_solid; k++) dz[k] = p.dz_s();
    for (int k = 0; k < p.nz_fluid; k++) dz[p.nz_solid + k] = p.dz_f();
    const std::vector<double>& T = rec.at("T").d;
    const std::vector<double>& gamma = rec.at("gamma").d;
    ThermalMetrics m = compute_thermal_metrics(T, gamma, dz, p);
    save_thermal_metrics(m, argv[3]);
    save_k_field(gamma, p, argv[3]);
    GradientField grad = compute_gradient_field(T, dz, p);
    save_gradient_vtk(grad, dz, p, std::string(argv[3]) + "/thermal_gradient_3d.vtk");
    FILE* o = std::fopen(argv[2], "wb");
    const double vals[] = {m.T_avg_base, m.T_avg_fluid, m.T_avg_solid, m.T_avg_global, m.T_std_base,
                           m.T_std_fluid, m.T_std_global, m.T_range_base, m.T_range_fluid, m.T_range_global,
                           m.T_uniformity_base, m.T_uniformity_global, m.grad_max, m.grad_avg, m.grad_max_base,
                           m.grad_avg_base, (double)m.grad_max_i, (double)m.grad_max_j, (double)m.grad_max_k,
                           p.dx(), p.dy()};
    char name[16] = {0};
    std::strncpy(name, "metrics", 16);
    const char t = 'd';
    const int64_t n = sizeof(vals) / sizeof(double);
    std::fwrite(name, 1, 16, o);
    std::fwrite(&t, 1, 1, o);
    std::fwrite(&n, 8, 1, o);
    std::fwrite(vals, 8, n, o);
    std::fclose(o);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "thermal_out: %s\n", e.what());
    return 1;
  }
  return 0;
}
