// Runs the reference's own thermal assembly (ThermalSolver3D::solve,
// ThermalSolver/thermal_solver.cpp:420-529; TEST INFRASTRUCTURE ONLY) and
// records the CSR matrix and right-hand side it builds.  The reference file
// includes AMGCL, which is absent, so oracle/Makefile compiles a scratch copy
// (oracle/_ref/thermal_src/, git-ignored) in which two mechanical edits are
// made: the AMGCL #include lines are dropped, and the AMGCL set-up and solve
// (:532-550) are replaced by one call that hands the assembled matrix and
// right-hand side to this harness and stands in for the solve.  Its main() is
// renamed so that this file's main() drives it the way the reference's main()
// does (:706-760).  The temperature is left at T_inlet, or, given a record
// "T" (Nz*Ny*Nx), set to that field by the stand-in solve, so that solve()
// prints the reference's temperature ranges and energy balance for it
// (:567-619); the harness then runs the reference's save_vtk (:622-662),
// which writes thermal_results_3d.vtk to the working directory.
//
//   thermal_asm case.bin out.bin
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

template <class Matrix>
void harness_capture(const Matrix& A, const std::vector<double>& b);
std::vector<double> g_T;  // the field the stand-in solve returns (empty: T stays at T_inlet)
inline std::pair<int, double> harness_solve(std::vector<double>& T) {
  if (!g_T.empty()) T = g_T;
  return {0, 0.0};
}

#define main reference_main
#include "thermal_solver.cpp"
#undef main

namespace {

std::vector<int32_t> g_ptr, g_col;
std::vector<double> g_val, g_b;

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

void put(FILE* o, const char* nm, char t, const void* data, int64_t n) {
  char name[16] = {0};
  std::strncpy(name, nm, 16);
  std::fwrite(name, 1, 16, o);
  std::fwrite(&t, 1, 1, o);
  std::fwrite(&n, 8, 1, o);
  std::fwrite(data, t == 'd' ? 8 : 4, n, o);
}

}  // namespace

template <class Matrix>
void harness_capture(const Matrix& A, const std::vector<double>& b) {
  g_ptr.assign(A.row_ptr.begin(), A.row_ptr.end());
  g_col.assign(A.col_idx.begin(), A.col_idx.end());
  g_val = A.values;
  g_b = b;
}

int main(int argc, char** argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: %s case.bin out.bin\n", argv[0]);
    return 2;
  }
  try {
    auto rec = read_records(argv[1]);
    const std::vector<int32_t>& ip = rec.at("ints").i;
    const std::vector<double>& dp = rec.at("reals").d;
    // ints: Nx Ny nz_solid nz_fluid k_interp_mode; reals: dx dy H_b H_t k_s k_f rho Cp T_inlet qk
    Params p;
    p.Nx = ip[0];
    p.Ny = ip[1];
    p.nz_solid = ip[2];
    p.nz_fluid = ip[3];
    p.k_interp_mode = ip[4];
    p.Lx = p.Nx * dp[0];  // main: p.Lx = cols * dx (thermal_solver.cpp:723)
    p.Ly = p.Ny * dp[1];
    p.H_b = dp[2];
    p.H_t = dp[3];
    p.k_s = dp[4];
    p.k_f = dp[5];
    p.rho = dp[6];
    p.Cp = dp[7];
    p.T_inlet = dp[8];
    p.qk = dp[9];
    ThermalSolver3D s(p);
    s.gamma = rec.at("gamma").d;
    s.u_xy = rec.at("u").d;
    s.v_xy = rec.at("v").d;
    s.q0 = rec.at("q0").d;
    auto t = rec.find("T");
    if (t != rec.end()) {
      if (t->second.d.size() != (size_t)p.n_dofs()) throw std::runtime_error("T record has the wrong size");
      g_T = t->second.d;
    }
    s.solve();
    if (t != rec.end()) s.save_vtk("thermal_results_3d.vtk");
    FILE* o = std::fopen(argv[2], "wb");
    if (!o) throw std::runtime_error("cannot write output");
    put(o, "row_ptr", 'i', g_ptr.data(), (int64_t)g_ptr.size());
    put(o, "col_idx", 'i', g_col.data(), (int64_t)g_col.size());
    put(o, "values", 'd', g_val.data(), (int64_t)g_val.size());
    put(o, "b", 'd', g_b.data(), (int64_t)g_b.size());
    const double dxy[2] = {p.dx(), p.dy()};
    put(o, "dxdy", 'd', dxy, 2);
    std::fclose(o);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "thermal_asm: %s\n", e.what());
    return 1;
  }
  return 0;
}
