// The reference's file formats at the drop-in boundary (host code of
// libcps.so): the case files a geometry export writes (fluid_params.txt,
// geometry_fluid.txt; SIMPLE.cpp:31-47, 517-584), the restart matrices
// u/v/p.txt (SIMPLE.cpp:203-232) and the output of saveAll (output.cpp:47-266:
// staggered and cell-centred text matrices, the thermal crop, the VTK file).
// Numbers are printed with the stream defaults the reference uses (six
// significant digits), so a file written here is byte-identical to the one
// the reference writes from the same values.
#include <algorithm>
#include <cmath>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/cps.h"

namespace {

thread_local std::string g_io_error;

cps_status io_fail(cps_status s, const std::string& m) {
  g_io_error = m;
  return s;
}

// Element (i, j) of a rows x cols host matrix in either layout.
inline double at(const double* a, int rows, int cols, int i, int j, int layout) {
  return layout == CPS_COL_MAJOR ? a[(size_t)j * rows + i] : a[(size_t)i * cols + j];
}

// Matrix of doubles, row-major, as the reference's Eigen temporaries.
struct Mat {
  int rows, cols;
  std::vector<double> a;
  Mat(int r, int c) : rows(r), cols(c), a((size_t)r * c, 0.0) {}
  double& operator()(int i, int j) { return a[(size_t)i * cols + j]; }
  double operator()(int i, int j) const { return a[(size_t)i * cols + j]; }
};

// saveMatrix (output.cpp:47-67): tab-separated rows.
bool save_matrix(const std::string& dir, const std::string& name, const Mat& m) {
  std::ofstream out(dir + "/" + name + ".txt");
  if (!out.is_open()) return false;
  for (int i = 0; i < m.rows; ++i) {
    for (int j = 0; j < m.cols; ++j) {
      out << m(i, j);
      if (j < m.cols - 1) out << "\t";
    }
    out << "\n";
  }
  return static_cast<bool>(out);
}

Mat from_host(const double* src, int rows, int cols, int layout) {
  Mat m(rows, cols);
  for (int i = 0; i < rows; ++i)
    for (int j = 0; j < cols; ++j) m(i, j) = at(src, rows, cols, i, j, layout);
  return m;
}

}  // namespace

extern "C" {

const char* cps_io_last_error(void) { return g_io_error.c_str(); }

cps_status cps_read_case_params(const char* path, cps_case_params* out) {
  if (!path || !out) return io_fail(CPS_ERR_ARG, "path and out are required");
  std::ifstream in(path);
  if (!in) return io_fail(CPS_ERR_ARG, std::string("could not open ") + path);
  cps_case_params p{};
  // loadParameters (SIMPLE.cpp:31-47): M N hy hx U_in N_in_buffer N_out_buffer [Ht [rho nu]]
  if (!(in >> p.M >> p.N >> p.hy >> p.hx >> p.U_in >> p.N_in_buffer >> p.N_out_buffer))
    return io_fail(CPS_ERR_ARG, std::string("invalid parameter file format: ") + path);
  double ht = 0.0;
  if (in >> ht) {
    p.Ht = ht;
    p.has_Ht = 1;
  }
  *out = p;
  return CPS_OK;
}

cps_status cps_read_geometry(const char* path, int M, int N, double* cellType, double* gamma, int* values_read) {
  if (!path || M <= 0 || N <= 0 || (!cellType && !gamma)) return io_fail(CPS_ERR_ARG, "bad arguments");
  // loadTopology (SIMPLE.cpp:517-551): cellType defaults to 0 (fluid); a
  // missing file leaves all fluid and a short file stops at its end.
  std::vector<double> ct((size_t)M * N, 0.0);
  int n = 0;
  std::ifstream in(path);
  const bool opened = static_cast<bool>(in);
  if (opened) {
    for (int i = 0; i < M && n == i * N; ++i)
      for (int j = 0; j < N; ++j) {
        double val;
        if (!(in >> val)) break;
        ct[(size_t)i * N + j] = val;
        ++n;
      }
  }
  if (values_read) *values_read = n;
  // loadDensityField (SIMPLE.cpp:556-584): gamma = 1 - cellType
  for (size_t k = 0; k < ct.size(); ++k) {
    if (cellType) cellType[k] = ct[k];
    if (gamma) gamma[k] = 1.0 - ct[k];
  }
  return opened ? CPS_OK : io_fail(CPS_OK, std::string("no geometry file ") + path + "; all fluid");
}

cps_status cps_read_restart(const char* dir, int M, int N, double* u, double* v, double* p, int* loaded) {
  if (!dir || M <= 0 || N <= 0 || !u || !v || !p) return io_fail(CPS_ERR_ARG, "bad arguments");
  // initializeMemory's restart loader (SIMPLE.cpp:203-226): a missing or
  // incomplete file leaves that matrix at zero.
  struct Item {
    const char* name;
    double* a;
    int rows, cols;
  } items[3] = {{"u", u, M + 1, N}, {"v", v, M, N + 1}, {"p", p, M + 1, N + 1}};
  int ok = 0;
  for (const Item& it : items) {
    const size_t n = (size_t)it.rows * it.cols;
    std::fill(it.a, it.a + n, 0.0);
    std::ifstream in(std::string(dir) + "/" + it.name + ".txt");
    if (!in) continue;
    bool complete = true;
    for (size_t k = 0; k < n && complete; ++k)
      if (!(in >> it.a[k])) complete = false;
    if (!complete) {
      std::fill(it.a, it.a + n, 0.0);
      continue;
    }
    ++ok;
  }
  if (loaded) *loaded = ok;
  return CPS_OK;
}

cps_status cps_save_all(const char* dir, int M, int N, double hx, double hy, int N_in_buffer, int N_out_buffer,
                        const double* u, const double* v, const double* p, const double* cellType,
                        const double* gamma, const double* alpha, int layout) {
  if (!dir || M < 2 || N < 2 || !u || !v || !p || !gamma || !alpha)
    return io_fail(CPS_ERR_ARG, "dir, M, N >= 2, u, v, p, gamma and alpha are required");
  if (layout != CPS_ROW_MAJOR && layout != CPS_COL_MAJOR) return io_fail(CPS_ERR_ARG, "bad layout");
  const std::string d(dir);
  const Mat U = from_host(u, M + 1, N, layout), V = from_host(v, M, N + 1, layout), P = from_host(p, M + 1, N + 1, layout);
  const Mat G = from_host(gamma, M, N, layout), A = from_host(alpha, M, N, layout);
  Mat C(M, N);
  for (int i = 0; i < M; ++i)
    for (int j = 0; j < N; ++j) C(i, j) = cellType ? at(cellType, M, N, i, j, layout) : 1.0 - G(i, j);
  if (!save_matrix(d, "u", U) || !save_matrix(d, "v", V) || !save_matrix(d, "p", P))
    return io_fail(CPS_ERR_ARG, "could not write to " + d);
  // cell-aligned fields (output.cpp:87-103)
  Mat uC(M, N), vC(M, N), pC(M, N);
  for (int i = 0; i < M; ++i)
    for (int j = 0; j < N; ++j) {
      uC(i, j) = 0.5 * (U(i, j) + U(i + 1, j));
      vC(i, j) = 0.5 * (V(i, j) + V(i, j + 1));
      const int pRow = std::max(1, std::min(i + 1, M - 1));
      const int pCol = std::max(1, std::min(j + 1, N - 1));
      pC(i, j) = P(pRow, pCol);
    }
  save_matrix(d, "u_full", uC);
  save_matrix(d, "v_full", vC);
  save_matrix(d, "pressure_full", pC);
  // pressure gradient (output.cpp:113-141)
  Mat gX(M, N), gY(M, N), gM(M, N);
  for (int i = 0; i < M; ++i)
    for (int j = 0; j < N; ++j) {
      if (j > 0 && j < N - 1) gX(i, j) = (pC(i, j + 1) - pC(i, j - 1)) / (2.0 * hx);
      else if (j == 0) gX(i, j) = (pC(i, j + 1) - pC(i, j)) / hx;
      else gX(i, j) = (pC(i, j) - pC(i, j - 1)) / hx;
      if (i > 0 && i < M - 1) gY(i, j) = (pC(i + 1, j) - pC(i - 1, j)) / (2.0 * hy);
      else if (i == 0) gY(i, j) = (pC(i + 1, j) - pC(i, j)) / hy;
      else gY(i, j) = (pC(i, j) - pC(i - 1, j)) / hy;
      gM(i, j) = std::sqrt(gX(i, j) * gX(i, j) + gY(i, j) * gY(i, j));
    }
  // thermal crop (output.cpp:146-171): skip the inlet and outlet buffers
  const int Nt = N - N_in_buffer - N_out_buffer;
  if (Nt > 0) {
    Mat uT(M, Nt), vT(M, Nt), pT(M, Nt), gT(M, Nt);
    for (int i = 0; i < M; ++i)
      for (int j = 0; j < Nt; ++j) {
        const int s = j + N_in_buffer;
        uT(i, j) = uC(i, s);
        vT(i, j) = vC(i, s);
        pT(i, j) = pC(i, s);
        gT(i, j) = gM(i, s);
      }
    save_matrix(d, "u_thermal", uT);
    save_matrix(d, "v_thermal", vT);
    save_matrix(d, "pressure_thermal", pT);
    save_matrix(d, "p_gradient", gT);
  }
  // VTK structured points (output.cpp:176-258)
  std::ofstream vtk(d + "/fluid_results.vtk");
  if (!vtk.is_open()) return io_fail(CPS_ERR_ARG, "could not write " + d + "/fluid_results.vtk");
  vtk << "# vtk DataFile Version 3.0\n";
  vtk << "SIMPLE CFD Results\n";
  vtk << "ASCII\n";
  vtk << "DATASET STRUCTURED_POINTS\n";
  vtk << "DIMENSIONS " << N << " " << M << " 1\n";
  vtk << "ORIGIN 0 0 0\n";
  vtk << "SPACING " << hx << " " << hy << " 1\n";
  vtk << "POINT_DATA " << N * M << "\n";
  auto scalars = [&](const char* name, const Mat& m) {
    vtk << "SCALARS " << name << " double 1\n";
    vtk << "LOOKUP_TABLE default\n";
    for (int i = 0; i < M; ++i)
      for (int j = 0; j < N; ++j) vtk << m(i, j) << "\n";
  };
  auto vectors = [&](const char* name, const Mat& x, const Mat& y) {
    vtk << "VECTORS " << name << " double\n";
    for (int i = 0; i < M; ++i)
      for (int j = 0; j < N; ++j) vtk << x(i, j) << " " << y(i, j) << " 0.0\n";
  };
  scalars("pressure", pC);
  vectors("velocity", uC, vC);
  scalars("cellType", C);
  scalars("Density", G);
  scalars("Alpha", A);
  scalars("PressureGradient", gM);
  vectors("pressure_gradient", gX, gY);
  return vtk ? CPS_OK : io_fail(CPS_ERR_ARG, "write failed: " + d + "/fluid_results.vtk");
}

cps_status cps_save_logs(const char* dir, int n, int iter0, const cps_step_out* hist, const double* dp,
                         const double* cfl, double cfl0) {
  if (!dir || n < 0 || (n > 0 && !hist)) return io_fail(CPS_ERR_ARG, "dir, n >= 0 and hist are required");
  const std::string d(dir);
  // initLogFiles (output.cpp:268-275)
  std::ofstream resid(d + "/residuals.txt"), dpf(d + "/pressure_drop_history.txt");
  if (!resid.is_open() || !dpf.is_open()) return io_fail(CPS_ERR_ARG, "could not write to " + d);
  resid << "Iter MassResid UResid VResid Core_dP_AfterInletBuffer(Pa) "
        << "Full_dP_FullSystem(Pa) CFL" << std::endl;
  dpf << "Iter Core_Total(Pa) Full_Total(Pa) Core_Static(Pa) Full_Static(Pa)" << std::endl;
  // writeIterationLogs (output.cpp:292-313), one row per outer iteration
  for (int k = 0; k < n; ++k) {
    const double* q = dp ? dp + (size_t)4 * k : nullptr;
    const double core = q ? q[0] : 0.0, full = q ? q[1] : 0.0, coreS = q ? q[2] : 0.0, fullS = q ? q[3] : 0.0;
    resid << iter0 + k << " " << hist[k].residMass << " " << hist[k].residU << " " << hist[k].residV << " " << core
          << " " << full << " " << (cfl ? cfl[k] : cfl0) << std::endl;
    dpf << iter0 + k << " " << core << " " << full << " " << coreS << " " << fullS << std::endl;
  }
  return (resid && dpf) ? CPS_OK : io_fail(CPS_ERR_ARG, "write failed in " + d);
}

}  // extern "C"
