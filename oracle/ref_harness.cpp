// Oracle harness around the reference solver's own code (TEST INFRASTRUCTURE
// ONLY -- never part of the product path).
//
// Built by oracle/Makefile from the reference sources where they lie, twice:
//   ref_f32  : the sources as shipped (FP32, Eigen::MatrixXf),
//   ref_f64  : a float->double mechanical promotion of a scratch copy.
// Outputs go to oracle/_ref/ only.
//
// The harness constructs the reference's `SIMPLE` object (SIMPLE.cpp:18-29; it
// reads ExportFiles/fluid_params.txt and geometry_fluid.txt from the working
// directory, which this harness writes first), sets the public configuration
// members the way SIMPLE.h documents them (SIMPLE.h:68-358), overwrites the
// geometry fields, and then drives the reference's own
// `SIMPLE::calculateStep` (iterations.cpp:82-526) in the loop that
// `runIterations` would run (SIMPLE.cpp:299-318) minus file I/O and printing.
//
// Jacobi sweep counts: calculateStep discards the count returned by
// solveU/VMomentumImplicit (iterations.cpp:125).  momentum_solver.cpp is
// compiled with -DsolveMomentumJacobi=harness_solveMomentumJacobi so that its
// call (momentum_solver.cpp:313) lands in the wrapper below, which calls the
// reference's unmodified solvers::cpu::solveMomentumJacobi
// (jacobi_solver.cpp:20-75) and records what it returns.
//
// I/O: a record file (see oracle/casefile.py): each record is a 16-byte
// NUL-padded name, a 1-byte type ('d' = float64, 'i' = int32), a little-endian
// int64 count, then the payload.  Grids are row-major (i-major) float64.
#include <sys/stat.h>
#include <unistd.h>

#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <optional>
#include <stdexcept>
#include <string>
#include <vector>

#include "SIMPLE.h"
#include "Utilities/solvers/cpu/jacobi_solver.h"
#ifdef CPS_DROPIN
#include "b200_dropin.h"
#endif

typedef decltype(SIMPLE::hx) real;                 // float as shipped, double when promoted
typedef decltype(SIMPLE::u) Matrix;                // Eigen::MatrixXf / MatrixXd

static std::vector<int> g_sweep_counts;

namespace solvers {
namespace cpu {
int harness_solveMomentumJacobi(int n, const std::vector<int>& row_ptr, const std::vector<int>& col_idx,
                                const std::vector<real>& values, const std::vector<real>& b,
                                std::vector<real>& x, const std::vector<int>& diagOffset, real tol,
                                int maxIter) {
  int it = solveMomentumJacobi(n, row_ptr, col_idx, values, b, x, diagOffset, tol, maxIter);
  g_sweep_counts.push_back(it);
  return it;
}
}  // namespace cpu
}  // namespace solvers

namespace {

struct Record {
  char type;
  std::vector<double> d;
  std::vector<int32_t> i;
};

std::map<std::string, Record> read_records(const char* path) {
  std::map<std::string, Record> recs;
  FILE* f = std::fopen(path, "rb");
  if (!f) throw std::runtime_error(std::string("cannot open ") + path);
  for (;;) {
    char name[17] = {0};
    if (std::fread(name, 1, 16, f) != 16) break;
    Record r;
    int64_t count = 0;
    if (std::fread(&r.type, 1, 1, f) != 1 || std::fread(&count, 8, 1, f) != 1) throw std::runtime_error("truncated");
    if (r.type == 'd') {
      r.d.resize(count);
      if (count && std::fread(r.d.data(), 8, count, f) != (size_t)count) throw std::runtime_error("truncated");
    } else if (r.type == 'i') {
      r.i.resize(count);
      if (count && std::fread(r.i.data(), 4, count, f) != (size_t)count) throw std::runtime_error("truncated");
    } else {
      throw std::runtime_error("bad record type");
    }
    recs[name] = std::move(r);
  }
  std::fclose(f);
  return recs;
}

struct Writer {
  FILE* f;
  explicit Writer(const char* path) : f(std::fopen(path, "wb")) {
    if (!f) throw std::runtime_error(std::string("cannot write ") + path);
  }
  ~Writer() { std::fclose(f); }
  void head(const char* name, char type, int64_t count) {
    char buf[16] = {0};
    std::strncpy(buf, name, 16);
    std::fwrite(buf, 1, 16, f);
    std::fwrite(&type, 1, 1, f);
    std::fwrite(&count, 8, 1, f);
  }
  void d(const char* name, const std::vector<double>& v) { head(name, 'd', v.size()); std::fwrite(v.data(), 8, v.size(), f); }
  void i(const char* name, const std::vector<int32_t>& v) { head(name, 'i', v.size()); std::fwrite(v.data(), 4, v.size(), f); }
  void matrix(const char* name, const Matrix& m) {
    std::vector<double> v(static_cast<size_t>(m.rows() * m.cols()));
    for (long r = 0; r < m.rows(); ++r)
      for (long c = 0; c < m.cols(); ++c) v[r * m.cols() + c] = static_cast<double>(m(r, c));
    d(name, v);
  }
};

double getd(std::map<std::string, Record>& recs, const char* key) {
  auto it = recs.find(key);
  if (it == recs.end() || it->second.d.empty()) throw std::runtime_error(std::string("missing ") + key);
  return it->second.d[0];
}
int geti(std::map<std::string, Record>& recs, const char* key) {
  auto it = recs.find(key);
  if (it == recs.end() || it->second.i.empty()) throw std::runtime_error(std::string("missing ") + key);
  return it->second.i[0];
}

void load_grid(std::map<std::string, Record>& recs, const char* key, Matrix& m) {
  auto it = recs.find(key);
  if (it == recs.end()) throw std::runtime_error(std::string("missing ") + key);
  const std::vector<double>& v = it->second.d;
  if ((long)v.size() != m.rows() * m.cols()) throw std::runtime_error(std::string("bad size for ") + key);
  for (long r = 0; r < m.rows(); ++r)
    for (long c = 0; c < m.cols(); ++c) m(r, c) = static_cast<real>(v[r * m.cols() + c]);
}

// Mass imbalance restricted to the pressure unknowns (i=1..M-1, j=1..N-2),
// evaluated with the reference's own expression (pressure_solver.cpp:476-480).
real mass_residual_dof(const SIMPLE& s) {
  real out = 0;
  for (int i = 1; i < s.M; ++i)
    for (int j = 1; j < s.N - 1; ++j) {
      real massE = s.rho * s.uStar(i, j) * s.hy;
      real massW = s.rho * s.uStar(i, j - 1) * s.hy;
      real massN = s.rho * s.vStar(i, j) * s.hx;
      real massS = s.rho * s.vStar(i - 1, j) * s.hx;
      real b = std::abs(massW - massE + massS - massN);
      if (b > out) out = b;
    }
  return out;
}

// The physical constants of a case (SIMPLE.h:334-335, 240-244; SIMPLE.cpp:65-66).
void configure_physics(SIMPLE& s, std::map<std::string, Record>& recs) {
  s.hx = static_cast<real>(getd(recs, "hx"));
  s.hy = static_cast<real>(getd(recs, "hy"));
  s.rho = static_cast<real>(getd(recs, "rho"));
  s.eta = static_cast<real>(getd(recs, "eta"));
  s.brinkmanKMin = static_cast<real>(getd(recs, "kmin"));
  s.brinkmanQ = static_cast<real>(getd(recs, "q"));
  s.brinkmanAlphaMax = s.eta / std::max(s.brinkmanKMin, static_cast<real>(1e-20));  // SIMPLE.cpp:65-66
}

// The solver configuration of a case: the public members SIMPLE.h documents
// (SIMPLE.h:68-358), set after construction as a driver would.
void configure_solver(SIMPLE& s, std::map<std::string, Record>& recs) {
  s.targetVel = static_cast<real>(getd(recs, "U_in"));
  s.inletVelocity = s.targetVel;
  s.convectionScheme = geti(recs, "conv");
  s.enableTwoPointFiveD = geti(recs, "twoFiveD") != 0;
  s.enableConvectionScaling = geti(recs, "convScale") != 0;
  s.Ht_channel = static_cast<real>(getd(recs, "Ht"));
  s.twoPointFiveDSinkMultiplier = static_cast<real>(getd(recs, "sinkMult"));
  s.uvAlpha = static_cast<real>(getd(recs, "uvAlpha"));
  s.pAlpha = static_cast<real>(getd(recs, "pAlpha"));
  s.pTol = static_cast<real>(getd(recs, "pTol"));
  s.maxPressureIter = geti(recs, "maxPIter");
  s.momentumTol = static_cast<real>(getd(recs, "momTol"));
  s.maxMomentumIter = geti(recs, "maxMomIter");
  s.pressureSolverType = recs.count("solverType") ? geti(recs, "solverType") : 1;  // 1 = Parallel CG
  s.momentumSolverType = recs.count("momType") ? geti(recs, "momType") : 1;  // iterations.cpp:109
  s.enablePseudoTimeStepping = false; // SIMPLE.h:262 default
  if (recs.count("pseudoI")) {
    // The pseudo-transient term and its CFL controllers (SIMPLE.h:255-313), in the
    // layout of oracle/simple_oracle_impl.h (ip[8..15], dp[11..27]).
    const std::vector<int32_t>& pi = recs["pseudoI"].i;
    const std::vector<double>& pd = recs["pseudoD"].d;
    if (pi.size() != 8 || pd.size() != 17) throw std::runtime_error("bad pseudo records");
    s.enablePseudoTimeStepping = pi[0] != 0;
    s.useLocalPseudoTime = pi[1] != 0;
    s.enableSER = pi[2] != 0;
    s.enableLineSearch = pi[3] != 0;
    s.enableCflRamp = pi[4] != 0;
    s.serUseMaxResid = pi[5] != 0;
    s.serMinIter = pi[6];
    s.lsMaxTries = pi[7];
    s.timeStepMultiplier = static_cast<real>(pd[0]);
    s.minPseudoSpeed = static_cast<real>(pd[1]);
    s.pseudoCFLInitial = static_cast<real>(pd[2]);
    s.pseudoCFLMax = static_cast<real>(pd[3]);
    s.cflRampStartRes = static_cast<real>(pd[4]);
    s.cflRampExponent = static_cast<real>(pd[5]);
    s.cflRampSmooth = static_cast<real>(pd[6]);
    s.serCFLMin = static_cast<real>(pd[7]);
    s.serCFLMax = static_cast<real>(pd[8]);
    s.serSmooth = static_cast<real>(pd[9]);
    s.serMaxIncrease = static_cast<real>(pd[10]);
    s.serMaxDecrease = static_cast<real>(pd[11]);
    s.lsAlphaMin = static_cast<real>(pd[12]);
    s.lsAlphaReduce = static_cast<real>(pd[13]);
    s.lsResidIncreaseTol = static_cast<real>(pd[14]);
    // The constructor's set-up with these values (SIMPLE.cpp:68-82): the global
    // pseudo time step from the domain length and the target velocity; the
    // starting CFL number.
    real domainLength = s.N * s.hx;
    real velRef = std::max(s.targetVel, static_cast<real>(1e-6));
    s.timeStep = s.timeStepMultiplier * domainLength / velRef;
    s.pseudoCFL = static_cast<real>(pd[16]);
    if (s.enableCflRamp) s.pseudoCFL = s.pseudoCFLInitial;
  }
  s.usePressureDropConvergence = false;
  s.saveStateInterval = 0;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: %s case.bin out.bin   (run inside a scratch directory)\n", argv[0]);
    return 2;
  }
  try {
    auto recs = read_records(argv[1]);
    const int M = geti(recs, "M"), N = geti(recs, "N");
    const int mode = geti(recs, "mode");  // 0 = iterate, 1 = alpha from gamma, 2 = runIterations, 3 = files,
                                          // 4 = a design loop in one process
    if (mode == 3) {
      // The reference's own file handling on files the caller put in ./ExportFiles:
      // the constructor reads fluid_params.txt and geometry_fluid.txt and builds
      // gamma and alpha (SIMPLE.cpp:18-29); with a "restart" record the restart
      // loader reads ./restart/{u,v,p}.txt (SIMPLE.cpp:203-232); with "save" the
      // fields given as records are written by saveAll (output.cpp:73-266).
      SIMPLE s;
      Writer w(argv[2]);
      w.matrix("cellType", s.cellType);
      w.matrix("gamma", s.gamma);  // after buildAlphaFromDensity's wall rows
      w.matrix("alpha", s.alpha);
      if (recs.count("restart")) {
        s.reuseInitialFields = true;
        s.restartDirectory = "restart";
        s.initializeMemory();
      }
      if (recs.count("save")) {
        load_grid(recs, "u0", s.u);
        load_grid(recs, "v0", s.v);
        load_grid(recs, "p0", s.p);
        s.saveAll();
      }
      w.i("MN", {s.M, s.N, s.N_in_buffer, s.N_out_buffer});
      w.d("params", {static_cast<double>(s.hx), static_cast<double>(s.hy), static_cast<double>(s.targetVel),
                     static_cast<double>(s.Ht_channel)});
      s.loadDensityField();  // gamma as the file gives it (SIMPLE.cpp:556-584)
      w.matrix("gammaLoaded", s.gamma);
      w.matrix("u", s.u);
      w.matrix("v", s.v);
      w.matrix("p", s.p);
      return 0;
    }
    // The constructor reads these two files from ./ExportFiles (SIMPLE.cpp:19-21).
    mkdir("ExportFiles", 0755);
    {
      FILE* f = std::fopen("ExportFiles/fluid_params.txt", "w");
      std::fprintf(f, "%d %d %.17g %.17g %.17g 0 0 %.17g\n", M, N, getd(recs, "hy"), getd(recs, "hx"),
                   getd(recs, "U_in"), getd(recs, "Ht"));
      std::fclose(f);
      f = std::fopen("ExportFiles/geometry_fluid.txt", "w");
      for (int i = 0; i < M; ++i) {
        for (int j = 0; j < N; ++j) std::fputs(j ? " 0" : "0", f);
        std::fputc('\n', f);
      }
      std::fclose(f);
    }
    if (mode == 4) {
      // A design loop in one process.  Object A runs maxOuter steps of design A
      // (alpha, gamma) from the zero state and is destroyed; a new object B runs
      // maxOuter steps of design B (alpha2, gamma2); then B's alpha and gamma
      // are set in place to design A's and u, v, p to zero (a new design on the
      // same object), and it runs maxOuter steps again.  Phase k writes its
      // err and pressure iterations as errK/pItersK and its fields as uK/vK/pK
      // (k = 1, 2, 3).  With the drop-in, the in-place edit is announced with
      // b200Invalidate, as a maintainer's driver would.
      const int maxOuter = geti(recs, "maxOuter");
      Writer w(argv[2]);
      auto phase = [&](SIMPLE& s, int k) {
        std::vector<double> err;
        std::vector<int32_t> pIt;
        for (int it = 0; it < maxOuter; ++it) {
          s.inletVelocity = s.targetVel;
          int pi = 0;
          err.push_back(static_cast<double>(s.calculateStep(pi)));
          pIt.push_back(pi);
        }
#ifdef CPS_DROPIN
        if (s.pressureSolverType >= 5) b200SyncFieldsToHost(s);
#endif
        const std::string n = std::to_string(k);
        w.d(("err" + n).c_str(), err);
        w.i(("pIters" + n).c_str(), pIt);
        w.matrix(("u" + n).c_str(), s.u);
        w.matrix(("v" + n).c_str(), s.v);
        w.matrix(("p" + n).c_str(), s.p);
      };
      auto setup = [&](SIMPLE& s, const char* alphaKey, const char* gammaKey) {
        omp_set_num_threads(geti(recs, "threads"));
        configure_physics(s, recs);
        configure_solver(s, recs);
        load_grid(recs, alphaKey, s.alpha);
        load_grid(recs, gammaKey, s.gamma);
      };
      // One storage for both objects, so that B is constructed at A's address
      // (the drop-in must tell the new object from the old one).
      std::optional<SIMPLE> obj;
      obj.emplace();
      setup(*obj, "alpha", "gamma");
      phase(*obj, 1);
      obj.reset();
      obj.emplace();
      SIMPLE& b = *obj;
      setup(b, "alpha2", "gamma2");
      phase(b, 2);
      load_grid(recs, "alpha", b.alpha);
      load_grid(recs, "gamma", b.gamma);
      b.u.setZero();
      b.v.setZero();
      b.p.setZero();
#ifdef CPS_DROPIN
      b200Invalidate(b);
#endif
      phase(b, 3);
#ifdef CPS_DROPIN
      b200Release();
#endif
      return 0;
    }
    SIMPLE s;
    omp_set_num_threads(geti(recs, "threads"));  // SIMPLE.cpp:89 forces numThreads=8

    configure_physics(s, recs);

    Writer w(argv[2]);
    if (mode == 1) {
      load_grid(recs, "gamma", s.gamma);
      s.buildAlphaFromDensity();  // SIMPLE.cpp:589-630
      w.matrix("alpha", s.alpha);
      w.matrix("gamma", s.gamma);
      return 0;
    }

    configure_solver(s, recs);

    load_grid(recs, "alpha", s.alpha);
    load_grid(recs, "gamma", s.gamma);
    if (recs.count("u0")) {
      load_grid(recs, "u0", s.u);
      load_grid(recs, "v0", s.v);
      load_grid(recs, "p0", s.p);
    }

    const int maxOuter = geti(recs, "maxOuter");
    const int stopOnConv = geti(recs, "stopOnConv");
    const double eps = getd(recs, "eps");
    std::vector<double> hU, hV, hMass, hMassDof, hErr, hCfl, hSer;
    std::vector<int32_t> hP, hJu, hJv;
    double elapsed = 0.0;
    if (mode == 2) {
      // The reference's own outer loop with its pressure-drop gate (SIMPLE.cpp:237-449); the
      // residual test is switched off (epsilon = 0) so that only the gate or maxIterations ends it.
      s.usePressureDropConvergence = true;
      s.dpConvergenceWindow = geti(recs, "dpWindow");
      s.dpConvergencePercent = static_cast<real>(getd(recs, "dpPercent"));
      s.usePressureDropSlopeGate = geti(recs, "dpSlopeGate") != 0;
      s.dpSlopeWindowIters = geti(recs, "dpSlopeWindow");
      s.dpSlopeMaxDelta = static_cast<real>(getd(recs, "dpSlopeMaxDelta"));
      s.rampSteps = geti(recs, "rampSteps");
      s.enableInletRamp = recs.count("inletRamp") && geti(recs, "inletRamp") != 0;
      s.xPlaneCoreInlet = static_cast<real>(getd(recs, "xCoreIn"));
      s.xPlaneCoreOutlet = static_cast<real>(getd(recs, "xCoreOut"));
      s.maxIterations = maxOuter;
      s.epsilon = 0;
      auto t0 = std::chrono::steady_clock::now();
      s.runIterations();
      elapsed = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      // its per-iteration log: iter, core total, full total, core static, full static dP
      std::vector<int32_t> dpIter;
      std::vector<double> dp;
      FILE* f = std::fopen("ExportFiles/pressure_drop_history.txt", "r");
      if (!f) throw std::runtime_error("no pressure_drop_history.txt");
      char line[512];
      if (!std::fgets(line, sizeof line, f)) line[0] = 0;  // header
      int it;
      double a, b, c, e;
      while (std::fscanf(f, "%d %lf %lf %lf %lf", &it, &a, &b, &c, &e) == 5) {
        dpIter.push_back(it);
        dp.insert(dp.end(), {a, b, c, e});
      }
      std::fclose(f);
      w.i("dpIter", dpIter);
      w.d("dp", dp);
    }
    if (mode == 0 && recs.count("inletRamp")) {
      s.enableInletRamp = geti(recs, "inletRamp") != 0;
      s.rampSteps = geti(recs, "rampSteps");
    }
    for (int it = 0; mode == 0 && it < maxOuter; ++it) {
      // SIMPLE.cpp:303-307
      if (s.enableInletRamp && s.rampSteps > 0 && it < s.rampSteps)
        s.inletVelocity = (static_cast<real>(it + 1) / s.rampSteps) * s.targetVel;
      else
        s.inletVelocity = s.targetVel;
      g_sweep_counts.clear();
      int pIt = 0;
      auto t0 = std::chrono::steady_clock::now();
      real err = s.calculateStep(pIt);
      // the CFL controllers after the step (SIMPLE.cpp:321-327); no-ops with the
      // pseudo-transient term off
      real monitoringResid = s.serUseMaxResid ? err : s.residMass;
      s.updateCflSER(monitoringResid, it);
      s.applyLineSearch(monitoringResid);
      s.updateCflRamp(monitoringResid);
      elapsed += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      hCfl.push_back(s.pseudoCFL);
      hSer.insert(hSer.end(), {(double)s.serResidPrev, (double)s.lsCurrentAlpha, (double)s.lsBacktrackCount});
#ifdef CPS_DROPIN
      if (s.pressureSolverType >= 5) b200SyncFieldsToHost(s);  // uStar/vStar for the residual below
#endif
      real massDof = mass_residual_dof(s);
      hU.push_back(s.residU);
      hV.push_back(s.residV);
      hMass.push_back(s.residMass);
      hMassDof.push_back(massDof);
      hErr.push_back(err);
      hP.push_back(pIt);
      hJu.push_back(g_sweep_counts.size() > 0 ? g_sweep_counts[0] : -1);
      hJv.push_back(g_sweep_counts.size() > 1 ? g_sweep_counts[1] : -1);
      double conv = std::max({(double)s.residU, (double)s.residV, (double)massDof});
      if (stopOnConv && conv <= eps) break;
    }
#ifdef CPS_DROPIN
    if (s.pressureSolverType >= 5) b200SyncFieldsToHost(s);  // fields live on the GPU between steps
#endif
    w.d("residU", hU);
    w.d("residV", hV);
    w.d("residMass", hMass);
    w.d("residMassDof", hMassDof);
    w.d("err", hErr);
    w.i("pIters", hP);
    w.i("uSweeps", hJu);
    w.i("vSweeps", hJv);
    w.d("elapsed", {elapsed});
    w.d("pseudoCFL", hCfl);  // after each step's controllers
    w.d("pseudoState", hSer);  // serResidPrev, lsCurrentAlpha, lsBacktrackCount after each step
    w.matrix("u", s.u);
    w.matrix("v", s.v);
    w.matrix("p", s.p);
    w.matrix("pStar", s.pStar);
    w.matrix("uStar", s.uStar);
    w.matrix("vStar", s.vStar);
    w.matrix("dE", s.dE);
    w.matrix("dN", s.dN);
    // Plane sampling with the reference's samplePlaneAtX (postprocessing.cpp:97-230):
    // full inlet/outlet (SIMPLE.cpp:256-257) and the two core planes.
    const double xs[4] = {0.0, static_cast<double>(N * s.hx), getd(recs, "xCoreIn"), getd(recs, "xCoreOut")};
    std::vector<double> planes;
    for (double x : xs) {
      PlaneMetrics m = samplePlaneAtX(s, static_cast<real>(x));
      planes.insert(planes.end(), {m.flowArea, m.massFlux, m.avgStatic, m.avgDynamic, m.avgTotal, m.valid ? 1.0 : 0.0});
    }
    w.d("planes", planes);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "ref_harness: %s\n", e.what());
    return 1;
  }
  return 0;
}
