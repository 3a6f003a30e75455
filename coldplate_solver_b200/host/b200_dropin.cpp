// B200 drop-in for SIMPLE::calculateStep (see b200_dropin.h).  Plain C++ over
// the C ABI of libcps.so (include/cps.h); compiled with the reference's own
// sources and compiler, against its Eigen matrices (column-major, float as
// shipped or double when promoted).
#include "b200_dropin.h"

#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "cps.h"

namespace {

typedef decltype(SIMPLE::hx) real;

struct DeviceDesign {
  cps_ctx* ctx = nullptr;
  int M = -1, N = -1;
};
DeviceDesign g_dev;

template <class Matrix>
std::vector<double> to_double(const Matrix& m) {  // column-major copy
  std::vector<double> out(static_cast<size_t>(m.rows() * m.cols()));
  for (long j = 0; j < m.cols(); ++j)
    for (long i = 0; i < m.rows(); ++i) out[static_cast<size_t>(j * m.rows() + i)] = static_cast<double>(m(i, j));
  return out;
}

template <class Matrix>
void from_double(const std::vector<double>& v, Matrix& m) {
  for (long j = 0; j < m.cols(); ++j)
    for (long i = 0; i < m.rows(); ++i) m(i, j) = static_cast<real>(v[static_cast<size_t>(j * m.rows() + i)]);
}

void check(cps_status st, const char* what) {
  if (st != CPS_OK) throw std::runtime_error(std::string("B200 path: ") + what + ": " + cps_last_error(g_dev.ctx));
}

// First call for a grid: build the device design from the SIMPLE registry
// (SIMPLE.h:68-358) and upload alpha, gamma and the current u, v, p.
void ensure_device(SIMPLE& s) {
  if (g_dev.ctx && g_dev.M == s.M && g_dev.N == s.N) return;
  b200Release();
  const std::vector<double> alpha = to_double(s.alpha), gamma = to_double(s.gamma);
  cps_desc d = {};
  d.M = s.M;
  d.N = s.N;
  d.hx = s.hx;
  d.hy = s.hy;
  d.rho = s.rho;
  d.eta = s.eta;
  d.uvAlpha = s.uvAlpha;
  d.pAlpha = s.pAlpha;
  d.pTol = s.pTol;
  d.maxPressureIter = s.maxPressureIter;
  d.momentumTol = s.momentumTol;
  d.maxMomentumIter = s.maxMomentumIter;
  d.convectionScheme = s.convectionScheme;
  d.momentum_explicit = s.momentumSolverType == 0 ? 1 : 0;
  d.enableTwoPointFiveD = s.enableTwoPointFiveD ? 1 : 0;
  d.enableConvectionScaling = s.enableConvectionScaling ? 1 : 0;
  d.Ht_channel = s.Ht_channel;
  d.twoPointFiveDSinkMultiplier = s.twoPointFiveDSinkMultiplier;
  d.precision = CPS_FP64;
  d.alpha = alpha.data();
  d.gamma = gamma.data();
  d.layout = CPS_COL_MAJOR;
  d.device = 0;
  d.grid_ctas = 0;
  cps_ctx* ctx = nullptr;
  if (cps_create(&d, &ctx) != CPS_OK)
    throw std::runtime_error(std::string("B200 path: cps_create: ") + cps_last_error(nullptr));
  g_dev.ctx = ctx;
  g_dev.M = s.M;
  g_dev.N = s.N;
  const std::vector<double> u = to_double(s.u), v = to_double(s.v), p = to_double(s.p);
  check(cps_upload_fields(ctx, u.data(), v.data(), p.data(), CPS_COL_MAJOR), "cps_upload_fields");
  if (s.enablePseudoTimeStepping) {
    // The pseudo-transient term with the global time step the constructor set
    // (SIMPLE.cpp:68-70); the CFL controllers stay the reference's own, on the
    // host (SIMPLE.cpp:321-327), and hand their CFL number to every step.
    cps_pseudo ps;
    cps_pseudo_defaults(&ps, static_cast<double>(s.targetVel));
    ps.enable = 1;
    ps.use_local = s.useLocalPseudoTime ? 1 : 0;
    ps.enable_ser = 0;
    ps.enable_line_search = 0;
    ps.enable_cfl_ramp = 0;
    ps.min_pseudo_speed = s.minPseudoSpeed;
    ps.pseudo_cfl = s.pseudoCFL;
    ps.time_step = s.timeStep;
    check(cps_set_pseudo(ctx, &ps), "cps_set_pseudo");
  }
}

}  // namespace

real b200StepDropIn(SIMPLE& s, int& pressureIterations) {
  ensure_device(s);
  if (s.enablePseudoTimeStepping) {
    cps_pseudo_state st = {static_cast<double>(s.pseudoCFL), 0.0, 1.0, 0, 0};
    check(cps_set_pseudo_state(g_dev.ctx, &st), "cps_set_pseudo_state");
  }
  cps_step_in in = {static_cast<double>(s.inletVelocity)};
  cps_step_out out = {};
  check(cps_step(g_dev.ctx, &in, &out), "cps_step");
  s.residU = static_cast<real>(out.residU);
  s.residV = static_cast<real>(out.residV);
  s.residMass = static_cast<real>(out.residMass);
  pressureIterations = out.pIters;
  return static_cast<real>(out.err);
}

void b200SyncFieldsToHost(SIMPLE& s) {
  if (!g_dev.ctx) return;
  std::vector<double> u(s.u.rows() * s.u.cols()), v(s.v.rows() * s.v.cols()), p(s.p.rows() * s.p.cols());
  std::vector<double> ps(p.size()), us(u.size()), vs(v.size()), de(u.size()), dn(v.size());
  check(cps_download_fields(g_dev.ctx, u.data(), v.data(), p.data(), ps.data(), us.data(), vs.data(), de.data(),
                            dn.data(), CPS_COL_MAJOR),
        "cps_download_fields");
  from_double(u, s.u);
  from_double(v, s.v);
  from_double(p, s.p);
  from_double(ps, s.pStar);
  from_double(us, s.uStar);
  from_double(vs, s.vStar);
  from_double(de, s.dE);
  from_double(dn, s.dN);
}

PlaneMetrics b200SamplePlaneAtX(const SIMPLE& s, real xPhysical) {
  (void)s;
  PlaneMetrics m;
  if (!g_dev.ctx) return m;
  cps_plane pl = {};
  check(cps_sample_plane(g_dev.ctx, static_cast<double>(xPhysical), &pl), "cps_sample_plane");
  m.flowArea = static_cast<real>(pl.flowArea);
  m.massFlux = static_cast<real>(pl.massFlux);
  m.avgStatic = static_cast<real>(pl.avgStatic);
  m.avgDynamic = static_cast<real>(pl.avgDynamic);
  m.avgTotal = static_cast<real>(pl.avgTotal);
  m.valid = pl.valid != 0;
  return m;
}

void b200Release() {
  if (g_dev.ctx) cps_destroy(g_dev.ctx);
  g_dev = DeviceDesign();
}
