// B200 drop-in for SIMPLE::calculateStep (see b200_dropin.h).  Plain C++ over
// the C ABI of libcps.so (include/cps.h); compiled with the reference's own
// sources and compiler, against its Eigen matrices (column-major, float as
// shipped or double when promoted).
#include "b200_dropin.h"

#include <cstdio>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "cps.h"

namespace {

typedef decltype(SIMPLE::hx) real;

// The solver parameters of SIMPLE (SIMPLE.h:68-358) a device design is built
// from; any change rebuilds it.
struct DesignParams {
  int M, N, convectionScheme, maxPressureIter, maxMomentumIter, momentumExplicit, twoPointFiveD, convScaling,
      precision, pseudo, useLocalPseudo;
  double hx, hy, rho, eta, uvAlpha, pAlpha, pTol, momentumTol, Ht, sinkMultiplier, minPseudoSpeed, timeStep;
};

DesignParams params_of(const SIMPLE& s) {
  DesignParams k;
  std::memset(&k, 0, sizeof(k));  // padding included, so the structs compare with memcmp
  k.M = s.M;
  k.N = s.N;
  k.convectionScheme = s.convectionScheme;
  k.maxPressureIter = s.maxPressureIter;
  k.maxMomentumIter = s.maxMomentumIter;
  k.momentumExplicit = s.momentumSolverType == 0 ? 1 : 0;
  k.twoPointFiveD = s.enableTwoPointFiveD ? 1 : 0;
  k.convScaling = s.enableConvectionScaling ? 1 : 0;
  k.precision = s.pressureSolverType == 6 ? CPS_MIXED : CPS_FP64;
  k.pseudo = s.enablePseudoTimeStepping ? 1 : 0;
  k.useLocalPseudo = s.useLocalPseudoTime ? 1 : 0;
  k.hx = s.hx;
  k.hy = s.hy;
  k.rho = s.rho;
  k.eta = s.eta;
  k.uvAlpha = s.uvAlpha;
  k.pAlpha = s.pAlpha;
  k.pTol = s.pTol;
  k.momentumTol = s.momentumTol;
  k.Ht = s.Ht_channel;
  k.sinkMultiplier = s.twoPointFiveDSinkMultiplier;
  k.minPseudoSpeed = s.minPseudoSpeed;
  k.timeStep = s.timeStep;
  return k;
}

// One SIMPLE object's device design.
struct DeviceDesign {
  cps_ctx* ctx = nullptr;
  DesignParams params{};
  bool stale = false;              // b200Invalidate: upload the host arrays before the next step
  real stamp[3] = {0, 0, 0};       // residU, residV, residMass as the last step left them
};

std::mutex g_mutex;
std::unordered_map<const SIMPLE*, DeviceDesign> g_designs;

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

void check(cps_ctx* ctx, cps_status st, const char* what) {
  if (st != CPS_OK) throw std::runtime_error(std::string("B200 path: ") + what + ": " + cps_last_error(ctx));
}

void set_stamp(DeviceDesign& e, const SIMPLE& s) {
  e.stamp[0] = s.residU;
  e.stamp[1] = s.residV;
  e.stamp[2] = s.residMass;
}

bool stamp_matches(const DeviceDesign& e, const SIMPLE& s) {
  return e.stamp[0] == s.residU && e.stamp[1] == s.residV && e.stamp[2] == s.residMass;
}

void release(DeviceDesign& e) {
  if (e.ctx) cps_destroy(e.ctx);
  e.ctx = nullptr;
}

void upload_all(DeviceDesign& e, const SIMPLE& s) {
  const std::vector<double> alpha = to_double(s.alpha), gamma = to_double(s.gamma);
  check(e.ctx, cps_upload_geometry(e.ctx, alpha.data(), gamma.data(), CPS_COL_MAJOR), "cps_upload_geometry");
  const std::vector<double> u = to_double(s.u), v = to_double(s.v), p = to_double(s.p);
  check(e.ctx, cps_upload_fields(e.ctx, u.data(), v.data(), p.data(), CPS_COL_MAJOR), "cps_upload_fields");
  e.stale = false;
  set_stamp(e, s);
}

// Build the device design of s from the host object (SIMPLE.h:68-358): the
// solver parameters, alpha, gamma and the current u, v, p.
void build(DeviceDesign& e, const SIMPLE& s, const DesignParams& k) {
  release(e);
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
  d.momentum_explicit = k.momentumExplicit;
  d.enableTwoPointFiveD = k.twoPointFiveD;
  d.enableConvectionScaling = k.convScaling;
  d.Ht_channel = s.Ht_channel;
  d.twoPointFiveDSinkMultiplier = s.twoPointFiveDSinkMultiplier;
  d.precision = k.precision;
  d.alpha = alpha.data();
  d.gamma = gamma.data();
  d.layout = CPS_COL_MAJOR;
  d.device = 0;
  d.grid_ctas = 0;
  cps_ctx* ctx = nullptr;
  if (cps_create(&d, &ctx) != CPS_OK)
    throw std::runtime_error(std::string("B200 path: cps_create: ") + cps_last_error(nullptr));
  e.ctx = ctx;
  e.params = k;
  const std::vector<double> u = to_double(s.u), v = to_double(s.v), p = to_double(s.p);
  check(ctx, cps_upload_fields(ctx, u.data(), v.data(), p.data(), CPS_COL_MAJOR), "cps_upload_fields");
  if (s.enablePseudoTimeStepping) {
    // The pseudo-transient term with the global time step the constructor set
    // (SIMPLE.cpp:68-70); the CFL controllers stay the reference's own, on the
    // host (SIMPLE.cpp:321-327), and hand their CFL number to every step.
    cps_pseudo ps;
    cps_pseudo_defaults(&ps, static_cast<double>(s.targetVel));
    ps.enable = 1;
    ps.use_local = k.useLocalPseudo;
    ps.enable_ser = 0;
    ps.enable_line_search = 0;
    ps.enable_cfl_ramp = 0;
    ps.min_pseudo_speed = s.minPseudoSpeed;
    ps.pseudo_cfl = s.pseudoCFL;
    ps.time_step = s.timeStep;
    check(ctx, cps_set_pseudo(ctx, &ps), "cps_set_pseudo");
  }
  e.stale = false;
  set_stamp(e, s);
}

// The device design of s, brought up to date with the host object.
DeviceDesign& current(const SIMPLE& s) {
  DeviceDesign& e = g_designs[&s];
  const DesignParams k = params_of(s);
  if (!e.ctx || !stamp_matches(e, s) || std::memcmp(&k, &e.params, sizeof(k)) != 0)
    build(e, s, k);
  else if (e.stale)
    upload_all(e, s);
  return e;
}

}  // namespace

real b200StepDropIn(SIMPLE& s, int& pressureIterations) {
  std::lock_guard<std::mutex> lock(g_mutex);
  DeviceDesign& e = current(s);
  if (s.enablePseudoTimeStepping) {
    cps_pseudo_state st = {static_cast<double>(s.pseudoCFL), 0.0, 1.0, 0, 0};
    check(e.ctx, cps_set_pseudo_state(e.ctx, &st), "cps_set_pseudo_state");
  }
  cps_step_in in = {static_cast<double>(s.inletVelocity)};
  cps_step_out out = {};
  check(e.ctx, cps_step(e.ctx, &in, &out), "cps_step");
  s.residU = static_cast<real>(out.residU);
  s.residV = static_cast<real>(out.residV);
  s.residMass = static_cast<real>(out.residMass);
  set_stamp(e, s);
  pressureIterations = out.pIters;
  return static_cast<real>(out.err);
}

void b200Invalidate(const SIMPLE& s) {
  std::lock_guard<std::mutex> lock(g_mutex);
  auto it = g_designs.find(&s);
  if (it != g_designs.end()) it->second.stale = true;
}

void b200SyncFieldsToHost(SIMPLE& s) {
  std::lock_guard<std::mutex> lock(g_mutex);
  auto it = g_designs.find(&s);
  if (it == g_designs.end() || !it->second.ctx || it->second.stale || !stamp_matches(it->second, s))
    return;  // the host object holds the current state
  cps_ctx* ctx = it->second.ctx;
  std::vector<double> u(s.u.rows() * s.u.cols()), v(s.v.rows() * s.v.cols()), p(s.p.rows() * s.p.cols());
  std::vector<double> ps(p.size()), us(u.size()), vs(v.size()), de(u.size()), dn(v.size());
  check(ctx, cps_download_fields(ctx, u.data(), v.data(), p.data(), ps.data(), us.data(), vs.data(), de.data(),
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
  std::lock_guard<std::mutex> lock(g_mutex);
  DeviceDesign& e = current(s);
  cps_plane pl = {};
  check(e.ctx, cps_sample_plane(e.ctx, static_cast<double>(xPhysical), &pl), "cps_sample_plane");
  PlaneMetrics m;
  m.flowArea = static_cast<real>(pl.flowArea);
  m.massFlux = static_cast<real>(pl.massFlux);
  m.avgStatic = static_cast<real>(pl.avgStatic);
  m.avgDynamic = static_cast<real>(pl.avgDynamic);
  m.avgTotal = static_cast<real>(pl.avgTotal);
  m.valid = pl.valid != 0;
  return m;
}

void b200Release(const SIMPLE& s) {
  std::lock_guard<std::mutex> lock(g_mutex);
  auto it = g_designs.find(&s);
  if (it == g_designs.end()) return;
  release(it->second);
  g_designs.erase(it);
}

void b200Release() {
  std::lock_guard<std::mutex> lock(g_mutex);
  for (auto& kv : g_designs) release(kv.second);
  g_designs.clear();
}
