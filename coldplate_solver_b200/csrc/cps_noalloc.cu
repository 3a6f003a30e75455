// cps_solve_noalloc: the single-design FP64 solve for callers that cannot
// allocate device memory.
//
// Who needs it: code that runs where cudaMalloc/cudaFree are not allowed or
// not safe -- inside a host application that owns all device memory through
// its own pool and forbids third-party allocations, a real-time loop that must
// not hit the driver's allocator (whose calls can synchronise the device and
// take unbounded time), or a plugin that is handed device buffers and a stream
// and nothing else.  Such a caller passes its own device buffers for the
// design's inputs and outputs; every other byte the kernel needs (the Jacobi
// and PCG vectors, coefficient planes, reduction ring, barrier, status and
// diagnostics) lives in one file-scope static device array, so this entry
// point allocates nothing.
//
// Limits and sharing:
//   * the scratch holds designs with (M + 1) * pitch <= kNoAllocMaxPlane
//     (131072 elements, e.g. a 250 x 500 cell grid with pitch 512); larger
//     designs are rejected with CPS_ERR_ARG before any device work;
//   * the array (about 27 MB) is held on every GPU that loads the library until
//     the process exits;
//   * all calls on a device share it and it keeps the last call's contents:
//     each call clears what must start at zero (barrier, status, counters), and
//     calls that overlap on the GPU (another stream, another host thread) race
//     on it -- serialise them;
//   * the array's name is only a host-side stand-in, never a device address:
//     every call looks the address up with cudaGetSymbolAddress in the
//     calling thread's current context (an allocation-free lookup), so a
//     call under a context of the caller's own, or after cudaDeviceReset,
//     gets that context's copy of the array; the first call in a process
//     also loads the kernel's module, so make it before any stream capture;
//   * the call runs on the caller's stream only and synchronises that stream
//     before it returns.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <string>

#include "../../include/cps.h"
#include "cps_device.cuh"

namespace {

constexpr size_t kNoAllocMaxPlane = 131072;  // (M + 1) * pitch elements
constexpr int kNoAllocInnerPlanes = 25;
constexpr int kNoAllocMaxCtas = 1024;
constexpr int kNoAllocHist = 4096;
constexpr size_t kPlanesBytes = kNoAllocInnerPlanes * kNoAllocMaxPlane * sizeof(double);
constexpr size_t kRingBytes = (size_t)cps::kRedSlots * kNoAllocMaxCtas * cps::kRedWidth * sizeof(double);
constexpr size_t kHistBytes = (size_t)kNoAllocHist * 8 * sizeof(double);
constexpr size_t kFlagsBytes = 256;  // barrier (8 B) at 0, status at 64, n_done at 68
constexpr size_t kScratchBytes = kPlanesBytes + kRingBytes + kHistBytes + kFlagsBytes;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Errors are returned as a status; the reason is printed to stderr on one line.
cps_status fail(cps_status s, const std::string& m) {
  std::fprintf(stderr, "cps_solve_noalloc: %s\n", m.c_str());
  return s;
}

}  // namespace

__global__ void __launch_bounds__(cps::kThreads, CPS_MIN_BLOCKS) cps_noalloc_kernel(cps::DesignView d, cps::RunControl rc,
                                                                      cps::GridBarrier* bar, double* red) {
  __shared__ double smem[cps::kRedWidth * 8];
  extern __shared__ __align__(128) char tile_smem[];
  cps::GridGroup g{bar, red, rc.status, blockIdx.x, gridDim.x, 0u, 0ull};  // no tensor maps: element-wise staging
  cps::SweepHint hint{2, 2, 2};
  for (int it = 0; it < rc.n_outer; ++it) {
    double out[8];
    const int r = cps::outer_iteration<double>(d, g, smem, tile_smem, out, it + 1 == rc.n_outer,
                                               rc.stop_on_conv != 0, rc.eps, 0, nullptr, nullptr, nullptr, &hint);
    if (r < 0) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      for (int k = 0; k < 8; ++k) rc.hist[(size_t)it * 8 + k] = out[k];
      *rc.n_done = it + 1;
    }
    if (r == 1) return;
  }
}

extern "C" cps_status cps_solve_noalloc(const cps_desc* desc, int pitch, const double* alpha, const double* gamma,
                                        double* u, double* v, double* p, double* pStar, double* uStar,
                                        double* vStar, double* dE, double* dN, double inletVelocity, int max_outer,
                                        double eps, cps_step_out* history, int* n_done, void* stream) {
  if (n_done) *n_done = 0;
  if (!desc) return fail(CPS_ERR_ARG, "desc is NULL");
  const cps_desc& d = *desc;
  if (d.M < 3 || d.N < 3) return fail(CPS_ERR_ARG, "grid too small: need M >= 3 and N >= 3");
  if (d.precision != CPS_FP64) return fail(CPS_ERR_ARG, "the allocation-free entry point is FP64 only");
  if (pitch < d.N + 1) return fail(CPS_ERR_ARG, "pitch must be >= N + 1 elements");
  if ((size_t)(d.M + 1) * (size_t)pitch > kNoAllocMaxPlane)
    return fail(CPS_ERR_ARG, "design too large for the static scratch: need (M + 1) * pitch <= 131072 elements");
  if (!(d.hx > 0) || !(d.hy > 0) || !(d.rho > 0) || !(d.eta > 0) || !(d.uvAlpha > 0) || !(d.pAlpha >= 0))
    return fail(CPS_ERR_ARG, "non-positive grid spacing, density, viscosity or relaxation");
  if (d.maxPressureIter < 0 || d.maxMomentumIter < 0 || max_outer < 0 || max_outer > kNoAllocHist)
    return fail(CPS_ERR_ARG, "iteration caps must be >= 0 and max_outer <= 4096");
  if (!alpha || !gamma || !u || !v || !p || !pStar || !uStar || !vStar || !dE || !dN)
    return fail(CPS_ERR_ARG, "every device buffer is required");
  if (max_outer == 0) return CPS_OK;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return fail(CPS_ERR_CUDA, "no device");
  // Set-up, with the caller's device current: the address of the static array
  // in the current context (its host-side name is not a device address), and
  // the co-resident CTAs of the cooperative launch.  None of these calls
  // allocates.
  unsigned char* scratch = nullptr;
  {
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess) return fail(CPS_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    scratch = static_cast<unsigned char*>(ptr);
  }
  int per_sm = 0, sms = 0;
  {
    cudaError_t e = cudaFuncSetAttribute((const void*)cps_noalloc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)cps::tile_smem_bytes<double>());
    if (e == cudaSuccess)
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cps_noalloc_kernel, cps::kThreads,
                                                        cps::tile_smem_bytes<double>());
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess || per_sm < 1) return fail(CPS_ERR_CUDA, "occupancy query failed");
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);

  // Design view over the caller's buffers and the static scratch (derived
  // constants in the reference's operation order, momentum_solver.cpp:166-191).
  cps::DesignView w = {};
  w.M = d.M; w.N = d.N; w.P = pitch;
  w.conv = d.convectionScheme; w.maxPIter = d.maxPressureIter; w.maxMomIter = d.maxMomentumIter;
  w.momExplicit = d.momentum_explicit != 0 ? 1 : 0;
  w.hx = d.hx; w.hy = d.hy; w.rho = d.rho; w.uvAlpha = d.uvAlpha; w.pAlpha = d.pAlpha; w.pTol = d.pTol;
  w.vol = d.hx * d.hy;
  w.De = d.eta * d.hy / d.hx;
  w.Dn = d.eta * d.hx / d.hy;
  const double sinkCoeff = (d.enableTwoPointFiveD && d.Ht_channel > 0.0)
                               ? d.twoPointFiveDSinkMultiplier * (5.0 * d.eta / (2.0 * d.Ht_channel * d.Ht_channel))
                               : 0.0;
  w.sinkDiag = sinkCoeff * w.vol;
  const double convScale = d.enableConvectionScaling ? (6.0 / 7.0) : 1.0;
  w.Fcx = convScale * d.rho * d.hy;
  w.Fcy = convScale * d.rho * d.hx;
  w.relax = (1.0 - d.uvAlpha) / d.uvAlpha;
  const double tolsq = d.momentumTol * d.momentumTol;
  w.thrU = tolsq * (double)((d.M - 1) * (d.N - 2));
  w.thrV = tolsq * (double)((d.M - 2) * (d.N - 1));
  w.Uin = inletVelocity;
  w.maxVel = 3.0 * std::max(std::fabs(inletVelocity), 0.1);  // iterations.cpp:104
  w.u = u; w.v = v; w.p = p; w.pc = pStar; w.us = uStar; w.vs = vStar; w.dE = dE; w.dN = dN;
  w.alpha = const_cast<double*>(alpha);
  w.gamma = const_cast<double*>(gamma);
  const size_t plane = (size_t)(d.M + 1) * pitch;
  w.planeStride = (long long)plane;
  double* base = reinterpret_cast<double*>(scratch);
  auto pl = [&](int k) { return base + (size_t)k * plane; };
  w.f64.cU = pl(0); w.f64.cV = pl(5);
  w.f64.bU = pl(10); w.f64.bV = pl(11);
  w.f64.xU0 = pl(12); w.f64.xU1 = pl(13); w.f64.xV0 = pl(14); w.f64.xV1 = pl(15);
  w.f64.px = pl(16); w.f64.pr = pl(17); w.f64.pz = pl(18); w.f64.pp0 = pl(19); w.f64.pp1 = pl(20);
  w.f64.pAp = pl(21); w.f64.pdiag = pl(22); w.f64.cx = pl(23); w.f64.cy = pl(24);

  double* ring = reinterpret_cast<double*>(scratch + kPlanesBytes);
  double* hist = reinterpret_cast<double*>(scratch + kPlanesBytes + kRingBytes);
  unsigned char* flags = scratch + kPlanesBytes + kRingBytes + kHistBytes;
  cps::GridBarrier* bar = reinterpret_cast<cps::GridBarrier*>(flags);
  int* status = reinterpret_cast<int*>(flags + 64);
  int* done = status + 1;

  // The grid cps_create picks for the same design: the fewest rounds of tiles
  // per CTA the co-resident CTAs allow, spread evenly.
  const int tiles = ((d.M - 1 + cps::kTileI - 1) / cps::kTileI) * ((d.N - 1 + cps::kTileJ - 1) / cps::kTileJ);
  const int cap = std::max(1, std::min(sms * per_sm, kNoAllocMaxCtas));
  const int rounds = (tiles + cap - 1) / cap;
  const int grid = std::max(1, std::min(std::min((tiles + rounds - 1) / rounds, cap), tiles));

  // The outputs the iteration writes only in part start from zero, as the
  // reference's fields do (SIMPLE.cpp:188-197); the shared scratch's barrier,
  // status and counter are cleared for this call.
  const size_t rows = (size_t)(d.M + 1) * pitch * sizeof(double);
  cudaError_t e = cudaSuccess;
  for (double* out : {pStar, uStar, vStar, dE, dN})
    if (e == cudaSuccess) e = cudaMemsetAsync(out, 0, rows, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(flags, 0, kFlagsBytes, st);
  if (e != cudaSuccess) return fail(CPS_ERR_CUDA, std::string("memset: ") + cudaGetErrorString(e));
  cps::RunControl rc{max_outer, eps > 0.0 ? 1 : 0, eps, hist, done, status};
  void* args[] = {&w, &rc, &bar, &ring};
  e = cudaLaunchCooperativeKernel((const void*)cps_noalloc_kernel, dim3(grid), dim3(cps::kThreads), args,
                                  cps::tile_smem_bytes<double>(), st);
  if (e != cudaSuccess) return fail(CPS_ERR_CUDA, std::string("cooperative launch: ") + cudaGetErrorString(e));
  int hflags[2] = {0, 0};
  e = cudaMemcpyAsync(hflags, status, sizeof(hflags), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return fail(CPS_ERR_CUDA, std::string("kernel: ") + cudaGetErrorString(e));
  const int nd = hflags[1];
  if (n_done) *n_done = nd;
  if (history && nd > 0) {
    double h[128 * 8];  // host stack staging, 128 iterations per copy, on the caller's stream
    for (int k0 = 0; k0 < nd; k0 += 128) {
      const int cnt = std::min(128, nd - k0);
      e = cudaMemcpyAsync(h, hist + (size_t)8 * k0, sizeof(double) * 8 * cnt, cudaMemcpyDeviceToHost, st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);
      if (e != cudaSuccess) return fail(CPS_ERR_CUDA, std::string("history copy: ") + cudaGetErrorString(e));
      for (int k = 0; k < cnt; ++k) {
        const double* r = h + 8 * k;
        cps_step_out& o = history[k0 + k];
        o.residU = r[0]; o.residV = r[1]; o.residMass = r[2]; o.residMassDof = r[3]; o.err = r[4];
        o.pIters = (int)r[5]; o.uSweeps = (int)r[6]; o.vSweeps = (int)r[7];
      }
    }
  }
  if (hflags[0] == cps::kStatusTimeout) return fail(CPS_ERR_TIMEOUT, "device grid barrier timed out");
  if (hflags[0] != cps::kStatusOk) return fail(CPS_ERR_DIVERGED, "residual is not finite (solution diverged)");
  return CPS_OK;
}
