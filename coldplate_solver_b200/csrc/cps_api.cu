// Host side of libcps.so: contexts, device memory, launches and the C ABI
// declared in include/cps.h.
//
// Memory: one cudaMalloc'd slab per context holds every field as a pitched
// row-major plane of (M+1) rows x P doubles, P = round_up(N+1, 32), plus the
// grid barrier, the reduction ring and the history buffer.  The fields stay
// resident between calls; per outer iteration only the 8 diagnostics of each
// step travel to the host (batched per cps_solve call).
//
// Launch: the outer iterations run in one persistent kernel launched
// cooperatively (all CTAs co-resident), synchronised by a software grid
// barrier whose waits are bounded (2 s) and report CPS_ERR_TIMEOUT instead of
// hanging.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/cps.h"
#include "cps_device.cuh"

namespace {

thread_local std::string g_create_error;

constexpr int kHistChunk = 4096;  // outer iterations per launch inside cps_solve

// Field planes held by a context, in slab order.
enum Plane {
  kU, kV, kP, kPc, kUs, kVs, kDE, kDN, kAlpha, kGamma,
  kCU0, kCU1, kCU2, kCU3, kCU4, kCV0, kCV1, kCV2, kCV3, kCV4,
  kBU, kBV, kXU0, kXU1, kXV0, kXV1,
  kPx, kPr, kPz, kPp0, kPp1, kPAp, kPdiag,
  kNumPlanes
};

size_t round_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

}  // namespace

struct cps_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int M = 0, N = 0, P = 0, R = 0;
  int precision = CPS_FP64;
  double momTol = 0.0;
  cps::DesignView view{};
  char* slab = nullptr;
  size_t slab_bytes = 0;
  size_t plane_elems = 0;
  cps::GridBarrier* bar = nullptr;
  double* red = nullptr;
  int* dstatus = nullptr;
  int* dndone = nullptr;
  double* dhist = nullptr;
  double* dplane = nullptr;
  double* hstage = nullptr;  // pinned, one plane of (M+1) x (N+1) doubles
  double* hhist = nullptr;   // pinned, kHistChunk * 8
  int* hflags = nullptr;     // pinned: status, n_done
  int grid = 0;
  std::string err;
};

__global__ void __launch_bounds__(cps::kThreads) cps_grid_kernel(cps::DesignView d, cps::RunControl rc,
                                                                cps::GridBarrier* bar, double* red) {
  __shared__ double smem[cps::kRedWidth * 8];
  cps::GridGroup g{bar, red, rc.status, blockIdx.x, gridDim.x, 0u};
  for (int it = 0; it < rc.n_outer; ++it) {
    double out[8];
    const int r = cps::outer_iteration(d, g, smem, out, it + 1 == rc.n_outer, rc.stop_on_conv != 0, rc.eps);
    if (r < 0) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      for (int k = 0; k < 8; ++k) rc.hist[(size_t)it * 8 + k] = out[k];
      *rc.n_done = it + 1;
    }
    if (r == 1) return;
  }
}

// samplePlaneAtX (postprocessing.cpp:62-230) for one plane, one CTA: every row's
// contribution is evaluated with the reference's expressions; the five sums are
// combined in a fixed tree order.
__global__ void __launch_bounds__(cps::kThreads) cps_plane_kernel(cps::DesignView d, double xPhysical, double* out) {
  __shared__ double smem[cps::kRedWidth * 8];
  const int M = d.M, N = d.N, P = d.P;
  const double hx = d.hx, hy = d.hy, rho = d.rho;
  const double xMin = 0.5 * hx, xMax = ((double)N - 0.5) * hx;
  const double xClamped = cps::maxd(xMin, cps::mind(xPhysical, xMax));
  const double jFloat = xClamped / hx - 0.5;
  int colLeft = (int)floor(jFloat);
  colLeft = colLeft < N - 2 ? colLeft : N - 2;
  colLeft = 0 < colLeft ? colLeft : 0;
  const int colRight = colLeft + 1;
  const double xLeft = ((double)colLeft + 0.5) * hx, xRight = ((double)colRight + 0.5) * hx;
  double t = (fabs(xRight - xLeft) < 1e-12) ? 0.0 : (xClamped - xLeft) / (xRight - xLeft);
  t = cps::maxd(0.0, cps::mind(1.0, t));
  double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};  // staticAreaSum, dynAreaSum, totalWeighted, area, fluxSum
  auto cl = [](int a, int lo, int hi) { return a < lo ? lo : (a > hi ? hi : a); };
  for (int i = 1 + threadIdx.x; i < M; i += blockDim.x) {
    const int cellRow = i - 1;
    if (d.gamma[(size_t)cellRow * P + colLeft] < 1.0 - 1e-6 || d.gamma[(size_t)cellRow * P + colRight] < 1.0 - 1e-6)
      continue;
    const double faceArea = hy;
    acc[3] += faceArea;
    const int pL = cl(colLeft + 1, 0, N), pR = cl(colRight + 1, 0, N);
    const double staticP = (1.0 - t) * d.p[(size_t)i * P + pL] + t * d.p[(size_t)i * P + pR];
    const int uL = cl(colLeft, 0, N - 1), uR = cl(colRight, 0, N - 1);
    const double uNormal = (1.0 - t) * d.u[(size_t)i * P + uL] + t * d.u[(size_t)i * P + uR];
    const int vL = cl(colLeft, 0, N), vR = cl(colRight, 0, N);
    const int vT = cl(i - 1, 0, M - 1), vB = cl(i, 0, M - 1);
    const double vTop = (1.0 - t) * d.v[(size_t)vT * P + vL] + t * d.v[(size_t)vT * P + vR];
    const double vBottom = (1.0 - t) * d.v[(size_t)vB * P + vL] + t * d.v[(size_t)vB * P + vR];
    const double vTangential = 0.5 * (vTop + vBottom);
    const double velMag = sqrt(uNormal * uNormal + vTangential * vTangential);
    const double dynP = 0.5 * rho * velMag * velMag;
    const double totalPAbs = staticP + dynP;
    acc[0] += staticP * faceArea;
    acc[1] += dynP * faceArea;
    const double fluxAbs = fabs(rho * uNormal * faceArea);
    if (fluxAbs > 0.0) {
      acc[4] += fluxAbs;
      acc[2] += totalPAbs * fluxAbs;
    }
  }
  cps::block_reduce<5, 0u>(acc, smem);
  if (threadIdx.x == 0) {
    const double area = acc[3], fluxSum = acc[4];
    double avgStatic = 0.0, avgDynamic = 0.0, avgTotal = 0.0, valid = 0.0;
    if (area > 0.0) { avgStatic = acc[0] / area; avgDynamic = acc[1] / area; valid = 1.0; }
    if (fluxSum > 0.0) avgTotal = acc[2] / fluxSum;
    else if (area > 0.0) avgTotal = avgStatic + avgDynamic;
    out[0] = area; out[1] = fluxSum; out[2] = avgStatic; out[3] = avgDynamic; out[4] = avgTotal; out[5] = valid;
  }
}

namespace {

bool cuda_ok(cps_ctx* ctx, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return true;
  std::string m = std::string(what) + ": " + cudaGetErrorString(e);
  if (ctx) ctx->err = m; else g_create_error = m;
  return false;
}

cps_status fail(cps_ctx* ctx, cps_status s, const std::string& msg) {
  if (ctx) ctx->err = msg; else g_create_error = msg;
  return s;
}

size_t footprint_bytes(int M, int N, size_t* plane_elems_out, int* P_out) {
  const int P = (int)round_up((size_t)N + 1, 32);
  const size_t plane = (size_t)(M + 1) * P;
  if (plane_elems_out) *plane_elems_out = plane;
  if (P_out) *P_out = P;
  size_t bytes = plane * sizeof(double) * kNumPlanes;
  bytes += 256;                                                // barrier + flags
  bytes += (size_t)cps::kRedSlots * 2048 * cps::kRedWidth * 8; // reduction ring (<= 2048 CTAs)
  bytes += (size_t)kHistChunk * 8 * 8 + 64;                    // history + plane metrics
  return round_up(bytes, 256);
}

cps_status validate(const cps_desc* d) {
  if (!d) return fail(nullptr, CPS_ERR_ARG, "desc is NULL");
  if (d->M < 3 || d->N < 3) return fail(nullptr, CPS_ERR_ARG, "grid too small: need M >= 3 and N >= 3");
  if ((long long)d->M * d->N > (1LL << 28)) return fail(nullptr, CPS_ERR_ARG, "grid too large");
  if (!(d->hx > 0) || !(d->hy > 0) || !(d->rho > 0) || !(d->eta > 0))
    return fail(nullptr, CPS_ERR_ARG, "hx, hy, rho and eta must be positive");
  if (!(d->uvAlpha > 0) || !(d->pAlpha >= 0)) return fail(nullptr, CPS_ERR_ARG, "bad relaxation factors");
  if (d->maxPressureIter < 0 || d->maxMomentumIter < 0) return fail(nullptr, CPS_ERR_ARG, "negative iteration cap");
  if (d->precision != CPS_FP64 && d->precision != CPS_MIXED) return fail(nullptr, CPS_ERR_ARG, "bad precision");
  if (d->layout != CPS_ROW_MAJOR && d->layout != CPS_COL_MAJOR) return fail(nullptr, CPS_ERR_ARG, "bad layout");
  if (!d->alpha || !d->gamma) return fail(nullptr, CPS_ERR_ARG, "alpha and gamma are required");
  return CPS_OK;
}

// Copy a host rows x cols matrix (row- or column-major) into a pitched device plane.
bool upload_plane(cps_ctx* c, double* dst, const double* src, int rows, int cols, int layout) {
  const double* rowmajor = src;
  if (layout == CPS_COL_MAJOR) {
    for (int i = 0; i < rows; ++i)
      for (int j = 0; j < cols; ++j) c->hstage[(size_t)i * cols + j] = src[(size_t)j * rows + i];
    rowmajor = c->hstage;
  } else {
    std::memcpy(c->hstage, src, sizeof(double) * (size_t)rows * cols);
    rowmajor = c->hstage;
  }
  if (!cuda_ok(c, cudaMemcpy2DAsync(dst, (size_t)c->P * 8, rowmajor, (size_t)cols * 8, (size_t)cols * 8, rows,
                                    cudaMemcpyHostToDevice, c->stream), "upload"))
    return false;
  return cuda_ok(c, cudaStreamSynchronize(c->stream), "upload sync");
}

bool download_plane(cps_ctx* c, double* dst, const double* src, int rows, int cols, int layout) {
  if (!dst) return true;
  if (!cuda_ok(c, cudaMemcpy2DAsync(c->hstage, (size_t)cols * 8, src, (size_t)c->P * 8, (size_t)cols * 8, rows,
                                    cudaMemcpyDeviceToHost, c->stream), "download"))
    return false;
  if (!cuda_ok(c, cudaStreamSynchronize(c->stream), "download sync")) return false;
  if (layout == CPS_COL_MAJOR) {
    for (int i = 0; i < rows; ++i)
      for (int j = 0; j < cols; ++j) dst[(size_t)j * rows + i] = c->hstage[(size_t)i * cols + j];
  } else {
    std::memcpy(dst, c->hstage, sizeof(double) * (size_t)rows * cols);
  }
  return true;
}

double* plane_ptr(cps_ctx* c, int k) { return reinterpret_cast<double*>(c->slab) + (size_t)k * c->plane_elems; }

void set_step_inputs(cps_ctx* c, double Uin) {
  c->view.Uin = Uin;
  c->view.maxVel = 3.0 * std::max(std::fabs(Uin), 0.1);  // iterations.cpp:104
}

cps_status run(cps_ctx* c, int n_outer, int stop_on_conv, double eps, cps_step_out* hist, int* n_done) {
  int done_total = 0;
  while (done_total < n_outer) {
    const int chunk = std::min(kHistChunk, n_outer - done_total);
    cps::RunControl rc{chunk, stop_on_conv, eps, c->dhist, c->dndone, c->dstatus};
    if (!cuda_ok(c, cudaMemsetAsync(c->dndone, 0, sizeof(int), c->stream), "memset")) return CPS_ERR_CUDA;
    void* args[] = {&c->view, &rc, &c->bar, &c->red};
    if (!cuda_ok(c, cudaLaunchCooperativeKernel((const void*)cps_grid_kernel, dim3(c->grid), dim3(cps::kThreads), args,
                                                0, c->stream), "cooperative launch"))
      return CPS_ERR_CUDA;
    if (!cuda_ok(c, cudaMemcpyAsync(c->hflags, c->dstatus, 2 * sizeof(int), cudaMemcpyDeviceToHost, c->stream), "d2h"))
      return CPS_ERR_CUDA;
    if (!cuda_ok(c, cudaMemcpyAsync(c->hhist, c->dhist, sizeof(double) * 8 * chunk, cudaMemcpyDeviceToHost, c->stream),
                 "d2h"))
      return CPS_ERR_CUDA;
    if (!cuda_ok(c, cudaStreamSynchronize(c->stream), "kernel")) return CPS_ERR_CUDA;
    const int status = c->hflags[0], nd = c->hflags[1];
    if (hist) {
      for (int k = 0; k < nd; ++k) {
        const double* h = c->hhist + (size_t)8 * k;
        cps_step_out& o = hist[done_total + k];
        o.residU = h[0]; o.residV = h[1]; o.residMass = h[2]; o.residMassDof = h[3]; o.err = h[4];
        o.pIters = (int)h[5]; o.uSweeps = (int)h[6]; o.vSweeps = (int)h[7];
      }
    }
    done_total += nd;
    if (n_done) *n_done = done_total;
    if (status != cps::kStatusOk) {
      // Reset the barrier and status so the context stays usable.
      cudaMemsetAsync(c->bar, 0, sizeof(cps::GridBarrier), c->stream);
      cudaMemsetAsync(c->dstatus, 0, sizeof(int), c->stream);
      cudaStreamSynchronize(c->stream);
      if (status == cps::kStatusTimeout) return fail(c, CPS_ERR_TIMEOUT, "device grid barrier timed out");
      return fail(c, CPS_ERR_DIVERGED, "residual is not finite (solution diverged)");
    }
    if (nd < chunk) break;  // converged
  }
  return CPS_OK;
}

}  // namespace

extern "C" {

const char* cps_version(void) { return "cps 0.1 (sm_100a)"; }

const char* cps_last_error(const cps_ctx* ctx) { return ctx ? ctx->err.c_str() : g_create_error.c_str(); }

cps_status cps_footprint(const cps_desc* desc, unsigned long long* bytes) {
  cps_status s = validate(desc);
  if (s != CPS_OK) return s;
  if (!bytes) return fail(nullptr, CPS_ERR_ARG, "bytes is NULL");
  *bytes = footprint_bytes(desc->M, desc->N, nullptr, nullptr);
  return CPS_OK;
}

cps_status cps_create(const cps_desc* d, cps_ctx** out) {
  if (!out) return fail(nullptr, CPS_ERR_ARG, "out is NULL");
  *out = nullptr;
  cps_status s = validate(d);
  if (s != CPS_OK) return s;
  if (d->precision != CPS_FP64) return fail(nullptr, CPS_ERR_ARG, "this entry point builds FP64 contexts only");
  cps_ctx* c = new (std::nothrow) cps_ctx();
  if (!c) return fail(nullptr, CPS_ERR_OOM, "host allocation failed");
  c->device = d->device;
  c->M = d->M;
  c->N = d->N;
  c->slab_bytes = footprint_bytes(d->M, d->N, &c->plane_elems, &c->P);
  c->R = d->M + 1;
  auto bail = [&](cps_status st) {
    g_create_error = c->err;
    cps_destroy(c);
    return st;
  };
  if (!cuda_ok(c, cudaSetDevice(d->device), "cudaSetDevice")) return bail(CPS_ERR_CUDA);
  if (!cuda_ok(c, cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "stream")) return bail(CPS_ERR_CUDA);
  cudaError_t e = cudaMalloc(&c->slab, c->slab_bytes);
  if (e != cudaSuccess) {
    cuda_ok(c, e, "cudaMalloc");
    return bail(CPS_ERR_OOM);
  }
  if (!cuda_ok(c, cudaMemsetAsync(c->slab, 0, c->slab_bytes, c->stream), "memset")) return bail(CPS_ERR_CUDA);
  const size_t stage = (size_t)(d->M + 1) * (d->N + 1);
  if (!cuda_ok(c, cudaMallocHost(&c->hstage, stage * sizeof(double)), "pinned alloc") ||
      !cuda_ok(c, cudaMallocHost(&c->hhist, (size_t)kHistChunk * 8 * sizeof(double)), "pinned alloc") ||
      !cuda_ok(c, cudaMallocHost(&c->hflags, 4 * sizeof(int)), "pinned alloc"))
    return bail(CPS_ERR_OOM);

  char* tail = c->slab + c->plane_elems * sizeof(double) * kNumPlanes;
  c->bar = reinterpret_cast<cps::GridBarrier*>(tail);
  c->dstatus = reinterpret_cast<int*>(tail + 64);  // [0] status, [1] n_done
  c->dndone = c->dstatus + 1;
  c->red = reinterpret_cast<double*>(tail + 256);
  c->dhist = c->red + (size_t)cps::kRedSlots * 2048 * cps::kRedWidth;
  c->dplane = c->dhist + (size_t)kHistChunk * 8;

  cps::DesignView& v = c->view;
  v.M = d->M; v.N = d->N; v.P = c->P;
  v.conv = d->convectionScheme; v.maxPIter = d->maxPressureIter; v.maxMomIter = d->maxMomentumIter;
  v.hx = d->hx; v.hy = d->hy; v.rho = d->rho; v.uvAlpha = d->uvAlpha; v.pAlpha = d->pAlpha; v.pTol = d->pTol;
  // Derived constants, evaluated in the reference's operation order
  // (momentum_solver.cpp:166-191, 220-222, 261; jacobi_solver.cpp:41, 63).
  v.vol = d->hx * d->hy;
  v.De = d->eta * d->hy / d->hx;
  v.Dn = d->eta * d->hx / d->hy;
  const double sinkCoeff = (d->enableTwoPointFiveD && d->Ht_channel > 0.0)
                               ? d->twoPointFiveDSinkMultiplier * (5.0 * d->eta / (2.0 * d->Ht_channel * d->Ht_channel))
                               : 0.0;
  v.sinkDiag = sinkCoeff * v.vol;
  const double convScale = d->enableConvectionScaling ? (6.0 / 7.0) : 1.0;
  v.Fcx = convScale * d->rho * d->hy;
  v.Fcy = convScale * d->rho * d->hx;
  v.relax = (1.0 - d->uvAlpha) / d->uvAlpha;
  const double tolsq = d->momentumTol * d->momentumTol;
  v.thrU = tolsq * (double)((d->M - 1) * (d->N - 2));
  v.thrV = tolsq * (double)((d->M - 2) * (d->N - 1));
  v.u = plane_ptr(c, kU); v.v = plane_ptr(c, kV); v.p = plane_ptr(c, kP); v.pc = plane_ptr(c, kPc);
  v.us = plane_ptr(c, kUs); v.vs = plane_ptr(c, kVs); v.dE = plane_ptr(c, kDE); v.dN = plane_ptr(c, kDN);
  v.alpha = plane_ptr(c, kAlpha); v.gamma = plane_ptr(c, kGamma);
  v.cU = plane_ptr(c, kCU0); v.cV = plane_ptr(c, kCV0);
  v.planeStride = (long long)c->plane_elems;
  v.bU = plane_ptr(c, kBU); v.bV = plane_ptr(c, kBV);
  v.xU0 = plane_ptr(c, kXU0); v.xU1 = plane_ptr(c, kXU1); v.xV0 = plane_ptr(c, kXV0); v.xV1 = plane_ptr(c, kXV1);
  v.px = plane_ptr(c, kPx); v.pr = plane_ptr(c, kPr); v.pz = plane_ptr(c, kPz); v.pp0 = plane_ptr(c, kPp0);
  v.pp1 = plane_ptr(c, kPp1); v.pAp = plane_ptr(c, kPAp); v.pdiag = plane_ptr(c, kPdiag);
  set_step_inputs(c, 0.0);

  if (!upload_plane(c, v.alpha, d->alpha, d->M, d->N, d->layout) ||
      !upload_plane(c, v.gamma, d->gamma, d->M, d->N, d->layout))
    return bail(CPS_ERR_CUDA);

  // Persistent grid: co-resident CTAs, at most one per tile of the design.
  int per_sm = 0, sms = 0;
  if (!cuda_ok(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cps_grid_kernel, cps::kThreads, 0),
               "occupancy") ||
      !cuda_ok(c, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d->device), "attribute"))
    return bail(CPS_ERR_CUDA);
  if (per_sm < 1) return bail(fail(c, CPS_ERR_CUDA, "persistent kernel does not fit on an SM"));
  const int tiles = ((d->M - 1 + cps::kTileI - 1) / cps::kTileI) * ((d->N - 1 + cps::kTileJ - 1) / cps::kTileJ);
  int grid = d->grid_ctas > 0 ? d->grid_ctas : std::min(sms * per_sm, std::max(1, (tiles + 1) / 2));
  grid = std::min(std::min(grid, sms * per_sm), 2048);
  grid = std::max(1, std::min(grid, tiles));
  c->grid = grid;
  c->precision = d->precision;
  *out = c;
  return CPS_OK;
}

void cps_destroy(cps_ctx* c) {
  if (!c) return;
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->slab) cudaFree(c->slab);
  if (c->hstage) cudaFreeHost(c->hstage);
  if (c->hhist) cudaFreeHost(c->hhist);
  if (c->hflags) cudaFreeHost(c->hflags);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

cps_status cps_upload_fields(cps_ctx* c, const double* u, const double* v, const double* p, int layout) {
  if (!c) return fail(nullptr, CPS_ERR_ARG, "ctx is NULL");
  if (layout != CPS_ROW_MAJOR && layout != CPS_COL_MAJOR) return fail(c, CPS_ERR_ARG, "bad layout");
  if (!cuda_ok(c, cudaSetDevice(c->device), "cudaSetDevice")) return CPS_ERR_CUDA;
  if (u && !upload_plane(c, c->view.u, u, c->M + 1, c->N, layout)) return CPS_ERR_CUDA;
  if (v && !upload_plane(c, c->view.v, v, c->M, c->N + 1, layout)) return CPS_ERR_CUDA;
  if (p && !upload_plane(c, c->view.p, p, c->M + 1, c->N + 1, layout)) return CPS_ERR_CUDA;
  return CPS_OK;
}

cps_status cps_step(cps_ctx* c, const cps_step_in* in, cps_step_out* out) {
  if (!c || !in) return fail(c, CPS_ERR_ARG, "ctx and in are required");
  if (!cuda_ok(c, cudaSetDevice(c->device), "cudaSetDevice")) return CPS_ERR_CUDA;
  set_step_inputs(c, in->inletVelocity);
  int nd = 0;
  cps_step_out tmp;
  cps_status s = run(c, 1, 0, 0.0, out ? out : &tmp, &nd);
  return s;
}

cps_status cps_solve(cps_ctx* c, double inletVelocity, int max_outer, double eps, cps_step_out* history,
                     int* n_done) {
  if (!c) return fail(nullptr, CPS_ERR_ARG, "ctx is NULL");
  if (max_outer < 0) return fail(c, CPS_ERR_ARG, "max_outer < 0");
  if (n_done) *n_done = 0;
  if (max_outer == 0) return CPS_OK;
  if (!cuda_ok(c, cudaSetDevice(c->device), "cudaSetDevice")) return CPS_ERR_CUDA;
  set_step_inputs(c, inletVelocity);
  return run(c, max_outer, eps > 0.0 ? 1 : 0, eps, history, n_done);
}

cps_status cps_sample_plane(cps_ctx* c, double x, cps_plane* out) {
  if (!c || !out) return fail(c, CPS_ERR_ARG, "ctx and out are required");
  if (!cuda_ok(c, cudaSetDevice(c->device), "cudaSetDevice")) return CPS_ERR_CUDA;
  cps_plane_kernel<<<1, cps::kThreads, 0, c->stream>>>(c->view, x, c->dplane);
  if (!cuda_ok(c, cudaGetLastError(), "plane launch")) return CPS_ERR_CUDA;
  if (!cuda_ok(c, cudaMemcpyAsync(c->hhist, c->dplane, 6 * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "d2h") ||
      !cuda_ok(c, cudaStreamSynchronize(c->stream), "plane"))
    return CPS_ERR_CUDA;
  out->flowArea = c->hhist[0]; out->massFlux = c->hhist[1]; out->avgStatic = c->hhist[2];
  out->avgDynamic = c->hhist[3]; out->avgTotal = c->hhist[4]; out->valid = c->hhist[5] != 0.0;
  return CPS_OK;
}

cps_status cps_download_fields(cps_ctx* c, double* u, double* v, double* p, double* pStar, double* uStar,
                               double* vStar, double* dE, double* dN, int layout) {
  if (!c) return fail(nullptr, CPS_ERR_ARG, "ctx is NULL");
  if (layout != CPS_ROW_MAJOR && layout != CPS_COL_MAJOR) return fail(c, CPS_ERR_ARG, "bad layout");
  if (!cuda_ok(c, cudaSetDevice(c->device), "cudaSetDevice")) return CPS_ERR_CUDA;
  const int M = c->M, N = c->N;
  const cps::DesignView& w = c->view;
  if (!download_plane(c, u, w.u, M + 1, N, layout) || !download_plane(c, v, w.v, M, N + 1, layout) ||
      !download_plane(c, p, w.p, M + 1, N + 1, layout) || !download_plane(c, pStar, w.pc, M + 1, N + 1, layout) ||
      !download_plane(c, uStar, w.us, M + 1, N, layout) || !download_plane(c, vStar, w.vs, M, N + 1, layout) ||
      !download_plane(c, dE, w.dE, M + 1, N, layout) || !download_plane(c, dN, w.dN, M, N + 1, layout))
    return CPS_ERR_CUDA;
  return CPS_OK;
}

}  // extern "C"
