// Device code for one SIMPLE outer iteration on a staggered MAC grid, sm_100a.
//
// Algorithm (each step cites the reference lines it reproduces):
//   A  momentum assembly for U and V fused with the first Jacobi sweep
//        momentum_solver.cpp:185-298, convection.cpp:53-186, SIMPLE.h:546-590,
//        jacobi_solver.cpp:44-58 (sweep 1 reads x0 = current u / v)
//   B  further Jacobi sweeps until the RMS stop rule or the cap
//        jacobi_solver.cpp:44-67 (stop test on the pre-update residual of the
//        sweep; that sweep's update is kept and counted)
//   C  scatter + clamp + max|dx| (momentum_solver.cpp:319-337), velocity BCs on
//        u*, v* (boundaries.cpp:48-106), mass imbalance (pressure_solver.cpp:
//        468-486) and PCG set-up (x0 = 0, r = b, z = r/diag, p = z;
//        pressure_solver.cpp:121-150, 693-732)
//   P1 PCG: p = z + beta p (folded into the SpMV) and Ap = A p, pAp
//   P2 PCG: x += alpha p, r -= alpha Ap, |r|^2, z = r/diag, r.z
//        pressure_solver.cpp:152-182 (|pAp| < 1e-20 and ||r|| < pTol stops,
//        counter semantics identical)
//   D  p' scatter with the outlet column p' = 0 (pressure_solver.cpp:796-805),
//        p += pAlpha p' and pressure BCs (iterations.cpp:456-467,
//        boundaries.cpp:111-134), velocity correction + BCs (iterations.cpp:
//        473-499)
//
// Matrix-free: no CSR is built.  The momentum coefficients of each unknown are
// stored once per outer iteration (5 per unknown) because the Jacobi sweeps
// reuse them; the pressure matrix is held as its two face-conductance planes
// (east and north faces) and its diagonal.
//
// Two arithmetic modes share this code through the storage type T of the
// inner-solve arrays:
//   T = double (plain FP64, the path checked against the reference).  Every product/sum that feeds
//     a stored value is evaluated in the reference's order and the unit is
//     compiled with --fmad=false, so per-point values equal the FP64
//     reference's; only the grid-wide sums (Jacobi RMS, PCG dots) are added
//     in a different (fixed, deterministic) order.
//   T = float (mixed).  Fields, momentum coefficients, the momentum defect
//     r0 = b - A u, the mass imbalance and every dot product / norm are FP64;
//     the Jacobi iterate is the correction delta (A delta = r0) and the PCG
//     vectors are stored in FP32.  Each outer iteration is one FP64 defect-
//     correction step, so the converged state is the FP64 fixed point.
//
// Two groups of CTAs can run a design: the whole grid (cooperative launch,
// software barrier with bounded waits) or one thread-block cluster (hardware
// cluster barrier, DSMEM reductions; used by the batched kernel).
//
// Layout: one pitched row-major plane per field in the reference's (i, j)
// index space; element (i, j) at base[i * P + j] with P >= N + 1 a multiple of
// 32 elements, so a warp's 32 consecutive j are one 256-byte (FP64) or
// 128-byte (FP32) segment.
//
// Phases A, C and D (and a Jacobi sweep 2 that re-assembles its rows) stage
// each tile's inputs, halo included, in shared memory kStageDepth tiles
// ahead: one TMA 2-D tile copy per window (cp.async.bulk.tensor, completing
// on the stage buffer's mbarrier; this GPU's own memory only, no multicast),
// or element-wise cp.async for designs without tensor maps.  C then evaluates
// u*, v* and z0 once per tile over the halo instead of once per neighbour.
// The Jacobi sweeps of B read global memory directly (a TMA-staged form is
// kept behind CPS_STAGE_SWEEPS=1; it measured no faster); P1 and P2 keep their
// state in registers or shared memory when it fits, else read global memory
// directly.  Per-point expressions and per-thread summation order are the
// same either way, so the results do not depend on staging.
#pragma once
#include <cuda_runtime.h>
#include <cooperative_groups.h>
#include <stdint.h>

namespace cps {

namespace cg = cooperative_groups;

constexpr int kThreads = 256;   // 8 warps
#ifndef CPS_TILE_J
#define CPS_TILE_J 32
#endif
constexpr int kTileJ = CPS_TILE_J;         // tile columns (16, 32 or 64; consecutive threads, consecutive j)
constexpr int kTileI = kThreads / kTileJ;  // tile rows; one point per thread
static_assert(kTileJ == 16 || kTileJ == 32 || kTileJ == 64, "tile width");
constexpr int kRedWidth = 8;    // doubles per CTA per reduction slot
constexpr int kPlaneSums = 20;  // the pressure-drop monitor's reduction (own ring region)
constexpr int kRedSlots = 4;    // ring of reduction slots (grid group)
// CTAs per SM the persistent kernels are compiled for (128 registers per
// thread at 2).
#ifndef CPS_MIN_BLOCKS
#define CPS_MIN_BLOCKS 2
#endif
constexpr int kStageDepth = 3;  // tiles whose shared-memory copies are in flight at once
// PCG with the CTA's unknowns in shared memory for designs of up to
// SmemTiles<T> tiles per CTA (0: the global-memory PCG there).
#ifndef CPS_SMEM_PCG
#define CPS_SMEM_PCG 1
#endif
#ifndef CPS_RESIDENT_TILES
#define CPS_RESIDENT_TILES 2
#endif
constexpr int kResidentTiles = CPS_RESIDENT_TILES;  // register-resident PCG up to this many tiles per CTA
constexpr unsigned long long kBarrierTimeoutNs = 2000000000ull;  // 2 s
constexpr unsigned long long kTmaTimeoutNs = 1000000000ull;      // a tile copy that has not landed after 1 s
constexpr unsigned long long kTmaDrainNs = 10000000ull;          // then wait up to 10 ms for the copies in flight

// An encoded TMA tensor map (CUtensorMap: 128 bytes, 64-byte aligned), built
// on the host by cuTensorMapEncodeTiled and kept in device memory.
struct alignas(64) TensorMap {
  unsigned long long w[16];
};

// The tensor maps of a design, one per (plane, window shape) the staged
// phases copy: phase A (and a re-assembling sweep 2), phase C, phase D, and
// the Jacobi sweeps of phase B (five coefficient planes, the source and the
// two iterate buffers of each component).
enum TmaMap : int {
  kTmU_A, kTmV_A, kTmP_A, kTmAlpha_A,
  kTmXU0_C, kTmXU1_C, kTmU_C, kTmDE_C, kTmXV0_C, kTmXV1_C, kTmV_C, kTmDN_C, kTmG_C,
  kTmPX_D, kTmP_D, kTmDE_D, kTmUS_D, kTmDN_D, kTmVS_D, kTmG_D,
  kTmCU_B, kTmBU_B = kTmCU_B + 5, kTmXU0_B, kTmXU1_B,
  kTmCV_B, kTmBV_B = kTmCV_B + 5, kTmXV0_B, kTmXV1_B,
  kTmCount
};

enum DeviceStatus : int { kStatusOk = 0, kStatusTimeout = 1, kStatusDiverged = 2 };

// Inner-solve arrays of one design in storage type T.
template <typename T>
struct Inner {
  T* cU;            // 5 planes (E, W, N, S, P) of U-momentum coefficients, stride planeStride
  T* cV;            // same for V
  T* bU;            // FP64 mode: source b; mixed: defect r0 = b - A u
  T* bV;
  T* xU0; T* xU1;   // Jacobi iterates (FP64: x; mixed: the correction delta)
  T* xV0; T* xV1;
  T* px; T* pr; T* pz; T* pp0; T* pp1; T* pAp;  // PCG vectors
  T* pdiag;         // pressure diagonal aP
  T* cx;            // rho dE hy: conductance of the east face of P-cell (i, j)
  T* cy;            // rho dN hx: conductance of the north face of P-cell (i, j)
};

// Device view of one design's grid, parameters and arrays.
struct DesignView {
  int M, N, P;
  int conv, maxPIter, maxMomIter;
  int pcgSingleReduction;  // 1: single-reduction PCG recurrences; 0: the reference's two-reduction PCG
  int momExplicit;         // 1: explicit point update of the momentum (momentumSolverType = 0)
  double hx, hy, rho, uvAlpha, pAlpha, pTol;
  double vol, De, Dn, sinkDiag, Fcx, Fcy, relax;  // Fcx = cs*rho*hy, Fcy = cs*rho*hx, relax = (1-uvA)/uvA
  double thrU, thrV;                              // momTol^2 * nU, momTol^2 * nV
  double Uin, maxVel;
  double *u, *v, *p, *pc, *us, *vs, *dE, *dN, *alpha, *gamma;
  long long planeStride;                          // elements between coefficient planes
  Inner<double> f64;
  Inner<float> f32;
  // Pressure-drop monitor and convergence gate of the outer loop (SIMPLE.cpp:269-408);
  // dpMonitor = 0 leaves the iteration as calculateStep alone.
  int dpMonitor;          // sample the four planes after every outer iteration
  int dpGate;             // usePressureDropConvergence
  int dpWindow;           // dpConvergenceWindow
  int dpSlopeGate;        // usePressureDropSlopeGate
  int dpSlopeWindow;      // dpSlopeWindowIters
  int dpRampSteps;        // rampSteps: the dP history starts at this iteration
  double dpPercent;       // dpConvergencePercent
  double dpSlopeMaxDelta; // dpSlopeMaxDelta
  double xPlane[4];       // core inlet, core outlet, x = 0, x = N hx
  double* dpHist;         // dpWindow circular slots, then dpSlopeWindow slots (slot = iter mod window)
  // Pseudo-transient term of the momentum equations and the outer loop's CFL
  // controllers (SIMPLE.h:255-313); pseudo = 0 leaves both out.
  int pseudo;             // enablePseudoTimeStepping
  int pseudoLocal;        // useLocalPseudoTime
  int serOn, lsOn, rampOn; // enableSER, enableLineSearch, enableCflRamp
  int serUseMax;          // serUseMaxResid: SER watches the step's error instead of residMass
  int serMinIter, lsMaxTries;
  double timeStep;        // timeStepMultiplier * N hx / max(targetVel, 1e-6) (SIMPLE.cpp:68-70)
  double minPseudoSpeed, hChar;  // hChar = min(hx, hy)
  double cflInitial, cflMax, rampStartRes, rampExponent, rampSmooth;
  double serCFLMin, serCFLMax, serSmooth, serMaxIncrease, serMaxDecrease;
  double lsAlphaMin, lsAlphaReduce, lsTol;
  double* pseudoState;    // pseudoCFL, serResidPrev, lsCurrentAlpha, lsBacktrackCount (across launches)
  // kTmCount tensor maps of this design's planes (TmaMap), or null: the staged
  // phases then copy element by element
  const TensorMap* tm;
  // with tensor maps: 1 stages the Jacobi sweeps' tiles too (phase B), 0 (the
  // default) loads them straight from global memory (no tensor maps: always)
  int stageSweeps;
};

// The CFL controllers' state while a design runs; every CTA keeps a copy in
// shared memory and updates it identically from the grid-reduced residuals.
struct PseudoRun {
  double cfl, prev, alpha;
  int count, pad;
};

// The Jacobi sweep counts of a design's last outer iteration, carried from one
// outer iteration to the next by every thread (the counts come from grid-wide
// reductions, so every thread holds the same values).
struct SweepHint {
  int kU, kV;
  int kP;  // the PCG's count (iterations after the first) of the last outer iteration
};

template <typename T> __device__ __forceinline__ const Inner<T>& inner(const DesignView& d);
template <> __device__ __forceinline__ const Inner<double>& inner<double>(const DesignView& d) { return d.f64; }
template <> __device__ __forceinline__ const Inner<float>& inner<float>(const DesignView& d) { return d.f32; }

// Per-launch control of the single-design (grid) kernel.
struct RunControl {
  int n_outer;        // outer iterations to run
  int stop_on_conv;   // stop once max(residU, residV, residMassDof) <= eps
  double eps;
  double* hist;       // n_outer x 8: residU, residV, residMass, residMassDof, err, pIters, uSweeps, vSweeps
  int* n_done;        // outer iterations completed by this launch
  int* status;        // DeviceStatus
  int iter0;          // the outer loop's iteration index of this launch's first iteration
  double* dplog;      // n_outer x 4 (core total, full total, core static, full static dP) or null
  int* dp_converged;  // set when the pressure-drop gate stopped the loop
};

// One entry of the batched (cluster) kernel's work list.
struct BatchItem {
  DesignView view;
  int n_outer;        // outer-iteration budget of this visit
  int stop_on_conv;
  double eps;
  double* hist;       // hist_cap x 8 (the first hist_cap iterations of the visit), may be null
  int hist_cap;
  int iter0;          // the outer loop's iteration index of the visit's first iteration
};
struct BatchResult {
  int n_done;         // outer iterations run in this visit
  int status;         // DeviceStatus
  int converged;
  int pad;
  double last[8];     // diagnostics of the last iteration
};

// Monotonic arrival counter of the grid barrier; zeroed before every launch.
struct GridBarrier {
  unsigned long long count;
};

// ---------------------------------------------------------------------------
// small helpers (std::max/min/clamp evaluated the way libstdc++ does)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double maxd(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double mind(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double clampd(double v, double lo, double hi) { return (v < lo) ? lo : (hi < v) ? hi : v; }

// ---------------------------------------------------------------------------
// Pseudo-transient term and CFL controllers
// ---------------------------------------------------------------------------
// rho vol / dt of the implicit assembly at a point whose current velocity is
// vel (momentum_solver.cpp:231-241).
__device__ __forceinline__ double trans_implicit(const DesignView& d, double cfl, double vel) {
  double dtLocal = maxd(d.timeStep, 1e-20);
  if (d.pseudoLocal) {
    const double speed = maxd(fabs(vel), d.minPseudoSpeed);
    dtLocal = mind(dtLocal, cfl * d.hChar / speed);
    dtLocal = maxd(dtLocal, 1e-20);
  }
  return d.rho * d.vol / dtLocal;
}

// The same coefficient of the explicit update, from computeLocalDt
// (iterations.cpp:207-217, 290-294).
__device__ __forceinline__ double trans_explicit(const DesignView& d, double cfl, double vel) {
  double dtLocal = d.timeStep;
  if (d.pseudoLocal) {
    const double speed = maxd(fabs(vel), d.minPseudoSpeed);
    dtLocal = mind(d.timeStep, cfl * d.hChar / speed);
  }
  return d.rho * d.vol / dtLocal;
}

// The outer loop's controllers after the step with index `iteration`
// (SIMPLE.cpp:321-327): updateCflSER (time_control.cpp:82-118),
// applyLineSearch (:127-166), updateCflRamp (:43-63), in that order; resid is
// the monitoring residual.  The ramp's power is CUDA's pow, which may differ
// from the host's in the last bit.
__device__ __forceinline__ void pseudo_update(const DesignView& d, PseudoRun& s, double resid, int iteration) {
  double cfl = s.cfl, prev = s.prev, alpha = s.alpha;
  int count = s.count;
  if (d.serOn && iteration >= d.serMinIter) {
    const double cur = maxd(resid, 1e-15);
    if (prev <= 0.0) {
      prev = cur;
    } else {
      double ratio = prev / cur;
      ratio = maxd(ratio, d.serMaxDecrease);
      ratio = mind(ratio, d.serMaxIncrease);
      double target = cfl * ratio;
      target = maxd(target, d.serCFLMin);
      target = mind(target, d.serCFLMax);
      cfl = (1.0 - d.serSmooth) * cfl + d.serSmooth * target;
      if (!isfinite(cfl) || cfl <= 0.0) cfl = d.serCFLMin;
      prev = cur;
    }
  }
  if (d.lsOn && d.serOn) {
    if (prev <= 0.0) {
      alpha = 1.0;
      count = 0;
    } else if (resid / prev > d.lsTol) {
      ++count;
      if (count <= d.lsMaxTries) {
        alpha = maxd(alpha * d.lsAlphaReduce, d.lsAlphaMin);
        cfl = maxd(cfl * d.lsAlphaReduce, d.serCFLMin);
      }
    } else {
      if (alpha < 1.0) alpha = mind(alpha * 1.1, 1.0);
      count = 0;
    }
  }
  if (d.rampOn && !d.serOn) {
    const double cur = maxd(resid, 1e-12);
    if (cur > d.rampStartRes) {
      cfl = d.cflInitial;
    } else {
      const double rawFactor = pow(d.rampStartRes / cur, d.rampExponent);
      const double target = mind(d.cflInitial * rawFactor, d.cflMax);
      cfl = (1.0 - d.rampSmooth) * cfl + d.rampSmooth * target;
      if (!isfinite(cfl) || cfl <= 0.0) cfl = d.cflInitial;
    }
  }
  s.cfl = cfl;
  s.prev = prev;
  s.alpha = alpha;
  s.count = count;
}

// Thread 0 loads a design's controller state at the start of its run; the
// caller synchronises the CTA before the state is read.
__device__ __forceinline__ void load_pseudo(const DesignView& d, PseudoRun& s) {
  if (threadIdx.x != 0) return;
  if (d.pseudo && d.pseudoState) {
    s.cfl = __ldcg(d.pseudoState);
    s.prev = __ldcg(d.pseudoState + 1);
    s.alpha = __ldcg(d.pseudoState + 2);
    s.count = (int)__ldcg(d.pseudoState + 3);
  } else {
    s.cfl = 0.0;
    s.prev = 0.0;
    s.alpha = 1.0;
    s.count = 0;
  }
}

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned long long atom_add_acq_rel_u64(unsigned long long* p, unsigned long long v) {
  unsigned long long old;
  asm volatile("atom.acq_rel.gpu.global.add.u64 %0, [%1], %2;" : "=l"(old) : "l"(p), "l"(v) : "memory");
  return old;
}
__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Asynchronous global -> shared copies of one 4- or 8-byte element (cp.async,
// cached at all levels; ordered after the grid barrier's acquire like any
// other load of this thread).
template <typename E>
__device__ __forceinline__ void cp_async_elem(E* smem_dst, const E* gsrc) {
  static_assert(sizeof(E) == 4 || sizeof(E) == 8, "4- or 8-byte elements");
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  if (sizeof(E) == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gsrc) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// mbarriers and TMA tile copies (sm_90+ PTX; CTA-local, no multicast).
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
  asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.shared::cta.b64 st, [%0];\n}" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Wait for the phase with the given parity to complete, at most `limit_ns`;
// false when the limit passed first.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity,
                                                  unsigned long long limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = globaltimer_ns();
  for (unsigned spins = 1;; ++spins) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((spins & 63u) == 0 && globaltimer_ns() - t0 > limit_ns) return false;
  }
}
// One 2-D tile of `map` at element coordinates (x, y) into shared memory;
// `bytes` (the box) is added to the barrier's expected transactions first.
// x times the element size must be a multiple of 16 bytes (checked on the host
// for every window shape).
__device__ __forceinline__ void tma_load_2d(void* dst, const TensorMap* map, int x, int y, unsigned long long* bar,
                                            unsigned bytes) {
  mbar_expect_tx(bar, bytes);
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
      ::"r"(smem_u32(dst)), "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void fence_proxy_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// The CTA's stage-buffer mbarriers and the parity of each one's next phase
// (one byte per buffer: thread 0 flips buffer b's byte while others may read
// another buffer's).  Shared memory rather than registers, so that the
// persistent kernels carry no extra live registers through their phases.
__shared__ unsigned long long s_tma_bar[kStageDepth];
__shared__ unsigned char s_tma_parity[kStageDepth];

// Initialised once per launch by thread 0 (one arrival per phase: the issuing
// thread's), made visible to the CTA and to the TMA unit.  Every persistent
// kernel that runs the staged phases calls it first.
__device__ __forceinline__ void tma_barriers_init() {
  if (threadIdx.x == 0) {
    for (int b = 0; b < kStageDepth; ++b) {
      mbar_init(s_tma_bar + b, 1);
      s_tma_parity[b] = 0;
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    fence_proxy_async_shared();
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// Block reduction of K values, fixed order (deterministic).  Bit k of MaxMask
// selects max instead of sum.  Result valid in every thread.
// ---------------------------------------------------------------------------
template <int K, unsigned MaxMask>
__device__ __forceinline__ void block_reduce(double (&v)[K], double* smem /* K*8 */) {
#pragma unroll
  for (int k = 0; k < K; ++k) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      double o = __shfl_xor_sync(0xffffffffu, v[k], off);
      v[k] = ((MaxMask >> k) & 1u) ? maxd(v[k], o) : v[k] + o;
    }
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) smem[k * 8 + warp] = v[k];
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < K; ++k) {
    double a = smem[k * 8 + 0];
#pragma unroll
    for (int w = 1; w < 8; ++w) a = ((MaxMask >> k) & 1u) ? maxd(a, smem[k * 8 + w]) : a + smem[k * 8 + w];
    v[k] = a;
  }
}

// ---------------------------------------------------------------------------
// Group of CTAs working on one design: the whole grid (cooperative launch)
// with a bounded software barrier.
// ---------------------------------------------------------------------------
struct GridGroup {
  GridBarrier* bar;
  double* red;        // kRedSlots * nblk * kRedWidth
  int* status;
  unsigned rank, nblk;
  unsigned redCount;  // reductions issued so far (same in every CTA)
  unsigned long long epoch;  // barriers passed in this launch

  // Arrive (release) and wait (acquire) for all nblk CTAs: barrier k is
  // complete once the counter reaches k * nblk.  The CTA's writes are ordered
  // before thread 0's release by __syncthreads (cumulativity), and thread 0's
  // acquire before the other threads' reads by the trailing __syncthreads.
  // Returns false (the CTA must return) on timeout or on an error raised elsewhere.
  __device__ bool sync() {
    __shared__ int s_ok;
    __syncthreads();
    ++epoch;
    if (threadIdx.x == 0) s_ok = arrive_and_wait();
    __syncthreads();
    return s_ok != 0;
  }

  // Thread 0 only: arrive at barrier number `epoch` and wait for the others.
  __device__ int arrive_and_wait() {
    const unsigned long long target = epoch * nblk;
    const unsigned long long old = atom_add_acq_rel_u64(&bar->count, 1ull);
    if (old + 1 >= target) return 1;
    const unsigned long long t0 = globaltimer_ns();
    unsigned spins = 0;
    while (ld_acquire_u64(&bar->count) < target) {
      if ((++spins & 255u) == 0) {
        if (*(volatile int*)status != kStatusOk) return 0;
        if (globaltimer_ns() - t0 > kBarrierTimeoutNs) {
          atomicCAS(status, kStatusOk, kStatusTimeout);
          return 0;
        }
      }
    }
    return 1;
  }

  // Publish this CTA's K values, synchronise, and combine all CTAs' values in
  // a fixed order.  Result valid in every thread of every CTA.
  //   CTA value: warp trees (shfl_xor), then the 8 warps in order.
  //   Grid value: lane l folds CTAs l, l+32, ... in order, then a warp tree
  //   (warp 0 for a single value; warp k for value k when there are several).
  //   The ring holds value k of CTA b at [k * nblk + b].
  // Two __syncthreads per single-value reduction: the first orders every
  // thread's tile writes before thread 0's release (cumulativity) and hands
  // the warp values to thread 0; the second hands the result (and thread 0's
  // acquire, through __syncwarp in warp 0) to the whole CTA.  Reductions of
  // 2..8 values take three (see below).
  template <int K, unsigned MaxMask>
  __device__ bool sync_reduce(double (&v)[K], double* smem) {
    static_assert(K <= kRedWidth, "ring slots hold kRedWidth values per CTA");
    double* slot = red + (size_t)(redCount % kRedSlots) * nblk * kRedWidth;
    ++redCount;
    return sync_reduce_at<K, MaxMask>(v, smem, slot);
  }

  // The same with the CTA partials in a region of K * nblk values of the
  // caller's choosing (one that no reduction in flight can be using).
  template <int K, unsigned MaxMask>
  __device__ bool sync_reduce_at(double (&v)[K], double* smem, double* slot) {
    __shared__ double s_res[kPlaneSums];
    __shared__ int s_ok;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < K; ++k) {
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const double o = __shfl_xor_sync(0xffffffffu, v[k], off);
        v[k] = ((MaxMask >> k) & 1u) ? maxd(v[k], o) : v[k] + o;
      }
    }
    if (lane == 0) {
#pragma unroll
      for (int k = 0; k < K; ++k) smem[k * 8 + warp] = v[k];
    }
    ++epoch;
    __syncthreads();
    if constexpr (K >= 2 && K <= kThreads / 32) {
      // Value k folded by warp k, all K at once: the same order per value as
      // below (CTAs lane, lane + 32, ... then a warp tree), but one L2 round
      // trip for the whole reduction instead of one per batch of 16/K CTAs
      // per lane.  A third __syncthreads hands thread 0's acquire to the
      // folding warps.
      if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
          double a = smem[k * 8 + 0];
#pragma unroll
          for (int w = 1; w < 8; ++w) a = ((MaxMask >> k) & 1u) ? maxd(a, smem[k * 8 + w]) : a + smem[k * 8 + w];
          slot[(size_t)k * nblk + rank] = a;
        }
        s_ok = arrive_and_wait();
      }
      __syncthreads();
      const int ok = s_ok;
      if (warp < K) {
        const bool isMax = ((MaxMask >> warp) & 1u) != 0;
        const double* src = slot + (size_t)warp * nblk;
        double acc = 0.0;
        if (ok) {
          constexpr int kB = 16;
          for (unsigned b0 = lane; b0 < nblk; b0 += 32u * kB) {
            double x[kB];
#pragma unroll
            for (int j = 0; j < kB; ++j) {
              const unsigned b = b0 + 32u * j;
              x[j] = b < nblk ? __ldcg(src + b) : 0.0;
            }
#pragma unroll
            for (int j = 0; j < kB; ++j) {
              if (b0 + 32u * j >= nblk) break;
              acc = isMax ? maxd(acc, x[j]) : acc + x[j];
            }
          }
#pragma unroll
          for (int off = 16; off > 0; off >>= 1) {
            const double o = __shfl_xor_sync(0xffffffffu, acc, off);
            acc = isMax ? maxd(acc, o) : acc + o;
          }
        }
        if (lane == 0) s_res[warp] = acc;
      }
      __syncthreads();
#pragma unroll
      for (int k = 0; k < K; ++k) v[k] = s_res[k];
      return ok != 0;
    }
    if (warp == 0) {
      int ok = 1;
      if (lane == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
          double a = smem[k * 8 + 0];
#pragma unroll
          for (int w = 1; w < 8; ++w) a = ((MaxMask >> k) & 1u) ? maxd(a, smem[k * 8 + w]) : a + smem[k * 8 + w];
          slot[(size_t)k * nblk + rank] = a;
        }
        ok = arrive_and_wait();
      }
      ok = __shfl_sync(0xffffffffu, ok, 0);
      __syncwarp();
      double acc[K];
#pragma unroll
      for (int k = 0; k < K; ++k) acc[k] = 0.0;
      if (ok) {
        // CTAs lane, lane + 32, ... in order, their values loaded kBatch at a
        // time before any is added (one L2 round trip per batch instead of
        // one per CTA; the order of the additions is unchanged).
        constexpr int kBatch = K >= 16 ? 1 : 16 / K;
        for (unsigned b0 = lane; b0 < nblk; b0 += 32u * kBatch) {
          double x[K][kBatch];
#pragma unroll
          for (int k = 0; k < K; ++k)
#pragma unroll
            for (int j = 0; j < kBatch; ++j) {
              const unsigned b = b0 + 32u * j;
              x[k][j] = b < nblk ? __ldcg(slot + (size_t)k * nblk + b) : 0.0;
            }
#pragma unroll
          for (int j = 0; j < kBatch; ++j) {
            if (b0 + 32u * j >= nblk) break;
#pragma unroll
            for (int k = 0; k < K; ++k)
              acc[k] = ((MaxMask >> k) & 1u) ? maxd(acc[k], x[k][j]) : acc[k] + x[k][j];
          }
        }
#pragma unroll
        for (int k = 0; k < K; ++k) {
#pragma unroll
          for (int off = 16; off > 0; off >>= 1) {
            const double o = __shfl_xor_sync(0xffffffffu, acc[k], off);
            acc[k] = ((MaxMask >> k) & 1u) ? maxd(acc[k], o) : acc[k] + o;
          }
        }
      }
      if (lane == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) s_res[k] = acc[k];
        s_ok = ok;
      }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = s_res[k];
    return s_ok != 0;
  }
};

// ---------------------------------------------------------------------------
// Group of CTAs working on one design: one thread-block cluster.  The cluster
// barrier is a hardware barrier with release/acquire semantics at cluster
// scope (no spin loop); partial sums travel through distributed shared memory.
// ---------------------------------------------------------------------------
struct ClusterGroup {
  double* redbuf;     // this CTA's shared-memory ring, 2 x kRedWidth
  int* status;        // the current design's status word
  unsigned rank, nblk;
  unsigned redCount;

  __device__ bool sync() {
    cg::this_cluster().sync();
    return true;
  }

  template <int K, unsigned MaxMask>
  __device__ bool sync_reduce(double (&v)[K], double* smem) {
    block_reduce<K, MaxMask>(v, smem);
    double* slot = redbuf + (redCount & 1u) * kRedWidth;
    ++redCount;
    if (threadIdx.x == 0) {
#pragma unroll
      for (int k = 0; k < K; ++k) slot[k] = v[k];
    }
    cg::cluster_group cl = cg::this_cluster();
    cl.sync();
    double acc[K];
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = 0.0;
    if (threadIdx.x < nblk) {
      const double* remote = cl.map_shared_rank(slot, threadIdx.x);
#pragma unroll
      for (int k = 0; k < K; ++k) acc[k] = remote[k];
    }
    block_reduce<K, MaxMask>(acc, smem);
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = acc[k];
    return true;
  }
};

// ---------------------------------------------------------------------------
// Tile staging.  Every phase walks the CTA's tiles (kTileI x kTileJ points,
// one point per thread) in a fixed order.  The values a tile reads, halo
// included, are first copied into shared memory -- one TMA 2-D tile copy per
// window completing on the stage buffer's mbarrier, or element-wise cp.async
// when the design has no tensor maps -- and the copies of the next tiles are
// issued before the current tile is evaluated; every point is then evaluated
// from shared memory with the same expressions as the reference.  Within one
// phase no point reads a value that another point of that phase writes, so
// staging a tile ahead of the writes of the tile before it is exact.
//
// A window's rows start at a 16-byte column: tiles start at column
// j0 = 1 + kTileJ t, so the first column j0 + C0 of a window sits kShift elements
// into its 16-byte group for every tile, and the window is stored from column
// j0 + C0 - kShift with a row pitch of kPitch elements (a multiple of 16 bytes).
// That is the TMA box, whose x coordinate is then 16-byte aligned as TMA
// requires; the element-wise copies use the same layout.
// ---------------------------------------------------------------------------
#define AT(a, i, j) (a)[(size_t)(i) * P + (j)]

// Rows [r0, r0 + NR) x columns [c0, c0 + NC) of a pitched plane whose rows
// 0..rmax and columns 0..P-1 exist, copied element by element into dst (row
// pitch PITCH, column c0 at SHIFT).  Elements outside the plane are not copied
// (and never read by the phases).
template <int NR, int NC, int PITCH, int SHIFT, typename E>
__device__ __forceinline__ void stage_region(E* dst, const E* src, int P, int rmax, int r0, int c0) {
  for (int k = threadIdx.x; k < NR * NC; k += kThreads) {
    const int r = k / NC, c = k - r * NC;
    const int gi = r0 + r, gj = c0 + c;
    if (gi >= 0 && gi <= rmax && gj >= 0 && gj < P) cp_async_elem(dst + r * PITCH + c + SHIFT, src + (size_t)gi * P + gj);
  }
}

// A tile's window onto one plane: rows i0+R0 .. i0+R0+NR-1 and columns
// j0+C0 .. j0+C0+NC-1, indexed by global (i, j).
template <typename E, int R0, int NR, int C0, int NC>
struct Staged {
  using Elem = E;
  static constexpr int kAlign = 16 / (int)sizeof(E);                     // elements per 16 bytes
  static constexpr int kShift = ((1 + C0) % kAlign + kAlign) % kAlign;    // column j0 + C0 within its 16-byte group
  static constexpr int kPitch = (NC + kShift + kAlign - 1) / kAlign * kAlign;
  static constexpr int kRows = NR;
  static constexpr int kElems = NR * NC;  // logical elements
  static constexpr unsigned kBoxBytes = (unsigned)(NR * kPitch * sizeof(E));
  static constexpr size_t kBytes = (kBoxBytes + 127) / 128 * 128;  // the next window stays 128-byte aligned
  E* s;
  int i0, j0;
  __device__ __forceinline__ E operator()(int i, int j) const {
    return s[(i - i0 - R0) * kPitch + (j - j0 - C0 + kShift)];
  }
  // the k-th logical element (row-major over NR x NC), for loops that fill a window
  __device__ __forceinline__ E& ref(int k) const {
    const int r = k / NC;
    return s[r * kPitch + (k - r * NC) + kShift];
  }
  // the window as one TMA tile copy of `map` (issued by one thread)
  __device__ __forceinline__ void tma(const TensorMap* map, unsigned long long* bar) const {
    tma_load_2d(s, map, j0 + C0 - kShift, i0 + R0, bar, kBoxBytes);
  }
  // the window element by element (every thread of the CTA)
  __device__ __forceinline__ void elems(const E* src, int P, int rmax) const {
    stage_region<NR, NC, kPitch, kShift>(s, src, P, rmax, i0 + R0, j0 + C0);
  }
  // (i, j) of the k-th logical element
  __device__ __forceinline__ void coords(int k, int& i, int& j) const {
    const int r = k / NC;
    i = i0 + R0 + r;
    j = j0 + C0 + (k - r * NC);
  }
};

// Column 0 of a plane (gamma's inlet column) for rows i0+R0 .. i0+R0+NR-1,
// copied as the 16-byte column pair 0..1.
template <int R0, int NR>
struct StagedCol0 {
  static constexpr int kPitch = 2;
  static constexpr int kRows = NR;
  static constexpr unsigned kBoxBytes = (unsigned)(NR * kPitch * sizeof(double));
  static constexpr size_t kBytes = (kBoxBytes + 127) / 128 * 128;
  double* s;
  int i0;
  __device__ __forceinline__ double operator()(int row) const { return s[(row - i0 - R0) * kPitch]; }
  __device__ __forceinline__ void tma(const TensorMap* map, unsigned long long* bar) const {
    tma_load_2d(s, map, 0, i0 + R0, bar, kBoxBytes);
  }
  __device__ __forceinline__ void elems(const double* src, int P, int rmax) const {
    stage_region<NR, 1, kPitch, 0>(s, src, P, rmax, i0 + R0, 0);
  }
};

// Carves consecutive windows out of one tile buffer.
struct Carver {
  char* p;
  template <class W>
  __device__ __forceinline__ W take(int i0, int j0) {
    W w{reinterpret_cast<typename W::Elem*>(p), i0, j0};
    p += W::kBytes;
    return w;
  }
  template <class W>
  __device__ __forceinline__ W take_col(int i0) {
    W w{reinterpret_cast<double*>(p), i0};
    p += W::kBytes;
    return w;
  }
};

// Walk the CTA's tiles t = rank, rank + nblk, ... (the order every phase uses
// for its per-thread sums).  Layout(buffer, i0, j0) names the tile's windows;
// with the design's tensor maps thread 0 issues a tile's copies with
// stage_tma(L, tm, bar) and arrives on the buffer's mbarrier, else every
// thread copies with stage_elems(L); compute(L, i, j, inside) evaluates the
// thread's point (i, j) (inside: the point lies in 1..M-1 x 1..N-1; every
// thread of the CTA calls compute, so compute may use __syncthreads).
// kStageDepth tiles are in flight.  Every thread waits for a TMA buffer's
// phase at most kTmaTimeoutNs; a copy that has not landed by then records
// kStatusTimeout, the CTA waits up to kTmaDrainNs for its other copies in
// flight and the walk returns false (the caller then stops).  tbuf is
// 128-byte aligned.
template <class Layout, class Group, class StageTma, class StageElems, class Compute>
__device__ __forceinline__ bool for_each_tile(const DesignView& d, Group& g, char* tbuf, StageTma&& stage_tma,
                                              StageElems&& stage_elems, Compute&& compute) {
  const unsigned rank = g.rank, nblk = g.nblk;
  const int tilesJ = (d.N - 1 + kTileJ - 1) / kTileJ;
  const int tilesI = (d.M - 1 + kTileI - 1) / kTileI;
  const int nt = tilesI * tilesJ;
  const TensorMap* tm = d.tm;
  auto buf = [&](int k) { return tbuf + (size_t)(k % kStageDepth) * Layout::kBytes; };
  auto at = [&](int t, int k) {
    return Layout(buf(k), 1 + (t / tilesJ) * kTileI, 1 + (t % tilesJ) * kTileJ);
  };
  auto issue = [&](int t, int k) {
    if (tm) {
      if (threadIdx.x == 0) {
        unsigned long long* bar = s_tma_bar + (k % kStageDepth);
        stage_tma(at(t, k), tm, bar);
        mbar_arrive(bar);
      }
    } else {
      stage_elems(at(t, k));
    }
  };
  if (tm) {
    // earlier generic-proxy accesses to the buffers come before the copies
    fence_proxy_async_shared();
    __syncthreads();
  }
#pragma unroll
  for (int k = 0; k < kStageDepth - 1; ++k) {
    const int t = (int)rank + k * (int)nblk;
    if (t < nt) issue(t, k);
    if (!tm) cp_async_commit();
  }
  int k = 0;
  for (int t = (int)rank; t < nt; t += (int)nblk, ++k) {
    const int tn = t + (kStageDepth - 1) * (int)nblk;
    if (tn < nt) issue(tn, k + kStageDepth - 1);
    bool late = false;
    if (tm) {
      const int b = k % kStageDepth;
      late = !mbar_wait_bounded(s_tma_bar + b, s_tma_parity[b], kTmaTimeoutNs);
    } else {
      cp_async_commit();
      cp_async_wait<kStageDepth - 1>();
    }
    if (__syncthreads_or(late)) {
      // a tile copy did not land: record it, wait (bounded) for this tile's
      // and the later tiles' copies still in flight, and stop
      if (threadIdx.x == 0 && g.status) atomicCAS(g.status, kStatusOk, kStatusTimeout);
      for (int q = 0; q < kStageDepth; ++q)
        if (t + q * (int)nblk < nt) {
          const int b = (k + q) % kStageDepth;
          mbar_wait_bounded(s_tma_bar + b, s_tma_parity[b], kTmaDrainNs);
        }
      return false;
    }
    const Layout L = at(t, k);
    const int i = L.i0 + (int)threadIdx.x / kTileJ, j = L.j0 + (int)threadIdx.x % kTileJ;
    compute(L, i, j, i <= d.M - 1 && j <= d.N - 1);
    __syncthreads();  // the buffer is restaged next round
    // every thread has waited on this buffer's phase; the next wait on it is
    // kStageDepth tiles later, after more barriers
    if (tm && threadIdx.x == 0) s_tma_parity[k % kStageDepth] ^= 1u;
  }
  return true;
}

// Tile iteration without staging: the same points in the same order, loads
// straight from global memory.
template <class F>
__device__ __forceinline__ void for_each_point(const DesignView& d, unsigned rank, unsigned nblk, F&& f) {
  const int tilesJ = (d.N - 1 + kTileJ - 1) / kTileJ;
  const int tilesI = (d.M - 1 + kTileI - 1) / kTileI;
  const int ty = (int)threadIdx.x / kTileJ, tx = (int)threadIdx.x % kTileJ;
  for (int t = rank; t < tilesI * tilesJ; t += nblk) {
    const int i = 1 + (t / tilesJ) * kTileI + ty;
    const int j = 1 + (t % tilesJ) * kTileJ + tx;
    if (i <= d.M - 1 && j <= d.N - 1) f(i, j);
  }
}

// ---------------------------------------------------------------------------
// Phase A: momentum assembly + Jacobi sweep 1
// ---------------------------------------------------------------------------
struct LayoutA {
  using WU = Staged<double, -2, kTileI + 4, -2, kTileJ + 4>;  // u, v: SOU reaches two cells
  using WP = Staged<double, 0, kTileI + 1, 0, kTileJ + 1>;
  using WA = Staged<double, -1, kTileI + 1, -1, kTileJ + 1>;
  static constexpr size_t kBytes = 2 * WU::kBytes + WP::kBytes + WA::kBytes;
  int i0, j0;
  WU u, v;
  WP p;
  WA a;
  __device__ __forceinline__ LayoutA(char* b, int i0_, int j0_) : i0(i0_), j0(j0_) {
    Carver c{b};
    u = c.take<WU>(i0, j0);
    v = c.take<WU>(i0, j0);
    p = c.take<WP>(i0, j0);
    a = c.take<WA>(i0, j0);
  }
};

// SOU deferred correction, convection.cpp:53-118 (U) and :121-186 (V); the two
// components' range guards differ and are kept as in the reference.
template <bool IsU, class X>
__device__ __forceinline__ double sou_correction(const DesignView& d, const X& x, int i, int j, double Fe, double Fw,
                                                 double Fn, double Fs) {
  const int M = d.M, N = d.N;
  double Sdc = 0.0;
  if (Fe >= 0.0) {
    if (j >= 2) Sdc -= Fe * ((1.5 * x(i, j) - 0.5 * x(i, j - 1)) - x(i, j));
  } else {
    if (IsU ? (j + 2 < N) : (j + 2 <= N)) Sdc -= Fe * ((1.5 * x(i, j + 1) - 0.5 * x(i, j + 2)) - x(i, j + 1));
  }
  if (Fw >= 0.0) {
    if (j >= 2) Sdc += Fw * ((1.5 * x(i, j - 1) - 0.5 * x(i, j - 2)) - x(i, j - 1));
  } else {
    if (IsU ? (j + 1 < N) : (j + 1 <= N)) Sdc += Fw * ((1.5 * x(i, j) - 0.5 * x(i, j + 1)) - x(i, j));
  }
  if (Fn >= 0.0) {
    if (i >= 1) Sdc -= Fn * ((1.5 * x(i, j) - 0.5 * x(i - 1, j)) - x(i, j));
  } else {
    if (IsU ? (i + 2 <= M) : (i + 2 < M)) Sdc -= Fn * ((1.5 * x(i + 1, j) - 0.5 * x(i + 2, j)) - x(i + 1, j));
  }
  if (Fs >= 0.0) {
    if (i >= 2) Sdc += Fs * ((1.5 * x(i - 1, j) - 0.5 * x(i - 2, j)) - x(i - 1, j));
  } else {
    if (IsU ? (i + 1 <= M) : (i + 1 < M)) Sdc += Fs * ((1.5 * x(i, j) - 0.5 * x(i + 1, j)) - x(i, j));
  }
  return Sdc;
}

// The momentum row of one unknown (momentum_solver.cpp:203-296): the
// coefficients of its unknown neighbours (negated; 0 where the neighbour is
// not an unknown), the relaxed diagonal aP, the source Sp with the neighbours
// that are not unknowns folded in at their current values, the current
// velocity, and h / aP0 (dE for U, dN for V) in dOut.  Phase A and the
// re-assembling sweep 2 both evaluate it from the same staged inputs, so they
// get the same bits.
struct MomRow {
  double cE, cW, cN, cS, aP, Sp, velCur;
  bool hasE, hasW, hasN, hasS;
};

template <bool IsU, bool Pseudo>
__device__ __forceinline__ MomRow momentum_row(const DesignView& d, const LayoutA& L, int i, int j, double cfl,
                                               double& dOut) {
  const int M = d.M, N = d.N;
  const auto& u = L.u;
  const auto& v = L.v;
  const double mv = d.maxVel;
  double alphaLocal, ue, uw, vn, vs;
  if (IsU) {
    alphaLocal = 0.5 * (L.a(i - 1, j - 1) + L.a(i - 1, j));
    ue = clampd(0.5 * (u(i, j) + u(i, j + 1)), -mv, mv);
    uw = clampd(0.5 * (u(i, j - 1) + u(i, j)), -mv, mv);
    vn = clampd(0.5 * (v(i, j) + v(i, j + 1)), -mv, mv);
    vs = clampd(0.5 * (v(i - 1, j) + v(i - 1, j + 1)), -mv, mv);
  } else {
    alphaLocal = 0.5 * (L.a(i - 1, j - 1) + L.a(i, j - 1));
    ue = clampd(0.5 * (u(i, j) + u(i + 1, j)), -mv, mv);
    uw = clampd(0.5 * (u(i, j - 1) + u(i + 1, j - 1)), -mv, mv);
    vn = clampd(0.5 * (v(i, j) + v(i + 1, j)), -mv, mv);
    vs = clampd(0.5 * (v(i - 1, j) + v(i, j)), -mv, mv);
  }
  const double Fe = d.Fcx * ue, Fw = d.Fcx * uw, Fn = d.Fcy * vn, Fs = d.Fcy * vs;
  const double aE = d.De + maxd(0.0, -Fe), aW = d.De + maxd(0.0, Fw);
  const double aN = d.Dn + maxd(0.0, -Fn), aS = d.Dn + maxd(0.0, Fs);
  const double sumA = aE + aW + aN + aS;
  const auto& X = IsU ? u : v;
  MomRow m;
  m.velCur = X(i, j);
  const double transCoeff = (Pseudo && d.pseudo) ? trans_implicit(d, cfl, m.velCur) : 0.0;
  const double brinkmanDrag = alphaLocal * d.vol;
  double aP0 = sumA + (Fe - Fw + Fn - Fs) + transCoeff + d.sinkDiag + brinkmanDrag;
  aP0 = maxd(aP0, 1e-10);
  m.aP = aP0 / d.uvAlpha;
  double Sp = IsU ? (L.p(i, j) - L.p(i, j + 1)) * d.hy : (L.p(i, j) - L.p(i + 1, j)) * d.hx;
  Sp += transCoeff * m.velCur;
  Sp += d.relax * aP0 * m.velCur;
  if (d.conv == 1) Sp += sou_correction<IsU>(d, X, i, j, Fe, Fw, Fn, Fs);
  dOut = (IsU ? d.hy : d.hx) / aP0;
  const int iHi = IsU ? M - 1 : M - 2, jHi = IsU ? N - 2 : N - 1;
  m.hasE = j + 1 <= jHi;
  m.hasW = j - 1 >= 1;
  m.hasN = i + 1 <= iHi;
  m.hasS = i - 1 >= 1;
  m.cE = m.cW = m.cN = m.cS = 0.0;
  if (m.hasE) m.cE = -aE; else Sp += aE * X(i, j + 1);
  if (m.hasW) m.cW = -aW; else Sp += aW * X(i, j - 1);
  if (m.hasN) m.cN = -aN; else Sp += aN * X(i + 1, j);
  if (m.hasS) m.cS = -aS; else Sp += aS * X(i - 1, j);
  m.Sp = Sp;
  return m;
}

// The row times the current velocities (sweep 1's x0), in the reference's CSR
// order S, W, P, E, N (jacobi_solver.cpp:49-55).
template <bool IsU>
__device__ __forceinline__ double row_times_current(const MomRow& m, const LayoutA& L, int i, int j) {
  const auto& X = IsU ? L.u : L.v;
  double Ax = 0.0;
  if (m.hasS) Ax += m.cS * X(i - 1, j);
  if (m.hasW) Ax += m.cW * X(i, j - 1);
  Ax += m.aP * m.velCur;
  if (m.hasE) Ax += m.cE * X(i, j + 1);
  if (m.hasN) Ax += m.cN * X(i + 1, j);
  return Ax;
}

// Stores the row of one unknown and its source (FP64: b = Sp; mixed: b = r0)
// in the storage type T the Jacobi sweeps read.
template <bool IsU, typename T>
__device__ __forceinline__ void store_row(const DesignView& d, size_t o, T cE, T cW, T cN, T cS, T aP, T b) {
  const Inner<T>& w = inner<T>(d);
  T* c = IsU ? w.cU : w.cV;
  const long long ps = d.planeStride;
  c[o] = cE;
  c[o + ps] = cW;
  c[o + 2 * ps] = cN;
  c[o + 3 * ps] = cS;
  c[o + 4 * ps] = aP;
  (IsU ? w.bU : w.bV)[o] = b;
}

// Momentum assembly at one unknown fused with Jacobi sweep 1
// (jacobi_solver.cpp:49-57, x0 = current velocity).  Stores dE or dN, the
// sweep's result and, with `storeRow`, the row for the sweeps after it (a
// second sweep re-assembles the row when it was not stored).  Returns the
// squared residual of sweep 1 (0 when no sweep is run).
//   FP64:  b = Sp, x1 = x0 + (b - A x0)/aP.
//   mixed: b = r0 = Sp - A x0 (FP64 defect), delta1 = r0/aP (delta0 = 0).
template <bool IsU, typename T, bool Pseudo>
__device__ __forceinline__ double assemble_point(const DesignView& d, const LayoutA& L, int i, int j, bool sweep,
                                                 double cfl, bool storeRow) {
  constexpr bool kMixed = sizeof(T) == 4;
  const Inner<T>& w = inner<T>(d);
  double dv;
  const MomRow m = momentum_row<IsU, Pseudo>(d, L, i, j, cfl, dv);
  const size_t o = (size_t)i * d.P + j;
  (IsU ? d.dE : d.dN)[o] = dv;
  if (!sweep) {
    (IsU ? w.xU0 : w.xV0)[o] = kMixed ? (T)0.0 : (T)m.velCur;
    return 0.0;
  }
  const double r = m.Sp - row_times_current<IsU>(m, L, i, j);
  if (storeRow)
    store_row<IsU, T>(d, o, (T)m.cE, (T)m.cW, (T)m.cN, (T)m.cS, (T)m.aP, kMixed ? (T)r : (T)m.Sp);
  if (kMixed) {
    (IsU ? w.xU1 : w.xV1)[o] = (T)(r / m.aP);
    return r * r;
  }
  (IsU ? w.xU1 : w.xV1)[o] = (T)(m.velCur + r / m.aP);
  return r * r;
}

// Jacobi sweep 2 at one unknown (jacobi_solver.cpp:49-57) with the row
// re-assembled from the staged inputs of phase A (the same bits phase A
// computed), in the storage type T the later sweeps read: the row and its
// source (FP64: b = Sp; mixed: b = r0) are stored for them when `store`.
template <bool IsU, typename T, bool Pseudo>
__device__ __forceinline__ double sweep2_point(const DesignView& d, const LayoutA& L, int i, int j, double cfl,
                                               const T* __restrict__ xin, T* __restrict__ xout, bool store) {
  constexpr bool kMixed = sizeof(T) == 4;
  const Inner<T>& w = inner<T>(d);
  const int P = d.P;
  double dv;
  const MomRow m = momentum_row<IsU, Pseudo>(d, L, i, j, cfl, dv);
  const size_t o = (size_t)i * P + j;
  const T cE = (T)m.cE, cW = (T)m.cW, cN = (T)m.cN, cS = (T)m.cS, aPt = (T)m.aP;
  const T bt = kMixed ? (T)(m.Sp - row_times_current<IsU>(m, L, i, j)) : (T)m.Sp;
  if (store) store_row<IsU, T>(d, o, cE, cW, cN, cS, aPt, bt);
  double Ax = 0.0;
  if (m.hasS) Ax += (double)cS * (double)xin[o - P];
  if (m.hasW) Ax += (double)cW * (double)xin[o - 1];
  const double aP = (double)aPt;
  const double x0 = (double)xin[o];
  Ax += aP * x0;
  if (m.hasE) Ax += (double)cE * (double)xin[o + 1];
  if (m.hasN) Ax += (double)cN * (double)xin[o + P];
  const double r = (double)bt - Ax;
  xout[o] = (T)(x0 + r / aP);
  return r * r;
}

// The explicit momentum update at one unknown (momentumSolverType = 0,
// iterations.cpp:254-412; with the pseudo-transient term off its coefficient
// is rho vol / inf = 0): the full coefficients, one point update from the
// current velocities, clamped to +-maxVel; d = h / max(aP0, 1e-12).  Its
// result goes where phase C reads the final Jacobi iterate (FP64: the value;
// mixed: its difference to the current velocity).
template <bool IsU, typename T, bool Pseudo>
__device__ __forceinline__ void explicit_point(const DesignView& d, const LayoutA& L, int i, int j, double cfl) {
  constexpr bool kMixed = sizeof(T) == 4;
  const Inner<T>& w = inner<T>(d);
  const int P = d.P;
  const auto& u = L.u;
  const auto& v = L.v;
  const double mv = d.maxVel;
  auto clampv = [&](double x) { return maxd(-mv, mind(mv, x)); };  // std::max(-maxVel, std::min(maxVel, x))
  double alphaLocal, ue, uw, vn, vs;
  if (IsU) {
    alphaLocal = 0.5 * (L.a(i - 1, j - 1) + L.a(i - 1, j));
    ue = clampv(0.5 * (u(i, j) + u(i, j + 1)));
    uw = clampv(0.5 * (u(i, j - 1) + u(i, j)));
    vn = clampv(0.5 * (v(i, j) + v(i, j + 1)));
    vs = clampv(0.5 * (v(i - 1, j) + v(i - 1, j + 1)));
  } else {
    alphaLocal = 0.5 * (L.a(i - 1, j - 1) + L.a(i, j - 1));
    ue = clampv(0.5 * (u(i, j) + u(i + 1, j)));
    uw = clampv(0.5 * (u(i, j - 1) + u(i + 1, j - 1)));
    vn = clampv(0.5 * (v(i, j) + v(i + 1, j)));
    vs = clampv(0.5 * (v(i - 1, j) + v(i, j)));
  }
  const double Fe = d.Fcx * ue, Fw = d.Fcx * uw, Fn = d.Fcy * vn, Fs = d.Fcy * vs;
  const double aE = d.De + maxd(0.0, -Fe), aW = d.De + maxd(0.0, Fw);
  const double aN = d.Dn + maxd(0.0, -Fn), aS = d.Dn + maxd(0.0, Fs);
  const auto& X = IsU ? u : v;
  const double Sdc = (d.conv == 1) ? sou_correction<IsU>(d, X, i, j, Fe, Fw, Fn, Fs) : 0.0;
  const double sumA = aE + aW + aN + aS;
  const double velCur = X(i, j);
  const double transCoeffLocal = (Pseudo && d.pseudo) ? trans_explicit(d, cfl, velCur) : 0.0;
  const double brinkmanDrag = alphaLocal * d.vol;
  double aP0 = sumA + (Fe - Fw + Fn - Fs) + transCoeffLocal + d.sinkDiag + brinkmanDrag;
  aP0 = maxd(aP0, 1e-10);
  const double dDenom = maxd(aP0, 1e-12);
  const size_t o = (size_t)i * P + j;
  double Sp;
  if (IsU) {
    d.dE[o] = d.hy / dDenom;
    Sp = (L.p(i, j) - L.p(i, j + 1)) * d.hy;
  } else {
    d.dN[o] = d.hx / dDenom;
    Sp = (L.p(i, j) - L.p(i + 1, j)) * d.hx;
  }
  Sp += transCoeffLocal * velCur;
  Sp += Sdc;
  const double aP = aP0 / d.uvAlpha;
  Sp += d.relax * aP0 * velCur;
  double xNew = (aE * X(i, j + 1) + aW * X(i, j - 1) + aN * X(i + 1, j) + aS * X(i - 1, j) + Sp) / aP;
  xNew = clampv(xNew);
  (IsU ? w.xU0 : w.xV0)[o] = kMixed ? (T)(xNew - velCur) : (T)xNew;
}

// ---------------------------------------------------------------------------
// Phase B: Jacobi sweep k >= 2 at one unknown (jacobi_solver.cpp:49-57),
// arithmetic in FP64 on the stored values, loaded straight from global memory
// (sweep_point).  With tensor maps and DesignView::stageSweeps a tile's five
// coefficient windows, its source window and its iterate window (halo 1) are
// staged by TMA instead (sweep_point_staged; 7 copies per active component,
// issued by one thread): the same expressions in the same order, the same
// bits, but not faster on B200 (the sweeps are not bound by their loads'
// latency), so it is off by default; element by element the fourteen
// windows cost more than they save.
// ---------------------------------------------------------------------------
template <typename T>
struct LayoutB {
  using WC = Staged<T, 0, kTileI, 0, kTileJ>;            // a coefficient plane or the source: the tile
  using WX = Staged<T, -1, kTileI + 2, -1, kTileJ + 2>;  // the iterate and its 1-point halo
  static constexpr size_t kComp = 6 * WC::kBytes + WX::kBytes;
  static constexpr size_t kBytes = 2 * kComp;
  int i0, j0;
  WC cu[5], bu, cv[5], bv;  // cu[k]: plane k of cU (aE, aW, aN, aS, aP), bu: bU
  WX xu, xv;
  __device__ __forceinline__ LayoutB(char* b, int i0_, int j0_) : i0(i0_), j0(j0_) {
    Carver c{b};
#pragma unroll
    for (int k = 0; k < 5; ++k) cu[k] = c.take<WC>(i0, j0);
    bu = c.take<WC>(i0, j0);
    xu = c.take<WX>(i0, j0);
#pragma unroll
    for (int k = 0; k < 5; ++k) cv[k] = c.take<WC>(i0, j0);
    bv = c.take<WC>(i0, j0);
    xv = c.take<WX>(i0, j0);
  }
};

template <bool IsU, typename T>
__device__ __forceinline__ double sweep_point_staged(const DesignView& d, const LayoutB<T>& L, int i, int j,
                                                     T* __restrict__ xout) {
  const int M = d.M, N = d.N, P = d.P;
  const int iHi = IsU ? M - 1 : M - 2, jHi = IsU ? N - 2 : N - 1;
  const auto* c = IsU ? L.cu : L.cv;
  const auto& X = IsU ? L.xu : L.xv;
  double Ax = 0.0;
  if (i - 1 >= 1) Ax += (double)c[3](i, j) * (double)X(i - 1, j);
  if (j - 1 >= 1) Ax += (double)c[1](i, j) * (double)X(i, j - 1);
  const double aP = (double)c[4](i, j);
  const double x0 = (double)X(i, j);
  Ax += aP * x0;
  if (j + 1 <= jHi) Ax += (double)c[0](i, j) * (double)X(i, j + 1);
  if (i + 1 <= iHi) Ax += (double)c[2](i, j) * (double)X(i + 1, j);
  const double r = (double)(IsU ? L.bu : L.bv)(i, j) - Ax;
  xout[(size_t)i * P + j] = (T)(x0 + r / aP);
  return r * r;
}

template <bool IsU, typename T>
__device__ __forceinline__ double sweep_point(const DesignView& d, int i, int j, const T* __restrict__ xin,
                                              T* __restrict__ xout) {
  const Inner<T>& w = inner<T>(d);
  const int M = d.M, N = d.N, P = d.P;
  const int iHi = IsU ? M - 1 : M - 2, jHi = IsU ? N - 2 : N - 1;
  const T* __restrict__ c = IsU ? w.cU : w.cV;
  const long long ps = d.planeStride;
  const size_t o = (size_t)i * P + j;
  double Ax = 0.0;
  if (i - 1 >= 1) Ax += (double)c[o + 3 * ps] * (double)xin[o - P];
  if (j - 1 >= 1) Ax += (double)c[o + ps] * (double)xin[o - 1];
  const double aP = (double)c[o + 4 * ps];
  const double x0 = (double)xin[o];
  Ax += aP * x0;
  if (j + 1 <= jHi) Ax += (double)c[o] * (double)xin[o + 1];
  if (i + 1 <= iHi) Ax += (double)c[o + 2 * ps] * (double)xin[o + P];
  const double r = (double)(IsU ? w.bU : w.bV)[o] - Ax;
  xout[o] = (T)(x0 + r / aP);
  return r * r;
}

// ---------------------------------------------------------------------------
// PCG as the reference runs it (pressure_solver.cpp:121-184): two grid-wide
// reductions per iteration (p.Ap, then |r|^2 and r.z).  Phase P1 forms
// p = z + beta p on the fly for the 5-point stencil and Ap; phase P2 updates
// x, r, z.  Both load straight from global memory, every load of a point
// issued before its first store so that the loads overlap (staging these two
// light phases through shared memory measured slower on B200).  Returns the
// reference's iteration count, or -1 if a wait failed.
// ---------------------------------------------------------------------------
template <typename T, class Group>
__device__ int pcg_two_reductions(const DesignView& d, Group& g, double* smem, double rz0, double pAp0) {
  const Inner<T>& w = inner<T>(d);
  const int M = d.M, N = d.N, P = d.P;
  double rz = rz0, beta = 0.0;
  int it = 0;
  for (; it < d.maxPIter; ++it) {
    const T* pold = (it & 1) ? w.pp0 : w.pp1;  // p_{it-1}
    T* pcur = (it & 1) ? w.pp1 : w.pp0;        // p_it
    const double bt = beta;
    double s1[1] = {pAp0};  // iteration 0's p = z, A p and p.Ap come from phase C
    if (it > 0) {
      s1[0] = 0.0;
      for_each_point(d, g.rank, g.nblk, [&](int i, int j) {
        if (j > N - 2) return;
        const size_t o = (size_t)i * P + j;
        // p_k at (i, j) and its unknown neighbours: p = z + beta p (pressure_solver.cpp:181)
        auto pk = [&](size_t q) -> double { return (double)(T)((double)w.pz[q] + bt * (double)pold[q]); };
        const double pc0 = pk(o);
        double Ap = 0.0;
        if (i > 1) Ap += -(double)w.cy[o - P] * pk(o - P);
        if (j > 1) Ap += -(double)w.cx[o - 1] * pk(o - 1);
        Ap += (double)w.pdiag[o] * pc0;
        if (j + 1 <= N - 2) Ap += -(double)w.cx[o] * pk(o + 1);
        if (i < M - 1) Ap += -(double)w.cy[o] * pk(o + P);
        pcur[o] = (T)pc0;
        const T apt = (T)Ap;
        w.pAp[o] = apt;
        s1[0] += pc0 * (double)apt;
      });
      if (!g.template sync_reduce<1, 0u>(s1, smem)) return -1;
    }
    const double pAp = s1[0];
    if (fabs(pAp) < 1e-20) break;
    const double alpha = rz / pAp;
    double s2[2] = {0.0, 0.0};  // |r|^2, r.z
    for_each_point(d, g.rank, g.nblk, [&](int i, int j) {
      if (j > N - 2) return;
      const size_t o = (size_t)i * P + j;
      const T xo = w.px[o], pc = pcur[o], ro = w.pr[o], ap = w.pAp[o], dgo = w.pdiag[o];
      w.px[o] = (T)((double)xo + alpha * (double)pc);
      const T rt = (T)((double)ro - alpha * (double)ap);
      w.pr[o] = rt;
      const double r = (double)rt;
      s2[0] += r * r;
      const double dg = (double)dgo;
      const T z = (T)((fabs(dg) > 1e-20) ? r / dg : r);
      w.pz[o] = z;
      s2[1] += r * (double)z;
    });
    if (!g.template sync_reduce<2, 0u>(s2, smem)) return -1;
    if (sqrt(s2[0]) < d.pTol) break;
    const double rzPrev = rz;
    rz = s2[1];
    beta = rz / rzPrev;
  }
  return it;
}

// ---------------------------------------------------------------------------
// The same PCG for groups in which a thread owns at most R unknowns (every
// CTA has at most R tiles): each thread keeps its unknowns' x, r, z, p, Ap,
// diagonal and face conductances in registers for the whole solve, so P2
// reads no memory (it stores x for phase D and z for the neighbours) and P1
// loads only the neighbours' z and p_{k-1} (and stores p_k for them).  The
// arithmetic, the points' order and so every sum are those of
// pcg_two_reductions.
// ---------------------------------------------------------------------------
template <typename T, int R, class Group>
__device__ int pcg_resident(const DesignView& d, Group& g, double* smem, double rz0, double pAp0) {
  const Inner<T>& w = inner<T>(d);
  const int M = d.M, N = d.N, P = d.P;
  const int tilesJ = (N - 1 + kTileJ - 1) / kTileJ;
  const int tilesI = (M - 1 + kTileI - 1) / kTileI;
  const int nt = tilesI * tilesJ;
  const int ty = (int)threadIdx.x / kTileJ, tx = (int)threadIdx.x % kTileJ;
  bool on[R];
  int ii[R], jj[R];
  size_t oo[R];
  T x[R], r[R], z[R], p[R], ap[R], dg[R], cE[R], cW[R], cN[R], cS[R];
#pragma unroll
  for (int u = 0; u < R; ++u) {
    const int t = (int)g.rank + u * (int)g.nblk;
    ii[u] = 1 + (t / tilesJ) * kTileI + ty;
    jj[u] = 1 + (t % tilesJ) * kTileJ + tx;
    on[u] = t < nt && ii[u] <= M - 1 && jj[u] <= N - 2;
    oo[u] = on[u] ? (size_t)ii[u] * P + jj[u] : 0;
    x[u] = r[u] = z[u] = p[u] = ap[u] = dg[u] = cE[u] = cW[u] = cN[u] = cS[u] = (T)0;
    if (on[u]) {
      const size_t o = oo[u];
      x[u] = w.px[o];
      r[u] = w.pr[o];
      z[u] = w.pz[o];
      p[u] = w.pp0[o];
      ap[u] = w.pAp[o];
      dg[u] = w.pdiag[o];
      cE[u] = w.cx[o];
      cN[u] = w.cy[o];
      if (jj[u] > 1) cW[u] = w.cx[o - 1];
      if (ii[u] > 1) cS[u] = w.cy[o - P];
    }
  }
  double rz = rz0, beta = 0.0;
  int it = 0;
  for (; it < d.maxPIter; ++it) {
    const T* pold = (it & 1) ? w.pp0 : w.pp1;  // p_{it-1}
    T* pcur = (it & 1) ? w.pp1 : w.pp0;        // p_it
    const double bt = beta;
    double s1[1] = {pAp0};  // iteration 0's p = z, A p and p.Ap come from phase C
    if (it > 0) {
      s1[0] = 0.0;
      T zn[R][4], pn[R][4];  // z and p_{k-1} at the S, W, E, N neighbours
#pragma unroll
      for (int u = 0; u < R; ++u) {
#pragma unroll
        for (int q = 0; q < 4; ++q) zn[u][q] = pn[u][q] = (T)0;
        if (on[u]) {
          const size_t o = oo[u];
          if (ii[u] > 1) { zn[u][0] = w.pz[o - P]; pn[u][0] = pold[o - P]; }
          if (jj[u] > 1) { zn[u][1] = w.pz[o - 1]; pn[u][1] = pold[o - 1]; }
          if (jj[u] + 1 <= N - 2) { zn[u][2] = w.pz[o + 1]; pn[u][2] = pold[o + 1]; }
          if (ii[u] < M - 1) { zn[u][3] = w.pz[o + P]; pn[u][3] = pold[o + P]; }
        }
      }
#pragma unroll
      for (int u = 0; u < R; ++u) {
        if (!on[u]) continue;
        const int i = ii[u], j = jj[u];
        // p = z + beta p (pressure_solver.cpp:181) at the point and its unknown neighbours
        auto pk = [&](T zq, T pq) -> double { return (double)(T)((double)zq + bt * (double)pq); };
        const double pc0 = pk(z[u], p[u]);
        double Ap = 0.0;
        if (i > 1) Ap += -(double)cS[u] * pk(zn[u][0], pn[u][0]);
        if (j > 1) Ap += -(double)cW[u] * pk(zn[u][1], pn[u][1]);
        Ap += (double)dg[u] * pc0;
        if (j + 1 <= N - 2) Ap += -(double)cE[u] * pk(zn[u][2], pn[u][2]);
        if (i < M - 1) Ap += -(double)cN[u] * pk(zn[u][3], pn[u][3]);
        p[u] = (T)pc0;
        pcur[oo[u]] = p[u];
        ap[u] = (T)Ap;
        s1[0] += pc0 * (double)ap[u];
      }
      if (!g.template sync_reduce<1, 0u>(s1, smem)) return -1;
    }
    const double pAp = s1[0];
    if (fabs(pAp) < 1e-20) break;
    const double alpha = rz / pAp;
    double s2[2] = {0.0, 0.0};  // |r|^2, r.z
#pragma unroll
    for (int u = 0; u < R; ++u) {
      if (!on[u]) continue;
      x[u] = (T)((double)x[u] + alpha * (double)p[u]);
      w.px[oo[u]] = x[u];
      const T rt = (T)((double)r[u] - alpha * (double)ap[u]);
      r[u] = rt;
      const double rr = (double)rt;
      s2[0] += rr * rr;
      const double dgd = (double)dg[u];
      const T zz = (T)((fabs(dgd) > 1e-20) ? rr / dgd : rr);
      z[u] = zz;
      w.pz[oo[u]] = zz;
      s2[1] += rr * (double)zz;
    }
    if (!g.template sync_reduce<2, 0u>(s2, smem)) return -1;
    if (sqrt(s2[0]) < d.pTol) break;
    const double rzPrev = rz;
    rz = s2[1];
    beta = rz / rzPrev;
  }
  return it;
}

// ---------------------------------------------------------------------------
// The same PCG with the CTA's unknowns in shared memory, for groups in which a
// CTA owns more tiles than fit in registers but at most R (SmemTiles<T>): r,
// z, p, Ap and the east/north face conductances of every point of the CTA's
// tiles (mixed: also the diagonal and x) are loaded once, and each PCG
// iteration then reads global memory only for the neighbours that lie in
// another tile (the ring around each tile: z and p_{k-1}, copied with
// cp.async for all tiles at once, each thread into halo slots only it reads).
//   P1 forms p_k = z + beta p_{k-1} once at each of the CTA's points, in
//   place, then (after a CTA barrier) Ap from it, and from z and p_{k-1} at the
//   halo with the same expression; P2 updates x, r, z and stores p_k and z to
//   global memory for the other tiles.
// FP64 forms the diagonal from the four conductances the way phase C did (the
// stored conductances are phase C's summands, added in its order), and keeps x
// at the thread's points in registers (x + alpha p, one rounding, as P2
// forms it), storing it every iteration so that the last store precedes the
// last grid barrier and phase D reads the final x.  The points, their order
// and every sum are those of pcg_two_reductions, so the iterates are the same
// bits.
// ---------------------------------------------------------------------------
constexpr int kHalo = 2 * kTileJ + 2 * kTileI;  // a tile's south row, north row, west column, east column

template <typename T>
struct SmemTiles {
  static constexpr int value = sizeof(T) == 8 ? 7 : 12;
};

template <typename T, int R>
struct PcgSmem {
  static constexpr int kM = sizeof(T) == 4 ? R : 1;  // arrays the mixed mode keeps in addition
  T r[R][kThreads], z[R][kThreads], p[R][kThreads], ap[R][kThreads], cE[R][kThreads], cN[R][kThreads];
  T dg[kM][kThreads], x[kM][kThreads];
  T zH[R][kHalo], pH[R][kHalo];      // z and p_{k-1} at the neighbours in other tiles
  T cWH[R][kTileI], cSH[R][kTileJ];  // the west / south conductances at the tile's west / south edge
};

template <typename T, int R, class Group>
__device__ int pcg_smem(const DesignView& d, Group& g, double* smem, char* tbuf, double rz0, double pAp0) {
  constexpr bool kMixed = sizeof(T) == 4;
  PcgSmem<T, R>& S = *reinterpret_cast<PcgSmem<T, R>*>(tbuf);
  const Inner<T>& w = inner<T>(d);
  const int M = d.M, N = d.N, P = d.P;
  const int tilesJ = (N - 1 + kTileJ - 1) / kTileJ;
  const int tilesI = (M - 1 + kTileI - 1) / kTileI;
  const int nt = tilesI * tilesJ;
  const int ty = (int)threadIdx.x / kTileJ, tx = (int)threadIdx.x % kTileJ, th = threadIdx.x;
  const int nk = (int)g.rank < nt ? (nt - 1 - (int)g.rank) / (int)g.nblk + 1 : 0;  // this CTA's tiles
  T* const pg = w.pp0;  // p_k in global memory for the other tiles (read by P1 of the next iteration)
  // the thread's point in its k-th tile; true: a pressure unknown
  auto point = [&](int k, int& i, int& j) {
    const int t = (int)g.rank + k * (int)g.nblk;
    i = 1 + (t / tilesJ) * kTileI + ty;
    j = 1 + (t % tilesJ) * kTileJ + tx;
    return i <= M - 1 && j <= N - 2;
  };
  // the west / south conductances of the thread's point in tile k
  auto cW = [&](int k, int j) -> T { return j > 1 ? (tx > 0 ? S.cE[k][th - 1] : S.cWH[k][ty]) : (T)0; };
  auto cS = [&](int k, int i) -> T { return i > 1 ? (ty > 0 ? S.cN[k][th - kTileJ] : S.cSH[k][tx]) : (T)0; };
  // the diagonal (pressure_solver.cpp:703-706 as phase C evaluates it)
  auto diag = [&](int k, int i, int j) -> double {
    if constexpr (kMixed) {
      return (double)S.dg[k][th];
    } else {
      double aP = (double)S.cE[k][th] + (double)cW(k, j) + (double)S.cN[k][th] + (double)cS(k, i);
      if (aP < 1e-20) aP = 1.0;
      return aP;
    }
  };
  // state from phase C: r0, z0, p0 = z0, A p0 and the conductances
  for (int k = 0; k < nk; ++k) {
    int i, j;
    if (!point(k, i, j)) continue;
    const size_t o = (size_t)i * P + j;
    cp_async_elem(&S.r[k][th], w.pr + o);
    cp_async_elem(&S.z[k][th], w.pz + o);
    cp_async_elem(&S.p[k][th], w.pp0 + o);
    cp_async_elem(&S.ap[k][th], w.pAp + o);
    cp_async_elem(&S.cE[k][th], w.cx + o);
    cp_async_elem(&S.cN[k][th], w.cy + o);
    if constexpr (kMixed) {
      cp_async_elem(&S.dg[k][th], w.pdiag + o);
      S.x[k][th] = (T)0;  // phase C's x0
    }
    if (tx == 0 && j > 1) cp_async_elem(&S.cWH[k][ty], w.cx + o - 1);
    if (ty == 0 && i > 1) cp_async_elem(&S.cSH[k][tx], w.cy + o - P);
  }
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  double rz = rz0, beta = 0.0;
  double xr[R];  // FP64: x at the thread's points (phase C's x0 = 0)
#pragma unroll
  for (int k = 0; k < R; ++k) xr[k] = 0.0;
  int it = 0;
  for (; it < d.maxPIter; ++it) {
    const double bt = beta;
    // p = z + beta p (pressure_solver.cpp:181)
    auto pk = [&](T zq, T pq) -> double { return (double)(T)((double)zq + bt * (double)pq); };
    double s1[1] = {pAp0};  // iteration 0's p = z, A p and p.Ap come from phase C
    if (it > 0) {
      s1[0] = 0.0;
      // the neighbours in other tiles, every tile's at once
      for (int k = 0; k < nk; ++k) {
        int i, j;
        if (!point(k, i, j)) continue;
        const size_t o = (size_t)i * P + j;
        if (ty == 0 && i > 1) {
          cp_async_elem(&S.zH[k][tx], w.pz + o - P);
          cp_async_elem(&S.pH[k][tx], pg + o - P);
        }
        if (ty == kTileI - 1 && i < M - 1) {
          cp_async_elem(&S.zH[k][kTileJ + tx], w.pz + o + P);
          cp_async_elem(&S.pH[k][kTileJ + tx], pg + o + P);
        }
        if (tx == 0 && j > 1) {
          cp_async_elem(&S.zH[k][2 * kTileJ + ty], w.pz + o - 1);
          cp_async_elem(&S.pH[k][2 * kTileJ + ty], pg + o - 1);
        }
        if (tx == kTileJ - 1 && j + 1 <= N - 2) {
          cp_async_elem(&S.zH[k][2 * kTileJ + kTileI + ty], w.pz + o + 1);
          cp_async_elem(&S.pH[k][2 * kTileJ + kTileI + ty], pg + o + 1);
        }
      }
      cp_async_commit();
      // p_it at the CTA's own points, formed once in place (the stencil below
      // and P2 read it; the value of forming it at every use)
      for (int k = 0; k < nk; ++k) {
        int i, j;
        if (!point(k, i, j)) continue;
        S.p[k][th] = (T)pk(S.z[k][th], S.p[k][th]);
      }
      cp_async_wait<0>();  // each thread reads only the halo slots it copied
      __syncthreads();     // and its tile's p_it after every thread has formed its own
      for (int k = 0; k < nk; ++k) {
        int i, j;
        if (!point(k, i, j)) continue;
        const double pc0 = (double)S.p[k][th];
        double Ap = 0.0;
        if (i > 1) {
          if (ty > 0) Ap += -(double)S.cN[k][th - kTileJ] * (double)S.p[k][th - kTileJ];
          else Ap += -(double)S.cSH[k][tx] * pk(S.zH[k][tx], S.pH[k][tx]);
        }
        if (j > 1) {
          if (tx > 0) Ap += -(double)S.cE[k][th - 1] * (double)S.p[k][th - 1];
          else Ap += -(double)S.cWH[k][ty] * pk(S.zH[k][2 * kTileJ + ty], S.pH[k][2 * kTileJ + ty]);
        }
        Ap += diag(k, i, j) * pc0;
        if (j + 1 <= N - 2) {
          const int q = 2 * kTileJ + kTileI + ty;
          Ap += -(double)S.cE[k][th] * (tx < kTileJ - 1 ? (double)S.p[k][th + 1] : pk(S.zH[k][q], S.pH[k][q]));
        }
        if (i < M - 1) {
          const int q = kTileJ + tx;
          Ap += -(double)S.cN[k][th] *
                (ty < kTileI - 1 ? (double)S.p[k][th + kTileJ] : pk(S.zH[k][q], S.pH[k][q]));
        }
        const T apt = (T)Ap;
        S.ap[k][th] = apt;
        s1[0] += pc0 * (double)apt;
      }
      if (!g.template sync_reduce<1, 0u>(s1, smem)) return -1;
    }
    const double pAp = s1[0];
    if (fabs(pAp) < 1e-20) break;
    const double alpha = rz / pAp;
    double s2[2] = {0.0, 0.0};  // |r|^2, r.z
#pragma unroll
    for (int k = 0; k < R; ++k) {  // unrolled: xr[k] stays in a register
      if (k >= nk) break;
      int i, j;
      if (!point(k, i, j)) continue;
      const size_t o = (size_t)i * P + j;
      const T pc = S.p[k][th];  // p_it (P1 formed it in place; iteration 0: p0 = z0)
      pg[o] = pc;
      if constexpr (kMixed) {
        const T xn = (T)((double)S.x[k][th] + alpha * (double)pc);
        S.x[k][th] = xn;
        w.px[o] = xn;
      } else {
        xr[k] = xr[k] + alpha * (double)pc;  // x += alpha p (pressure_solver.cpp:164)
        w.px[o] = xr[k];
      }
      const T rt = (T)((double)S.r[k][th] - alpha * (double)S.ap[k][th]);
      S.r[k][th] = rt;
      const double r = (double)rt;
      s2[0] += r * r;
      const double dgd = diag(k, i, j);
      const T zt = (T)((fabs(dgd) > 1e-20) ? r / dgd : r);
      S.z[k][th] = zt;
      w.pz[o] = zt;
      s2[1] += r * (double)zt;
    }
    if (!g.template sync_reduce<2, 0u>(s2, smem)) return -1;
    if (sqrt(s2[0]) < d.pTol) break;
    const double rzPrev = rz;
    rz = s2[1];
    beta = rz / rzPrev;
  }
  return it;
}

// ---------------------------------------------------------------------------
// Single-reduction Jacobi-PCG (Chronopoulos-Gear recurrences), selected per
// design by pcgSingleReduction: the same Krylov iterates as the reference's PCG in exact
// arithmetic, with one grid-wide reduction per iteration instead of two.
//   u0 = M^-1 r0, w0 = A u0, gamma0 = (r0,u0), delta0 = (w0,u0), alpha0 = gamma0/delta0
//   iteration k: p_k = u_k + beta_k p_{k-1};  s_k = w_k + beta_k s_{k-1}  (= A p_k)
//                x += alpha_k p_k;  r_{k+1} = r_k - alpha_k s_k;  u_{k+1} = M^-1 r_{k+1}
//                w_{k+1} = A u_{k+1};  |r_{k+1}|^2, gamma_{k+1}, delta_{k+1}  (one reduction)
//                beta_{k+1} = gamma_{k+1}/gamma_k
//                alpha_{k+1} = gamma_{k+1} / (delta_{k+1} - beta_{k+1} gamma_{k+1} / alpha_k)
// The neighbours' s_k, r_{k+1}, u_{k+1} needed by w_{k+1} = A u_{k+1} are
// recomputed from the previous iteration's planes, so each iteration is one
// phase.  Stop rules and counter as the reference (pressure_solver.cpp:152-182):
// ||r_{k+1}|| < pTol stops with count k; the (p, Ap) < 1e-20 test of iteration
// k+1 is the denominator of alpha_{k+1} and stops with count k+1.
// Plane use: x = px, r = pr/pz, s = pp0/pp1, w = pAp/cU[0], u = cU[1],
// p = cU[2]; the momentum coefficient planes are free after phase C.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T* cg1_u(const Inner<T>& w, long long ps) { return w.cU + ps; }

template <typename T, class Group>
__device__ int pcg_single_reduction(const DesignView& d, Group& g, double* smem, double gamma0, double delta0) {
  const Inner<T>& w = inner<T>(d);
  const int M = d.M, N = d.N, P = d.P;
  const long long ps = d.planeStride;
  T* const rb[2] = {w.pr, w.pz};
  T* const sb[2] = {w.pp0, w.pp1};
  T* const wb[2] = {w.pAp, w.cU};
  T* const ub = w.cU + ps;
  T* const pb = w.cU + 2 * ps;
  if (d.maxPIter <= 0) return 0;
  auto inv_diag = [&](size_t q, double r) -> double {
    const double dg = (double)w.pdiag[q];
    return (fabs(dg) > 1e-20) ? r / dg : r;
  };
  // w0 = A u0 and delta0 = (w0, u0) come from phase C
  double gam = gamma0;
  double denom = delta0;
  if (fabs(denom) < 1e-20) return 0;
  double alpha = gam / denom, beta = 0.0;
  int k = 0;
  for (; k < d.maxPIter; ++k) {
    const T* rin = rb[k & 1];
    T* rout = rb[(k + 1) & 1];
    const T* sin = sb[(k + 1) & 1];  // s_{k-1}
    T* sout = sb[k & 1];             // s_k
    const T* win = wb[k & 1];        // w_k
    T* wout = wb[(k + 1) & 1];       // w_{k+1}
    const double a = alpha, bt = beta;
    const bool first = (k == 0);
    double red[3] = {0.0, 0.0, 0.0};  // |r|^2, gamma, delta
    for_each_point(d, g.rank, g.nblk, [&](int i, int j) {
      if (j > N - 2) return;
      const size_t o = (size_t)i * P + j;
      // s_k, r_{k+1}, u_{k+1} at q (identical arithmetic at the owner and its neighbours)
      auto s_at = [&](size_t q) -> T {
        return first ? win[q] : (T)((double)win[q] + bt * (double)sin[q]);
      };
      auto r_at = [&](size_t q, T sq) -> T { return (T)((double)rin[q] - a * (double)sq); };
      auto u_at = [&](size_t q) -> double {
        const T rq = r_at(q, s_at(q));
        return (double)(T)inv_diag(q, (double)rq);
      };
      const T sc = s_at(o);
      const T rc = r_at(o, sc);
      const double uc = (double)(T)inv_diag(o, (double)rc);
      const T pk = first ? ub[o] : (T)((double)ub[o] + bt * (double)pb[o]);
      w.px[o] = (T)((double)w.px[o] + a * (double)pk);
      double Au = 0.0;
      if (i > 1) Au += -(double)w.cy[o - P] * u_at(o - P);
      if (j > 1) Au += -(double)w.cx[o - 1] * u_at(o - 1);
      Au += (double)w.pdiag[o] * uc;
      if (j + 1 <= N - 2) Au += -(double)w.cx[o] * u_at(o + 1);
      if (i < M - 1) Au += -(double)w.cy[o] * u_at(o + P);
      const T wt = (T)Au;
      pb[o] = pk;
      sout[o] = sc;
      rout[o] = rc;
      ub[o] = (T)uc;
      wout[o] = wt;
      const double rr = (double)rc;
      red[0] += rr * rr;
      red[1] += rr * uc;
      red[2] += (double)wt * uc;
    });
    if (!g.template sync_reduce<3, 0u>(red, smem)) return -1;
    if (sqrt(red[0]) < d.pTol) break;
    if (k + 1 >= d.maxPIter) { k = d.maxPIter; break; }
    const double gNew = red[1];
    const double bNew = gNew / gam;
    denom = red[2] - bNew * gNew / alpha;
    if (fabs(denom) < 1e-20) { ++k; break; }
    alpha = gNew / denom;
    beta = bNew;
    gam = gNew;
  }
  return k;
}


// ---------------------------------------------------------------------------
// Phase D: p' scatter with the outlet column p' = 0 (pressure_solver.cpp:
// 796-805), p += pAlpha p' and pressure BCs (iterations.cpp:456-467,
// boundaries.cpp:111-134), velocity correction and BCs (iterations.cpp:473-499).
// Reads p' (own point, E and N), p, dE, u*, dN, v* and gamma's inlet column;
// writes p', p, u, v and boundary copies, none of which a point of this phase
// reads.
// ---------------------------------------------------------------------------
template <typename T>
struct LayoutD {
  using WX = Staged<T, 0, kTileI + 1, 0, kTileJ + 1>;
  using WO = Staged<double, 0, kTileI, 0, kTileJ>;
  using WG = StagedCol0<-1, kTileI>;
  static constexpr size_t kBytes = WX::kBytes + 5 * WO::kBytes + WG::kBytes;
  int i0, j0;
  WX px;
  WO p, dE, us, dN, vs;
  WG g0;
  __device__ __forceinline__ LayoutD(char* b, int i0_, int j0_) : i0(i0_), j0(j0_) {
    Carver c{b};
    px = c.take<WX>(i0, j0);
    p = c.take<WO>(i0, j0);
    dE = c.take<WO>(i0, j0);
    us = c.take<WO>(i0, j0);
    dN = c.take<WO>(i0, j0);
    vs = c.take<WO>(i0, j0);
    g0 = c.take_col<WG>(i0);
  }
};

template <typename T, class Group>
__device__ bool correct_fields(const DesignView& d, Group& g, char* tbuf) {
  const Inner<T>& w = inner<T>(d);
  const int M = d.M, N = d.N, P = d.P;
  return for_each_tile<LayoutD<T>>(
      d, g, tbuf,
      [](const LayoutD<T>& L, const TensorMap* tm, unsigned long long* bar) {
        L.px.tma(tm + kTmPX_D, bar);
        L.p.tma(tm + kTmP_D, bar);
        L.dE.tma(tm + kTmDE_D, bar);
        L.us.tma(tm + kTmUS_D, bar);
        L.dN.tma(tm + kTmDN_D, bar);
        L.vs.tma(tm + kTmVS_D, bar);
        if (L.j0 == 1) L.g0.tma(tm + kTmG_D, bar);
      },
      [&](const LayoutD<T>& L) {
        L.px.elems(w.px, P, M);
        L.p.elems(d.p, P, M);
        L.dE.elems(d.dE, P, M);
        L.us.elems(d.us, P, M);
        L.dN.elems(d.dN, P, M);
        L.vs.elems(d.vs, P, M);
        if (L.j0 == 1) L.g0.elems(d.gamma, P, M - 1);
      },
      [&](const LayoutD<T>& L, int i, int j, bool inside) {
        if (!inside) return;
        const size_t o = (size_t)i * P + j;
        const double pcv = (j == N - 1) ? 0.0 : (double)L.px(i, j);
        d.pc[o] = pcv;
        const double pn = L.p(i, j) + d.pAlpha * pcv;
        d.p[o] = pn;
        if (i == 1) d.p[o - P] = pn;
        if (i == M - 1) d.p[o + P] = pn;
        if (j == 1) d.p[o - 1] = pn;
        if (j == N - 1) d.p[o + 1] = 0.0;
        const double mv = d.maxVel;
        if (j <= N - 2) {
          const double pcE = (j + 1 == N - 1) ? 0.0 : (double)L.px(i, j + 1);
          double du = L.dE(i, j) * (pcv - pcE);
          du = maxd(-mv, mind(mv, du));
          double un = L.us(i, j) + du;
          un = maxd(-mv, mind(mv, un));
          d.u[o] = un;
          if (j == N - 2) d.u[o + 1] = un;
        }
        if (i <= M - 2) {
          const double pcN = (j == N - 1) ? 0.0 : (double)L.px(i + 1, j);
          double dv = L.dN(i, j) * (pcv - pcN);
          dv = maxd(-mv, mind(mv, dv));
          double vn = L.vs(i, j) + dv;
          vn = maxd(-mv, mind(mv, vn));
          d.v[o] = vn;
          if (j == N - 1) d.v[o + 1] = vn;
        }
        // walls, inlet (boundaries.cpp:57-94)
        if (i == 1) {
          d.u[o - P] = 0.0;
          d.v[o - P] = 0.0;
          if (j == 1) { d.u[o - P - 1] = 0.0; d.v[o - P - 1] = 0.0; }
          if (j == N - 1) d.v[o - P + 1] = 0.0;
        }
        if (i == M - 1) {
          d.u[o + P] = 0.0;
          d.v[o] = 0.0;
          if (j == 1) { d.u[o + P - 1] = 0.0; d.v[o - 1] = 0.0; }
          if (j == N - 1) d.v[o + 1] = 0.0;
        }
        if (j == 1) {
          d.u[o - 1] = (L.g0(i - 1) > 0.5) ? d.Uin : 0.0;
          d.v[o - 1] = 0.0;
        }
      });
}

// ---------------------------------------------------------------------------
// Phase C: scatter + clamp + max|dx| (momentum_solver.cpp:319-337), velocity
// BCs on u*, v* (boundaries.cpp:48-106), mass imbalance (pressure_solver.cpp:
// 468-486), pressure matrix (pressure_solver.cpp:693-732) and PCG set-up
// (x0 = 0, r = b, z = r/diag, p = z; pressure_solver.cpp:121-150) with the
// first PCG product A p0 (pressure_solver.cpp:153-156).
// u* and v* are evaluated once per tile over the halo the tile needs, then z0
// over the tile and a one-cell ring, so the neighbours' z0 entering A p0 cost
// no extra memory traffic.
// ---------------------------------------------------------------------------
template <typename T>
struct LayoutC {
  using WUx = Staged<T, -1, kTileI + 2, -2, kTileJ + 3>;       // final U iterate
  using WUd = Staged<double, -1, kTileI + 2, -2, kTileJ + 3>;  // u (mixed: u + delta; both: residual), dE
  using WVx = Staged<T, -2, kTileI + 3, -1, kTileJ + 2>;       // final V iterate
  using WVd = Staged<double, -2, kTileI + 3, -1, kTileJ + 2>;  // v, dN
  using WG = StagedCol0<-2, kTileI + 2>;                      // gamma(i-1, 0) for u*(i, 0)
  using WZ = Staged<double, -1, kTileI + 2, -1, kTileJ + 2>;
  static constexpr size_t kBytes = WUx::kBytes + 2 * WUd::kBytes + WVx::kBytes + 2 * WVd::kBytes + WG::kBytes;
  // evaluated windows after the staging buffers (not double buffered)
  static constexpr size_t kExtraBytes = WUd::kBytes + WVd::kBytes + WZ::kBytes;
  int i0, j0;
  WUx xu;
  WUd u, dE;
  WVx xv;
  WVd v, dN;
  WG g0;
  __device__ __forceinline__ LayoutC(char* b, int i0_, int j0_) : i0(i0_), j0(j0_) {
    Carver c{b};
    xu = c.take<WUx>(i0, j0);
    u = c.take<WUd>(i0, j0);
    dE = c.take<WUd>(i0, j0);
    xv = c.take<WVx>(i0, j0);
    v = c.take<WVd>(i0, j0);
    dN = c.take<WVd>(i0, j0);
    g0 = c.take_col<WG>(i0);
  }
};

// Final Jacobi value at a U/V unknown: FP64 the iterate, mixed u + delta.
template <typename T>
__device__ __forceinline__ double final_velocity(double vel, T xf) {
  if (sizeof(T) == 4) return vel + (double)xf;
  return (double)xf;
}

// Returns false when a wait failed.  rc: residU, residV, residMass,
// residMassDof, non-finite flag (max); r.z, p.Ap (sum).
template <typename T, class Group>
__device__ bool mass_phase(const DesignView& d, Group& g, double* smem, char* tbuf, const T* xfU, const T* xfV,
                           int mapXU, int mapXV, double (&rc)[7]) {
  const Inner<T>& w = inner<T>(d);
  const int M = d.M, N = d.N, P = d.P;
  using L_t = LayoutC<T>;
  char* ext = tbuf + (size_t)kStageDepth * L_t::kBytes;
  const double mv = d.maxVel;
  const bool ok = for_each_tile<L_t>(
      d, g, tbuf,
      [mapXU, mapXV](const L_t& L, const TensorMap* tm, unsigned long long* bar) {
        L.xu.tma(tm + mapXU, bar);
        L.u.tma(tm + kTmU_C, bar);
        L.dE.tma(tm + kTmDE_C, bar);
        L.xv.tma(tm + mapXV, bar);
        L.v.tma(tm + kTmV_C, bar);
        L.dN.tma(tm + kTmDN_C, bar);
        if (L.j0 <= 2) L.g0.tma(tm + kTmG_C, bar);
      },
      [&](const L_t& L) {
        L.xu.elems(xfU, P, M);
        L.u.elems(d.u, P, M);
        L.dE.elems(d.dE, P, M);
        L.xv.elems(xfV, P, M);
        L.v.elems(d.v, P, M);
        L.dN.elems(d.dN, P, M);
        if (L.j0 <= 2) L.g0.elems(d.gamma, P, M - 1);
      },
      [&](const L_t& L, int i, int j, bool inside) {
        Carver c{ext};
        const auto us = c.take<typename L_t::WUd>(L.i0, L.j0);  // u* after scatter, clamp and BCs
        const auto vs = c.take<typename L_t::WVd>(L.i0, L.j0);  // v*
        const auto z0 = c.take<typename L_t::WZ>(L.i0, L.j0);   // z0 = r0/diag at the P-unknowns
        // u*(ii, jj) as momentum_solver.cpp:326 + boundaries.cpp:57-103 leave it
        for (int k = threadIdx.x; k < us.kElems; k += kThreads) {
          int ii, jj;
          us.coords(k, ii, jj);
          double val = 0.0;
          if (ii >= 1 && ii <= M - 1 && jj >= 0) {
            if (jj == 0) {
              val = (L.g0(ii - 1) > 0.5) ? d.Uin : 0.0;
            } else {
              const int jc = (jj >= N - 1) ? N - 2 : jj;
              val = clampd(final_velocity<T>(L.u(ii, jc), L.xu(ii, jc)), -mv, mv);
            }
          }
          us.ref(k) = val;
        }
        for (int k = threadIdx.x; k < vs.kElems; k += kThreads) {
          int ii, jj;
          vs.coords(k, ii, jj);
          double val = 0.0;
          if (ii >= 1 && ii <= M - 2 && jj >= 1) {
            const int jc = (jj >= N) ? N - 1 : jj;
            val = clampd(final_velocity<T>(L.v(ii, jc), L.xv(ii, jc)), -mv, mv);
          }
          vs.ref(k) = val;
        }
        __syncthreads();
        // z0 at every P-unknown of the tile and its one-cell ring
        for (int k = threadIdx.x; k < z0.kElems; k += kThreads) {
          int ii, jj;
          z0.coords(k, ii, jj);
          double z = 0.0;
          if (ii >= 1 && ii <= M - 1 && jj >= 1 && jj <= N - 2) {
            const double mE = d.rho * us(ii, jj) * d.hy;
            const double mW = d.rho * us(ii, jj - 1) * d.hy;
            const double mN = d.rho * vs(ii, jj) * d.hx;
            const double mS = d.rho * vs(ii - 1, jj) * d.hx;
            const double b = mW - mE + mS - mN;
            const double aE = (jj < N - 1) ? d.rho * L.dE(ii, jj) * d.hy : 0.0;
            const double aW = (jj > 1) ? d.rho * L.dE(ii, jj - 1) * d.hy : 0.0;
            const double aN = (ii < M - 1) ? d.rho * L.dN(ii, jj) * d.hx : 0.0;
            const double aS = (ii > 1) ? d.rho * L.dN(ii - 1, jj) * d.hx : 0.0;
            double aP = aE + aW + aN + aS;
            if (aP < 1e-20) aP = 1.0;
            const double rr = (double)(T)b, dd = (double)(T)aP;
            z = (double)(T)((fabs(dd) > 1e-20) ? rr / dd : rr);
          }
          z0.ref(k) = z;
        }
        __syncthreads();
        if (!inside) return;
        const size_t o = (size_t)i * P + j;
        if (j <= N - 2) {
          const double val = us(i, j);
          d.us[o] = val;
          rc[0] = maxd(rc[0], fabs(val - L.u(i, j)));
          if (!isfinite(val)) rc[4] = 1.0;
          if (j == N - 2) d.us[o + 1] = val;
        }
        if (j == 1) d.us[o - 1] = us(i, 0);
        if (i <= M - 2) {
          const double val = vs(i, j);
          d.vs[o] = val;
          rc[1] = maxd(rc[1], fabs(val - L.v(i, j)));
          if (!isfinite(val)) rc[4] = 1.0;
          if (j == N - 1) d.vs[o + 1] = val;
        }
        const double massE = d.rho * us(i, j) * d.hy;
        const double massW = d.rho * us(i, j - 1) * d.hy;
        const double massN = d.rho * vs(i, j) * d.hx;
        const double massS = d.rho * vs(i - 1, j) * d.hx;
        const double b = massW - massE + massS - massN;
        const double ab = fabs(b);
        if (!isfinite(ab)) rc[4] = 1.0;
        if (ab > rc[2]) rc[2] = ab;
        if (j <= N - 2) {
          if (ab > rc[3]) rc[3] = ab;
          // pressure_solver.cpp:698-703
          const double aE = (j < N - 1) ? d.rho * L.dE(i, j) * d.hy : 0.0;
          const double aW = (j > 1) ? d.rho * L.dE(i, j - 1) * d.hy : 0.0;
          const double aN = (i < M - 1) ? d.rho * L.dN(i, j) * d.hx : 0.0;
          const double aS = (i > 1) ? d.rho * L.dN(i - 1, j) * d.hx : 0.0;
          double aP = aE + aW + aN + aS;
          if (aP < 1e-20) aP = 1.0;
          const T dg = (T)aP;
          w.pdiag[o] = dg;
          w.cx[o] = (T)aE;
          w.cy[o] = (T)aN;
          const T rt = (T)b;
          w.pr[o] = rt;
          w.px[o] = (T)0.0;
          const double rr = (double)rt, dd = (double)dg;
          const T z = (T)((fabs(dd) > 1e-20) ? rr / dd : rr);
          if (d.pcgSingleReduction) {
            w.cU[o + d.planeStride] = z;  // u0 = M^-1 r0 of the single-reduction recurrences
          } else {
            w.pz[o] = z;
            w.pp0[o] = z;
          }
          rc[5] += rr * (double)z;
          // first PCG product: A p0 with p0 = z0, in CSR order S, W, P, E, N
          const double zc = (double)z;
          double Ap = 0.0;
          if (i > 1) Ap += -(double)(T)aS * z0(i - 1, j);
          if (j > 1) Ap += -(double)(T)aW * z0(i, j - 1);
          Ap += (double)dg * zc;
          if (j + 1 <= N - 2) Ap += -(double)(T)aE * z0(i, j + 1);
          if (i < M - 1) Ap += -(double)(T)aN * z0(i + 1, j);
          const T apt = (T)Ap;
          w.pAp[o] = apt;  // FP64: A p0; mixed: w0 = A u0 (the same plane)
          rc[6] += zc * (double)apt;
        }
      });
  if (!ok) return false;
  return g.template sync_reduce<7, 0x1Fu>(rc, smem);
}

// ---------------------------------------------------------------------------
// samplePlaneAtX (postprocessing.cpp:62-230), split into the interpolation
// set-up of a plane, one row's five contributions and the metrics from the
// five sums (staticAreaSum, dynAreaSum, totalWeighted, area, fluxSum).
// ---------------------------------------------------------------------------
struct PlaneSetup {
  int colLeft, colRight;
  double t;
};

__device__ __forceinline__ PlaneSetup plane_setup(const DesignView& d, double xPhysical) {
  const int N = d.N;
  const double hx = d.hx;
  const double xMin = 0.5 * hx, xMax = ((double)N - 0.5) * hx;
  const double xClamped = maxd(xMin, mind(xPhysical, xMax));
  const double jFloat = xClamped / hx - 0.5;
  int colLeft = (int)floor(jFloat);
  colLeft = colLeft < N - 2 ? colLeft : N - 2;
  colLeft = 0 < colLeft ? colLeft : 0;
  const int colRight = colLeft + 1;
  const double xLeft = ((double)colLeft + 0.5) * hx, xRight = ((double)colRight + 0.5) * hx;
  double t = (fabs(xRight - xLeft) < 1e-12) ? 0.0 : (xClamped - xLeft) / (xRight - xLeft);
  t = maxd(0.0, mind(1.0, t));
  return PlaneSetup{colLeft, colRight, t};
}

// Row i (1..M-1) of the plane, added into acc in the reference's order.
__device__ __forceinline__ void plane_row(const DesignView& d, const PlaneSetup& s, int i, double* acc) {
  const int M = d.M, N = d.N, P = d.P;
  const double hy = d.hy, rho = d.rho, t = s.t;
  const int colLeft = s.colLeft, colRight = s.colRight;
  auto cl = [](int a, int lo, int hi) { return a < lo ? lo : (a > hi ? hi : a); };
  const int cellRow = i - 1;
  if (d.gamma[(size_t)cellRow * P + colLeft] < 1.0 - 1e-6 || d.gamma[(size_t)cellRow * P + colRight] < 1.0 - 1e-6)
    return;
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

// out: area, fluxSum, avgStatic, avgDynamic, avgTotal, valid (PlaneMetrics)
__device__ __forceinline__ void plane_metrics(const double* acc, double* out) {
  const double area = acc[3], fluxSum = acc[4];
  double avgStatic = 0.0, avgDynamic = 0.0, avgTotal = 0.0, valid = 0.0;
  if (area > 0.0) { avgStatic = acc[0] / area; avgDynamic = acc[1] / area; valid = 1.0; }
  if (fluxSum > 0.0) avgTotal = acc[2] / fluxSum;
  else if (area > 0.0) avgTotal = avgStatic + avgDynamic;
  out[0] = area; out[1] = fluxSum; out[2] = avgStatic; out[3] = avgDynamic; out[4] = avgTotal; out[5] = valid;
}

// ---------------------------------------------------------------------------
// After an outer iteration: the four planes (core inlet/outlet, x = 0 and
// x = N hx, SIMPLE.cpp:338-344) sampled by the whole group, the four
// pressure drops (:347-353) and the pressure-drop convergence gate
// (:356-408).  Rows are spread over the group's threads and the twenty sums
// reduced once, so every CTA holds the same drops and evaluates the gate
// identically: the history slots are a function of the iteration index
// (value k of the window goes to slot k mod window, the slope window holds
// the last dpSlopeWindow iterations) and CTA 0 writes this iteration's slots.
// The window statistics are the reference's formulas; their sums are grouped
// in a fixed lane-strided order, as the plane sums are.  Returns false when a
// wait failed.
// ---------------------------------------------------------------------------
template <class Group>
__device__ bool dp_phase(const DesignView& d, Group& g, double* smem, char* tbuf, int iter, double* dplog,
                         bool& converged) {
  PlaneSetup ps[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) ps[q] = plane_setup(d, d.xPlane[q]);
  double acc[kPlaneSums];
#pragma unroll
  for (int k = 0; k < kPlaneSums; ++k) acc[k] = 0.0;
  const int first = (int)g.rank * kThreads + (int)threadIdx.x, step = (int)g.nblk * kThreads;
#pragma unroll
  for (int q = 0; q < 4; ++q)
    for (int i = 1 + first; i <= d.M - 1; i += step) plane_row(d, ps[q], i, acc + 5 * q);
  // the plane sums use the ring region after the kRedSlots slots, which no
  // other reduction touches
  if (!g.template sync_reduce_at<kPlaneSums, 0u>(acc, smem, g.red + (size_t)kRedSlots * g.nblk * kRedWidth))
    return false;
  double m[4][6];
#pragma unroll
  for (int q = 0; q < 4; ++q) plane_metrics(acc + 5 * q, m[q]);
  const double coreTotal = m[0][4] - m[1][4], fullTotal = m[2][4] - m[3][4];
  const double coreStatic = m[0][2] - m[1][2], fullStatic = m[2][2] - m[3][2];
  const bool writer = g.rank == 0 && threadIdx.x == 0;
  if (writer && dplog) {
    dplog[0] = coreTotal;
    dplog[1] = fullTotal;
    dplog[2] = coreStatic;
    dplog[3] = fullStatic;
  }
  converged = false;
  const int W = d.dpWindow, S = d.dpSlopeWindow;
  const bool slope = d.dpSlopeGate && S > 0;
  const double v = coreTotal;
  if (d.dpGate && iter >= d.dpRampSteps && iter - d.dpRampSteps + 1 >= W) {
    // Warp 0 evaluates the statistics: lane-strided sums in a fixed order and a
    // warp tree (deterministic, the same in every CTA), the window values staged
    // in shared memory once; the other warps wait at one barrier.
    __shared__ int s_conv;
    const int lane = threadIdx.x & 31;
    if (threadIdx.x < 32) {
      double* win = reinterpret_cast<double*>(tbuf);
      double* sl = win + W;
      const int cur = (iter - d.dpRampSteps) % W;
      const bool slopeFull = slope && iter + 1 >= S;
      for (int k = lane; k < W; k += 32) win[k] = (k == cur) ? v : __ldcg(d.dpHist + k);
      if (slopeFull)
        for (int k = lane; k < S; k += 32) sl[k] = (k == S - 1) ? v : __ldcg(d.dpHist + W + (iter - S + 1 + k) % S);
      __syncwarp();
      auto warp_sum = [](double x) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
        return x;
      };
      double sum = 0.0;
      for (int k = lane; k < W; k += 32) sum += win[k];
      const double mean = warp_sum(sum) / double(W);
      double varSum = 0.0;
      for (int k = lane; k < W; k += 32) {
        const double diff = win[k] - mean;
        varSum += diff * diff;
      }
      const double stdDev = sqrt(warp_sum(varSum) / double(W));
      const double denom = maxd(fabs(mean), 1.0);
      const double stdPercent = (stdDev / denom) * 100.0;
      const double latestDeltaPercent = (fabs(v - mean) / denom) * 100.0;
      bool slopeGatePassed = true;
      if (slopeFull) {
        // least-squares slope over (iteration - first iteration, dP), SIMPLE.cpp:276-294
        double sumX = 0.0, sumY = 0.0, sumXX = 0.0, sumXY = 0.0;
        for (int k = lane; k < S; k += 32) {
          const double x = (double)k, y = sl[k];
          sumX += x;
          sumY += y;
          sumXX += x * x;
          sumXY += x * y;
        }
        sumX = warp_sum(sumX);
        sumY = warp_sum(sumY);
        sumXX = warp_sum(sumXX);
        sumXY = warp_sum(sumXY);
        const double n = (double)S;
        const double den = n * sumXX - sumX * sumX;
        const double slopeVal = (fabs(den) < 1e-12) ? 0.0 : (n * sumXY - sumX * sumY) / den;
        slopeGatePassed = fabs(slopeVal) <= d.dpSlopeMaxDelta / (double)S;
      }
      if (lane == 0) s_conv = (stdPercent < d.dpPercent && latestDeltaPercent < d.dpPercent && slopeGatePassed) ? 1 : 0;
    }
    __syncthreads();
    converged = s_conv != 0;
  }
  if (writer) {
    if (slope) d.dpHist[W + iter % S] = v;
    if (d.dpGate && iter >= d.dpRampSteps) d.dpHist[(iter - d.dpRampSteps) % W] = v;
  }
  return true;
}

// Dynamic shared memory a persistent kernel needs for storage type T (the
// tile buffers).
template <typename T>
constexpr size_t tile_smem_bytes() {
  constexpr size_t a = kStageDepth * LayoutA::kBytes;
  constexpr size_t c = kStageDepth * LayoutC<T>::kBytes + LayoutC<T>::kExtraBytes;
  constexpr size_t dd = kStageDepth * LayoutD<T>::kBytes;
  constexpr size_t bb = kStageDepth * LayoutB<T>::kBytes;
  constexpr size_t m0 = a > c ? a : c;
  constexpr size_t m = m0 > bb ? m0 : bb;
  constexpr size_t t = m > dd ? m : dd;
  constexpr size_t q = CPS_SMEM_PCG ? sizeof(PcgSmem<T, SmemTiles<T>::value>) : 0;  // the PCG reuses the buffers
  return t > q ? t : q;
}

// The kernels declare their dynamic shared memory (the tile buffers, where
// TMA tile copies land) 128-byte aligned.  Checked once at the start of a
// launch: a CTA whose buffer is not aligned records kStatusTimeout (the host
// reports a failed device wait) and the launch does no work.
__device__ __forceinline__ bool tile_buffer_aligned(const char* dyn, int* status) {
  const bool bad = (smem_u32(dyn) & 127u) != 0;
  if (bad && threadIdx.x == 0 && status) atomicCAS(status, kStatusOk, kStatusTimeout);
  return !__syncthreads_or(bad);
}

// ---------------------------------------------------------------------------
// One outer iteration for one design on group g; out[8] receives the step
// diagnostics.  tbuf: tile_smem_bytes<T>() of shared memory.  iter is the
// outer loop's iteration index of this step.  With Monitor (compiled in for
// the single-design kernel only) and d.dpMonitor, dplog (may be null) receives
// its four pressure drops and *dpConverged is set when the pressure-drop gate
// ends the loop.  pr (may be null) holds the CTA's copy of the CFL
// controllers' state when d.pseudo; Pseudo = false compiles the
// pseudo-transient term and the controllers out.  Returns 0 to continue with another outer
// iteration, 1 when this one is the last (iteration budget, convergence, the
// pressure-drop gate, or a non-finite residual), -1 when the group must stop
// because a device-side wait failed.
// ---------------------------------------------------------------------------
template <typename T, class Group, bool Monitor = false, bool Pseudo = true>
__device__ int outer_iteration(const DesignView& d, Group& g, double* smem, char* tbuf, double (&out)[8],
                               bool lastIter, bool stopOnConv, double eps, int iter = 0, double* dplog = nullptr,
                               int* dpConverged = nullptr, PseudoRun* pr = nullptr, SweepHint* hint = nullptr) {
  const Inner<T>& w = inner<T>(d);
  const int M = d.M, N = d.N, P = d.P;
  // ---- A: assembly + sweep 1 (or the explicit update) ----
  const double cfl = (Pseudo && d.pseudo && pr) ? pr->cfl : 0.0;
  const bool expl = d.momExplicit != 0;
  const bool anySweep = !expl && d.maxMomIter > 0;
  // Rows are stored in phase A when the last outer iteration needed a second
  // sweep of that component (the sweep counts change slowly); otherwise a
  // second sweep re-assembles them.  Both give the same bits.
  const bool canSweep2 = anySweep && d.maxMomIter > 1;
  const bool storeU = canSweep2 && (!hint || hint->kU >= 2);
  const bool storeV = canSweep2 && (!hint || hint->kV >= 2);
  double red2[2] = {0.0, 0.0};
  const auto tmaA = [](const LayoutA& L, const TensorMap* tm, unsigned long long* bar) {
    L.u.tma(tm + kTmU_A, bar);
    L.v.tma(tm + kTmV_A, bar);
    L.p.tma(tm + kTmP_A, bar);
    L.a.tma(tm + kTmAlpha_A, bar);
  };
  const auto elemsA = [&](const LayoutA& L) {
    L.u.elems(d.u, P, M);
    L.v.elems(d.v, P, M);
    L.p.elems(d.p, P, M);
    L.a.elems(d.alpha, P, M - 1);
  };
  const bool okA = for_each_tile<LayoutA>(
      d, g, tbuf, tmaA, elemsA,
      [&](const LayoutA& L, int i, int j, bool inside) {
        if (!inside) return;
        if (expl) {
          if (j <= N - 2) explicit_point<true, T, Pseudo>(d, L, i, j, cfl);
          if (i <= M - 2) explicit_point<false, T, Pseudo>(d, L, i, j, cfl);
          return;
        }
        if (j <= N - 2) red2[0] += assemble_point<true, T, Pseudo>(d, L, i, j, anySweep, cfl, storeU);
        if (i <= M - 2) red2[1] += assemble_point<false, T, Pseudo>(d, L, i, j, anySweep, cfl, storeV);
      });
  if (!okA || !g.template sync_reduce<2, 0u>(red2, smem)) return -1;
  int kU = anySweep ? 1 : 0, kV = kU;
  bool actU = anySweep && !(red2[0] < d.thrU) && kU < d.maxMomIter;
  bool actV = anySweep && !(red2[1] < d.thrV) && kV < d.maxMomIter;
  // ---- B: sweeps 2.. ----
  while (actU || actV) {
    const int k = (actU ? kU : kV) + 1;  // both active components are at the same sweep
    const T* xinU = (k & 1) ? w.xU0 : w.xU1;
    T* xoutU = (k & 1) ? w.xU1 : w.xU0;
    const T* xinV = (k & 1) ? w.xV0 : w.xV1;
    T* xoutV = (k & 1) ? w.xV1 : w.xV0;
    double s[2] = {0.0, 0.0};
    const bool au = actU, av = actV;
    bool okB = true;
    if (k == 2 && ((au && !storeU) || (av && !storeV))) {
      // sweep 2 of a component whose rows phase A did not store re-assembles
      // them from the same staged inputs and stores them for the sweeps after it
      const bool store = d.maxMomIter > 2;
      okB = for_each_tile<LayoutA>(
          d, g, tbuf, tmaA, elemsA,
          [&](const LayoutA& L, int i, int j, bool inside) {
            if (!inside) return;
            if (au && j <= N - 2)
              s[0] += storeU ? sweep_point<true, T>(d, i, j, xinU, xoutU)
                             : sweep2_point<true, T, Pseudo>(d, L, i, j, cfl, xinU, xoutU, store);
            if (av && i <= M - 2)
              s[1] += storeV ? sweep_point<false, T>(d, i, j, xinV, xoutV)
                             : sweep2_point<false, T, Pseudo>(d, L, i, j, cfl, xinV, xoutV, store);
          });
    } else if (d.tm && d.stageSweeps) {
      using LB = LayoutB<T>;
      const long long ps = d.planeStride;
      const int mapXU = (k & 1) ? kTmXU0_B : kTmXU1_B, mapXV = (k & 1) ? kTmXV0_B : kTmXV1_B;
      okB = for_each_tile<LB>(
          d, g, tbuf,
          [au, av, mapXU, mapXV](const LB& L, const TensorMap* tm, unsigned long long* bar) {
            if (au) {
#pragma unroll
              for (int q = 0; q < 5; ++q) L.cu[q].tma(tm + kTmCU_B + q, bar);
              L.bu.tma(tm + kTmBU_B, bar);
              L.xu.tma(tm + mapXU, bar);
            }
            if (av) {
#pragma unroll
              for (int q = 0; q < 5; ++q) L.cv[q].tma(tm + kTmCV_B + q, bar);
              L.bv.tma(tm + kTmBV_B, bar);
              L.xv.tma(tm + mapXV, bar);
            }
          },
          [&](const LB& L) {
            if (au) {
              for (int q = 0; q < 5; ++q) L.cu[q].elems(w.cU + q * ps, P, M);
              L.bu.elems(w.bU, P, M);
              L.xu.elems(xinU, P, M);
            }
            if (av) {
              for (int q = 0; q < 5; ++q) L.cv[q].elems(w.cV + q * ps, P, M);
              L.bv.elems(w.bV, P, M);
              L.xv.elems(xinV, P, M);
            }
          },
          [&](const LB& L, int i, int j, bool inside) {
            if (!inside) return;
            if (au && j <= N - 2) s[0] += sweep_point_staged<true, T>(d, L, i, j, xoutU);
            if (av && i <= M - 2) s[1] += sweep_point_staged<false, T>(d, L, i, j, xoutV);
          });
    } else {
      for_each_point(d, g.rank, g.nblk, [&](int i, int j) {
        if (au && j <= N - 2) s[0] += sweep_point<true, T>(d, i, j, xinU, xoutU);
        if (av && i <= M - 2) s[1] += sweep_point<false, T>(d, i, j, xinV, xoutV);
      });
    }
    if (!okB || !g.template sync_reduce<2, 0u>(s, smem)) return -1;
    if (au) { kU = k; actU = !(s[0] < d.thrU) && kU < d.maxMomIter; }
    if (av) { kV = k; actV = !(s[1] < d.thrV) && kV < d.maxMomIter; }
  }
  if (hint) {
    hint->kU = kU;
    hint->kV = kV;
  }
  const T* xfU = (kU & 1) ? w.xU1 : w.xU0;
  const T* xfV = (kV & 1) ? w.xV1 : w.xV0;
  // ---- C: scatter, BCs, mass residual, PCG set-up ----
  double rc[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  if (!mass_phase<T>(d, g, smem, tbuf, xfU, xfV, (kU & 1) ? kTmXU1_C : kTmXU0_C, (kV & 1) ? kTmXV1_C : kTmXV0_C, rc))
    return -1;
  out[0] = rc[0];
  out[1] = rc[1];
  out[2] = rc[2];
  out[3] = rc[3];
  out[6] = kU;
  out[7] = kV;
  // std::max({residU, residV, residMass}) (iterations.cpp:525); the stop test
  // uses the mass imbalance over the pressure unknowns.
  double e = out[0];
  if (e < out[1]) e = out[1];
  if (e < out[2]) e = out[2];
  out[4] = e;
  const double conv = maxd(maxd(out[0], out[1]), out[3]);
  // The max reductions drop NaN the way std::max does, so non-finite values
  // are flagged explicitly.
  const bool finite = isfinite(e) && isfinite(out[3]) && rc[4] == 0.0;
  if (!finite && g.rank == 0 && threadIdx.x == 0 && g.status) atomicCAS(g.status, kStatusOk, kStatusDiverged);
  const bool stop = lastIter || !finite || (stopOnConv && conv <= eps);
  // The CFL controllers (SIMPLE.cpp:321-327).  Every CTA's thread 0 updates its
  // copy from the same reduced residuals; the barriers before the next phase A
  // publish it to the CTA.
  if (Pseudo && d.pseudo && pr && threadIdx.x == 0) {
    pseudo_update(d, *pr, d.serUseMax ? out[4] : out[2], iter);
    if (g.rank == 0 && d.pseudoState) {
      d.pseudoState[0] = pr->cfl;
      d.pseudoState[1] = pr->prev;
      d.pseudoState[2] = pr->alpha;
      d.pseudoState[3] = (double)pr->count;
    }
  }
  // ---- P: Jacobi-preconditioned CG ----
  if (d.pcgSingleReduction) {
    const int its = pcg_single_reduction<T>(d, g, smem, rc[5], rc[6]);
    if (its < 0) return -1;
    out[5] = its;
  } else {
    const int tiles = ((M - 1 + kTileI - 1) / kTileI) * ((N - 1 + kTileJ - 1) / kTileJ);
    constexpr int kS = SmemTiles<T>::value;
    int its;
    if (tiles <= kResidentTiles * (int)g.nblk)
      its = pcg_resident<T, kResidentTiles>(d, g, smem, rc[5], rc[6]);
    else if (CPS_SMEM_PCG && tiles <= kS * (int)g.nblk && (!hint || hint->kP >= 2))
      // the shared-memory form pays when the PCG runs several iterations (its
      // loading costs about one); the last outer iteration's count decides
      its = pcg_smem<T, kS>(d, g, smem, tbuf, rc[5], rc[6]);
    else
      its = pcg_two_reductions<T>(d, g, smem, rc[5], rc[6]);
    if (its < 0) return -1;
    out[5] = its;
    if (hint) hint->kP = its;
  }
  // ---- D: pressure and velocity correction ----
  if (!correct_fields<T>(d, g, tbuf)) return -1;
  if constexpr (Monitor) {
    if (d.dpMonitor) {
      // ---- pressure-drop monitor and gate; its reduction is the barrier before the next A ----
      bool gateStop = false;
      if (!g.sync() || !dp_phase(d, g, smem, tbuf, iter, dplog, gateStop)) return -1;
      if (gateStop && dpConverged && g.rank == 0 && threadIdx.x == 0) *dpConverged = 1;
      return (stop || gateStop) ? 1 : 0;
    }
  }
  if (!stop) return g.sync() ? 0 : -1;
  return 1;
}

#undef AT

}  // namespace cps
