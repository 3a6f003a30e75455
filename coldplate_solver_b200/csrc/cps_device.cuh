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
// reuse them; the pressure coefficients are rebuilt on the fly from dE, dN.
// Every product/sum that feeds a stored value is evaluated in the reference's
// order, and this translation unit is compiled with --fmad=false, so per-point
// values equal the FP64 reference's; only the grid-wide sums (Jacobi RMS, PCG
// dots) are summed in a different (fixed, deterministic) order.
//
// Layout: one pitched row-major array per field in the reference's (i, j)
// index space; element (i, j) at base[i * P + j] with P >= N + 1 a multiple of
// 32 doubles, so a warp's 32 consecutive j are one 256-byte segment.
#pragma once
#include <cuda_runtime.h>
#include <cooperative_groups.h>
#include <stdint.h>

namespace cps {

namespace cg = cooperative_groups;

constexpr int kThreads = 256;   // 8 warps
constexpr int kTileI = 8;       // tile rows (one warp per row)
constexpr int kTileJ = 32;      // tile columns (one lane per column)
constexpr int kRedWidth = 8;    // doubles per CTA per reduction
constexpr int kRedSlots = 4;    // ring of reduction slots
constexpr unsigned long long kBarrierTimeoutNs = 2000000000ull;  // 2 s

enum DeviceStatus : int { kStatusOk = 0, kStatusTimeout = 1, kStatusDiverged = 2 };

// Device view of one design's grid, parameters and arrays.
struct DesignView {
  int M, N, P;
  int conv, maxPIter, maxMomIter;
  double hx, hy, rho, uvAlpha, pAlpha, pTol;
  double vol, De, Dn, sinkDiag, Fcx, Fcy, relax;  // Fcx = cs*rho*hy, Fcy = cs*rho*hx, relax = (1-uvA)/uvA
  double thrU, thrV;                              // momTol^2 * nU, momTol^2 * nV
  double Uin, maxVel;
  double *u, *v, *p, *pc, *us, *vs, *dE, *dN, *alpha, *gamma;
  double *cU, *cV;          // 5 planes each (E, W, N, S, P), plane stride = planeStride
  double *bU, *bV;
  double *xU0, *xU1, *xV0, *xV1;
  double *px, *pr, *pz, *pp0, *pp1, *pAp, *pdiag;
  long long planeStride;    // elements between coefficient planes
};

// Per-launch control shared by all CTAs.
struct RunControl {
  int n_outer;        // outer iterations to run
  int stop_on_conv;   // stop once max(residU, residV, residMassDof) <= eps
  double eps;
  double* hist;       // n_outer x 8: residU, residV, residMass, residMassDof, err, pIters, uSweeps, vSweeps
  int* n_done;        // outer iterations completed by this launch
  int* status;        // DeviceStatus
};

struct GridBarrier {
  unsigned int count;
  unsigned int gen;
};

// ---------------------------------------------------------------------------
// small helpers (std::max/min/clamp evaluated the way libstdc++ does)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double maxd(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double mind(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double clampd(double v, double lo, double hi) { return (v < lo) ? lo : (hi < v) ? hi : v; }

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u32(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
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

  // Returns false (and the CTA must return) on timeout or on an error raised elsewhere.
  __device__ bool sync() {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
      int ok = 1;
      __threadfence();
      const unsigned g = ld_acquire_u32(&bar->gen);
      const unsigned arrived = atomicAdd(&bar->count, 1u);
      if (arrived == nblk - 1) {
        atomicExch(&bar->count, 0u);
        __threadfence();
        st_release_u32(&bar->gen, g + 1);
      } else {
        const unsigned long long t0 = globaltimer_ns();
        unsigned spins = 0;
        while (ld_acquire_u32(&bar->gen) == g) {
          if ((++spins & 255u) == 0) {
            if (*(volatile int*)status != kStatusOk) { ok = 0; break; }
            if (globaltimer_ns() - t0 > kBarrierTimeoutNs) {
              atomicCAS(status, kStatusOk, kStatusTimeout);
              ok = 0;
              break;
            }
          }
        }
      }
      __threadfence();
      s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
  }

  // Publish this CTA's K values, synchronise, and combine all CTAs' values in
  // CTA order.  Result valid in every thread of every CTA.
  template <int K, unsigned MaxMask>
  __device__ bool sync_reduce(double (&v)[K], double* smem) {
    block_reduce<K, MaxMask>(v, smem);
    double* slot = red + (size_t)(redCount % kRedSlots) * nblk * kRedWidth;
    ++redCount;
    if (threadIdx.x == 0) {
#pragma unroll
      for (int k = 0; k < K; ++k) slot[rank * kRedWidth + k] = v[k];
    }
    if (!sync()) return false;
    double acc[K];
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = ((MaxMask >> k) & 1u) ? 0.0 : 0.0;
    bool first = true;
    for (unsigned b = threadIdx.x; b < nblk; b += kThreads) {
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const double x = __ldcg(slot + b * kRedWidth + k);
        acc[k] = first ? x : (((MaxMask >> k) & 1u) ? maxd(acc[k], x) : acc[k] + x);
      }
      first = false;
    }
    block_reduce<K, MaxMask>(acc, smem);
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = acc[k];
    return true;
  }
};

// ---------------------------------------------------------------------------
// Per-point kernels
// ---------------------------------------------------------------------------
#define AT(a, i, j) (a)[(size_t)(i) * P + (j)]

// SOU deferred correction, convection.cpp:53-118 (U) and :121-186 (V); the two
// components' range guards differ and are kept as in the reference.
template <bool IsU>
__device__ __forceinline__ double sou_correction(const DesignView& d, const double* __restrict__ x, int i, int j,
                                                 double Fe, double Fw, double Fn, double Fs) {
  const int M = d.M, N = d.N, P = d.P;
  double Sdc = 0.0;
  if (Fe >= 0.0) {
    if (j >= 2) Sdc -= Fe * ((1.5 * AT(x, i, j) - 0.5 * AT(x, i, j - 1)) - AT(x, i, j));
  } else {
    if (IsU ? (j + 2 < N) : (j + 2 <= N)) Sdc -= Fe * ((1.5 * AT(x, i, j + 1) - 0.5 * AT(x, i, j + 2)) - AT(x, i, j + 1));
  }
  if (Fw >= 0.0) {
    if (j >= 2) Sdc += Fw * ((1.5 * AT(x, i, j - 1) - 0.5 * AT(x, i, j - 2)) - AT(x, i, j - 1));
  } else {
    if (IsU ? (j + 1 < N) : (j + 1 <= N)) Sdc += Fw * ((1.5 * AT(x, i, j) - 0.5 * AT(x, i, j + 1)) - AT(x, i, j));
  }
  if (Fn >= 0.0) {
    if (i >= 1) Sdc -= Fn * ((1.5 * AT(x, i, j) - 0.5 * AT(x, i - 1, j)) - AT(x, i, j));
  } else {
    if (IsU ? (i + 2 <= M) : (i + 2 < M)) Sdc -= Fn * ((1.5 * AT(x, i + 1, j) - 0.5 * AT(x, i + 2, j)) - AT(x, i + 1, j));
  }
  if (Fs >= 0.0) {
    if (i >= 2) Sdc += Fs * ((1.5 * AT(x, i - 1, j) - 0.5 * AT(x, i - 2, j)) - AT(x, i - 1, j));
  } else {
    if (IsU ? (i + 1 <= M) : (i + 1 < M)) Sdc += Fs * ((1.5 * AT(x, i, j) - 0.5 * AT(x, i + 1, j)) - AT(x, i, j));
  }
  return Sdc;
}

// Momentum assembly at one unknown (momentum_solver.cpp:203-296) fused with
// Jacobi sweep 1 (jacobi_solver.cpp:49-57, x0 = current velocity).  Returns the
// squared residual of sweep 1 (0 when no sweep is run).
template <bool IsU>
__device__ __forceinline__ double assemble_point(const DesignView& d, int i, int j, bool sweep) {
  const int M = d.M, N = d.N, P = d.P;
  const double* __restrict__ u = d.u;
  const double* __restrict__ v = d.v;
  const double* __restrict__ p = d.p;
  const double* __restrict__ A = d.alpha;
  const double mv = d.maxVel;
  double alphaLocal, ue, uw, vn, vs;
  if (IsU) {
    alphaLocal = 0.5 * (AT(A, i - 1, j - 1) + AT(A, i - 1, j));
    ue = clampd(0.5 * (AT(u, i, j) + AT(u, i, j + 1)), -mv, mv);
    uw = clampd(0.5 * (AT(u, i, j - 1) + AT(u, i, j)), -mv, mv);
    vn = clampd(0.5 * (AT(v, i, j) + AT(v, i, j + 1)), -mv, mv);
    vs = clampd(0.5 * (AT(v, i - 1, j) + AT(v, i - 1, j + 1)), -mv, mv);
  } else {
    alphaLocal = 0.5 * (AT(A, i - 1, j - 1) + AT(A, i, j - 1));
    ue = clampd(0.5 * (AT(u, i, j) + AT(u, i + 1, j)), -mv, mv);
    uw = clampd(0.5 * (AT(u, i, j - 1) + AT(u, i + 1, j - 1)), -mv, mv);
    vn = clampd(0.5 * (AT(v, i, j) + AT(v, i + 1, j)), -mv, mv);
    vs = clampd(0.5 * (AT(v, i - 1, j) + AT(v, i, j)), -mv, mv);
  }
  const double Fe = d.Fcx * ue, Fw = d.Fcx * uw, Fn = d.Fcy * vn, Fs = d.Fcy * vs;
  const double aE = d.De + maxd(0.0, -Fe), aW = d.De + maxd(0.0, Fw);
  const double aN = d.Dn + maxd(0.0, -Fn), aS = d.Dn + maxd(0.0, Fs);
  const double sumA = aE + aW + aN + aS;
  const double transCoeff = 0.0;  // pseudo-transient off
  const double brinkmanDrag = alphaLocal * d.vol;
  double aP0 = sumA + (Fe - Fw + Fn - Fs) + transCoeff + d.sinkDiag + brinkmanDrag;
  aP0 = maxd(aP0, 1e-10);
  const double aP = aP0 / d.uvAlpha;
  const double* __restrict__ X = IsU ? u : v;
  const double velCur = AT(X, i, j);
  double Sp = IsU ? (AT(p, i, j) - AT(p, i, j + 1)) * d.hy : (AT(p, i, j) - AT(p, i + 1, j)) * d.hx;
  Sp += transCoeff * velCur;
  Sp += d.relax * aP0 * velCur;
  if (d.conv == 1) Sp += sou_correction<IsU>(d, X, i, j, Fe, Fw, Fn, Fs);
  if (IsU) AT(d.dE, i, j) = d.hy / aP0; else AT(d.dN, i, j) = d.hx / aP0;
  const int iHi = IsU ? M - 1 : M - 2, jHi = IsU ? N - 2 : N - 1;
  const bool hasE = j + 1 <= jHi, hasW = j - 1 >= 1, hasN = i + 1 <= iHi, hasS = i - 1 >= 1;
  const double xE = AT(X, i, j + 1), xW = AT(X, i, j - 1), xN = AT(X, i + 1, j), xS = AT(X, i - 1, j);
  double cE = 0.0, cW = 0.0, cN = 0.0, cS = 0.0;
  if (hasE) cE = -aE; else Sp += aE * xE;
  if (hasW) cW = -aW; else Sp += aW * xW;
  if (hasN) cN = -aN; else Sp += aN * xN;
  if (hasS) cS = -aS; else Sp += aS * xS;
  double* c = IsU ? d.cU : d.cV;
  const long long ps = d.planeStride;
  const size_t o = (size_t)i * P + j;
  c[o] = cE;
  c[o + ps] = cW;
  c[o + 2 * ps] = cN;
  c[o + 3 * ps] = cS;
  c[o + 4 * ps] = aP;
  (IsU ? d.bU : d.bV)[o] = Sp;
  if (!sweep) {
    (IsU ? d.xU0 : d.xV0)[o] = velCur;
    return 0.0;
  }
  double Ax = 0.0;
  if (hasS) Ax += cS * xS;
  if (hasW) Ax += cW * xW;
  Ax += aP * velCur;
  if (hasE) Ax += cE * xE;
  if (hasN) Ax += cN * xN;
  const double r = Sp - Ax;
  (IsU ? d.xU1 : d.xV1)[o] = velCur + r / aP;
  return r * r;
}

// Jacobi sweep k >= 2 at one unknown (jacobi_solver.cpp:49-57).
template <bool IsU>
__device__ __forceinline__ double sweep_point(const DesignView& d, int i, int j, const double* __restrict__ xin,
                                              double* __restrict__ xout) {
  const int M = d.M, N = d.N, P = d.P;
  const int iHi = IsU ? M - 1 : M - 2, jHi = IsU ? N - 2 : N - 1;
  const double* __restrict__ c = IsU ? d.cU : d.cV;
  const long long ps = d.planeStride;
  const size_t o = (size_t)i * P + j;
  double Ax = 0.0;
  if (i - 1 >= 1) Ax += __ldg(c + o + 3 * ps) * xin[o - P];
  if (j - 1 >= 1) Ax += __ldg(c + o + ps) * xin[o - 1];
  const double aP = c[o + 4 * ps];
  const double x0 = xin[o];
  Ax += aP * x0;
  if (j + 1 <= jHi) Ax += c[o] * xin[o + 1];
  if (i + 1 <= iHi) Ax += c[o + 2 * ps] * xin[o + P];
  const double r = (IsU ? d.bU : d.bV)[o] - Ax;
  xout[o] = x0 + r / aP;
  return r * r;
}

// u* after scatter + clamp + velocity BCs, evaluated from the final Jacobi
// iterate (momentum_solver.cpp:326, boundaries.cpp:57-103).
__device__ __forceinline__ double ustar_at(const DesignView& d, const double* __restrict__ xU, int i, int j) {
  const int M = d.M, N = d.N, P = d.P;
  if (i <= 0 || i >= M) return 0.0;
  if (j == 0) return (AT(d.gamma, i - 1, 0) > 0.5) ? d.Uin : 0.0;
  if (j >= N - 1) j = N - 2;
  return clampd(AT(xU, i, j), -d.maxVel, d.maxVel);
}
__device__ __forceinline__ double vstar_at(const DesignView& d, const double* __restrict__ xV, int i, int j) {
  const int M = d.M, N = d.N, P = d.P;
  if (i <= 0 || i >= M - 1 || j == 0) return 0.0;
  if (j >= N) j = N - 1;
  return clampd(AT(xV, i, j), -d.maxVel, d.maxVel);
}

// Pressure-correction coefficients of P-unknown (i, j) (pressure_solver.cpp:698-703).
struct PCoef {
  double aE, aW, aN, aS, aP;
};
__device__ __forceinline__ PCoef pcoef(const DesignView& d, int i, int j) {
  const int M = d.M, N = d.N, P = d.P;
  PCoef c;
  c.aE = (j < N - 1) ? d.rho * AT(d.dE, i, j) * d.hy : 0.0;
  c.aW = (j > 1) ? d.rho * AT(d.dE, i, j - 1) * d.hy : 0.0;
  c.aN = (i < M - 1) ? d.rho * AT(d.dN, i, j) * d.hx : 0.0;
  c.aS = (i > 1) ? d.rho * AT(d.dN, i - 1, j) * d.hx : 0.0;
  c.aP = c.aE + c.aW + c.aN + c.aS;
  if (c.aP < 1e-20) c.aP = 1.0;
  return c;
}

// ---------------------------------------------------------------------------
// Tile iteration over the region i = 1..M-1, j = 1..N-1 shared by all phases.
// ---------------------------------------------------------------------------
template <class F>
__device__ __forceinline__ void for_each_point(const DesignView& d, unsigned rank, unsigned nblk, F&& f) {
  const int tilesJ = (d.N - 1 + kTileJ - 1) / kTileJ;
  const int tilesI = (d.M - 1 + kTileI - 1) / kTileI;
  const int ty = threadIdx.x >> 5, tx = threadIdx.x & 31;
  for (int t = rank; t < tilesI * tilesJ; t += nblk) {
    const int i = 1 + (t / tilesJ) * kTileI + ty;
    const int j = 1 + (t % tilesJ) * kTileJ + tx;
    if (i <= d.M - 1 && j <= d.N - 1) f(i, j);
  }
}

// ---------------------------------------------------------------------------
// One outer iteration for one design on group g.  Returns false if the group
// must stop (device error).  out[8] receives the step diagnostics.
// ---------------------------------------------------------------------------
// Returns 0 to continue with another outer iteration, 1 when this one is the
// last (iteration budget, convergence, or a non-finite residual), -1 when the
// group must stop because a device-side wait failed.
template <class Group>
__device__ int outer_iteration(const DesignView& d, Group& g, double* smem, double (&out)[8], bool lastIter,
                               bool stopOnConv, double eps) {
  const int M = d.M, N = d.N, P = d.P;
  // ---- A: assembly + sweep 1 ----
  const bool anySweep = d.maxMomIter > 0;
  double red2[2] = {0.0, 0.0};
  for_each_point(d, g.rank, g.nblk, [&](int i, int j) {
    if (j <= N - 2) red2[0] += assemble_point<true>(d, i, j, anySweep);
    if (i <= M - 2) red2[1] += assemble_point<false>(d, i, j, anySweep);
  });
  if (!g.template sync_reduce<2, 0u>(red2, smem)) return -1;
  int kU = anySweep ? 1 : 0, kV = kU;
  bool actU = anySweep && !(red2[0] < d.thrU) && kU < d.maxMomIter;
  bool actV = anySweep && !(red2[1] < d.thrV) && kV < d.maxMomIter;
  // ---- B: sweeps 2.. ----
  while (actU || actV) {
    const int k = (actU ? kU : kV) + 1;  // both active components are at the same sweep
    const double* xinU = (k & 1) ? d.xU0 : d.xU1;
    double* xoutU = (k & 1) ? d.xU1 : d.xU0;
    const double* xinV = (k & 1) ? d.xV0 : d.xV1;
    double* xoutV = (k & 1) ? d.xV1 : d.xV0;
    double s[2] = {0.0, 0.0};
    const bool au = actU, av = actV;
    for_each_point(d, g.rank, g.nblk, [&](int i, int j) {
      if (au && j <= N - 2) s[0] += sweep_point<true>(d, i, j, xinU, xoutU);
      if (av && i <= M - 2) s[1] += sweep_point<false>(d, i, j, xinV, xoutV);
    });
    if (!g.template sync_reduce<2, 0u>(s, smem)) return -1;
    if (au) { kU = k; actU = !(s[0] < d.thrU) && kU < d.maxMomIter; }
    if (av) { kV = k; actV = !(s[1] < d.thrV) && kV < d.maxMomIter; }
  }
  const double* xfU = (kU & 1) ? d.xU1 : d.xU0;
  const double* xfV = (kV & 1) ? d.xV1 : d.xV0;
  // ---- C: scatter, BCs, mass residual, PCG set-up ----
  // residU, residV, residMass, residMassDof, non-finite flag (max); r.z (sum)
  double rc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  for_each_point(d, g.rank, g.nblk, [&](int i, int j) {
    const size_t o = (size_t)i * P + j;
    if (j <= N - 2) {
      const double val = clampd(xfU[o], -d.maxVel, d.maxVel);
      d.us[o] = val;
      rc[0] = maxd(rc[0], fabs(val - d.u[o]));
      if (!isfinite(val)) rc[4] = 1.0;
      if (j == N - 2) d.us[o + 1] = val;
    }
    if (j == 1) d.us[o - 1] = ustar_at(d, xfU, i, 0);
    if (i <= M - 2) {
      const double val = clampd(xfV[o], -d.maxVel, d.maxVel);
      d.vs[o] = val;
      rc[1] = maxd(rc[1], fabs(val - d.v[o]));
      if (!isfinite(val)) rc[4] = 1.0;
      if (j == N - 1) d.vs[o + 1] = val;
    }
    const double massE = d.rho * ustar_at(d, xfU, i, j) * d.hy;
    const double massW = d.rho * ustar_at(d, xfU, i, j - 1) * d.hy;
    const double massN = d.rho * vstar_at(d, xfV, i, j) * d.hx;
    const double massS = d.rho * vstar_at(d, xfV, i - 1, j) * d.hx;
    const double b = massW - massE + massS - massN;
    const double ab = fabs(b);
    if (!isfinite(ab)) rc[4] = 1.0;
    if (ab > rc[2]) rc[2] = ab;
    if (j <= N - 2) {
      if (ab > rc[3]) rc[3] = ab;
      const PCoef c = pcoef(d, i, j);
      d.pdiag[o] = c.aP;
      d.pr[o] = b;
      d.px[o] = 0.0;
      const double z = (fabs(c.aP) > 1e-20) ? b / c.aP : b;
      d.pz[o] = z;
      d.pp0[o] = z;
      rc[5] += b * z;
    }
  });
  if (!g.template sync_reduce<6, 0x1Fu>(rc, smem)) return -1;
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
  if (!finite && g.rank == 0 && threadIdx.x == 0) atomicCAS(g.status, kStatusOk, kStatusDiverged);
  const bool stop = lastIter || !finite || (stopOnConv && conv <= eps);
  // ---- P: Jacobi-preconditioned CG ----
  double rz = rc[5], beta = 0.0;
  int it = 0;
  for (; it < d.maxPIter; ++it) {
    const double* pold = (it & 1) ? d.pp0 : d.pp1;  // p_{it-1}
    double* pcur = (it & 1) ? d.pp1 : d.pp0;        // p_it
    const int k = it;
    const double bt = beta;
    double s1[1] = {0.0};
    for_each_point(d, g.rank, g.nblk, [&](int i, int j) {
      if (j > N - 2) return;
      const size_t o = (size_t)i * P + j;
      // p_k at (i, j) and its unknown neighbours: p = z + beta p (pressure_solver.cpp:181)
      auto pk = [&](size_t q) -> double { return k == 0 ? d.pp0[q] : d.pz[q] + bt * pold[q]; };
      const PCoef c = pcoef(d, i, j);
      const double pc0 = pk(o);
      double Ap = 0.0;
      if (i > 1) Ap += -c.aS * pk(o - P);
      if (j > 1) Ap += -c.aW * pk(o - 1);
      Ap += c.aP * pc0;
      if (j + 1 <= N - 2) Ap += -c.aE * pk(o + 1);
      if (i < M - 1) Ap += -c.aN * pk(o + P);
      if (k > 0) pcur[o] = pc0;
      d.pAp[o] = Ap;
      s1[0] += pc0 * Ap;
    });
    if (!g.template sync_reduce<1, 0u>(s1, smem)) return -1;
    const double pAp = s1[0];
    if (fabs(pAp) < 1e-20) break;
    const double alpha = rz / pAp;
    double s2[2] = {0.0, 0.0};  // |r|^2, r.z
    for_each_point(d, g.rank, g.nblk, [&](int i, int j) {
      if (j > N - 2) return;
      const size_t o = (size_t)i * P + j;
      d.px[o] = d.px[o] + alpha * pcur[o];
      const double r = d.pr[o] - alpha * d.pAp[o];
      d.pr[o] = r;
      s2[0] += r * r;
      const double dg = d.pdiag[o];
      const double z = (fabs(dg) > 1e-20) ? r / dg : r;
      d.pz[o] = z;
      s2[1] += r * z;
    });
    if (!g.template sync_reduce<2, 0u>(s2, smem)) return -1;
    if (sqrt(s2[0]) < d.pTol) break;
    const double rzPrev = rz;
    rz = s2[1];
    beta = rz / rzPrev;
  }
  out[5] = it;
  // ---- D: pressure and velocity correction ----
  for_each_point(d, g.rank, g.nblk, [&](int i, int j) {
    const size_t o = (size_t)i * P + j;
    const double pcv = (j == N - 1) ? 0.0 : d.px[o];
    d.pc[o] = pcv;
    const double pn = d.p[o] + d.pAlpha * pcv;
    d.p[o] = pn;
    if (i == 1) d.p[o - P] = pn;
    if (i == M - 1) d.p[o + P] = pn;
    if (j == 1) d.p[o - 1] = pn;
    if (j == N - 1) d.p[o + 1] = 0.0;
    const double mv = d.maxVel;
    if (j <= N - 2) {
      const double pcE = (j + 1 == N - 1) ? 0.0 : d.px[o + 1];
      double du = d.dE[o] * (pcv - pcE);
      du = maxd(-mv, mind(mv, du));
      double un = d.us[o] + du;
      un = maxd(-mv, mind(mv, un));
      d.u[o] = un;
      if (j == N - 2) d.u[o + 1] = un;
    }
    if (i <= M - 2) {
      const double pcN = (j == N - 1) ? 0.0 : d.px[o + P];
      double dv = d.dN[o] * (pcv - pcN);
      dv = maxd(-mv, mind(mv, dv));
      double vn = d.vs[o] + dv;
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
      d.u[o - 1] = (AT(d.gamma, i - 1, 0) > 0.5) ? d.Uin : 0.0;
      d.v[o - 1] = 0.0;
    }
  });
  if (!stop) return g.sync() ? 0 : -1;
  return 1;
}

#undef AT

}  // namespace cps
