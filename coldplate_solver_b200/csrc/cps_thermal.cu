// The 3-D conjugate-heat-transfer solve (include/cps_thermal.h) on one GPU.
//
// Assembly: one thread per cell evaluates the reference's per-cell formulas
// (ThermalSolver/thermal_solver.cpp:438-517) in their operation order and
// writes seven coefficient planes and the right-hand side; an off-diagonal
// plane holds the merged CSR entry (diffusion plus upwind advection) of
// SparseMatrix::from_coo.  Nothing is assembled on the host.
//
// Preconditioner: structured aggregation multigrid.  Level l+1 aggregates
// 2 x 2 x 1 cells of level l (in-plane only: the z layers have different
// thicknesses and conductivities and stay separate), and its operator is the
// exact Galerkin product P^T A P of the piecewise-constant prolongation, which
// on a 7-point stencil is again a 7-point stencil (in-aggregate couplings fold
// into the diagonal).  Levels run down to one column of Nz cells, solved
// exactly (tridiagonal).  V-cycle: damped Jacobi before and after the coarse
// correction, the correction over-scaled (unsmoothed aggregation needs it).
//
// Krylov: BiCGStab (the system is non-symmetric: upwind advection), right
// preconditioned by one V-cycle per application, in one persistent
// cooperative kernel with the bounded software grid barrier and the
// fixed-order grid reductions of the flow solver: no host round trip per
// iteration, run-to-run identical results.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/cps_thermal.h"
#include "cps_device.cuh"

namespace cpt {

constexpr int kMaxLevels = 16;
constexpr int kMaxNz = 64;
constexpr int kMaxCtas = 2048;
enum Plane { kW = 0, kE, kS, kN, kB, kT, kD };

struct Level {
  int nx, ny, nz, n;
  double* c[7];    // W E S N B T diagonal
  double* x0;      // iterate / correction (coarse levels)
  double* x1;      // Jacobi partner
  double* b;       // restricted residual (coarse levels)
};

struct View {
  int nlev, maxiter, sweeps;
  double rtol, omega, alpha;
  Level lv[kMaxLevels];
  double *rhs, *T, *r, *rhat, *p, *v, *s, *t;  // level-0 Krylov vectors
  double *ph0, *ph1, *sh0, *sh1;               // level-0 V-cycle buffers for M^-1 p and M^-1 s
  double* out;                                 // iterations, converged, rel residual, true rel residual
};

struct Inputs {
  int Nx, Ny, nzs, nzf;
  double dx, dy, Hb, Ht, ks, kf, rhoCp, Tin, qk;
  int mode;
  const double *gamma, *u, *v, *q0;
};

__device__ __forceinline__ double maxd(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double mind(double a, double b) { return (b < a) ? b : a; }

// kval (thermal_solver.cpp:283-312)
__device__ __forceinline__ double kval(const Inputs& in, int i, int j, int k) {
  if (k < in.nzs) return in.ks;
  double g = in.gamma[j * in.Nx + i];
  g = maxd(0.0, mind(1.0, g));
  if (in.mode == 1) {
    const double num = 1.0 - g;
    const double den = 1.0 + in.qk * g;
    return in.kf + (in.ks - in.kf) * num / den;
  }
  if (in.mode == 2) return in.ks * in.kf / ((1.0 - g) * in.kf + g * in.ks + 1e-30);
  return in.ks * (1.0 - g) + in.kf * g;
}

__device__ __forceinline__ int region(const Inputs& in, int i, int j, int k) {
  if (k < in.nzs) return 0;
  return in.gamma[j * in.Nx + i] > 0.01 ? 1 : 0;
}

__device__ __forceinline__ double harm(double a, double b) { return 2 * a * b / (a + b + 1e-30); }

__device__ __forceinline__ double dz_of(const Inputs& in, int k) {
  return k < in.nzs ? in.Hb / in.nzs : in.Ht / in.nzf;
}

// pois (thermal_solver.cpp:336-340)
__device__ __forceinline__ double pois(const Inputs& in, int k) {
  if (k < in.nzs) return 0;
  const double z = (k - in.nzs + 0.5) * (in.Ht / in.nzf) / in.Ht;
  return 4.0 * z * (1 - z);
}

// One row of the system (thermal_solver.cpp:443-517), one thread per cell.
__global__ void assemble_kernel(Inputs in, Level L, double* rhs) {
  const int Nx = in.Nx, Ny = in.Ny, Nz = in.nzs + in.nzf;
  const int n = Nx * Ny * Nz;
  for (int P = blockIdx.x * blockDim.x + threadIdx.x; P < n; P += gridDim.x * blockDim.x) {
    const int i = P % Nx, j = (P / Nx) % Ny, k = P / (Nx * Ny);
    const double dx = in.dx, dy = in.dy, rhoCp = in.rhoCp, T_in = in.Tin;
    const double dz_k = dz_of(in, k), Ax = dy * dz_k, Ay = dx * dz_k, Az_cell = dx * dy;
    double diag = 0, bP = 0;
    const double kP = kval(in, i, j, k), po = pois(in, k);
    double g = (k < in.nzs) ? 0.0 : in.gamma[j * Nx + i];
    g = maxd(0.0, mind(1.0, g));
    const double uP = (g > 0.01) ? in.u[j * Nx + i] * po : 0.0;
    const double vP = (g > 0.01) ? in.v[j * Nx + i] * po : 0.0;
    const int rP = region(in, i, j, k);
    double cW = 0, cE = 0, cS = 0, cN = 0, cB = 0, cT = 0;
    if (i > 0) {
      const double D = harm(kP, kval(in, i - 1, j, k)) * Ax / dx;
      diag += D;
      cW = -D;
      if (rP == 1 && region(in, i - 1, j, k) == 1) {
        const double uW = in.u[j * Nx + i - 1] * po, F = rhoCp * 0.5 * (uP + uW) * Ax;
        diag += maxd(-F, 0.0);
        cW = cW + -maxd(F, 0.0);
      }
    } else if (rP == 1) {
      const double D_bc = 2.0 * kP * Ax / dx, F_bc = rhoCp * uP * Ax;
      diag += D_bc;
      bP += D_bc * T_in;
      if (F_bc > 0) bP += F_bc * T_in; else diag += -F_bc;
    }
    if (i < Nx - 1) {
      const double D = harm(kP, kval(in, i + 1, j, k)) * Ax / dx;
      diag += D;
      cE = -D;
      if (rP == 1 && region(in, i + 1, j, k) == 1) {
        const double uE = in.u[j * Nx + i + 1] * po, F = rhoCp * 0.5 * (uP + uE) * Ax;
        diag += maxd(F, 0.0);
        cE = cE + -maxd(-F, 0.0);
      }
    } else if (rP == 1 && uP > 0) {
      diag += rhoCp * uP * Ax;
    }
    if (j > 0) {
      const double D = harm(kP, kval(in, i, j - 1, k)) * Ay / dy;
      diag += D;
      cS = -D;
      if (rP == 1 && region(in, i, j - 1, k) == 1) {
        const double vS = in.v[(j - 1) * Nx + i] * po, F = rhoCp * 0.5 * (vP + vS) * Ay;
        diag += maxd(-F, 0.0);
        cS = cS + -maxd(F, 0.0);
      }
    }
    if (j < Ny - 1) {
      const double D = harm(kP, kval(in, i, j + 1, k)) * Ay / dy;
      diag += D;
      cN = -D;
      if (rP == 1 && region(in, i, j + 1, k) == 1) {
        const double vN = in.v[(j + 1) * Nx + i] * po, F = rhoCp * 0.5 * (vP + vN) * Ay;
        diag += maxd(F, 0.0);
        cN = cN + -maxd(-F, 0.0);
      }
    } else if (rP == 1 && vP > 0) {
      diag += rhoCp * vP * Ay;
    }
    if (k > 0) {
      const double kN = kval(in, i, j, k - 1), dz_P = dz_k, dz_N = dz_of(in, k - 1);
      const double kf = (dz_P + dz_N) / (dz_P / kP + dz_N / kN);
      const double D = kf * Az_cell / (0.5 * (dz_P + dz_N));
      diag += D;
      cB = -D;
    } else {
      bP += in.q0[j * Nx + i] * Az_cell;
    }
    if (k < Nz - 1) {
      const double kN = kval(in, i, j, k + 1), dz_P = dz_k, dz_N = dz_of(in, k + 1);
      const double kf = (dz_P + dz_N) / (dz_P / kP + dz_N / kN);
      const double D = kf * Az_cell / (0.5 * (dz_P + dz_N));
      diag += D;
      cT = -D;
    }
    L.c[kW][P] = cW;
    L.c[kE][P] = cE;
    L.c[kS][P] = cS;
    L.c[kN][P] = cN;
    L.c[kB][P] = cB;
    L.c[kT][P] = cT;
    L.c[kD][P] = diag + 1e-12;
    rhs[P] = bP;
  }
}

// Galerkin operator of level f's 2 x 2 x 1 aggregates, one thread per coarse cell.
__global__ void coarsen_kernel(Level F, Level C) {
  const int cplane = C.nx * C.ny, fplane = F.nx * F.ny;
  for (int Q = blockIdx.x * blockDim.x + threadIdx.x; Q < C.n; Q += gridDim.x * blockDim.x) {
    const int I = Q % C.nx, J = (Q / C.nx) % C.ny, k = Q / cplane;
    double a[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int bb = 0; bb < 2; ++bb)
      for (int aa = 0; aa < 2; ++aa) {
        const int i = 2 * I + aa, j = 2 * J + bb;
        if (i >= F.nx || j >= F.ny) continue;
        const int f = k * fplane + j * F.nx + i;
        a[kD] += F.c[kD][f];
        a[kB] += F.c[kB][f];
        a[kT] += F.c[kT][f];
        if (i > 0) { if ((i - 1) / 2 == I) a[kD] += F.c[kW][f]; else a[kW] += F.c[kW][f]; }
        if (i < F.nx - 1) { if ((i + 1) / 2 == I) a[kD] += F.c[kE][f]; else a[kE] += F.c[kE][f]; }
        if (j > 0) { if ((j - 1) / 2 == J) a[kD] += F.c[kS][f]; else a[kS] += F.c[kS][f]; }
        if (j < F.ny - 1) { if ((j + 1) / 2 == J) a[kD] += F.c[kN][f]; else a[kN] += F.c[kN][f]; }
      }
    for (int p = 0; p < 7; ++p) C.c[p][Q] = a[p];
  }
}

// (A x)[P] on level L, the entries in CSR column order.
__device__ __forceinline__ double apply(const Level& L, const double* __restrict__ x, int P) {
  const int nx = L.nx, plane = L.nx * L.ny;
  const int i = P % nx, j = (P / nx) % L.ny, k = P / plane;
  double s = 0.0;
  if (k > 0) s += L.c[kB][P] * x[P - plane];
  if (j > 0) s += L.c[kS][P] * x[P - nx];
  if (i > 0) s += L.c[kW][P] * x[P - 1];
  s += L.c[kD][P] * x[P];
  if (i < nx - 1) s += L.c[kE][P] * x[P + 1];
  if (j < L.ny - 1) s += L.c[kN][P] * x[P + nx];
  if (k < L.nz - 1) s += L.c[kT][P] * x[P + plane];
  return s;
}

struct Loop {
  int start, stride;
  __device__ Loop() : start(blockIdx.x * blockDim.x + threadIdx.x), stride(gridDim.x * blockDim.x) {}
};

// Levels with at most this many cells run inside CTA 0 alone (block-stride
// loops, CTA barriers): below it a grid barrier costs more than the work.
constexpr int kLocalCells = 2048;

// Where a phase runs: the whole grid (grid-stride loops, grid barrier) or,
// with Local, CTA 0 alone (block-stride loops, __syncthreads).
template <bool Local>
struct Exec {
  int start, stride;
  cps::GridGroup* g;
  __device__ explicit Exec(cps::GridGroup* gg) : g(gg) {
    start = Local ? (int)threadIdx.x : (int)(blockIdx.x * blockDim.x + threadIdx.x);
    stride = Local ? (int)blockDim.x : (int)(gridDim.x * blockDim.x);
  }
  __device__ bool sync() {
    if (Local) {
      __syncthreads();
      return true;
    }
    return g->sync();
  }
};

// The first level at or below which every level is small enough for CTA 0.
__device__ __forceinline__ int local_from(const View& tv) {
  int l = tv.nlev - 1;
  while (l > 0 && tv.lv[l - 1].n <= kLocalCells) --l;
  return l;
}

// One V-cycle over levels [l0, nlev) on rhs0 (level l0), iterate buffers
// a0/a1 of level l0.  Every non-coarsest level's result ends in its second
// buffer (2 sweeps - 1 swaps in all), the coarsest's in its first; so the
// caller knows where the result is without being told.  The grid instance
// hands the small levels to CTA 0 and waits at one grid barrier.
template <bool Local>
__device__ double* vcycle_from(const View& tv, cps::GridGroup& g, int l0, const double* rhs0, double* a0, double* a1,
                               bool& ok) {
  Exec<Local> ex(&g);
  double* cur[kMaxLevels];
  double* oth[kMaxLevels];
  const double w = tv.omega;
  const double* rhs = rhs0;
  const int last = tv.nlev - 1;
  const int split = Local ? last + 1 : local_from(tv);  // grid instance: levels >= split go to CTA 0
  int l = l0;
  for (; l < last && (Local || l < split); ++l) {
    const Level& L = tv.lv[l];
    double* xa = l == l0 ? a0 : L.x0;
    double* xb = l == l0 ? a1 : L.x1;
    for (int P = ex.start; P < L.n; P += ex.stride) xa[P] = w * rhs[P] / L.c[kD][P];
    if (!ex.sync()) { ok = false; return a0; }
    for (int sw = 1; sw < tv.sweeps; ++sw) {
      for (int P = ex.start; P < L.n; P += ex.stride) xb[P] = xa[P] + w * (rhs[P] - apply(L, xa, P)) / L.c[kD][P];
      double* tmp = xa; xa = xb; xb = tmp;
      if (!ex.sync()) { ok = false; return a0; }
    }
    const Level& C = tv.lv[l + 1];
    const int fplane = L.nx * L.ny, cplane = C.nx * C.ny;
    for (int Q = ex.start; Q < C.n; Q += ex.stride) {
      const int I = Q % C.nx, J = (Q / C.nx) % C.ny, k = Q / cplane;
      double acc = 0.0;
      for (int bb = 0; bb < 2; ++bb)
        for (int aa = 0; aa < 2; ++aa) {
          const int i = 2 * I + aa, j = 2 * J + bb;
          if (i >= L.nx || j >= L.ny) continue;
          const int f = k * fplane + j * L.nx + i;
          acc += rhs[f] - apply(L, xa, f);
        }
      C.b[Q] = acc;
    }
    if (!ex.sync()) { ok = false; return a0; }
    cur[l] = xa;
    oth[l] = xb;
    rhs = C.b;
  }
  // l is now the first level this instance does not descend from
  if (!Local && l < last) {
    // levels [l, last] inside CTA 0; the rest of the grid waits at the barrier
    double* x0 = l == l0 ? a0 : tv.lv[l].x0;
    double* x1 = l == l0 ? a1 : tv.lv[l].x1;
    if (g.rank == 0) vcycle_from<true>(tv, g, l, rhs, x0, x1, ok);
    if (!g.sync()) { ok = false; return a0; }
    cur[l] = x1;
  } else {
    // coarsest: one column of nz cells, tridiagonal in z (Thomas algorithm)
    const Level& Z = tv.lv[last];
    double* xz = last == l0 ? a0 : Z.x0;
    if ((Local || g.rank == 0) && threadIdx.x == 0) {
      double cp[kMaxNz], dp[kMaxNz];
      const int nz = Z.nz;
      for (int k = 0; k < nz; ++k) {
        const double a = k > 0 ? Z.c[kB][k] : 0.0;
        const double m = Z.c[kD][k] - (k > 0 ? a * cp[k - 1] : 0.0);
        cp[k] = Z.c[kT][k] / m;
        dp[k] = (rhs[k] - (k > 0 ? a * dp[k - 1] : 0.0)) / m;
      }
      xz[nz - 1] = dp[nz - 1];
      for (int k = nz - 2; k >= 0; --k) xz[k] = dp[k] - cp[k] * xz[k + 1];
    }
    if (!ex.sync()) { ok = false; return a0; }
    cur[last] = xz;
    l = last;
  }
  for (int m = l - 1; m >= l0; --m) {
    const Level& L = tv.lv[m];
    const Level& C = tv.lv[m + 1];
    const double* rhsl = m == l0 ? rhs0 : L.b;
    double* xa = cur[m];
    double* xb = oth[m];
    const double* e = cur[m + 1];
    const int fplane = L.nx * L.ny, cplane = C.nx * C.ny;
    const double alpha = tv.alpha;
    // First post-smoothing sweep with the coarse correction folded in: every
    // value it reads is x + alpha e(parent), computed as the separate
    // prolongation pass would have stored it (the same operations, so the same
    // bits), which saves that pass and its barrier.
    for (int P = ex.start; P < L.n; P += ex.stride) {
      const int i = P % L.nx, j = (P / L.nx) % L.ny, k = P / fplane;
      auto xc = [&](int q, int ii, int jj, int kk) { return xa[q] + alpha * e[kk * cplane + (jj >> 1) * C.nx + (ii >> 1)]; };
      double s = 0.0;  // A x in apply()'s order
      if (k > 0) s += L.c[kB][P] * xc(P - fplane, i, j, k - 1);
      if (j > 0) s += L.c[kS][P] * xc(P - L.nx, i, j - 1, k);
      if (i > 0) s += L.c[kW][P] * xc(P - 1, i - 1, j, k);
      const double xP = xc(P, i, j, k);
      s += L.c[kD][P] * xP;
      if (i < L.nx - 1) s += L.c[kE][P] * xc(P + 1, i + 1, j, k);
      if (j < L.ny - 1) s += L.c[kN][P] * xc(P + L.nx, i, j + 1, k);
      if (k < L.nz - 1) s += L.c[kT][P] * xc(P + fplane, i, j, k + 1);
      xb[P] = xP + w * (rhsl[P] - s) / L.c[kD][P];
    }
    { double* tmp = xa; xa = xb; xb = tmp; }
    if (!ex.sync()) { ok = false; return a0; }
    for (int sw = 1; sw < tv.sweeps; ++sw) {
      for (int P = ex.start; P < L.n; P += ex.stride) xb[P] = xa[P] + w * (rhsl[P] - apply(L, xa, P)) / L.c[kD][P];
      double* tmp = xa; xa = xb; xb = tmp;
      if (!ex.sync()) { ok = false; return a0; }
    }
    cur[m] = xa;
  }
  return cur[l0];
}

__device__ double* vcycle(const View& tv, cps::GridGroup& g, const double* rhs0, double* a0, double* a1, bool& ok) {
  return vcycle_from<false>(tv, g, 0, rhs0, a0, a1, ok);
}

// BiCGStab, right-preconditioned by the V-cycle, from T = T_inlet.
// Three CTAs per SM (80 registers, no spills): the fine-level phases are
// bound by memory latency, and 24 warps per SM keep more loads in flight than
// 16 (B200, 1000 x 500 x 9 cells: 98 -> 84 ms per solve; four per SM spill
// and gain nothing more).
#ifndef CPT_MIN_BLOCKS
#define CPT_MIN_BLOCKS 3
#endif
__global__ void __launch_bounds__(cps::kThreads, CPT_MIN_BLOCKS) solve_kernel(View tv, double T_in, int warm, cps::GridBarrier* bar,
                                                                 double* red, int* status) {
  __shared__ double smem[cps::kRedWidth * 8];
  cps::GridGroup g{bar, red, status, blockIdx.x, gridDim.x, 0u, 0ull};
  const Loop lp;
  const Level& L = tv.lv[0];
  const int n = L.n;
  bool ok = true;
  double q2[2] = {0.0, 0.0};
  if (!warm) {
    for (int P = lp.start; P < n; P += lp.stride) tv.T[P] = T_in;
    if (!g.sync()) return;
  }
  for (int P = lp.start; P < n; P += lp.stride) {
    const double r = tv.rhs[P] - apply(L, tv.T, P);
    tv.r[P] = r;
    tv.rhat[P] = r;
    tv.p[P] = 0.0;
    tv.v[P] = 0.0;
    q2[0] += r * r;
    q2[1] += tv.rhs[P] * tv.rhs[P];
  }
  if (!g.sync_reduce<2, 0u>(q2, smem)) return;
  double bnorm = sqrt(q2[1]);
  if (!(bnorm > 0.0)) bnorm = 1.0;
  double rr = q2[0], rho = 1.0, alpha = 1.0, omega = 1.0, rho_new = q2[0];
  int it = 0;
  bool conv = sqrt(rr) <= tv.rtol * bnorm;
  while (!conv && it < tv.maxiter) {
    const double beta = (rho_new / rho) * (alpha / omega);
    for (int P = lp.start; P < n; P += lp.stride) tv.p[P] = tv.r[P] + beta * (tv.p[P] - omega * tv.v[P]);
    if (!g.sync()) return;
    double* ph = vcycle(tv, g, tv.p, tv.ph0, tv.ph1, ok);
    if (!ok) return;
    double q1[1] = {0.0};
    for (int P = lp.start; P < n; P += lp.stride) {
      const double vv = apply(L, ph, P);
      tv.v[P] = vv;
      q1[0] += tv.rhat[P] * vv;
    }
    if (!g.sync_reduce<1, 0u>(q1, smem)) return;
    alpha = rho_new / q1[0];
    double qs[1] = {0.0};
    for (int P = lp.start; P < n; P += lp.stride) {
      const double s = tv.r[P] - alpha * tv.v[P];
      tv.s[P] = s;
      qs[0] += s * s;
    }
    if (!g.sync_reduce<1, 0u>(qs, smem)) return;
    if (sqrt(qs[0]) <= tv.rtol * bnorm) {
      for (int P = lp.start; P < n; P += lp.stride) tv.T[P] += alpha * ph[P];
      rr = qs[0];
      ++it;
      conv = true;
      break;
    }
    double* sh = vcycle(tv, g, tv.s, tv.sh0, tv.sh1, ok);
    if (!ok) return;
    double q3[2] = {0.0, 0.0};
    for (int P = lp.start; P < n; P += lp.stride) {
      const double tt = apply(L, sh, P);
      tv.t[P] = tt;
      q3[0] += tt * tv.s[P];
      q3[1] += tt * tt;
    }
    if (!g.sync_reduce<2, 0u>(q3, smem)) return;
    omega = q3[1] > 0.0 ? q3[0] / q3[1] : 0.0;
    double q4[2] = {0.0, 0.0};
    for (int P = lp.start; P < n; P += lp.stride) {
      tv.T[P] += alpha * ph[P] + omega * sh[P];
      const double r = tv.s[P] - omega * tv.t[P];
      tv.r[P] = r;
      q4[0] += tv.rhat[P] * r;
      q4[1] += r * r;
    }
    if (!g.sync_reduce<2, 0u>(q4, smem)) return;
    rho = rho_new;
    rho_new = q4[0];
    rr = q4[1];
    ++it;
    conv = sqrt(rr) <= tv.rtol * bnorm;
    if (!isfinite(rr) || rho_new == 0.0 || omega == 0.0) break;  // breakdown: report what was reached
  }
  if (!g.sync()) return;
  double qt[1] = {0.0};
  for (int P = lp.start; P < n; P += lp.stride) {
    const double r = tv.rhs[P] - apply(L, tv.T, P);
    qt[0] += r * r;
  }
  if (!g.sync_reduce<1, 0u>(qt, smem)) return;
  if (g.rank == 0 && threadIdx.x == 0) {
    tv.out[0] = it;
    tv.out[1] = conv ? 1.0 : 0.0;
    tv.out[2] = sqrt(rr) / bnorm;
    tv.out[3] = sqrt(qt[0]) / bnorm;
    if (!isfinite(rr)) atomicCAS(status, cps::kStatusOk, cps::kStatusDiverged);
  }
}

}  // namespace cpt

struct cps_thermal {
  int device = 0;
  cudaStream_t stream = nullptr;
  cps_thermal_desc desc{};
  cpt::Inputs in{};
  cpt::View view{};
  char* slab = nullptr;
  double *dgamma = nullptr, *du = nullptr, *dv = nullptr, *dq = nullptr;
  cps::GridBarrier* bar = nullptr;
  double* red = nullptr;
  int* status = nullptr;
  double* hout = nullptr;  // pinned: out[4] + status
  int grid = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double kernel_ms = 0.0;
  std::string err;
};

namespace {

thread_local std::string g_thermal_error;

cps_status tfail(cps_thermal* t, cps_status s, const std::string& m) {
  if (t) t->err = m;
  g_thermal_error = m;
  return s;
}

bool tcuda(cps_thermal* t, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return true;
  tfail(t, CPS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return false;
}

// Upload the 2-D inputs (q0 NULL: the uniform flux) and assemble level 0 and
// the hierarchy, in stream order.
cps_status assemble(cps_thermal* t, const double* gamma, const double* u, const double* v, const double* q0) {
  const size_t n2 = (size_t)t->desc.Nx * t->desc.Ny, bytes = n2 * sizeof(double);
  if (gamma && !tcuda(t, cudaMemcpyAsync(t->dgamma, gamma, bytes, cudaMemcpyHostToDevice, t->stream), "h2d"))
    return CPS_ERR_CUDA;
  if (u && !tcuda(t, cudaMemcpyAsync(t->du, u, bytes, cudaMemcpyHostToDevice, t->stream), "h2d")) return CPS_ERR_CUDA;
  if (v && !tcuda(t, cudaMemcpyAsync(t->dv, v, bytes, cudaMemcpyHostToDevice, t->stream), "h2d")) return CPS_ERR_CUDA;
  if (q0) {
    if (!tcuda(t, cudaMemcpyAsync(t->dq, q0, bytes, cudaMemcpyHostToDevice, t->stream), "h2d")) return CPS_ERR_CUDA;
  }
  if (!tcuda(t, cudaStreamSynchronize(t->stream), "h2d")) return CPS_ERR_CUDA;
  const cpt::View& tv = t->view;
  const int n0 = tv.lv[0].n;
  cpt::assemble_kernel<<<std::min(4096, (n0 + 255) / 256), 256, 0, t->stream>>>(t->in, tv.lv[0], tv.rhs);
  if (!tcuda(t, cudaGetLastError(), "assemble launch")) return CPS_ERR_CUDA;
  for (int l = 1; l < tv.nlev; ++l) {
    const int nc = tv.lv[l].n;
    cpt::coarsen_kernel<<<std::min(4096, (nc + 255) / 256), 256, 0, t->stream>>>(tv.lv[l - 1], tv.lv[l]);
    if (!tcuda(t, cudaGetLastError(), "coarsen launch")) return CPS_ERR_CUDA;
  }
  if (!tcuda(t, cudaStreamSynchronize(t->stream), "assembly")) return CPS_ERR_CUDA;
  return CPS_OK;
}

}  // namespace

extern "C" {

cps_status cps_thermal_defaults(cps_thermal_desc* d) {
  if (!d) return tfail(nullptr, CPS_ERR_ARG, "desc is NULL");
  std::memset(d, 0, sizeof(*d));
  // Params (thermal_solver.cpp:147-193)
  d->nz_solid = 2;
  d->nz_fluid = 7;
  d->H_b = 0.0005;
  d->H_t = 0.004;
  d->k_s = 400.0;
  d->k_f = 0.6;
  d->rho = 998.0;
  d->Cp = 4180.0;
  d->T_inlet = 30.0;
  d->rtol = 1e-6;
  d->maxiter = 1000;
  d->k_interp_mode = 1;
  d->qk = 1.0;
  return CPS_OK;
}

cps_status cps_thermal_create(const cps_thermal_desc* d, cps_thermal** out) {
  if (!d || !out) return tfail(nullptr, CPS_ERR_ARG, "desc and out are required");
  *out = nullptr;
  if (d->Nx < 1 || d->Ny < 1 || d->nz_solid < 1 || d->nz_fluid < 1 || d->nz_solid + d->nz_fluid > cpt::kMaxNz)
    return tfail(nullptr, CPS_ERR_ARG, "need Nx, Ny, nz_solid, nz_fluid >= 1 and nz_solid + nz_fluid <= 64");
  const long long n0ll = (long long)d->Nx * d->Ny * (d->nz_solid + d->nz_fluid);
  if (n0ll > (1LL << 30)) return tfail(nullptr, CPS_ERR_ARG, "grid too large (more than 2^30 cells)");
  const double reals[] = {d->dx, d->dy, d->H_b, d->H_t, d->k_s, d->k_f, d->rho, d->Cp, d->rtol};
  for (double x : reals)
    if (!(x > 0.0) || !std::isfinite(x)) return tfail(nullptr, CPS_ERR_ARG, "dx, dy, H_b, H_t, k_s, k_f, rho, Cp, rtol must be > 0");
  if (!d->gamma || !d->u || !d->v) return tfail(nullptr, CPS_ERR_ARG, "gamma, u and v are required");
  if (d->k_interp_mode < 0 || d->k_interp_mode > 2) return tfail(nullptr, CPS_ERR_ARG, "k_interp_mode must be 0, 1 or 2");
  if (d->maxiter < 0) return tfail(nullptr, CPS_ERR_ARG, "maxiter < 0");
  cps_thermal* t = new (std::nothrow) cps_thermal();
  if (!t) return tfail(nullptr, CPS_ERR_OOM, "host allocation failed");
  auto bail = [&](cps_status s) {
    g_thermal_error = t->err;
    cps_thermal_destroy(t);
    return s;
  };
  t->desc = *d;
  t->device = d->device;
  const int Nz = d->nz_solid + d->nz_fluid;
  // levels: 2 x 2 in-plane aggregation down to one column
  cpt::View& tv = t->view;
  tv.nlev = 0;
  {
    int nx = d->Nx, ny = d->Ny;
    for (;;) {
      if (tv.nlev == cpt::kMaxLevels) return bail(tfail(t, CPS_ERR_ARG, "grid needs more than 16 multigrid levels"));
      cpt::Level& L = tv.lv[tv.nlev++];
      L.nx = nx;
      L.ny = ny;
      L.nz = Nz;
      L.n = nx * ny * Nz;
      if (nx == 1 && ny == 1) break;
      nx = (nx + 1) / 2;
      ny = (ny + 1) / 2;
    }
  }
  const size_t n0 = (size_t)tv.lv[0].n, n2 = (size_t)d->Nx * d->Ny;
  auto al = [](size_t elems) { return (elems * sizeof(double) + 255) / 256 * 256; };
  size_t bytes = al(n0) * (7 + 1 + 1 + 6 + 4);
  for (int l = 1; l < tv.nlev; ++l) bytes += al(tv.lv[l].n) * 10;
  bytes += al(n2) * 4 + 256 + al((size_t)cps::kRedSlots * cps::kRedWidth * cpt::kMaxCtas) + 256;
  if (!tcuda(t, cudaSetDevice(d->device), "cudaSetDevice") ||
      !tcuda(t, cudaStreamCreateWithFlags(&t->stream, cudaStreamNonBlocking), "stream"))
    return bail(CPS_ERR_CUDA);
  if (cudaMalloc(&t->slab, bytes) != cudaSuccess) return bail(tfail(t, CPS_ERR_OOM, "device allocation failed"));
  if (!tcuda(t, cudaMemsetAsync(t->slab, 0, bytes, t->stream), "memset") ||
      !tcuda(t, cudaMallocHost(&t->hout, 8 * sizeof(double)), "pinned alloc") ||
      !tcuda(t, cudaEventCreate(&t->ev0), "event") || !tcuda(t, cudaEventCreate(&t->ev1), "event"))
    return bail(CPS_ERR_CUDA);
  char* cur = t->slab;
  auto take = [&](size_t elems) {
    double* p = reinterpret_cast<double*>(cur);
    cur += al(elems);
    return p;
  };
  for (int p = 0; p < 7; ++p) tv.lv[0].c[p] = take(n0);
  tv.rhs = take(n0);
  tv.T = take(n0);
  tv.r = take(n0);
  tv.rhat = take(n0);
  tv.p = take(n0);
  tv.v = take(n0);
  tv.s = take(n0);
  tv.t = take(n0);
  tv.ph0 = take(n0);
  tv.ph1 = take(n0);
  tv.sh0 = take(n0);
  tv.sh1 = take(n0);
  tv.lv[0].x0 = tv.lv[0].x1 = tv.lv[0].b = nullptr;
  for (int l = 1; l < tv.nlev; ++l) {
    cpt::Level& L = tv.lv[l];
    for (int p = 0; p < 7; ++p) L.c[p] = take(L.n);
    L.x0 = take(L.n);
    L.x1 = take(L.n);
    L.b = take(L.n);
  }
  t->dgamma = take(n2);
  t->du = take(n2);
  t->dv = take(n2);
  t->dq = take(n2);
  tv.out = take(32);
  t->bar = reinterpret_cast<cps::GridBarrier*>(tv.out + 8);
  t->status = reinterpret_cast<int*>(tv.out + 16);
  t->red = take((size_t)cps::kRedSlots * cps::kRedWidth * cpt::kMaxCtas);
  tv.maxiter = d->maxiter;
  tv.rtol = d->rtol;
  tv.sweeps = d->mg_sweeps > 0 ? d->mg_sweeps : 2;
  tv.omega = d->mg_omega > 0.0 ? d->mg_omega : 0.8;
  tv.alpha = d->mg_overcorrect > 0.0 ? d->mg_overcorrect : 1.7;
  cpt::Inputs& in = t->in;
  in.Nx = d->Nx;
  in.Ny = d->Ny;
  in.nzs = d->nz_solid;
  in.nzf = d->nz_fluid;
  in.dx = d->dx;
  in.dy = d->dy;
  in.Hb = d->H_b;
  in.Ht = d->H_t;
  in.ks = d->k_s;
  in.kf = d->k_f;
  in.rhoCp = d->rho * d->Cp;
  in.Tin = d->T_inlet;
  in.qk = d->qk;
  in.mode = d->k_interp_mode;
  in.gamma = t->dgamma;
  in.u = t->du;
  in.v = t->dv;
  in.q0 = t->dq;
  if (!d->q0) {
    // main: s.q0.assign(Ny*Nx, qf) (thermal_solver.cpp:760).  On the handle's
    // stream, after the slab's memset: that stream does not order against the
    // legacy default stream.
    std::vector<double> q(n2, d->q);
    if (!tcuda(t, cudaMemcpyAsync(t->dq, q.data(), n2 * sizeof(double), cudaMemcpyHostToDevice, t->stream), "h2d") ||
        !tcuda(t, cudaStreamSynchronize(t->stream), "h2d"))
      return bail(CPS_ERR_CUDA);
  }
  const cps_status st = assemble(t, d->gamma, d->u, d->v, d->q0);
  if (st != CPS_OK) return bail(st);
  int per_sm = 0, sms = 0;
  if (!tcuda(t, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)cpt::solve_kernel, cps::kThreads, 0),
             "occupancy") ||
      !tcuda(t, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d->device), "attribute"))
    return bail(CPS_ERR_CUDA);
  if (per_sm < 1) return bail(tfail(t, CPS_ERR_CUDA, "solve kernel does not fit on an SM"));
  t->grid = std::max(1, std::min({sms * per_sm, cpt::kMaxCtas, (tv.lv[0].n + cps::kThreads - 1) / cps::kThreads}));
  *out = t;
  return CPS_OK;
}

cps_status cps_thermal_update(cps_thermal* t, const double* gamma, const double* u, const double* v,
                              const double* q0) {
  if (!t) return tfail(nullptr, CPS_ERR_ARG, "handle is NULL");
  if (!tcuda(t, cudaSetDevice(t->device), "cudaSetDevice")) return CPS_ERR_CUDA;
  return assemble(t, gamma, u, v, q0);
}

}  // extern "C"

namespace {

// One solve launch: from T = T_inlet, or (warm) from the handle's current temperature.
cps_status solve_launch(cps_thermal* t, int warm, cps_thermal_result* res) {
  cpt::View& tv = t->view;
  if (!tcuda(t, cudaMemsetAsync(tv.out, 0, 32 * sizeof(double), t->stream), "memset")) return CPS_ERR_CUDA;
  double T_in = t->desc.T_inlet;
  void* args[] = {&tv, &T_in, &warm, &t->bar, &t->red, &t->status};
  if (!tcuda(t, cudaEventRecord(t->ev0, t->stream), "event") ||
      !tcuda(t, cudaLaunchCooperativeKernel((const void*)cpt::solve_kernel, dim3(t->grid), dim3(cps::kThreads), args, 0,
                                            t->stream), "cooperative launch") ||
      !tcuda(t, cudaEventRecord(t->ev1, t->stream), "event") ||
      !tcuda(t, cudaMemcpyAsync(t->hout, tv.out, 4 * sizeof(double), cudaMemcpyDeviceToHost, t->stream), "d2h") ||
      !tcuda(t, cudaMemcpyAsync(t->hout + 4, t->status, sizeof(int), cudaMemcpyDeviceToHost, t->stream), "d2h") ||
      !tcuda(t, cudaStreamSynchronize(t->stream), "solve kernel"))
    return CPS_ERR_CUDA;
  float ms = 0.0f;
  if (cudaEventElapsedTime(&ms, t->ev0, t->ev1) == cudaSuccess) t->kernel_ms += ms;
  int status = 0;
  std::memcpy(&status, t->hout + 4, sizeof(int));
  if (res) {
    res->iterations = (int)t->hout[0];
    res->converged = t->hout[1] != 0.0;
    res->rel_residual = t->hout[2];
    res->true_rel_residual = t->hout[3];
  }
  if (status == cps::kStatusTimeout) return tfail(t, CPS_ERR_TIMEOUT, "device grid barrier timed out");
  if (status == cps::kStatusDiverged) return tfail(t, CPS_ERR_DIVERGED, "residual is not finite");
  return CPS_OK;
}

}  // namespace

extern "C" {

cps_status cps_thermal_solve(cps_thermal* t, cps_thermal_result* res) {
  if (!t) return tfail(nullptr, CPS_ERR_ARG, "handle is NULL");
  if (!tcuda(t, cudaSetDevice(t->device), "cudaSetDevice")) return CPS_ERR_CUDA;
  return solve_launch(t, 0, res);
}

cps_status cps_thermal_solve_from(cps_thermal* t, const double* T0, cps_thermal_result* res) {
  if (!t) return tfail(nullptr, CPS_ERR_ARG, "handle is NULL");
  if (!tcuda(t, cudaSetDevice(t->device), "cudaSetDevice")) return CPS_ERR_CUDA;
  if (T0) {
    const size_t n = (size_t)t->view.lv[0].n;
    if (!tcuda(t, cudaMemcpyAsync(t->view.T, T0, n * sizeof(double), cudaMemcpyHostToDevice, t->stream), "h2d"))
      return CPS_ERR_CUDA;
  }
  return solve_launch(t, 1, res);
}

cps_status cps_thermal_download(cps_thermal* t, double* T) {
  if (!t || !T) return tfail(t, CPS_ERR_ARG, "handle and T are required");
  if (!tcuda(t, cudaSetDevice(t->device), "cudaSetDevice")) return CPS_ERR_CUDA;
  const size_t n = (size_t)t->view.lv[0].n;
  if (!tcuda(t, cudaMemcpyAsync(T, t->view.T, n * sizeof(double), cudaMemcpyDeviceToHost, t->stream), "d2h") ||
      !tcuda(t, cudaStreamSynchronize(t->stream), "d2h"))
    return CPS_ERR_CUDA;
  return CPS_OK;
}

cps_status cps_thermal_system(cps_thermal* t, double* planes, double* b) {
  if (!t) return tfail(nullptr, CPS_ERR_ARG, "handle is NULL");
  if (!tcuda(t, cudaSetDevice(t->device), "cudaSetDevice")) return CPS_ERR_CUDA;
  const size_t n = (size_t)t->view.lv[0].n;
  for (int p = 0; planes && p < 7; ++p)
    if (!tcuda(t, cudaMemcpyAsync(planes + p * n, t->view.lv[0].c[p], n * sizeof(double), cudaMemcpyDeviceToHost,
                                  t->stream), "d2h"))
      return CPS_ERR_CUDA;
  if (b && !tcuda(t, cudaMemcpyAsync(b, t->view.rhs, n * sizeof(double), cudaMemcpyDeviceToHost, t->stream), "d2h"))
    return CPS_ERR_CUDA;
  if (!tcuda(t, cudaStreamSynchronize(t->stream), "d2h")) return CPS_ERR_CUDA;
  return CPS_OK;
}

cps_status cps_thermal_timing(cps_thermal* t, double* kernel_ms, int* levels, int reset) {
  if (!t) return tfail(nullptr, CPS_ERR_ARG, "handle is NULL");
  if (kernel_ms) *kernel_ms = t->kernel_ms;
  if (levels) *levels = t->view.nlev;
  if (reset) t->kernel_ms = 0.0;
  return CPS_OK;
}

void cps_thermal_destroy(cps_thermal* t) {
  if (!t) return;
  if (t->stream) cudaStreamSynchronize(t->stream);
  if (t->slab) cudaFree(t->slab);
  if (t->hout) cudaFreeHost(t->hout);
  if (t->ev0) cudaEventDestroy(t->ev0);
  if (t->ev1) cudaEventDestroy(t->ev1);
  if (t->stream) cudaStreamDestroy(t->stream);
  delete t;
}

const char* cps_thermal_last_error(const cps_thermal* t) { return t ? t->err.c_str() : g_thermal_error.c_str(); }

}  // extern "C"
