/*
 * CPU restatement of one SIMPLE outer iteration of the reference solver
 * (TEST INFRASTRUCTURE ONLY: the oracle the CUDA path is checked against; no
 * product code calls it).
 *
 * This file is included twice by simple_oracle.c, with REAL = double (prefix
 * orc64_) and REAL = float (prefix orc32_).  Every function follows the cited
 * reference lines operation by operation, in the same evaluation order, so
 * that with one OpenMP thread in the reference (sequential reductions) the two
 * agree bit for bit.  Compile with -ffp-contract=off.
 *
 * Index space and storage: the reference's own (i,j) index space
 * (SIMPLE.h:393-440), stored row-major here:
 *   u, uStar, dE   (M+1) x N        U(i,j)  = u[i*N + j]
 *   v, vStar, dN   M x (N+1)        V(i,j)  = v[i*(N+1) + j]
 *   p, pStar       (M+1) x (N+1)    P(i,j)  = p[i*(N+1) + j]
 *   alpha, gamma   M x N            A(i,j)  = alpha[i*N + j]
 * Unknowns (momentum_solver.cpp:52-74, pressure_solver.cpp:438-458):
 *   U-DOF i=1..M-1, j=1..N-2;  V-DOF i=1..M-2, j=1..N-1;  P-DOF i=1..M-1, j=1..N-2,
 * numbered i-major (row = (i-1)*(cols) + (j-1)).
 */

#define CAT_(a, b) a##b
#define CAT(a, b) CAT_(a, b)
#define FN(name) CAT(PREFIX, name)

/* std::max / std::min / std::clamp exactly as libstdc++ evaluates them. */
static inline REAL FN(max_)(REAL a, REAL b) { return (a < b) ? b : a; }
static inline REAL FN(min_)(REAL a, REAL b) { return (b < a) ? b : a; }
static inline REAL FN(clamp_)(REAL v, REAL lo, REAL hi) { return (v < lo) ? lo : (hi < v) ? hi : v; }

/* Parameter layout (ip, dp), shared with coldplate_solver_b200/geometry.py:
 *   ip[0..7]   M N conv twoFiveD convScale maxPIter maxMomIter momType
 *   ip[8..15]  pseudo-transient (SIMPLE.h:255-313): enablePseudoTimeStepping useLocalPseudoTime
 *              enableSER enableLineSearch enableCflRamp serUseMaxResid serMinIter lsMaxTries
 *   ip[16..17] inlet ramp of the outer loop (SIMPLE.h:345-346): enableInletRamp rampSteps
 *   dp[0..10]  hx hy rho eta uvAlpha pAlpha Uin Ht sinkMult pTol momTol
 *   dp[11..26] timeStepMultiplier minPseudoSpeed pseudoCFLInitial pseudoCFLMax cflRampStartRes
 *              cflRampExponent cflRampSmooth serCFLMin serCFLMax serSmooth serMaxIncrease
 *              serMaxDecrease lsAlphaMin lsAlphaReduce lsResidIncreaseTol targetVel
 *   dp[27]     pseudoCFL: the CFL number the step uses (the controllers' current state) */
typedef struct {
  int M, N, conv, twoFiveD, convScale, maxPIter, maxMomIter, momType;
  int pseudo, pseudoLocal, serOn, lsOn, rampOn, serUseMax, serMinIter, lsMaxTries;
  REAL hx, hy, rho, eta, uvAlpha, pAlpha, Uin, Ht, sinkMult, pTol, momTol;
  REAL timeStep, minPseudoSpeed, cflInitial, cflMax, rampStartRes, rampExponent, rampSmooth;
  REAL serCFLMin, serCFLMax, serSmooth, serMaxIncrease, serMaxDecrease, lsAlphaMin, lsAlphaReduce, lsTol;
  REAL pseudoCFL;
} FN(params);

static void FN(unpack)(const int* ip, const double* dp, FN(params) * s) {
  s->M = ip[0]; s->N = ip[1]; s->conv = ip[2]; s->twoFiveD = ip[3]; s->convScale = ip[4];
  s->maxPIter = ip[5]; s->maxMomIter = ip[6]; s->momType = ip[7];
  s->pseudo = ip[8]; s->pseudoLocal = ip[9]; s->serOn = ip[10]; s->lsOn = ip[11]; s->rampOn = ip[12];
  s->serUseMax = ip[13]; s->serMinIter = ip[14]; s->lsMaxTries = ip[15];
  s->hx = (REAL)dp[0]; s->hy = (REAL)dp[1]; s->rho = (REAL)dp[2]; s->eta = (REAL)dp[3];
  s->uvAlpha = (REAL)dp[4]; s->pAlpha = (REAL)dp[5]; s->Uin = (REAL)dp[6]; s->Ht = (REAL)dp[7];
  s->sinkMult = (REAL)dp[8]; s->pTol = (REAL)dp[9]; s->momTol = (REAL)dp[10];
  s->minPseudoSpeed = (REAL)dp[12]; s->cflInitial = (REAL)dp[13]; s->cflMax = (REAL)dp[14];
  s->rampStartRes = (REAL)dp[15]; s->rampExponent = (REAL)dp[16]; s->rampSmooth = (REAL)dp[17];
  s->serCFLMin = (REAL)dp[18]; s->serCFLMax = (REAL)dp[19]; s->serSmooth = (REAL)dp[20];
  s->serMaxIncrease = (REAL)dp[21]; s->serMaxDecrease = (REAL)dp[22]; s->lsAlphaMin = (REAL)dp[23];
  s->lsAlphaReduce = (REAL)dp[24]; s->lsTol = (REAL)dp[25]; s->pseudoCFL = (REAL)dp[27];
  { /* SIMPLE.cpp:68-70: the global pseudo time step from the domain length and the target velocity */
    const REAL domainLength = (REAL)s->N * s->hx;
    const REAL velRef = FN(max_)((REAL)dp[26], (REAL)1e-6);
    s->timeStep = (REAL)dp[11] * domainLength / velRef;
  }
}

/* The pseudo-transient coefficient rho vol / dt of the implicit assembly at a
 * point whose current velocity is vel (momentum_solver.cpp:231-241); 0 with
 * the pseudo-transient term off. */
static REAL FN(trans_implicit)(const FN(params) * s, REAL vel) {
  if (!s->pseudo) return 0;
  const REAL vol = s->hx * s->hy, hChar = FN(min_)(s->hx, s->hy);
  REAL dtLocal = FN(max_)(s->timeStep, (REAL)1e-20);
  if (s->pseudoLocal) {
    const REAL speed = FN(max_)((REAL)fabs(vel), s->minPseudoSpeed);
    dtLocal = FN(min_)(dtLocal, s->pseudoCFL * hChar / speed);
    dtLocal = FN(max_)(dtLocal, (REAL)1e-20);
  }
  return s->rho * vol / dtLocal;
}

/* The same coefficient in the explicit update, from computeLocalDt
 * (iterations.cpp:189-217, 290-294): dt = +inf with the term off. */
static REAL FN(trans_explicit)(const FN(params) * s, REAL vel) {
  const REAL vol = s->hx * s->hy, hChar = FN(min_)(s->hx, s->hy);
  REAL dtLocal;
  if (!s->pseudo) dtLocal = (REAL)INFINITY;
  else if (!s->pseudoLocal) dtLocal = s->timeStep;
  else {
    const REAL speed = FN(max_)((REAL)fabs(vel), s->minPseudoSpeed);
    const REAL dtCfl = s->pseudoCFL * hChar / speed;
    dtLocal = FN(min_)(s->timeStep, dtCfl);
  }
  return s->rho * vol / dtLocal;
}

/* The outer loop's CFL controllers after one step (SIMPLE.cpp:321-327):
 * updateCflSER (time_control.cpp:82-118), applyLineSearch (:127-166) and
 * updateCflRamp (:43-63), in that order.  st = {pseudoCFL, serResidPrev,
 * lsCurrentAlpha, lsBacktrackCount}; resid = the monitoring residual
 * (serUseMaxResid ? the step's error : residMass); iteration = the outer
 * loop's index of the step. */
void FN(pseudo_update)(const int* ip, const double* dp, double* st, double resid_d, int iteration) {
  FN(params) s;
  FN(unpack)(ip, dp, &s);
  if (!s.pseudo) return;
  REAL cfl = (REAL)st[0], prev = (REAL)st[1], alpha = (REAL)st[2];
  int count = (int)st[3];
  const REAL resid = (REAL)resid_d;
  if (s.serOn && iteration >= s.serMinIter) {
    const REAL cur = FN(max_)(resid, (REAL)1e-15);
    if (prev <= 0) {
      prev = cur;
    } else {
      REAL ratio = prev / cur;
      ratio = FN(max_)(ratio, s.serMaxDecrease);
      ratio = FN(min_)(ratio, s.serMaxIncrease);
      REAL target = cfl * ratio;
      target = FN(max_)(target, s.serCFLMin);
      target = FN(min_)(target, s.serCFLMax);
      cfl = ((REAL)1 - s.serSmooth) * cfl + s.serSmooth * target;
      if (!isfinite(cfl) || cfl <= 0) cfl = s.serCFLMin;
      prev = cur;
    }
  }
  if (s.lsOn && s.serOn) {
    if (prev <= 0) {
      alpha = 1;
      count = 0;
    } else {
      const REAL ratio = resid / prev;
      if (ratio > s.lsTol) {
        count++;
        if (count <= s.lsMaxTries) {
          alpha *= s.lsAlphaReduce;
          alpha = FN(max_)(alpha, s.lsAlphaMin);
          cfl *= s.lsAlphaReduce;
          cfl = FN(max_)(cfl, s.serCFLMin);
        }
      } else {
        if (alpha < 1) alpha = FN(min_)(alpha * (REAL)1.1, (REAL)1);
        count = 0;
      }
    }
  }
  if (s.rampOn && !s.serOn) {
    const REAL cur = FN(max_)(resid, (REAL)1e-12);
    if (cur > s.rampStartRes) {
      cfl = s.cflInitial;
    } else {
      const REAL ratio = s.rampStartRes / cur;
      const REAL rawFactor = sizeof(REAL) == 4 ? (REAL)powf((float)ratio, (float)s.rampExponent)
                                               : (REAL)pow((double)ratio, (double)s.rampExponent);
      const REAL target = FN(min_)(s.cflInitial * rawFactor, s.cflMax);
      cfl = ((REAL)1 - s.rampSmooth) * cfl + s.rampSmooth * target;
      if (!isfinite(cfl) || cfl <= 0) cfl = s.cflInitial;
    }
  }
  st[0] = cfl; st[1] = prev; st[2] = alpha; st[3] = count;
}

/* SIMPLE.cpp:589-630 buildAlphaFromDensity: RAMP alpha from gamma, then rows 0
 * and M-2 forced solid (alpha = alpha_max, gamma = 0). */
void FN(build_alpha)(int M, int N, double amax_d, double q_d, REAL* gamma, REAL* alpha) {
  const REAL amax = (REAL)amax_d, q = (REAL)q_d;
  for (int i = 0; i < M; ++i)
    for (int j = 0; j < N; ++j) {
      REAL g = gamma[i * N + j];
      alpha[i * N + j] = amax * ((REAL)1 - g) / ((REAL)1 + q * g + (REAL)1e-10);
    }
  if (M >= 2) {
    for (int j = 0; j < N; ++j) {
      alpha[0 * N + j] = amax;
      alpha[(M - 2) * N + j] = amax;
      gamma[0 * N + j] = 0;
      gamma[(M - 2) * N + j] = 0;
    }
  }
}

/* convection.cpp:53-118 computeSOUCorrectionU. */
static REAL FN(sou_u)(const FN(params) * s, const REAL* u, int i, int j, REAL Fe, REAL Fw, REAL Fn, REAL Fs) {
  const int M = s->M, N = s->N;
#define UU(a, b) u[(a) * N + (b)]
  REAL Sdc = 0;
  if (Fe >= 0) {
    if (j >= 2) { REAL s_ = (REAL)1.5 * UU(i, j) - (REAL)0.5 * UU(i, j - 1); REAL f_ = UU(i, j); Sdc -= Fe * (s_ - f_); }
  } else {
    if (j + 2 < N) { REAL s_ = (REAL)1.5 * UU(i, j + 1) - (REAL)0.5 * UU(i, j + 2); REAL f_ = UU(i, j + 1); Sdc -= Fe * (s_ - f_); }
  }
  if (Fw >= 0) {
    if (j >= 2) { REAL s_ = (REAL)1.5 * UU(i, j - 1) - (REAL)0.5 * UU(i, j - 2); REAL f_ = UU(i, j - 1); Sdc += Fw * (s_ - f_); }
  } else {
    if (j + 1 < N) { REAL s_ = (REAL)1.5 * UU(i, j) - (REAL)0.5 * UU(i, j + 1); REAL f_ = UU(i, j); Sdc += Fw * (s_ - f_); }
  }
  if (Fn >= 0) {
    if (i >= 1) { REAL s_ = (REAL)1.5 * UU(i, j) - (REAL)0.5 * UU(i - 1, j); REAL f_ = UU(i, j); Sdc -= Fn * (s_ - f_); }
  } else {
    if (i + 2 <= M) { REAL s_ = (REAL)1.5 * UU(i + 1, j) - (REAL)0.5 * UU(i + 2, j); REAL f_ = UU(i + 1, j); Sdc -= Fn * (s_ - f_); }
  }
  if (Fs >= 0) {
    if (i >= 2) { REAL s_ = (REAL)1.5 * UU(i - 1, j) - (REAL)0.5 * UU(i - 2, j); REAL f_ = UU(i - 1, j); Sdc += Fs * (s_ - f_); }
  } else {
    if (i + 1 <= M) { REAL s_ = (REAL)1.5 * UU(i, j) - (REAL)0.5 * UU(i + 1, j); REAL f_ = UU(i, j); Sdc += Fs * (s_ - f_); }
  }
#undef UU
  return Sdc;
}

/* convection.cpp:121-186 computeSOUCorrectionV (note its guards differ from U's). */
static REAL FN(sou_v)(const FN(params) * s, const REAL* v, int i, int j, REAL Fe, REAL Fw, REAL Fn, REAL Fs) {
  const int M = s->M, N = s->N;
#define VV(a, b) v[(a) * (N + 1) + (b)]
  REAL Sdc = 0;
  if (Fe >= 0) {
    if (j >= 2) { REAL s_ = (REAL)1.5 * VV(i, j) - (REAL)0.5 * VV(i, j - 1); REAL f_ = VV(i, j); Sdc -= Fe * (s_ - f_); }
  } else {
    if (j + 2 <= N) { REAL s_ = (REAL)1.5 * VV(i, j + 1) - (REAL)0.5 * VV(i, j + 2); REAL f_ = VV(i, j + 1); Sdc -= Fe * (s_ - f_); }
  }
  if (Fw >= 0) {
    if (j >= 2) { REAL s_ = (REAL)1.5 * VV(i, j - 1) - (REAL)0.5 * VV(i, j - 2); REAL f_ = VV(i, j - 1); Sdc += Fw * (s_ - f_); }
  } else {
    if (j + 1 <= N) { REAL s_ = (REAL)1.5 * VV(i, j) - (REAL)0.5 * VV(i, j + 1); REAL f_ = VV(i, j); Sdc += Fw * (s_ - f_); }
  }
  if (Fn >= 0) {
    if (i >= 1) { REAL s_ = (REAL)1.5 * VV(i, j) - (REAL)0.5 * VV(i - 1, j); REAL f_ = VV(i, j); Sdc -= Fn * (s_ - f_); }
  } else {
    if (i + 2 < M) { REAL s_ = (REAL)1.5 * VV(i + 1, j) - (REAL)0.5 * VV(i + 2, j); REAL f_ = VV(i + 1, j); Sdc -= Fn * (s_ - f_); }
  }
  if (Fs >= 0) {
    if (i >= 2) { REAL s_ = (REAL)1.5 * VV(i - 1, j) - (REAL)0.5 * VV(i - 2, j); REAL f_ = VV(i - 1, j); Sdc += Fs * (s_ - f_); }
  } else {
    if (i + 1 < M) { REAL s_ = (REAL)1.5 * VV(i, j) - (REAL)0.5 * VV(i + 1, j); REAL f_ = VV(i, j); Sdc += Fs * (s_ - f_); }
  }
#undef VV
  return Sdc;
}

/* One momentum component: assembly (momentum_solver.cpp:185-298), Jacobi
 * (jacobi_solver.cpp:20-75) and scatter/clamp/residual (momentum_solver.cpp:318-337).
 * The CSR of the reference is replaced by the 5-point structure it encodes; each
 * row's products are summed in the CSR column order, which for an i-major
 * numbering is S, W, P, E, N.  Writes xStar (uStar or vStar) at the DOFs and d
 * (dE or dN); returns the sweep count, *resid = max |x - vel|. */
static int FN(momentum)(const FN(params) * s, int isU, const REAL* u, const REAL* v, const REAL* p,
                        const REAL* alpha, REAL* xStar, REAL* d, REAL* resid) {
  const int M = s->M, N = s->N;
  const REAL hx = s->hx, hy = s->hy, vol = hx * hy, rho = s->rho, eta = s->eta;
  const int i0 = 1, i1 = isU ? M - 1 : M - 2;  /* inclusive DOF row range */
  const int j0 = 1, j1 = isU ? N - 2 : N - 1;  /* inclusive DOF column range */
  const int cols = j1 - j0 + 1;
  const int n = (i1 >= i0 && j1 >= j0) ? (i1 - i0 + 1) * cols : 0;
  *resid = 0;
  if (n == 0) return 0;
  const int xc = isU ? N : N + 1; /* row length of the component's own grid */
  const REAL* x_old = isU ? u : v;
#define U_(a, b) u[(a) * N + (b)]
#define V_(a, b) v[(a) * (N + 1) + (b)]
#define P_(a, b) p[(a) * (N + 1) + (b)]
#define A_(a, b) alpha[(a) * N + (b)]
  const REAL maxVel = (REAL)3 * FN(max_)((REAL)fabs(s->Uin), (REAL)0.1);
  const REAL sinkCoeff = (s->twoFiveD && s->Ht > 0) ? s->sinkMult * ((REAL)5 * eta / ((REAL)2 * s->Ht * s->Ht)) : (REAL)0;
  const REAL sinkDiag = sinkCoeff * vol;
  const REAL De = eta * hy / hx, Dn = eta * hx / hy;

  REAL *cE = malloc(sizeof(REAL) * n), *cW = malloc(sizeof(REAL) * n), *cN = malloc(sizeof(REAL) * n),
       *cS = malloc(sizeof(REAL) * n), *cP = malloc(sizeof(REAL) * n), *b = malloc(sizeof(REAL) * n),
       *xa = malloc(sizeof(REAL) * n), *xb = malloc(sizeof(REAL) * n);
  for (int i = i0; i <= i1; ++i)
    for (int j = j0; j <= j1; ++j) {
      const int row = (i - i0) * cols + (j - j0);
      REAL alphaLocal, ue, uw, vn, vs;
      if (isU) { /* SIMPLE.h:546-566 alphaAtU; momentum_solver.cpp:207-211 */
        alphaLocal = (REAL)0.5 * (A_(i - 1, j - 1) + A_(i - 1, j));
        ue = FN(clamp_)((REAL)0.5 * (U_(i, j) + U_(i, j + 1)), -maxVel, maxVel);
        uw = FN(clamp_)((REAL)0.5 * (U_(i, j - 1) + U_(i, j)), -maxVel, maxVel);
        vn = FN(clamp_)((REAL)0.5 * (V_(i, j) + V_(i, j + 1)), -maxVel, maxVel);
        vs = FN(clamp_)((REAL)0.5 * (V_(i - 1, j) + V_(i - 1, j + 1)), -maxVel, maxVel);
      } else { /* SIMPLE.h:570-590 alphaAtV; momentum_solver.cpp:213-216 */
        alphaLocal = (REAL)0.5 * (A_(i - 1, j - 1) + A_(i, j - 1));
        ue = FN(clamp_)((REAL)0.5 * (U_(i, j) + U_(i + 1, j)), -maxVel, maxVel);
        uw = FN(clamp_)((REAL)0.5 * (U_(i, j - 1) + U_(i + 1, j - 1)), -maxVel, maxVel);
        vn = FN(clamp_)((REAL)0.5 * (V_(i, j) + V_(i + 1, j)), -maxVel, maxVel);
        vs = FN(clamp_)((REAL)0.5 * (V_(i - 1, j) + V_(i, j)), -maxVel, maxVel);
      }
      const REAL convScale = s->convScale ? ((REAL)6 / (REAL)7) : (REAL)1; /* :220 */
      const REAL Fe = convScale * rho * hy * ue, Fw = convScale * rho * hy * uw;
      const REAL Fn = convScale * rho * hx * vn, Fs = convScale * rho * hx * vs;
      const REAL aE = De + FN(max_)(0, -Fe), aW = De + FN(max_)(0, Fw);
      const REAL aN = Dn + FN(max_)(0, -Fn), aS = Dn + FN(max_)(0, Fs);
      const REAL sumA = aE + aW + aN + aS;
      const REAL velCur = isU ? U_(i, j) : V_(i, j);
      const REAL transCoeff = FN(trans_implicit)(s, velCur); /* :231-241 */
      const REAL brinkmanDrag = alphaLocal * vol;
      REAL aP0 = sumA + (Fe - Fw + Fn - Fs) + transCoeff + sinkDiag + brinkmanDrag; /* :246 */
      aP0 = FN(max_)(aP0, (REAL)1e-10);
      const REAL aP = aP0 / s->uvAlpha;
      REAL Sp;
      if (isU) Sp = (P_(i, j) - P_(i, j + 1)) * hy;
      else     Sp = (P_(i, j) - P_(i + 1, j)) * hx;
      Sp += transCoeff * velCur; /* uOld == u at this point (iterations.cpp:118) */
      Sp += ((REAL)1 - s->uvAlpha) / s->uvAlpha * aP0 * velCur;
      if (s->conv == 1) Sp += isU ? FN(sou_u)(s, u, i, j, Fe, Fw, Fn, Fs) : FN(sou_v)(s, v, i, j, Fe, Fw, Fn, Fs);
      if (isU) d[i * N + j] = hy / aP0; else d[i * (N + 1) + j] = hx / aP0;
      /* :276-295 neighbours that are unknowns become matrix entries; the others
       * are folded into the source with their current values, in E, W, N, S order. */
      const REAL xE = x_old[i * xc + j + 1], xW = x_old[i * xc + j - 1];
      const REAL xN = x_old[(i + 1) * xc + j], xS = x_old[(i - 1) * xc + j];
      cP[row] = aP;
      if (j + 1 <= j1) cE[row] = -aE; else { cE[row] = 0; Sp += aE * xE; }
      if (j - 1 >= j0) cW[row] = -aW; else { cW[row] = 0; Sp += aW * xW; }
      if (i + 1 <= i1) cN[row] = -aN; else { cN[row] = 0; Sp += aN * xN; }
      if (i - 1 >= i0) cS[row] = -aS; else { cS[row] = 0; Sp += aS * xS; }
      xa[row] = velCur;
      b[row] = Sp;
    }

  /* jacobi_solver.cpp:38-67 */
  REAL *xc_ = xa, *xn_ = xb;
  const REAL tol_sq = s->momTol * s->momTol;
  int iter = 0;
  for (; iter < s->maxMomIter; ++iter) {
    REAL total = 0;
    for (int i = i0; i <= i1; ++i)
      for (int j = j0; j <= j1; ++j) {
        const int row = (i - i0) * cols + (j - j0);
        REAL Ax = 0;
        if (i - 1 >= i0) Ax += cS[row] * xc_[row - cols];
        if (j - 1 >= j0) Ax += cW[row] * xc_[row - 1];
        Ax += cP[row] * xc_[row];
        if (j + 1 <= j1) Ax += cE[row] * xc_[row + 1];
        if (i + 1 <= i1) Ax += cN[row] * xc_[row + cols];
        const REAL r = b[row] - Ax;
        total += r * r;
        xn_[row] = xc_[row] + r / cP[row];
      }
    REAL* t = xc_; xc_ = xn_; xn_ = t;
    if (total < tol_sq * n) { iter++; break; }
  }

  /* momentum_solver.cpp:319-337 */
  REAL res = 0;
  for (int i = i0; i <= i1; ++i)
    for (int j = j0; j <= j1; ++j) {
      const int row = (i - i0) * cols + (j - j0);
      const REAL newVal = FN(clamp_)(xc_[row], -maxVel, maxVel);
      res = FN(max_)(res, (REAL)fabs(newVal - x_old[i * xc + j]));
      xStar[i * xc + j] = newVal;
    }
  *resid = res;
#undef U_
#undef V_
#undef P_
#undef A_
  free(cE); free(cW); free(cN); free(cS); free(cP); free(b); free(xa); free(xb);
  return iter;
}

/* The explicit momentum update of calculateStep with momentumSolverType = 0
 * (iterations.cpp:176-441): one point update
 * per unknown from the current velocities with the full coefficients, clamped
 * to +-maxVel; d = h / max(aP0, 1e-12).  Writes xStar and d at the unknowns;
 * *resid = max |xNew - vel|. */
static void FN(momentum_explicit)(const FN(params) * s, int isU, const REAL* u, const REAL* v, const REAL* p,
                                  const REAL* alpha, REAL* xStar, REAL* d, REAL* resid) {
  const int M = s->M, N = s->N;
  const REAL hx = s->hx, hy = s->hy, vol = hx * hy, rho = s->rho, eta = s->eta;
  const int i1 = isU ? M - 1 : M - 2, j1 = isU ? N - 2 : N - 1;
  const int xc = isU ? N : N + 1;
  const REAL* x_old = isU ? u : v;
#define U_(a, b) u[(a) * N + (b)]
#define V_(a, b) v[(a) * (N + 1) + (b)]
#define P_(a, b) p[(a) * (N + 1) + (b)]
#define A_(a, b) alpha[(a) * N + (b)]
  const REAL maxVel = (REAL)3 * FN(max_)((REAL)fabs(s->Uin), (REAL)0.1);
  const REAL convScale = s->convScale ? ((REAL)6 / (REAL)7) : (REAL)1;                 /* :233 */
  const REAL sinkCoeff = (s->twoFiveD && s->Ht > 0) ? s->sinkMult * ((REAL)5 * eta / ((REAL)2 * s->Ht * s->Ht)) : (REAL)0;
  const REAL sinkDiag = sinkCoeff * vol;                                                 /* :240 */
  REAL res = 0;
  for (int i = 1; i <= i1; ++i)
    for (int j = 1; j <= j1; ++j) {
      REAL alphaLocal, ue, uw, vn, vs;
      if (isU) { /* :262-271 */
        alphaLocal = (REAL)0.5 * (A_(i - 1, j - 1) + A_(i - 1, j));
        ue = FN(max_)(-maxVel, FN(min_)(maxVel, (REAL)0.5 * (U_(i, j) + U_(i, j + 1))));
        uw = FN(max_)(-maxVel, FN(min_)(maxVel, (REAL)0.5 * (U_(i, j - 1) + U_(i, j))));
        vn = FN(max_)(-maxVel, FN(min_)(maxVel, (REAL)0.5 * (V_(i, j) + V_(i, j + 1))));
        vs = FN(max_)(-maxVel, FN(min_)(maxVel, (REAL)0.5 * (V_(i - 1, j) + V_(i - 1, j + 1))));
      } else { /* :350-359 */
        alphaLocal = (REAL)0.5 * (A_(i - 1, j - 1) + A_(i, j - 1));
        ue = FN(max_)(-maxVel, FN(min_)(maxVel, (REAL)0.5 * (U_(i, j) + U_(i + 1, j))));
        uw = FN(max_)(-maxVel, FN(min_)(maxVel, (REAL)0.5 * (U_(i, j - 1) + U_(i + 1, j - 1))));
        vn = FN(max_)(-maxVel, FN(min_)(maxVel, (REAL)0.5 * (V_(i, j) + V_(i + 1, j))));
        vs = FN(max_)(-maxVel, FN(min_)(maxVel, (REAL)0.5 * (V_(i - 1, j) + V_(i, j))));
      }
      const REAL De = eta * hy / hx, Dn = eta * hx / hy;
      const REAL Fe = convScale * rho * hy * ue, Fw = convScale * rho * hy * uw;
      const REAL Fn = convScale * rho * hx * vn, Fs = convScale * rho * hx * vs;
      const REAL aE = De + FN(max_)(0, -Fe), aW = De + FN(max_)(0, Fw);
      const REAL aN = Dn + FN(max_)(0, -Fn), aS = Dn + FN(max_)(0, Fs);
      const REAL Sdc = (s->conv == 1) ? (isU ? FN(sou_u)(s, u, i, j, Fe, Fw, Fn, Fs) : FN(sou_v)(s, v, i, j, Fe, Fw, Fn, Fs))
                                      : (REAL)0;
      const REAL sumA = aE + aW + aN + aS;
      const REAL velCur = x_old[i * xc + j];
      const REAL transCoeffLocal = FN(trans_explicit)(s, velCur); /* :290-294 */
      const REAL brinkmanDrag = alphaLocal * vol;
      REAL aP0 = sumA + (Fe - Fw + Fn - Fs) + transCoeffLocal + sinkDiag + brinkmanDrag;
      aP0 = FN(max_)(aP0, (REAL)1e-10);
      const REAL dDenom = FN(max_)(aP0, (REAL)1e-12);
      REAL Sp;
      if (isU) { d[i * N + j] = hy / dDenom; Sp = (P_(i, j) - P_(i, j + 1)) * hy; }
      else     { d[i * (N + 1) + j] = hx / dDenom; Sp = (P_(i, j) - P_(i + 1, j)) * hx; }
      Sp += transCoeffLocal * velCur; /* uOld == u (:220) */
      Sp += Sdc;
      const REAL aP = aP0 / s->uvAlpha;
      Sp += ((REAL)1 - s->uvAlpha) / s->uvAlpha * aP0 * velCur;
      REAL xNew = (aE * x_old[i * xc + j + 1] + aW * x_old[i * xc + j - 1] + aN * x_old[(i + 1) * xc + j] +
                   aS * x_old[(i - 1) * xc + j] + Sp) / aP;
      xNew = FN(max_)(-maxVel, FN(min_)(maxVel, xNew));
      const REAL diff = (REAL)fabs(xNew - velCur);
      if (diff > res) res = diff;
      xStar[i * xc + j] = xNew;
    }
  *resid = res;
#undef U_
#undef V_
#undef P_
#undef A_
}

/* boundaries.cpp:48-106 setVelocityBoundaryConditions. */
void FN(velocity_bc)(int M, int N, double Uin_d, const REAL* gamma, REAL* uIn, REAL* vIn) {
  const REAL Uin = (REAL)Uin_d;
  for (int j = 0; j < N; ++j) uIn[0 * N + j] = 0;
  for (int j = 0; j < N + 1; ++j) vIn[0 * (N + 1) + j] = 0;
  for (int j = 0; j < N; ++j) uIn[M * N + j] = 0;
  for (int j = 0; j < N + 1; ++j) vIn[(M - 1) * (N + 1) + j] = 0;
  for (int i = 1; i < M; ++i) uIn[i * N + 0] = (gamma[(i - 1) * N + 0] > (REAL)0.5) ? Uin : (REAL)0;
  for (int i = 0; i < M; ++i) vIn[i * (N + 1) + 0] = 0;
  for (int i = 0; i < M + 1; ++i) uIn[i * N + N - 1] = uIn[i * N + N - 2];
  for (int i = 0; i < M; ++i) vIn[i * (N + 1) + N] = vIn[i * (N + 1) + N - 1];
}

/* boundaries.cpp:111-134 setPressureBoundaryConditions. */
static void FN(pressure_bc)(int M, int N, REAL* p) {
  const int W = N + 1;
  for (int j = 1; j < N; ++j) { p[0 * W + j] = p[1 * W + j]; p[M * W + j] = p[(M - 1) * W + j]; }
  for (int i = 1; i < M; ++i) p[i * W + 0] = p[i * W + 1];
  for (int i = 1; i < M; ++i) p[i * W + N] = 0;
}

/* Mass imbalance of one cell (pressure_solver.cpp:476-480, 726-730), no abs. */
static inline REAL FN(mass_b)(const FN(params) * s, const REAL* uStar, const REAL* vStar, int i, int j) {
  const int N = s->N;
  const REAL massE = s->rho * uStar[i * N + j] * s->hy;
  const REAL massW = s->rho * uStar[i * N + j - 1] * s->hy;
  const REAL massN = s->rho * vStar[i * (N + 1) + j] * s->hx;
  const REAL massS = s->rho * vStar[(i - 1) * (N + 1) + j] * s->hx;
  return massW - massE + massS - massN;
}

/* Pressure correction: mass residual (pressure_solver.cpp:463-486), P-DOF matrix
 * and RHS (:693-732), Jacobi-PCG (:121-184) and scatter (:796-805).  Writes
 * pStar; returns the PCG count; *residMass over i=1..M-1, j=1..N-1 and
 * *residMassDof over the unknowns (j<=N-2). */
static int FN(pressure)(const FN(params) * s, const REAL* uStar, const REAL* vStar, const REAL* dE,
                        const REAL* dN, REAL* pStar, REAL* residMass, REAL* residMassDof) {
  const int M = s->M, N = s->N, W = N + 1;
  const REAL rho = s->rho, hx = s->hx, hy = s->hy;
  for (int k = 0; k < (M + 1) * W; ++k) pStar[k] = 0;
  REAL rm = 0, rmd = 0;
  for (int i = 1; i < M; ++i)
    for (int j = 1; j < N; ++j) {
      const REAL b = (REAL)fabs(FN(mass_b)(s, uStar, vStar, i, j));
      if (b > rm) rm = b;
      if (j < N - 1 && b > rmd) rmd = b;
    }
  *residMass = rm;
  *residMassDof = rmd;
  const int i0 = 1, i1 = M - 1, j0 = 1, j1 = N - 2, cols = j1 - j0 + 1;
  const int n = (i1 >= i0 && j1 >= j0) ? (i1 - i0 + 1) * cols : 0;
  if (n == 0) return 0;
  REAL *cE = malloc(sizeof(REAL) * n), *cW = malloc(sizeof(REAL) * n), *cN = malloc(sizeof(REAL) * n),
       *cS = malloc(sizeof(REAL) * n), *cP = malloc(sizeof(REAL) * n), *bb = malloc(sizeof(REAL) * n),
       *x = malloc(sizeof(REAL) * n), *r = malloc(sizeof(REAL) * n), *z = malloc(sizeof(REAL) * n),
       *pp = malloc(sizeof(REAL) * n), *Ap = malloc(sizeof(REAL) * n);
  for (int i = i0; i <= i1; ++i)
    for (int j = j0; j <= j1; ++j) {
      const int row = (i - i0) * cols + (j - j0);
      const REAL aE = (j < N - 1) ? rho * dE[i * N + j] * hy : (REAL)0;
      const REAL aW = (j > 1) ? rho * dE[i * N + j - 1] * hy : (REAL)0;
      const REAL aN = (i < M - 1) ? rho * dN[i * W + j] * hx : (REAL)0;
      const REAL aS = (i > 1) ? rho * dN[(i - 1) * W + j] * hx : (REAL)0;
      REAL aP = aE + aW + aN + aS;
      if (aP < (REAL)1e-20) aP = 1;
      cP[row] = aP;
      cE[row] = (j + 1 <= j1) ? -aE : (REAL)0;
      cW[row] = (j - 1 >= j0) ? -aW : (REAL)0;
      cN[row] = (i + 1 <= i1) ? -aN : (REAL)0;
      cS[row] = (i - 1 >= i0) ? -aS : (REAL)0;
      bb[row] = FN(mass_b)(s, uStar, vStar, i, j);
      x[row] = 0; /* pStar(i,j) after setZero */
    }
#define SPMV(dst, src)                                               \
  for (int i = i0; i <= i1; ++i)                                     \
    for (int j = j0; j <= j1; ++j) {                                 \
      const int row = (i - i0) * cols + (j - j0);                    \
      REAL sum = 0;                                                  \
      if (i - 1 >= i0) sum += cS[row] * (src)[row - cols];           \
      if (j - 1 >= j0) sum += cW[row] * (src)[row - 1];              \
      sum += cP[row] * (src)[row];                                   \
      if (j + 1 <= j1) sum += cE[row] * (src)[row + 1];              \
      if (i + 1 <= i1) sum += cN[row] * (src)[row + cols];           \
      (dst)[row] = sum;                                              \
    }
  SPMV(Ap, x);
  for (int k = 0; k < n; ++k) r[k] = bb[k] - Ap[k];
  for (int k = 0; k < n; ++k) z[k] = ((REAL)fabs(cP[k]) > (REAL)1e-20) ? r[k] / cP[k] : r[k];
  for (int k = 0; k < n; ++k) pp[k] = z[k];
  REAL rz = 0;
  for (int k = 0; k < n; ++k) rz += r[k] * z[k];
  int iter = 0;
  for (; iter < s->maxPIter; ++iter) {
    SPMV(Ap, pp);
    REAL pAp = 0;
    for (int k = 0; k < n; ++k) pAp += pp[k] * Ap[k];
    if ((REAL)fabs(pAp) < (REAL)1e-20) break;
    const REAL alpha = rz / pAp;
    for (int k = 0; k < n; ++k) { x[k] += alpha * pp[k]; r[k] -= alpha * Ap[k]; }
    REAL err = 0;
    for (int k = 0; k < n; ++k) err += r[k] * r[k];
    if ((REAL)sqrt(err) < s->pTol) break;
    for (int k = 0; k < n; ++k) z[k] = ((REAL)fabs(cP[k]) > (REAL)1e-20) ? r[k] / cP[k] : r[k];
    const REAL rz_prev = rz;
    rz = 0;
    for (int k = 0; k < n; ++k) rz += r[k] * z[k];
    const REAL beta = rz / rz_prev;
    for (int k = 0; k < n; ++k) pp[k] = z[k] + beta * pp[k];
  }
#undef SPMV
  for (int i = i0; i <= i1; ++i)
    for (int j = j0; j <= j1; ++j) pStar[i * W + j] = x[(i - i0) * cols + (j - j0)];
  for (int i = 1; i < M; ++i) pStar[i * W + N - 1] = 0;
  free(cE); free(cW); free(cN); free(cS); free(cP); free(bb); free(x); free(r); free(z); free(pp); free(Ap);
  return iter;
}

/* iterations.cpp:82-526 calculateStep with momentumSolverType 1 (implicit
 * Jacobi) or 0 (explicit point update) and the Parallel-CG pressure solver.  `stop_after`: 1 = after the momentum solve and
 * its BCs (uStar, vStar, dE, dN final), 2 = after the pressure solve (pStar
 * final), 3 = whole step.  diag[0..7] = residU, residV, residMass,
 * residMassDof, returned error, PCG count, U sweeps, V sweeps. */
int FN(step)(const int* ip, const double* dp, int stop_after, REAL* u, REAL* v, REAL* p, REAL* pStar,
             REAL* uStar, REAL* vStar, REAL* dE, REAL* dN, const REAL* alpha, const REAL* gamma,
             double* diag) {
  FN(params) s;
  FN(unpack)(ip, dp, &s);
  const int M = s.M, N = s.N, W = N + 1;
  if (M < 3 || N < 3) return -1;
  const REAL maxVel = (REAL)3 * FN(max_)((REAL)fabs(s.Uin), (REAL)0.1); /* :104 */
  REAL residU, residV, residMass, residMassDof;
  int su = -1, sv = -1; /* no Jacobi solve in the explicit path */
  if (s.momType == 0) {
    FN(momentum_explicit)(&s, 1, u, v, p, alpha, uStar, dE, &residU);
    FN(momentum_explicit)(&s, 0, u, v, p, alpha, vStar, dN, &residV);
  } else {
    su = FN(momentum)(&s, 1, u, v, p, alpha, uStar, dE, &residU);
    sv = FN(momentum)(&s, 0, u, v, p, alpha, vStar, dN, &residV);
  }
  FN(velocity_bc)(M, N, dp[6], gamma, uStar, vStar); /* :134 */
  diag[0] = residU; diag[1] = residV; diag[6] = su; diag[7] = sv;
  if (stop_after == 1) return 0;
  const int pit = FN(pressure)(&s, uStar, vStar, dE, dN, pStar, &residMass, &residMassDof);
  diag[2] = residMass; diag[3] = residMassDof; diag[5] = pit;
  if (stop_after == 2) return 0;
  /* :456-467 */
  for (int i = 1; i < M; ++i)
    for (int j = 1; j < N; ++j) p[i * W + j] += s.pAlpha * pStar[i * W + j];
  FN(pressure_bc)(M, N, p);
  /* :473-499 */
  for (int i = 1; i < M; ++i)
    for (int j = 1; j < N - 1; ++j) {
      REAL du = dE[i * N + j] * (pStar[i * W + j] - pStar[i * W + j + 1]);
      du = FN(max_)(-maxVel, FN(min_)(maxVel, du));
      u[i * N + j] = uStar[i * N + j] + du;
      u[i * N + j] = FN(max_)(-maxVel, FN(min_)(maxVel, u[i * N + j]));
    }
  for (int i = 1; i < M - 1; ++i)
    for (int j = 1; j < N; ++j) {
      REAL dv = dN[i * W + j] * (pStar[i * W + j] - pStar[(i + 1) * W + j]);
      dv = FN(max_)(-maxVel, FN(min_)(maxVel, dv));
      v[i * W + j] = vStar[i * W + j] + dv;
      v[i * W + j] = FN(max_)(-maxVel, FN(min_)(maxVel, v[i * W + j]));
    }
  FN(velocity_bc)(M, N, dp[6], gamma, u, v);
  /* :525 std::max({residU, residV, residMass}) */
  REAL e = residU;
  if (e < residV) e = residV;
  if (e < residMass) e = residMass;
  diag[4] = e;
  return 0;
}

/* The inlet velocity of outer iteration `iteration` (SIMPLE.cpp:303-307): the
 * ramp (iter + 1) / rampSteps of the target velocity dp[6] while it runs. */
double FN(inlet_velocity)(const int* ip, const double* dp, int iteration) {
  const int on = ip[16], steps = ip[17];
  if (on && steps > 0 && iteration < steps) return (double)(((REAL)(iteration + 1) / (REAL)steps) * (REAL)dp[6]);
  return dp[6];
}

/* Outer loop (SIMPLE.cpp:299-327 without logging or the dP window): at most
 * max_outer steps, stopping once max(residU, residV, residMassDof) <= eps when
 * stop_on_conv.  hist is max_outer x 8 (the step diagnostics); returns steps run. */
int FN(solve)(const int* ip, const double* dp, int max_outer, double eps, int stop_on_conv, REAL* u, REAL* v,
              REAL* p, REAL* pStar, REAL* uStar, REAL* vStar, REAL* dE, REAL* dN, const REAL* alpha,
              const REAL* gamma, double* hist) {
  /* the controllers' state starts as the constructor leaves it (SIMPLE.cpp:78-82, SIMPLE.h:280-292) */
  double dpl[28], st[4] = {dp[27], 0.0, 1.0, 0.0};
  for (int k = 0; k < 28; ++k) dpl[k] = dp[k];
  int it = 0;
  for (; it < max_outer; ++it) {
    double* h = hist + 8 * it;
    dpl[6] = FN(inlet_velocity)(ip, dp, it);
    dpl[27] = st[0];
    if (FN(step)(ip, dpl, 3, u, v, p, pStar, uStar, vStar, dE, dN, alpha, gamma, h) != 0) return -1;
    FN(pseudo_update)(ip, dpl, st, ip[13] ? h[4] : h[2], it); /* SIMPLE.cpp:323-326 */
    double conv = h[0];
    if (conv < h[1]) conv = h[1];
    if (conv < h[3]) conv = h[3];
    if (stop_on_conv && conv <= eps) { ++it; break; }
  }
  return it;
}

/* postprocessing.cpp:62-90 findBracketingColumns and :97-230 samplePlaneAtX.
 * out[0..5] = flowArea, massFlux, avgStatic, avgDynamic, avgTotal, valid. */
void FN(sample_plane)(int M, int N, double hx_d, double hy_d, double rho_d, double x_d, const REAL* u,
                      const REAL* v, const REAL* p, const REAL* gamma, double* out) {
  const REAL hx = (REAL)hx_d, hy = (REAL)hy_d, rho = (REAL)rho_d, xPhysical = (REAL)x_d;
  for (int k = 0; k < 6; ++k) out[k] = 0;
  if (M <= 0 || N <= 0 || hx <= 0 || hy <= 0) return;
  const REAL xMin = (REAL)0.5 * hx;
  const REAL xMax = ((REAL)N - (REAL)0.5) * hx;
  const REAL xClamped = FN(max_)(xMin, FN(min_)(xPhysical, xMax));
  const REAL jFloat = xClamped / hx - (REAL)0.5;
  int colLeft = (int)floor(jFloat);
  colLeft = colLeft < N - 2 ? colLeft : N - 2;
  colLeft = 0 < colLeft ? colLeft : 0;
  const int colRight = colLeft + 1;
  const REAL xLeft = ((REAL)colLeft + (REAL)0.5) * hx, xRight = ((REAL)colRight + (REAL)0.5) * hx;
  REAL t = ((REAL)fabs(xRight - xLeft) < (REAL)1e-12) ? (REAL)0 : (xClamped - xLeft) / (xRight - xLeft);
  t = FN(max_)(0, FN(min_)(1, t));
  REAL staticAreaSum = 0, dynAreaSum = 0, totalWeighted = 0, area = 0, fluxSum = 0;
#define CLAMPI(a, lo, hi) ((a) < (lo) ? (lo) : ((a) > (hi) ? (hi) : (a)))
  for (int i = 1; i < M; ++i) {
    const int cellRow = i - 1;
    if (colLeft < 0 || colLeft >= N || colRight < 0 || colRight >= N) continue;
    const REAL pureFluidTol = (REAL)1e-6;
    if (gamma[cellRow * N + colLeft] < (REAL)1 - pureFluidTol || gamma[cellRow * N + colRight] < (REAL)1 - pureFluidTol)
      continue;
    const REAL faceArea = hy;
    area += faceArea;
    const int pL = CLAMPI(colLeft + 1, 0, N), pR = CLAMPI(colRight + 1, 0, N);
    const REAL staticP = ((REAL)1 - t) * p[i * (N + 1) + pL] + t * p[i * (N + 1) + pR];
    const int uL = CLAMPI(colLeft, 0, N - 1), uR = CLAMPI(colRight, 0, N - 1);
    const REAL uNormal = ((REAL)1 - t) * u[i * N + uL] + t * u[i * N + uR];
    const int vL = CLAMPI(colLeft, 0, N), vR = CLAMPI(colRight, 0, N);
    const int vTopRow = CLAMPI(i - 1, 0, M - 1), vBotRow = CLAMPI(i, 0, M - 1);
    const REAL vTop = ((REAL)1 - t) * v[vTopRow * (N + 1) + vL] + t * v[vTopRow * (N + 1) + vR];
    const REAL vBottom = ((REAL)1 - t) * v[vBotRow * (N + 1) + vL] + t * v[vBotRow * (N + 1) + vR];
    const REAL vTangential = (REAL)0.5 * (vTop + vBottom);
    const REAL velMag = (REAL)sqrt(uNormal * uNormal + vTangential * vTangential);
    const REAL dynP = (REAL)0.5 * rho * velMag * velMag;
    const REAL totalPAbs = staticP + dynP;
    staticAreaSum += staticP * faceArea;
    dynAreaSum += dynP * faceArea;
    const REAL flux = rho * uNormal * faceArea;
    const REAL fluxAbs = (REAL)fabs(flux);
    if (fluxAbs > 0) { fluxSum += fluxAbs; totalWeighted += totalPAbs * fluxAbs; }
  }
#undef CLAMPI
  out[0] = area;
  out[1] = fluxSum;
  REAL avgStatic = 0, avgDynamic = 0, avgTotal = 0;
  if (area > 0) { avgStatic = staticAreaSum / area; avgDynamic = dynAreaSum / area; out[5] = 1; }
  if (fluxSum > 0) avgTotal = totalWeighted / fluxSum;
  else if (area > 0) avgTotal = avgStatic + avgDynamic;
  out[2] = avgStatic; out[3] = avgDynamic; out[4] = avgTotal;
}

#undef FN
