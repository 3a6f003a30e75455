/*
 * cps.h -- C ABI of the B200 SIMPLE outer-iteration engine (libcps.so).
 *
 * Plain C types only: host pointers, sizes, doubles.  The caller owns every
 * host buffer; a context owns its device memory.  Every call returns a
 * cps_status (0 = OK, negative = error) and never exits the process; the
 * message of the last failure is available from cps_last_error().
 *
 * Which reference interfaces these entry points replace (paths inside the
 * reference project):
 *   - the per-call GPU solver ABI  namespace amgcl_cuda { initialize();
 *     cleanup(); solve(); solveMomentumU(); solveMomentumV(); }
 *     (Utilities/solvers/gpu/cuda_solver.hpp:18-57), which took host
 *     std::vectors, uploaded a CSR matrix three times per outer iteration and
 *     reported no errors;
 *   - the outer-iteration seam SIMPLE::calculateStep(int&)
 *     (Utilities/iterations.cpp:82-526), selected by a new value of the
 *     pressureSolverType registry member (SIMPLE.h:145);
 *   - SIMPLE::runIterations's residual stop rule (SIMPLE.cpp:299-318) and
 *     samplePlaneAtX (Utilities/postprocessing.cpp:97-230).
 * Fields stay resident on the device between steps; only the residual
 * diagnostics leave the GPU per outer iteration.
 *
 * Threading: one context per host thread, or external synchronisation.
 */
#ifndef CPS_H
#define CPS_H

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  CPS_OK = 0,
  CPS_ERR_ARG = -1,       /* invalid argument or size */
  CPS_ERR_OOM = -2,       /* device allocation failed */
  CPS_ERR_CUDA = -3,      /* CUDA runtime error */
  CPS_ERR_TIMEOUT = -4,   /* a bounded device-side wait expired */
  CPS_ERR_DIVERGED = -5,  /* residual became NaN or Inf */
  CPS_ERR_STATE = -6      /* call not valid in the context's current state */
} cps_status;

/* Field storage order of host arrays. */
enum { CPS_ROW_MAJOR = 0, CPS_COL_MAJOR = 1 /* Eigen::MatrixX? default */ };

/* Arithmetic of the inner solves. */
enum {
  CPS_FP64 = 0,  /* plain FP64, the drop-in judge path */
  CPS_MIXED = 1  /* FP32 Jacobi and PCG inside FP64 defect correction */
};

/* One design (reference member names, SIMPLE.h:68-358). */
typedef struct {
  int M, N;                       /* cell rows (y) and columns (x) */
  double hx, hy;                  /* cell size [m] */
  double rho, eta;                /* SIMPLE.h:334-335 */
  double uvAlpha, pAlpha;         /* SIMPLE.h:357-358 */
  double pTol;                    /* SIMPLE.h:153 (absolute ||r||_2) */
  int maxPressureIter;            /* SIMPLE.h:152 */
  double momentumTol;             /* SIMPLE.h:176 (RMS) */
  int maxMomentumIter;            /* SIMPLE.h:177 */
  int convectionScheme;           /* SIMPLE.h:193: 0 FOU, 1 SOU */
  int enableTwoPointFiveD;        /* SIMPLE.h:205 */
  int enableConvectionScaling;    /* SIMPLE.h:206 */
  double Ht_channel;              /* SIMPLE.h:207 */
  double twoPointFiveDSinkMultiplier; /* SIMPLE.h:208 */
  int precision;                  /* CPS_FP64 or CPS_MIXED */
  const double* alpha;            /* host M x N Brinkman alpha (SIMPLE.h:439) */
  const double* gamma;            /* host M x N density (SIMPLE.h:440) */
  int layout;                     /* CPS_ROW_MAJOR or CPS_COL_MAJOR for alpha/gamma */
  int device;                     /* CUDA device ordinal */
  int grid_ctas;                  /* CTAs of the persistent kernel; 0 = automatic */
} cps_desc;

/* Per-step inputs (SIMPLE.h:344 inletVelocity; SIMPLE.cpp:303-307). */
typedef struct {
  double inletVelocity;
} cps_step_in;

/* Per-step diagnostics (iterations.cpp:125-127, 451, 525). */
typedef struct {
  double residU;        /* max |u* - u| over U unknowns */
  double residV;        /* max |v* - v| over V unknowns */
  double residMass;     /* max mass imbalance, i=1..M-1, j=1..N-1 (reference definition) */
  double residMassDof;  /* the same over the pressure unknowns only (j <= N-2) */
  double err;           /* max(residU, residV, residMass), calculateStep's return value */
  int pIters;           /* PCG count as the reference reports it */
  int uSweeps, vSweeps; /* Jacobi sweeps of the U and V solves */
} cps_step_out;

/* Plane metrics of samplePlaneAtX (SIMPLE.h:679-686). */
typedef struct {
  double flowArea, massFlux, avgStatic, avgDynamic, avgTotal;
  int valid;
} cps_plane;

typedef struct cps_ctx cps_ctx;

/* Replaces amgcl_cuda::initialize + the per-call allocations
 * (cuda_solver.hpp:18; SIMPLE.cpp:18-29, 178-201, 589-630): allocates the
 * design's device state, uploads alpha and gamma, zeroes all fields. */
cps_status cps_create(const cps_desc* desc, cps_ctx** out);

/* Replaces amgcl_cuda::cleanup (cuda_solver.hpp:21). NULL is ignored. */
void cps_destroy(cps_ctx* ctx);

/* Upload u (M+1 x N), v (M x N+1), p (M+1 x N+1); any may be NULL to keep the
 * device copy (restart fields, SIMPLE.cpp:203-232). */
cps_status cps_upload_fields(cps_ctx* ctx, const double* u, const double* v, const double* p, int layout);

/* One outer iteration (SIMPLE::calculateStep, iterations.cpp:82-526). */
cps_status cps_step(cps_ctx* ctx, const cps_step_in* in, cps_step_out* out);

/* Up to max_outer outer iterations on the device without host round trips,
 * stopping after the first iteration with max(residU, residV, residMassDof)
 * <= eps when eps > 0.  history (may be NULL) receives max_outer entries;
 * *n_done the number of iterations run. */
cps_status cps_solve(cps_ctx* ctx, double inletVelocity, int max_outer, double eps, cps_step_out* history,
                     int* n_done);

/* samplePlaneAtX at physical x (postprocessing.cpp:97-230), on the device. */
cps_status cps_sample_plane(cps_ctx* ctx, double x, cps_plane* out);

/* Download fields; each pointer may be NULL.  Shapes as in the reference:
 * u, uStar, dE (M+1 x N); v, vStar, dN (M x N+1); p, pStar (M+1 x N+1). */
cps_status cps_download_fields(cps_ctx* ctx, double* u, double* v, double* p, double* pStar, double* uStar,
                               double* vStar, double* dE, double* dN, int layout);

/* Device bytes held by a context created from desc (admission control). */
cps_status cps_footprint(const cps_desc* desc, unsigned long long* bytes);

/* Message of the last failed call on ctx (or of the last failed cps_create
 * on this thread when ctx is NULL). */
const char* cps_last_error(const cps_ctx* ctx);

/* Library version string. */
const char* cps_version(void);

#ifdef __cplusplus
}
#endif

#endif /* CPS_H */
