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
  CPS_FP64 = 0,  /* plain FP64, the path checked bit-closely against the reference */
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
  int pcg_variant;                /* CPS_PCG_REFERENCE (two reductions per iteration, as
                                     pressure_solver.cpp:121-184) or CPS_PCG_SINGLE_REDUCTION
                                     (Chronopoulos-Gear recurrences: one reduction per iteration) */
  int momentum_explicit;          /* 0: implicit Jacobi momentum (momentumSolverType = 1, SIMPLE.h:172);
                                     1: the explicit point update (momentumSolverType = 0,
                                     iterations.cpp:176-441) */
} cps_desc;

/* PCG recurrences (same Krylov iterates in exact arithmetic). */
enum { CPS_PCG_REFERENCE = 0, CPS_PCG_SINGLE_REDUCTION = 1 };

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

/* Replace alpha and gamma (M x N) of an existing context: the outputs of the
 * reference's loadTopology/loadDensityField/buildAlphaFromDensity
 * (SIMPLE.cpp:517-630) for a new design of the same grid. */
cps_status cps_upload_geometry(cps_ctx* ctx, const double* alpha, const double* gamma, int layout);

/* Zero u, v, p and every derived field on the device: the state cps_create
 * leaves (SIMPLE.cpp:184-197), without a host copy.  Also restarts the
 * outer-loop iteration index (inlet ramp, serMinIter, pressure-drop window)
 * and the CFL controllers' state, as a fresh solve of the reference does. */
cps_status cps_reset_fields(cps_ctx* ctx);

/* The cudaStream_t (as void*) every call of this context issues its work on,
 * for callers that time or order work against it. */
cps_status cps_get_stream(cps_ctx* ctx, void** stream);

/* Device time of the outer-iteration kernel launches issued since the last
 * reset, measured with CUDA events on the launching stream; reset != 0
 * clears the counters after reading. */
cps_status cps_kernel_timing(cps_ctx* ctx, double* kernel_ms, long long* launches, long long* outer_iterations,
                             int reset);

/* Pressure-drop monitor and convergence gate of the outer loop
 * (SIMPLE::runIterations, SIMPLE.cpp:269-408): after every outer iteration the
 * four planes core inlet/outlet, x = 0 and x = N hx are sampled as
 * samplePlaneAtX does (postprocessing.cpp:97-230) and, with gate set, the loop
 * stops once the core total-pressure drop settles: over the last `window`
 * values (collected from iteration ramp_steps on) std/|mean| and
 * |latest - mean|/|mean| (|mean| floored at 1) are both below percent %, and,
 * with slope_gate, the least-squares slope over the last slope_window
 * iterations is at most slope_max_delta / slope_window. */
typedef struct {
  int    gate;             /* usePressureDropConvergence (SIMPLE.h:98) */
  int    window;           /* dpConvergenceWindow (SIMPLE.h:99) */
  double percent;          /* dpConvergencePercent (SIMPLE.h:100) */
  int    slope_gate;       /* usePressureDropSlopeGate (SIMPLE.h:101) */
  int    slope_window;     /* dpSlopeWindowIters (SIMPLE.h:102) */
  double slope_max_delta;  /* dpSlopeMaxDelta (SIMPLE.h:103) */
  int    ramp_steps;       /* rampSteps (SIMPLE.h:346): the window starts at this iteration */
  double x_core_in;        /* xPlaneCoreInlet [m] */
  double x_core_out;       /* xPlaneCoreOutlet [m] */
} cps_dp_monitor;

/* Attach (m != NULL) or detach (NULL) the pressure-drop monitor of ctx and
 * restart the outer-loop iteration count at 0 (as does cps_reset_fields).
 * window + slope_window is limited by the kernel's shared memory (reported in
 * the error message when exceeded). */
cps_status cps_set_dp_monitor(cps_ctx* ctx, const cps_dp_monitor* m);

/* cps_solve with the monitor attached: also fills dp_history (may be NULL;
 * max_outer x 4 doubles: core total, full total, core static, full static
 * pressure drop of each iteration, the columns of the reference's
 * pressure_drop_history.txt) and sets *dp_converged when the gate ended the
 * loop.  The residual stop (eps > 0) and the gate both apply, as in the
 * reference's loop condition. */
cps_status cps_solve_monitored(cps_ctx* ctx, double inletVelocity, int max_outer, double eps, cps_step_out* history,
                               double* dp_history, int* n_done, int* dp_converged);

/* Pseudo-transient term of the momentum equations and the outer loop's CFL
 * controllers (SIMPLE.h:255-313; momentum_solver.cpp:231-241 and
 * iterations.cpp:189-217 for the term, time_control.cpp:43-166 with
 * SIMPLE.cpp:321-327 for the controllers).  With enable set, every momentum
 * unknown gets rho hx hy / dt on its diagonal and times its current velocity
 * in its source, dt = min(time_step, pseudo_cfl min(hx, hy) / max(|vel|,
 * min_pseudo_speed)) with use_local (else time_step), and after every outer
 * iteration SER (Switched Evolution Relaxation), its line search and the
 * residual ramp update pseudo_cfl from residMass (or, with
 * ser_use_max_resid, the step's error).  time_step =
 * time_step_multiplier * N hx / max(target_velocity, 1e-6) (SIMPLE.cpp:68-70)
 * unless given. */
typedef struct {
  int    enable;                /* enablePseudoTimeStepping (SIMPLE.h:262) */
  int    use_local;             /* useLocalPseudoTime */
  int    enable_ser;            /* enableSER */
  int    enable_line_search;    /* enableLineSearch */
  int    enable_cfl_ramp;       /* enableCflRamp (ignored while SER is on) */
  int    ser_use_max_resid;     /* serUseMaxResid */
  int    ser_min_iter;          /* serMinIter */
  int    ls_max_tries;          /* lsMaxTries */
  double target_velocity;       /* targetVel [m/s] */
  double time_step_multiplier;  /* timeStepMultiplier */
  double min_pseudo_speed;      /* minPseudoSpeed [m/s] */
  double pseudo_cfl;            /* pseudoCFL: the starting CFL number when the ramp is off */
  double cfl_initial;           /* pseudoCFLInitial: the starting CFL number when the ramp is on */
  double cfl_max;               /* pseudoCFLMax */
  double cfl_ramp_start_res;    /* cflRampStartRes */
  double cfl_ramp_exponent;     /* cflRampExponent */
  double cfl_ramp_smooth;       /* cflRampSmooth */
  double ser_cfl_min;           /* serCFLMin */
  double ser_cfl_max;           /* serCFLMax */
  double ser_smooth;            /* serSmooth */
  double ser_max_increase;      /* serMaxIncrease */
  double ser_max_decrease;      /* serMaxDecrease */
  double ls_alpha_min;          /* lsAlphaMin */
  double ls_alpha_reduce;       /* lsAlphaReduce */
  double ls_resid_increase_tol; /* lsResidIncreaseTol */
  double time_step;             /* > 0: the global pseudo time step timeStep [s] itself, in place of the formula */
} cps_pseudo;

/* The controllers' state carried from one outer iteration to the next. */
typedef struct {
  double pseudo_cfl;      /* pseudoCFL: the CFL number of the next step */
  double ser_resid_prev;  /* serResidPrev */
  double ls_alpha;        /* lsCurrentAlpha */
  int    ls_backtracks;   /* lsBacktrackCount */
  int    pad;
} cps_pseudo_state;

/* The reference's defaults (SIMPLE.h:255-313), enable = 0. */
cps_status cps_pseudo_defaults(cps_pseudo* p, double target_velocity);

/* Switch the term and controllers on (p->enable) or off (p == NULL or
 * !p->enable) for every later step, solve and batch of ctx; resets the
 * controllers' state to its start (pseudo_cfl = cfl_initial with the ramp on,
 * else pseudo_cfl; ser_resid_prev 0; ls_alpha 1; ls_backtracks 0).  The
 * outer-loop iteration index that serMinIter counts restarts at 0 with
 * cps_reset_fields. */
cps_status cps_set_pseudo(cps_ctx* ctx, const cps_pseudo* p);

/* Read or overwrite the controllers' state (a caller that runs the
 * controllers itself, such as the reference's own outer loop, sets the CFL
 * number before each cps_step). */
cps_status cps_get_pseudo_state(cps_ctx* ctx, cps_pseudo_state* state);
cps_status cps_set_pseudo_state(cps_ctx* ctx, const cps_pseudo_state* state);

/* The outer loop's inlet velocity ramp (enableInletRamp && rampSteps > 0,
 * SIMPLE.cpp:303-307): in cps_solve and cps_solve_monitored, outer iteration
 * iter < ramp_steps runs with inlet velocity ((iter + 1) / ramp_steps) times
 * the call's inletVelocity (iter: the context's outer-loop index, restarted by
 * cps_reset_fields).  Those iterations run one launch each.  ramp_steps = 0
 * switches it off.  cps_step and cps_batch_solve take their inlet velocities
 * from the caller as given. */
cps_status cps_set_inlet_ramp(cps_ctx* ctx, int ramp_steps);

/* Options of a batched solve. */
typedef struct {
  int cluster_ctas;   /* CTAs of the thread-block cluster that runs one design (1..16; 0 = 8) */
  int max_clusters;   /* upper bound on concurrent clusters (0 = as many as fit) */
  int max_outer;      /* outer-iteration budget of every design in this call */
  double eps;         /* stop a design once max(residU, residV, residMassDof) <= eps (0 = never) */
  int order_by_size;  /* start the largest designs first */
  int group_ctas;     /* > 0: run designs on groups of this many CTAs of one cooperative launch (software
                         group barrier, bounded waits) instead of on thread-block clusters */
  int tiles_per_cta;  /* > 0 (overrides group_ctas and cluster_ctas): give each design a group of
                         ceil(tiles / tiles_per_cta) CTAs (a tile is 8 x 32 points; at most the device's
                         co-resident CTAs) and run the groups in waves, one cooperative launch per wave,
                         packed largest first so that each wave fills the device */
} cps_batch_opts;

/* Per-design outcome of a batched solve. */
typedef struct {
  int n_done;         /* outer iterations run in this call */
  int converged;      /* the eps test passed on the last iteration */
  int status;         /* CPS_OK or CPS_ERR_DIVERGED */
  cps_step_out last;  /* diagnostics of the last iteration */
} cps_batch_result;

/* Many designs in one persistent launch: each design runs on one thread-block
 * cluster (hardware cluster barrier) or, with group_ctas > 0, on one group of
 * CTAs of a cooperative launch (software group barrier), until it meets eps
 * or spends max_outer outer iterations; clusters/groups take designs from a
 * device work queue, so designs of uneven size share the GPU.  With
 * tiles_per_cta > 0 each design's group is sized to the design instead, and
 * the designs run in as few launches (waves) as the co-resident CTAs allow.  Every context must be
 * on the same device with the same precision.  Has no reference counterpart:
 * the reference solves one design per process (SIMPLE.cpp:638-642).
 * inletVelocity: n values or NULL to keep each context's last value.
 * *kernel_ms (may be NULL) receives the launch's device time. */
cps_status cps_batch_solve(cps_ctx* const* ctxs, int n, const double* inletVelocity, const cps_batch_opts* opts,
                           cps_batch_result* results, double* kernel_ms);

/* The first n (<= 4096) diagnostics of the last cps_solve launch chunk or
 * cps_batch_solve visit of this context. */
cps_status cps_get_history(cps_ctx* ctx, int n, cps_step_out* history);

/* Allocation-free FP64 solve of one design, for callers that cannot call
 * cudaMalloc (an application that owns all device memory through its own
 * pool, a real-time loop that must not enter the driver's allocator, a plugin
 * handed only buffers and a stream).  No counterpart in the reference.
 *
 * The caller passes device buffers, all with row pitch `pitch` (>= N+1
 * doubles): alpha, gamma (M rows, inputs), u, v, p ((M+1) rows, inputs and
 * outputs), and pStar, uStar, vStar, dE, dN ((M+1) rows, outputs, zeroed by
 * the call first).  Runs up to max_outer (<= 4096) outer iterations on
 * `stream` (a cudaStream_t; NULL = default stream), stopping when
 * max(residU, residV, residMassDof) <= eps (eps > 0); history (host, may be
 * NULL) and *n_done as for cps_solve; desc's alpha/gamma/layout/device/
 * grid_ctas/pcg_variant are ignored (the reference's PCG is used) and
 * precision must be CPS_FP64.
 *
 * All scratch lives in one static device array of about 27 MB per GPU, held
 * until the process exits; designs need (M+1)*pitch <= 131072 elements or are
 * rejected with CPS_ERR_ARG (reason printed to stderr).  Every call on a device
 * shares that array: calls overlapping on the GPU race, so serialise them.
 * Each call looks the array's device address up in the calling thread's
 * current context (an allocation-free lookup), so it works under whichever
 * context the caller has made current; the first call in a process also
 * loads the kernel's module, so make it before any stream capture.  Elements
 * outside the logical matrices (the columns past each width, row M of the v
 * plane) are never read and may hold anything.  The call works on `stream`
 * only and synchronises it before returning; its grid is the one cps_create
 * would pick for the same design. */
cps_status cps_solve_noalloc(const cps_desc* desc, int pitch, const double* alpha, const double* gamma, double* u,
                             double* v, double* p, double* pStar, double* uStar, double* vStar, double* dE,
                             double* dN, double inletVelocity, int max_outer, double eps, cps_step_out* history,
                             int* n_done, void* stream);

/* Device bytes held by a context created from desc (admission control). */
cps_status cps_footprint(const cps_desc* desc, unsigned long long* bytes);

/* ---- The reference's files at the boundary (host code, no GPU) ---- */

/* fluid_params.txt as SIMPLE::loadParameters reads it (SIMPLE.cpp:31-47):
 * "M N hy hx U_in N_in_buffer N_out_buffer [Ht ...]". */
typedef struct {
  int M, N;
  double hx, hy, U_in;
  int N_in_buffer, N_out_buffer;
  double Ht;       /* the optional out-of-plane height */
  int has_Ht;
} cps_case_params;
cps_status cps_read_case_params(const char* path, cps_case_params* out);

/* geometry_fluid.txt as loadTopology + loadDensityField read it
 * (SIMPLE.cpp:517-584): M x N cellType values (0 fluid, 1 solid), row-major
 * into cellType and/or gamma = 1 - cellType (either may be NULL); a missing
 * file means all fluid (CPS_OK, message in cps_io_last_error) and a short
 * one stops at its end (*values_read, may be NULL, counts what was read). */
cps_status cps_read_geometry(const char* path, int M, int N, double* cellType, double* gamma, int* values_read);

/* Restart matrices dir/u.txt ((M+1) x N), v.txt (M x (N+1)), p.txt
 * ((M+1) x (N+1)), row-major, as the restart loader reads them
 * (SIMPLE.cpp:203-226): a missing or incomplete file leaves its matrix zero;
 * *loaded (may be NULL) counts the complete ones. */
cps_status cps_read_restart(const char* dir, int M, int N, double* u, double* v, double* p, int* loaded);

/* SIMPLE::saveAll (output.cpp:73-266) into dir: u, v, p (staggered),
 * u_full, v_full, pressure_full (cell-centred), u_thermal, v_thermal,
 * pressure_thermal, p_gradient (without the inlet/outlet buffer columns) as
 * tab-separated text, and fluid_results.vtk; numbers printed as the
 * reference prints them.  cellType may be NULL (then 1 - gamma). */
cps_status cps_save_all(const char* dir, int M, int N, double hx, double hy, int N_in_buffer, int N_out_buffer,
                        const double* u, const double* v, const double* p, const double* cellType,
                        const double* gamma, const double* alpha, int layout);

/* The outer loop's two logs as runIterations writes them (initLogFiles and
 * writeIterationLogs, output.cpp:268-313): dir/residuals.txt (iteration,
 * mass, U and V residuals, core and full total-pressure drop, CFL number)
 * and dir/pressure_drop_history.txt (iteration, core total, full total,
 * core static, full static drop), one row per outer iteration numbered from
 * iter0, numbers as the reference prints them.  hist: n rows of a solve's
 * history (residMass, residU, residV are logged); dp: n x 4 drops in that
 * order (cps_solve_monitored's), or NULL to log 0; cfl: n CFL numbers, or
 * NULL to log cfl0 on every row (pseudoCFL, constant while pseudo-time
 * stepping is off). */
cps_status cps_save_logs(const char* dir, int n, int iter0, const cps_step_out* hist, const double* dp,
                         const double* cfl, double cfl0);

/* Message of the last failed (or warning) file call on this thread. */
const char* cps_io_last_error(void);

/* Self-test of the persistent kernels' failure detection: launches `ctas`
 * CTAs (1..1024) on `device` that wait at the grid barrier the persistent
 * kernels use, told to expect one CTA more than the launch has, so the wait
 * can end only by its time limit (2 s of %globaltimer), after which the
 * kernel records a timeout status and every CTA returns.  Returns
 * CPS_ERR_TIMEOUT, the expected outcome, with the kernel's run time in
 * *kernel_ms (may be NULL) and the message in cps_last_error(NULL); CPS_OK
 * would mean the barrier let the CTAs through short of their count. */
cps_status cps_barrier_selftest(int device, int ctas, double* kernel_ms);

/* Message of the last failed call on ctx (or of the last failed cps_create
 * on this thread when ctx is NULL). */
const char* cps_last_error(const cps_ctx* ctx);

/* Library version string. */
const char* cps_version(void);

/* The tile shape this build of the library evaluates (points per tile:
 * *rows x *cols, one point per thread of a 256-thread CTA).  The shape is a
 * compile-time constant of the kernels; libcps.so is built with 8 x 32 tiles,
 * libcps_t16.so with 16 x 16 and libcps_t64.so with 4 x 64, all with this same
 * ABI.  The shape changes only which points a CTA evaluates together (and so
 * the grouping of the grid-wide sums), not the per-point arithmetic. */
cps_status cps_tile_shape(int* rows, int* cols);

#ifdef __cplusplus
}
#endif

#endif /* CPS_H */
