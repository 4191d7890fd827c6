/*
 * rq_b200.h -- C ABI of the B200-native forward model for Bayesian calibration
 * of RANS (k-omega SST) closure coefficients.
 *
 * Plain C types only: host pointers and sizes in, host buffers out (the
 * *_device variants take device pointers and a CUDA stream as void*). Every
 * entry point returns RQ_OK or a negative RQ_E_* code; rq_last_error() gives
 * the message of the calling thread's last failure. No C++ exception crosses
 * this boundary.
 *
 * Reference interfaces replaced (paths in the reference project):
 *   rq_problem_create / rq_problem_destroy
 *       ForwardBatch(mesh, parameters, observations, boundaries, nu, settings, U, p, k, omega)
 *       rans-uq/include/ForwardBatch.hpp:34-49, ForwardModel ctor rans-uq/src/ForwardModel.cpp:8-18
 *   rq_evaluate_batch
 *       ForwardBatch::evaluate(theta rows, workers)              rans-uq/include/ForwardBatch.hpp:52-124
 *       (per row: ForwardModel::evaluateWithDiagnostics        rans-uq/src/ForwardModel.cpp:35-137)
 *   rq_evaluate_multi
 *       several ForwardBatch::evaluate calls (one per mesh class) fused into one launch
 *   rq_solve
 *       SIMPLESolver::initUniform + solve(FlowFields&, Workspace&) rans-uq/src/SIMPLESolver.cpp:267-298, 1193-1716
 *   rq_resample_indices, rq_predictive_moments, rq_conformal_quantile, rq_split_conformal
 *       cfdr.statistics resample_posterior / predictive_summary / conformal_quantile /
 *       split_conformal_intervals                     rans-uq/python/cfdr/statistics.py:235-378
 *   rq_evaluate_cached, rq_warm_cache_*
 *       ForwardModel::evaluateWithDiagnostics with its WarmStartCache rans-uq/src/ForwardModel.cpp:35-137,
 *       rans-uq/include/ForwardModel.hpp:21-157 (size, clear, setByteBudget, byteBudget, retainedBytes)
 *   rq_linear_solve
 *       makeSolver(name)->solve(LinearSystem, x, maxIter, tol)  core/include/LinearSolver.hpp:137-153, 988-998
 *   rq_mesh_geometry
 *       Mesh::makePeriodicChannel2D / makeCurvedChannelPeriodic2D + computeWallDistance
 *       core/src/Mesh.cpp:490-741, 431-463
 *   rq_mesh_save_binary
 *       Mesh::saveBinary (MSH2)                                   core/src/Mesh.cpp:751-811
 */
#ifndef RQ_B200_H
#define RQ_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- return codes */
#define RQ_OK 0
#define RQ_E_INVALID -1      /* invalid argument (the reference throws std::invalid_argument) */
#define RQ_E_CUDA -2         /* CUDA runtime failure (no device, launch error, ...)          */
#define RQ_E_OOM -3          /* device memory exhausted (the reference's bad_alloc)            */
#define RQ_E_UNSUPPORTED -4  /* outside the GPU path's scope (see the message)                */

/* ---- EvaluationStatus, same values and order (core/include/EvaluationTypes.hpp:6) */
#define RQ_CONVERGED 0
#define RQ_UNCONVERGED 1
#define RQ_DIVERGED 2
#define RQ_INVALID_PARAMETERS 3
#define RQ_UNKNOWN 4

/* ---- linear solver kinds: the reference factory names "AMG", "PCG", "BiCGSTAB" */
#define RQ_SOLVER_AMG 0
#define RQ_SOLVER_PCG 1
#define RQ_SOLVER_BICGSTAB 2

/* ---- inner-solve precision */
#define RQ_PREC_FP64 0   /* plain form: every inner solve in FP64 */
#define RQ_PREC_MIXED 1  /* FP32 Krylov/AMG sweeps with FP64 residual refinement */

/* mesh kinds */
#define RQ_MESH_PERIODIC_CHANNEL 0 /* Mesh::makePeriodicChannel2D(nx, ny, lx, h, re_tau, yplus) */
#define RQ_MESH_CURVED_PERIODIC 1  /* Mesh::makeCurvedChannelPeriodic2D(x_nodes, y_bottom, y_top, ny, re, yplus) */

typedef struct rq_mesh_desc {
    int32_t kind, nx, ny, pad;
    double lx, h, re_tau, yplus;        /* channel */
    const double *x_nodes;              /* curved: nx+1 x nodes */
    const double *y_bottom;             /* curved: nx+1 bottom samples (periodic) */
    double y_top, re;                   /* curved */
} rq_mesh_desc;

/* FlowBoundaryConditions::channelDefaults(mesh, u_in, k_in, omega_in): on the
   streamwise-periodic meshes every boundary is a no-slip k-omega wall. */
typedef struct rq_bc_desc {
    double u_in, k_in, omega_in;
} rq_bc_desc;

/* SolverSettings (core/include/FlowFields.hpp:70-241), hot-path subset. */
typedef struct rq_settings {
    int32_t max_iterations;      /* 500     */
    int32_t inner_iterations;    /* 200     */
    int32_t convergence_window;  /* 25      */
    int32_t monitor_interval;    /* 10      */
    int32_t turb_start_iter;     /* 5       */
    int32_t turb_update_interval;/* 1       */
    int32_t nut_floor_iters;     /* 500     */
    int32_t pressure_solver;     /* RQ_SOLVER_AMG */
    int32_t precision;           /* RQ_PREC_FP64 */
    int32_t block_threads;       /* 0 = the class's launch shape (default rule, or what
                                    rq_problem_tune / rq_problem_set_launch chose) */
    double convergence_tol;      /* 1e-5    */
    double inner_tolerance;      /* 1e-3    */
    double divergence_limit;     /* 1e6     */
    double alpha_u, alpha_p, alpha_k, alpha_omega; /* 0.7 0.3 0.5 0.5 */
    double body_force[3];        /* 0 0 0   */
    double k_min, k_max, omega_min; /* 1e-10 1e10 1e-6 */
} rq_settings;

/* Velocity-profile probes (ObservationOperator::addVelocityProfile). */
typedef struct rq_obs_desc {
    int32_t n_obs, component;      /* component 0 = x, 1 = y */
    const double *x, *y;           /* probe locations */
    const double *observed;        /* y_obs */
    const double *sigma_obs;       /* observation std */
    const double *sigma_model;     /* model discrepancy std (may be NULL) */
} rq_obs_desc;

/* One batch row (ForwardBatchRow, rans-uq/include/ForwardBatch.hpp:8-14). */
typedef struct rq_row_out {
    int32_t status;        /* RQ_CONVERGED ... RQ_UNKNOWN */
    int32_t iterations;    /* EvaluationResult::simpleIters */
    int32_t stalled;
    int32_t converged;
    double loglik;         /* -1e30 invalid, -1e6 diverged/unknown */
    double final_worst;    /* ConvergenceHistory::finalWorstMeasure */
    double contraction_rate;
} rq_row_out;

/* Solver result (SolverResult, core/include/LinearSolver.hpp:137-143). */
typedef struct rq_solver_result {
    int32_t iterations, converged;
    double final_res, initial_res;
} rq_solver_result;

/* LDU system (LinearSystem, core/include/LinearSolver.hpp:20-116). */
typedef struct rq_ldu {
    int32_t n_cells, n_faces;
    const double *diag, *upper, *lower, *source;
    const int32_t *owner, *neighbour;
} rq_ldu;

typedef struct rq_problem rq_problem;

const char *rq_last_error(void);
int rq_version(void);

/* Fills s with the reference's SolverSettings defaults. */
int rq_default_settings(rq_settings *s);

/* Builds a mesh class on the device. init = {Ux, Uy, Uz, p, k, omega} (cold start);
   active = InferenceParameterSet active indices (0..10), base = the 11 coefficients
   that fill the inactive ones (SSTCoefficients order). The class lives on the
   device current at this call: every later call on the problem (and on servers and
   warm-start caches built from it) must be made with that device current, else it
   returns RQ_E_INVALID; the destroy calls switch to it themselves. */
int rq_problem_create(const rq_mesh_desc *mesh, const rq_bc_desc *bc, double nu,
                      const rq_settings *settings, const rq_obs_desc *obs, const double init[6],
                      const int32_t *active, int32_t n_active, const double base[11],
                      rq_problem **out);
int rq_problem_destroy(rq_problem *p);
int rq_problem_info(const rq_problem *p, int32_t *n_cells, int32_t *n_obs, int32_t *n_active,
                    int32_t *amg_levels);

/* Device workspace one solve of this mesh class uses (a batch CTA's slot, a serving
   request's pool region), in bytes. */
int rq_problem_workspace_bytes(const rq_problem *p, uint64_t *bytes);

/* Launch shape of a mesh class: the CTA size of its solves and the shared-memory
   arena each CTA places the solve's hottest arrays in. */
typedef struct rq_launch_shape {
    int32_t block_threads;   /* 64, 128, 256, 512, 768 or 1024 */
    int32_t arena_kb;        /* arena per CTA in KiB; 0 = none; -1 = the default rule (half
                                the SM's shared memory up to 768 cells, none above) */
    double us_per_iteration; /* measured by rq_problem_tune; 0 when not measured */
} rq_launch_shape;

/* Autotuner of the launch shape per mesh class (no reference counterpart). For every
   candidate (NULL = the built-in set: 256, 512, 768 threads x arena none / default /
   largest that fits) it times one solve at theta (n_active values, host) capped at
   `iters` outer iterations with the GPU's own timer, writes the measured time per
   outer iteration into measured[k] (NULL allowed; candidates that do not fit on an SM
   get a negative time), applies the fastest to the problem and returns it in *chosen.
   Results do not depend on the arena; the CTA size changes only the order of the
   block sums (agreement to rounding). Blocks until the timings are in. */
int rq_problem_tune(rq_problem *p, const double *theta, int32_t iters,
                    const rq_launch_shape *candidates, int32_t n_candidates,
                    rq_launch_shape *measured, rq_launch_shape *chosen);
/* Applies a launch shape (for example one the tuner chose earlier, from a cache);
   RQ_E_INVALID when the CTA size is not one of the six or it does not fit on an SM. */
int rq_problem_set_launch(rq_problem *p, const rq_launch_shape *shape);
int rq_problem_get_launch(const rq_problem *p, rq_launch_shape *shape);

/* theta: n rows x n_active (host). rows: n (host). predictions: n x n_obs (host,
   NaN where the reference returns none). fields (optional, host): n x 11 x n_cells,
   blocks Ux Uy Uz p k omega nuT F1 F2 Pk CDkw. history (optional): n x hist_cap x 11. */
int rq_evaluate_batch(rq_problem *p, const double *theta, int64_t n, rq_row_out *rows,
                      double *predictions, double *fields, double *history, int32_t hist_cap);

/* Several mesh classes in one persistent launch: row i uses problems[problem_of_row[i]];
   theta rows are padded to max n_active (row stride = theta_stride doubles),
   predictions to max n_obs (stride = pred_stride). */
int rq_evaluate_multi(rq_problem *const *problems, int32_t n_problems,
                      const int32_t *problem_of_row, const double *theta, int32_t theta_stride,
                      int64_t n, rq_row_out *rows, double *predictions, int32_t pred_stride);

/* Same on device buffers (device theta, rows, predictions) on a CUDA stream (cudaStream_t as
   void*), queued without waiting. clock_ns_dev (optional, device): 12 int64 per row -- the
   solve's start and end on the GPU global timer (ns), its inner Krylov iterations, its
   inner pressure-correction iterations, then SM cycles spent per stage: set-up, closure,
   momentum, pressure assembly, pressure solve, AMG refresh, turbulence, bookkeeping. */
int rq_evaluate_multi_device(rq_problem *const *problems, int32_t n_problems,
                             const int32_t *problem_of_row_host, const double *theta_dev,
                             int32_t theta_stride, int64_t n, rq_row_out *rows_dev,
                             double *predictions_dev, int32_t pred_stride, void *stream,
                             int64_t *clock_ns_dev);

/* One solve from a cold start with all eleven coefficients. */
int rq_solve(rq_problem *p, const double coeffs[11], rq_row_out *row, double *predictions,
             double *fields, double *history, int32_t hist_cap);

/* Mesh geometry as built for the device (nCells x 4: cx, cy, volume, wall distance). */
int rq_mesh_geometry(const rq_mesh_desc *mesh, int32_t *n_cells, double *cells);

/* Mesh::saveBinary (core/src/Mesh.cpp:751-811; Mesh.hpp:264-268): the generated mesh
   written to `path` in the reference's MSH2 binary layout (native byte order, int32
   indices, IEEE binary64 geometry, the periodic shift after each face's weight),
   byte-identical to the reference's file for the same generator call, so the
   reference's Mesh::loadBinary and tools read it. Host only (no device work). */
int rq_mesh_save_binary(const rq_mesh_desc *mesh, const char *path);

/* The linear solvers of the forward model on one LDU system, in FP64
   (ILinearSolver::solve, core/include/LinearSolver.hpp:137-153; kinds RQ_SOLVER_*
   for the factory names "AMG", "PCG", "BiCGSTAB" of makeSolver, :988-998;
   "GaussSeidel" returns RQ_E_UNSUPPORTED). x: initial guess in, solution out
   (host). The AMG is this project's device variant: greedy strength-0.25
   aggregation of the matrix, damped-Jacobi V-cycle, dense coarsest inverse. */
int rq_linear_solve(const rq_ldu *A, double *x, int32_t max_iter, double tol, int32_t kind,
                    rq_solver_result *result);
/* Many systems in one persistent launch (one CTA per system, largest first).
   x[s]: per-system initial guess in, solution out (host). precision RQ_PREC_MIXED:
   FP32 PCG corrections inside an FP64 residual-refinement loop (AMG and PCG kinds;
   BiCGSTAB stays FP64); result iterations count the inner FP32 iterations. */
int rq_linear_solve_batch(const rq_ldu *systems, int32_t n_systems, double *const *x,
                          int32_t max_iter, double tol, int32_t kind, int32_t precision,
                          rq_solver_result *results);
/* The same with the set-up kept on the device between solves: create builds and
   uploads every system's operator and hierarchy once; solve runs them from x
   (or from zero when x is NULL); solve_device queues a zero-start solve on a
   CUDA stream (void*) and returns; results copies results and solutions back. */
typedef struct rq_linsys rq_linsys;
int rq_linsys_create(const rq_ldu *systems, int32_t n_systems, int32_t kind, int32_t precision,
                     rq_linsys **out);
int rq_linsys_solve(rq_linsys *L, int32_t max_iter, double tol, double *const *x,
                    rq_solver_result *results);
int rq_linsys_solve_device(rq_linsys *L, int32_t max_iter, double tol, void *stream);
int rq_linsys_results(rq_linsys *L, rq_solver_result *results, double *const *x);
int rq_linsys_info(const rq_linsys *L, int32_t *n_systems, int64_t *total_rows, int64_t *total_nnz,
                   int32_t *max_levels);
int rq_linsys_destroy(rq_linsys *L);

/* One draw without any device allocation (no counterpart in the reference). For
   callers that must not allocate GPU memory once they are running: a sampler
   embedded in a host application whose memory budget was fixed at start-up, or
   a latency-bound loop where cudaMalloc would stall the device to synchronise.
   theta_dev (n_active doubles), row_dev (one rq_row_out) and predictions_dev
   (n_obs doubles) are the caller's device buffers; the solve's scratch is a fixed
   8 MiB array in the library (held on every GPU that loads it until exit), so
   mesh classes needing more (above about 17000 cells) are rejected with
   RQ_E_INVALID. The problem must come from rq_problem_create (which does
   allocate, and which also resolves the scratch array's device address on its
   device), so the call itself only launches. It must be made with the problem's
   device current (RQ_E_INVALID otherwise). Queued on `stream` (cudaStream_t as
   void*) without waiting. Nothing in the scratch needs to start at zero (a
   solve writes every array before reading it), but every call shares it:
   calls whose solves overlap on the GPU race and corrupt each other. Like every
   handle, the problem does not survive a reset of its device. */
int rq_evaluate_noalloc(rq_problem *p, const double *theta_dev, rq_row_out *row_dev,
                        double *predictions_dev, void *stream);

/* Normalised importance weights of a finite posterior, in FP64 on the GPU
   (cfdr.statistics.posterior_weights, rans-uq/python/cfdr/statistics.py:217-232):
   w_i = exp(l_i - log_q_i - m) / sum_j exp(l_j - log_q_j - m), m the maximum;
   log_q may be NULL (an independent prior design). A non-finite log-likelihood
   is RQ_E_INVALID, as the reference raises. log_evidence (optional) receives
   m + log(sum), the log-sum-exp. */
int rq_posterior_weights(const double *loglik, const double *log_q, int64_t n, double *weights,
                         double *log_evidence);
/* The same with the two parts of the log-sum-exp kept apart: max_out = m and
   sum_out = sum_j exp(l_j - log_q_j - m), for combining shards of one ensemble held
   by several ranks without the rounding of m + log(sum). */
int rq_posterior_weights_parts(const double *loglik, const double *log_q, int64_t n,
                               double *weights, double *max_out, double *sum_out);
/* The same on device buffers on a stream, queued without waiting; out3_dev
   receives {m, sum, number of non-finite terms} (weights are unset when the count
   is nonzero). */
int rq_posterior_weights_device(const double *loglik_dev, const double *log_q_dev, int64_t n,
                                double *weights_dev, double *out3_dev, void *stream);

/* ---- serving loop (no reference counterpart: the reference evaluates fixed
   batches only, ForwardBatch.hpp:52-124). A server owns a persistent kernel whose
   CTAs (slots = min(SMs x resident CTAs, max_slots if > 0)) claim requests in
   submission order as they are admitted; a CTA takes the next request as soon as
   its solve retires. Each admitted request solves in its own region of a device
   workspace pool sized for its mesh class; a request is admitted once its region
   fits in the pool (in submission order) and its region returns to the pool when
   its solve retires, so admission follows free memory as solves come and go.
   Requests and results live in pinned host memory mapped into the device, so a
   request needs no copy and a result is visible to rq_server_poll as soon as its
   done flag is raised. The problems must outlive the server. CTAs leave after
   idle_timeout_s without requests; submit / poll / wait launch more CTAs beside
   the ones still running whenever admitted requests wait and fewer CTAs than slots
   run. capacity bounds the requests over the server's lifetime. rq_server_create
   sizes the pool at 80 % of the free device memory (at most what the slots can use
   at once). */
typedef struct rq_server rq_server;
int rq_server_create(rq_problem *const *problems, int32_t n_problems, int32_t capacity,
                     double idle_timeout_s, int32_t max_slots, rq_server **out);
/* The same with the workspace pool's size given (pool_bytes 0 = the default above);
   RQ_E_OOM when it cannot hold one solve of the largest class. */
int rq_server_create_pooled(rq_problem *const *problems, int32_t n_problems, int32_t capacity,
                            double idle_timeout_s, int32_t max_slots, uint64_t pool_bytes,
                            rq_server **out);
/* theta: the problem's n_active values (host, copied). ticket: request index. */
int rq_server_submit(rq_server *s, int32_t problem, const double *theta, int64_t *ticket);
/* done = 1 once the request's row, predictions and clock record (12 int64, as
   rq_evaluate_multi_device) are final; the optional outputs are filled then. */
int rq_server_poll(rq_server *s, int64_t ticket, int32_t *done, rq_row_out *row,
                   double *predictions, int64_t *clock12);
/* Waits until every submitted request is done or timeout_s passes. */
int rq_server_wait(rq_server *s, double timeout_s, int64_t *completed);
/* No more submissions: the kernel drains what was submitted and leaves. */
int rq_server_close(rq_server *s);
int rq_server_info(rq_server *s, int32_t *slots, int64_t *submitted, int64_t *completed,
                   int32_t *launches);
/* The pool: its bytes, the bytes held by admitted requests whose solves have not
   retired, requests submitted but not yet admitted, and CTAs running now. */
int rq_server_memory(rq_server *s, uint64_t *pool_bytes, uint64_t *in_use_bytes,
                     int64_t *waiting, int32_t *running_ctas);
/* Cancels requests not yet claimed, waits for the solves in flight, frees. */
int rq_server_destroy(rq_server *s);

/* ---- statistics of a finished ensemble on the GPU (cfdr.statistics,
   rans-uq/python/cfdr/statistics.py), each with numpy's rounding so the results equal
   the reference's. Host buffers; the random draws stay with the caller (the
   reference's per-sample PCG64 streams).
   rq_resample_indices: resample_posterior's pick (:235-259) for uniforms[j], the first
   draw of output j's "posterior-resample" stream: numpy's Generator.choice(n, p=weights),
   i.e. cdf = cumsum(weights) in index order, cdf /= cdf[n-1], indices[j] = number of cdf
   values <= uniforms[j]. weights must pass choice's admission (nonnegative, Kahan sum
   within sqrt(eps) of 1) or RQ_E_INVALID. */
int rq_resample_indices(const double *weights, int64_t n, const double *uniforms, int64_t m,
                        int64_t *indices);
/* predictive_summary's latent moments (:277-339): mean and population variance (ddof 0)
   of each column of the row-major n x d matrix, summed in numpy's order. */
int rq_predictive_moments(const double *latent, int64_t n, int32_t d, double *mean,
                          double *variance);
/* conformal_quantile (:349-355): the ceil((n+1)(1-alpha))-th smallest score, +inf when
   that rank exceeds n. */
int rq_conformal_quantile(const double *scores, int64_t n, double alpha, double *quantile);
/* split_conformal_intervals (:358-378): radius = conformal quantile of |y - prediction|
   over the calibration set; lower/upper = test_pred -/+ radius (m values each). */
int rq_split_conformal(const double *cal_y, const double *cal_pred, int64_t n,
                       const double *test_pred, int64_t m, double alpha, double *lower,
                       double *upper);

/* ---- warm starts: the sequential model's cache of converged states
   (WarmStartCache, rans-uq/include/ForwardModel.hpp:21-157; the model's own is
   (50, 0.5, 64 MiB), ForwardModel.cpp:14). Entries stay in device memory; the byte
   count is the reference's payload count (entryBytes, :39-47: theta, the vector
   field and eight scalar fields, each over cells plus boundary faces), so eviction
   happens after the same calls. */
typedef struct rq_warm_cache rq_warm_cache;
/* max_size < 0 or a negative / non-finite threshold: RQ_E_INVALID (the reference throws). */
int rq_warm_cache_create(rq_problem *p, int32_t max_size, double threshold, uint64_t byte_budget,
                         rq_warm_cache **out);
int rq_warm_cache_destroy(rq_warm_cache *c);
/* size, retainedBytes, byteBudget */
int rq_warm_cache_info(rq_warm_cache *c, int32_t *size, uint64_t *retained_bytes,
                       uint64_t *byte_budget);
int rq_warm_cache_clear(rq_warm_cache *c);
/* setByteBudget: evicts oldest entries until the retained bytes fit. */
int rq_warm_cache_set_byte_budget(rq_warm_cache *c, uint64_t byte_budget);
/* ForwardModel::evaluateWithDiagnostics with the cache (rans-uq/src/ForwardModel.cpp:35-137):
   an admitted theta (n_active values, host) starts from the nearest cached state closer
   than the threshold (strictly; ties keep the older entry), else cold; a Converged solve
   is stored (replacing an entry with the same theta). row, predictions (n_obs) and the
   optional fields (11 x n_cells; NaN unless the row is Converged or Unconverged) are
   host buffers; used_warm_start (optional) reports ForwardEvaluationResult::usedWarmStart.
   Snapshot (evaluateWithDiagnostics(theta, snapshot = true); OwnedFlowSnapshot,
   ForwardModel.hpp:162-186), optional, written only for a Converged or Unconverged row
   (the rows the reference snapshots). On these nx x ny periodic meshes there are
   2 nx ny - nx internal faces and 2 nx wall faces (Mesh.cpp:620-625):
   boundary = 11 x 2nx values over the wall faces in the mesh's face order (bottom row,
   then top row), blocks as fields; face_fluxes = 2 nx ny + nx owner-outward fluxes in the
   mesh's face order; turb_established = FlowFields::turbEstablished. */
int rq_evaluate_cached(rq_warm_cache *c, const double *theta, rq_row_out *row,
                       double *predictions, double *fields, double *boundary,
                       double *face_fluxes, int32_t *turb_established,
                       int32_t *used_warm_start);

#ifdef __cplusplus
}
#endif
#endif
