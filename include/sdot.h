/*
 * sdot.h -- C ABI of libsdot_cuda.so, the B200 (sm_100a) implementation of
 * SemiDiscreteOT's entropic semi-discrete dual evaluation and its solver.
 *
 * Plain C: pointers, sizes and status codes; no exceptions, no C++ or torch
 * types cross this boundary.  Host pointers passed in are caller-owned and
 * copied; device state is library-owned.  One context per host thread (a
 * context owns its CUDA stream).  Unless stated otherwise every array uses the
 * caller's ordering (the library reorders internally and maps back).
 *
 * Each entry point cites the reference interface it replaces
 * (paths relative to the SemiDiscreteOT source tree).
 */
#ifndef SDOT_H
#define SDOT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SDOT_ABI_VERSION 1

typedef enum {
    SDOT_OK = 0,
    SDOT_EINVAL = 1,       /* bad argument / inconsistent sizes */
    SDOT_ENOMEM = 2,       /* device allocation failed */
    SDOT_ENONFINITE = 3,   /* NaN/Inf in inputs or in the evaluated functional */
    SDOT_ELINESEARCH = 4,  /* line search could not satisfy the Wolfe conditions */
    SDOT_EMAXITER = 5,     /* solver stopped at max_iterations without converging */
    SDOT_EBUDGET = 6,      /* request exceeds the context's device-memory budget */
    SDOT_ETIMEOUT = 7,     /* a bounded device wait expired */
    SDOT_ECUDA = 8,        /* CUDA runtime error (message in sdot_last_error) */
    SDOT_ESTATE = 9        /* call made in the wrong state (e.g. no source set) */
} sdot_status;

/* Arithmetic of the two exponential sweeps.
 *   SDOT_PREC_FP64  : both sweeps in FP64 (value 1e-10 rel., gradient ~1e-14).
 *   SDOT_PREC_HYBRID: value sweep FP64, gradient sweep FP32 exp2 with FP64
 *                     accumulation (gradient error <= ~3e-6 * max nu_j).
 *   SDOT_PREC_MIXED : accepted and currently run as SDOT_PREC_HYBRID (an FP32
 *                     value sweep cannot meet the 1e-10 relative value bound,
 *                     so the value sweep stays FP64).                       */
typedef enum { SDOT_PREC_FP64 = 0, SDOT_PREC_HYBRID = 1, SDOT_PREC_MIXED = 2 } sdot_precision;

typedef enum { SDOT_THRESH_POINTWISE = 0, SDOT_THRESH_INTEGRAL = 1, SDOT_THRESH_GEOMETRIC = 2 } sdot_threshold_type;
typedef enum { SDOT_CONTROL_L1NORM = 0, SDOT_CONTROL_COMPONENTWISE = 1, SDOT_CONTROL_LINF = 2 } sdot_control_type;
typedef enum { SDOT_LS_UPSTREAM = 0, SDOT_LS_VENDORED = 1 } sdot_line_search;

typedef struct {
    int device;                 /* CUDA device ordinal */
    int precision;              /* sdot_precision */
    size_t memory_budget;       /* bytes of device memory the context may hold (0 = unlimited) */
    int verbose;                /* print per-iteration lines like VerboseSolverControl */
} sdot_options;

/* Mirrors SotParameterManager::SolverParameters
 * (include/SemiDiscreteOT/utils/ParameterManager.h:56-72) plus the line
 * search variant. */
typedef struct {
    unsigned max_iterations;    /* max_iterations (default 1000) */
    double tolerance;           /* tolerance (default 1) */
    int control_type;           /* solver_control_type: l1norm | componentwise | linf */
    double epsilon;             /* epsilon (default 1e-3) */
    double tau;                 /* tau (default 1e-8); <= 0 disables truncation */
    int threshold_type;         /* distance_threshold_type */
    int use_log_sum_exp;        /* use_log_sum_exp_trick (default false) */
    int line_search;            /* sdot_line_search: deal.II SolverBFGS (default) or the vendored copy */
} sdot_solver_params;

typedef struct {
    double value;               /* J(psi) */
    double C_global;            /* sum_q rho_q JxW_q / S_q */
    double threshold;           /* distance threshold used */
    int64_t n_pairs;            /* sum over q of |candidates(cell(q))| */
    double device_ms;           /* device time of the evaluation (CUDA events) */
} sdot_eval_info;

typedef struct {
    unsigned iterations;        /* like get_last_iteration_count() */
    int converged;              /* like get_convergence_status() */
    int64_t n_evaluations;
    double last_value;
    double last_check_value;
    int64_t total_pairs;
    double device_ms;
} sdot_solve_info;

typedef struct sdot_ctx sdot_ctx;
typedef struct sdot_server sdot_server;

/* Library identity: ABI version and the sm architecture it was built for. */
int sdot_abi_version(void);
const char *sdot_build_info(void);

/* Human-readable text of the last error on this context (never NULL). */
const char *sdot_last_error(const sdot_ctx *ctx);

/* Replaces SotSolver::SotSolver(const MPI_Comm&)
 * (include/SemiDiscreteOT/solvers/SotSolver.h:176; src/solvers/SotSolver.cc:3-20). */
sdot_status sdot_create(sdot_ctx **ctx, const sdot_options *opts);
void sdot_destroy(sdot_ctx *ctx);

/* Replaces SotSolver::setup_source(dof_handler, mapping, fe, density,
 * quadrature_order) (SotSolver.h:186-190; SotSolver.cc:43-51).  deal.II objects
 * cannot cross a C ABI, so the source arrives flattened exactly as
 * SemiDiscreteOT::save_discrete_measures writes it (src/core/SemiDiscreteOT.cc
 * :2489-2558): quadrature points x (n_q*dim, row-major), JxW and the density
 * value at each point, grouped by cell: cell c owns points
 * [cell_offsets[c], cell_offsets[c+1]) and has centre cell_centers[c*dim..]
 * (TriaAccessor::center(), used by the truncation query at SotSolver.cc:801). */
sdot_status sdot_set_source(sdot_ctx *ctx, int dim, int64_t n_q, const double *x,
                            const double *jxw, const double *density, int64_t n_cells,
                            const int64_t *cell_offsets, const double *cell_centers);

/* Replaces SotSolver::setup_target(points, density) (SotSolver.h:197-198;
 * SotSolver.cc:53-60).  Like the reference, the weights are NOT normalised. */
sdot_status sdot_set_target(sdot_ctx *ctx, int64_t n, const double *y, const double *nu);

/* Replaces SotSolver::configure(params) (SotSolver.h:204; SotSolver.cc:62-69). */
sdot_status sdot_configure(sdot_ctx *ctx, const sdot_solver_params *params);
/* Defaults of SolverParameters (ParameterManager.h:56-72). */
void sdot_default_params(sdot_solver_params *params);

/* Replaces SotSolver::evaluate_functional(psi, gradient_out) (SotSolver.h:336-337;
 * SotSolver.cc:217-377): returns J(psi) in *value and grad_j =
 * sum_q w_q pi_qj - nu_j in grad (host arrays of n_targets doubles).  Updates
 * the persistent state read by the integral/geometric thresholds, like the
 * reference's members global_functional and C_global. */
sdot_status sdot_evaluate(sdot_ctx *ctx, const double *psi, double *grad, double *value,
                          sdot_eval_info *info);

/* Same evaluation on device pointers (internal ordering is NOT applied: psi
 * and grad are in the caller's ordering, resident on the context's device);
 * no host synchronisation beyond reading the scalar value. */
sdot_status sdot_evaluate_device(sdot_ctx *ctx, const double *psi_dev, double *grad_dev,
                                 double *value, sdot_eval_info *info);

/* Replaces SotSolver::solve(potential, params) (SotSolver.h:211-212;
 * SotSolver.cc:105-215): L-BFGS (history 5) with the strong-Wolfe line search
 * of deal.II SolverBFGS, driven on the device.  psi is read as the initial
 * potential and overwritten with the result.  Like the reference,
 * non-convergence is not an error: it returns SDOT_OK with converged = 0
 * (query sdot_get_convergence_status); SDOT_ELINESEARCH corresponds to the
 * exception the upstream line search throws. */
sdot_status sdot_solve(sdot_ctx *ctx, double *psi, const sdot_solver_params *params,
                       sdot_solve_info *info);

/* Replaces the declared-only SotSolver::compute_hessian(potential, hessian_out)
 * (SotSolver.h:343-344): dense row-major n_targets x n_targets matrix
 * H = (1/eps) sum_q w_q (diag(pi_q) - pi_q pi_q^T) into host memory H. */
sdot_status sdot_hessian(sdot_ctx *ctx, const double *psi, double *H);

/* Hessian on device memory, by method:
 *   SDOT_HESS_FP64  : the FP64 kernel of sdot_hessian (any threshold);
 *   SDOT_HESS_TENSOR: tcgen05 tensor cores, H = (diag(sum w pi) - P_w^T P)/eps
 *                     with P regenerated tile by tile (never stored), BF16
 *                     hi+lo operands (three products), FP32 accumulation in
 *                     tensor memory drained into FP64 every few thousand
 *                     points; relative Frobenius error ~1e-5 against FP64.
 *                     Needs an untruncated evaluation (tau <= 0, or a
 *                     threshold above the domain diameter) and rho*JxW >= 0;
 *   SDOT_HESS_AUTO  : SDOT_HESS_TENSOR when it applies, else SDOT_HESS_FP64.
 * Same matrix as sdot_hessian (the declared-only SotSolver::compute_hessian,
 * SotSolver.h:343-344), evaluated at psi_dev (device, caller order, n_targets
 * doubles).  H_dev: device, n_targets^2 entries row-major in the caller's
 * order, double (out_f32 = 0) or float (out_f32 = 1, tensor method only).
 * Like an evaluation, it updates the state read by the thresholds. */
typedef enum { SDOT_HESS_AUTO = 0, SDOT_HESS_FP64 = 1, SDOT_HESS_TENSOR = 2 } sdot_hessian_method;
typedef struct {
    int method;                 /* method used */
    double eval_ms;             /* device time of the evaluation at psi */
    double hessian_ms;          /* device time of the Hessian (set-up kernels included) */
    double kernel_ms;           /* main Hessian kernel alone (tensor method: needs sdot_set_profiling) */
    int64_t tiles;              /* tensor method: 128 x 256 output tiles computed */
} sdot_hessian_info;
sdot_status sdot_hessian_device(sdot_ctx *ctx, const double *psi_dev, void *H_dev, int method, int out_f32,
                                sdot_hessian_info *info);
/* Tuning of the tensor method: stages of 64 points accumulated in FP32 before
 * each FP64 drain (default 64). */
sdot_status sdot_set_hessian_chunk(sdot_ctx *ctx, int stages);
/* Bound of the tensor method's device-side waits (no reference counterpart:
 * the reference has no device code).  The kernel's stage loop waits on
 * mbarriers for its tensor-core products; a wait that takes more than
 * `clocks` SM clock cycles makes the kernel stop, wait (with the default
 * bound) for the products already issued, release its tensor memory and
 * report SDOT_ETIMEOUT, leaving the context usable.  clocks <= 0 restores
 * the default, 2e9 cycles (about 1 s at 1.965 GHz).  A bound below the
 * products' own latency (a few thousand cycles) makes every call time out:
 * that is how the failure path is tested. */
sdot_status sdot_set_hessian_wait_limit(sdot_ctx *ctx, int64_t clocks);
/* Operand generation of the tensor method (no reference counterpart).  When
 * the source's cells are 2 x 2 x 2 Gauss grids (3D, QGauss(2)) and the
 * per-dimension factors stay within 2^24, each generated row takes one ex2
 * per cell and one per dimension instead of one per point: the 8 values of a
 * cell are products of those factors and a per-point factor formed once per
 * point.  factored = 1 (default) uses it where it applies, 0 never, < 0 leaves
 * the setting; *last_factored (may be NULL) tells whether the last tensor
 * Hessian of the context used it. */
sdot_status sdot_set_hessian_generation(sdot_ctx *ctx, int factored, int *last_factored);
/* Whole tensor Hessians on SM pairs (no reference counterpart): 256 x 256
 * tiles whose products run over two SMs (tcgen05 cta_group::2, a cluster of
 * two CTAs), so that each SM generates two thirds of the operand rows it
 * would alone.  pairs = 2 (default): SM pairs, each CTA's operand generation
 * split into two groups of warps that take alternate stages, with a warp of
 * its own issuing the products; 1: SM pairs, one generating group; 0: single
 * SMs (128 x 256 tiles); < 0 leaves the setting.  *last_pairs (may be NULL)
 * receives the mode the last tensor Hessian of the context ran in.  A range
 * of tiles (sdot_hessian_tiles_device) always runs on single SMs. */
sdot_status sdot_set_hessian_pairs(sdot_ctx *ctx, int pairs, int *last_pairs);

/* The tensor-core Hessian in pieces, for sharding it over GPUs by output tiles
 * (no reference counterpart: the reference's Hessian is declared only,
 * SotSolver.h:343-344).  The upper triangle is covered by
 * sdot_hessian_tile_count tiles of 128 x 256 entries, each entry (a <= b) in
 * exactly one tile.  sdot_hessian_tiles_device evaluates at psi_dev like
 * sdot_hessian_device, then computes tiles [tile_begin, tile_end) only,
 * writing their entries and the mirrored ones of H_dev and leaving every other
 * entry untouched: with H_dev zeroed first, the matrices of disjoint ranges sum
 * to the full Hessian, and each one's product with x to its share of H x.
 * sdot_hessian_matvec_device: y = H x with FP64 accumulation over an n x n
 * row-major H (float when f32, else double), the product the Newton CG uses;
 * it returns after the product is complete. */
sdot_status sdot_hessian_tile_count(sdot_ctx *ctx, int64_t *count);
sdot_status sdot_hessian_tiles_device(sdot_ctx *ctx, const double *psi_dev, void *H_dev, int out_f32,
                                      int64_t tile_begin, int64_t tile_end, sdot_hessian_info *info);
sdot_status sdot_hessian_matvec_device(sdot_ctx *ctx, const void *H_dev, int f32, const double *x_dev,
                                       double *y_dev);

/* Newton solver with the tensor-core Hessian.  The reference declares the
 * Hessian (SotSolver::compute_hessian, SotSolver.h:343-344) but solves only
 * with deal.II SolverBFGS (SotSolver::solve, SotSolver.cc:105-215); this is
 * the second-order solve the Hessian is for, with solve()'s parameters,
 * convergence control (l1norm / componentwise / linf) and in-place potential
 * update.  Each iteration: FP64 evaluation; Hessian by hessian_method
 * (sdot_hessian_method; the tensor Hessian is stored in FP32); H p = -g by
 * Jacobi-preconditioned CG with FP64 vectors, the constant null vector
 * projected out and the true residual recomputed in FP64 every 64 steps;
 * Armijo backtracking on J in FP64.  Non-convergence within max_iterations is
 * SDOT_OK with converged = 0, like sdot_solve.  n_targets <= 46340.  The
 * evaluations use the context's precision: create it with SDOT_PREC_FP64 for
 * tolerances below the FP32-exponential gradient error (~5e-6 max nu_j). */
typedef struct {
    unsigned iterations;        /* Newton steps taken */
    int converged;
    int64_t n_evaluations;      /* functional evaluations (line search included) */
    int64_t cg_iterations;      /* CG iterations over all steps */
    double last_value;
    double last_check_value;
    int64_t total_pairs;
    double eval_ms;             /* device time in evaluations */
    double hessian_ms;          /* device time in Hessians */
    double cg_ms;               /* device time in CG */
    int hessian_method;         /* method of the last Hessian */
    int64_t n_hessians;         /* Hessians computed (see sdot_set_newton_hessian_reuse) */
} sdot_newton_info;
sdot_status sdot_solve_newton(sdot_ctx *ctx, double *psi, const sdot_solver_params *params, int hessian_method,
                              sdot_newton_info *info);
/* Lagged Hessians for sdot_solve_newton (no reference counterpart): the
 * Hessian of an earlier step is kept while the previous Newton step was a
 * full step (no halving) and reduced the gradient's 2-norm at least by the
 * factor `contraction` (0 < contraction < 1); otherwise it is recomputed.
 * 0 recomputes it every step; the default is 0.1 (config 3, N = 20,000: 3
 * Hessians instead of 4, 1.56 s instead of 2.01 s).  Convergence is still
 * decided on the FP64 gradient; only the search directions change. */
sdot_status sdot_set_newton_hessian_reuse(sdot_ctx *ctx, double contraction);

/* Replaces SoftmaxRefinement::compute_refinement (src/solvers/SoftmaxRefinement.cc
 * :61-280), the softmax transfer of potentials from a coarse target level to
 * its children used by SemiDiscreteOT::assign_potentials_by_hierarchy
 * (SemiDiscreteOT.cc:748-828).  The context's source is the source measure
 * and its target measure (sdot_set_target) is the COARSE level; psi_coarse
 * holds its potentials (caller order).  Fine level: n_fine points y_fine and
 * the children of coarse target i at child_indices[child_offsets[i] ..
 * child_offsets[i+1]) (each fine target the child of at most one coarse
 * target).  epsilon is the regularisation (lambda), threshold the distance
 * threshold r (the reference passes the last solve's), use_log_sum_exp the
 * reference's flag.  psi_fine[k] = -epsilon log(sum) where the sum of
 * contributions is positive, else 0.  Up to 32 quadrature points per cell. */
sdot_status sdot_softmax_refinement(sdot_ctx *ctx, const double *psi_coarse, double epsilon, double threshold,
                                    int use_log_sum_exp, int64_t n_fine, const double *y_fine,
                                    const int64_t *child_offsets, const int64_t *child_indices, double *psi_fine);

/* Replaces SotSolver::evaluate_weighted_barycenters for the euclidean distance
 * (SotSolver.cc:584-660) through compute_weighted_barycenters_euclidean
 * (:871-971).  Evaluates at psi (caller order) with the configured parameters
 * (threshold recomputed as there), then
 *   barycenters[j*dim + d] = sum_q rho_q JxW_q pi_qj x_q[d] / nu_j,
 *   pi_qj = nu_j e^(t_qj) / sum_i nu_i e^(t_qi) over the candidates of cell(q),
 * skipped points (no candidate or zero sum) excluded.  n_targets x dim out. */
sdot_status sdot_weighted_barycenters(sdot_ctx *ctx, const double *psi, double *barycenters);

/* Replaces SotSolver::get_potential_conditioned_density (SotSolver.cc:973-1046).
 * For each of n_points query points (the reference's DoF support points) with
 * the source density there, and each requested target k = indices[i]:
 *   out[i*n_points + p] = density(p) e^(t_k(p) - m) / sum_j nu_j e^(t_j(p) - m)
 * when target k lies within `threshold` of the point, else 0 (also 0 when the
 * point has no candidate).  t_j(p) = (psi_j - |p - y_j|^2 / 2) / epsilon; m the
 * largest t over the candidates.  The reference uses its current epsilon and
 * last distance threshold; pass them. */
sdot_status sdot_conditioned_densities(sdot_ctx *ctx, const double *psi, double epsilon, double threshold,
                                       int64_t n_points, const double *points, const double *density_at_points,
                                       int64_t n_indices, const int64_t *indices, double *out);

/* ---- batched solves (no single reference counterpart: many SotSolver::solve
 * calls, SotSolver.cc:105-215, each over an epsilon-scaling sequence as in
 * SemiDiscreteOT.cc:878-922, advanced together on one GPU) ----
 * A batch holds untruncated problems (tau <= 0, pointwise threshold) of one
 * dimension and uneven sizes, packed in device memory.  Every batched
 * evaluation runs all active problems in four launches (persistent sweeps
 * over (problem, block) work units, largest first); each problem keeps its
 * own L-BFGS state, line search (deal.II rules, as sdot_solve) and
 * convergence control from its sdot_solver_params.  Sources use the
 * flattened quadrature layout of sdot_set_source without the cell structure
 * (the untruncated path never queries cells).  psi arrays concatenate the
 * problems in the order they were added, each in its caller order. */
typedef struct sdot_batch sdot_batch;
typedef struct {
    double epsilon_scaling_factor;  /* EpsilonScalingHandler factor (> 1; default 10) */
    int epsilon_scaling_steps;      /* levels eps f^(s-1), ..., eps (1 = no scaling) */
    double intermediate_tolerance;  /* tolerance of the levels before the last (<= 0: each problem's own) */
    int mixed_precision;            /* 1: FP32-exponential gradient sweeps until a problem meets its tolerance,
                                       then FP64 sweeps until it meets the same tolerance in FP64 */
} sdot_batch_options;
typedef struct {
    int n_problems;
    int converged;                  /* problems that met their tolerance (in FP64) */
    int64_t rounds;                 /* batched evaluations */
    int64_t evaluations;            /* problem evaluations over all rounds */
    int64_t total_pairs;
    double eval_ms;                 /* device time in batched evaluations */
    double solve_ms;                /* device time of the whole solve */
} sdot_batch_info;
sdot_status sdot_batch_create(sdot_batch **batch, int device, int dim);
void sdot_batch_destroy(sdot_batch *batch);
const char *sdot_batch_last_error(const sdot_batch *batch);
int sdot_batch_size(const sdot_batch *batch);
/* Print each problem's iterations and line-search trials (like VerboseSolverControl). */
sdot_status sdot_batch_set_verbose(sdot_batch *batch, int verbose);
/* Adds one problem (copied); its index is written to *index. */
sdot_status sdot_batch_add(sdot_batch *batch, int64_t n_q, const double *x, const double *jxw, const double *density,
                           int64_t n_t, const double *y, const double *nu, const sdot_solver_params *params,
                           int *index);
/* One batched evaluation at psi (host, concatenated): gradients (host,
 * concatenated) and each problem's J(psi) in values[n_problems]; fp32 != 0
 * runs the gradient sweep with FP32 exponentials. */
sdot_status sdot_batch_evaluate(sdot_batch *batch, const double *psi, double *grad, double *values, int fp32);
/* Solves every problem; psi (host, concatenated) holds the initial
 * potentials and receives the results.  Non-convergence is reported per
 * problem (sdot_batch_problem_info), not as an error; a line-search failure
 * is SDOT_ELINESEARCH after all other problems have finished. */
sdot_status sdot_batch_solve(sdot_batch *batch, double *psi, const sdot_batch_options *opts, sdot_batch_info *info);
sdot_status sdot_batch_problem_info(const sdot_batch *batch, int index, sdot_solve_info *info);
/* Launch shape of the batched sweeps (no reference counterpart): shape[0]
 * and shape[1] are the persistent CTAs per SM of the value and gradient
 * sweeps, shape[2] the gradient sweep's slice target (each problem's points
 * are cut into slices until its (target block, slice) units number about
 * shape[2] per SM; 8 gives the single-problem path's slicing).  Default
 * {8, 8, 8}; each value in [1, 64].  The slicing changes only the order in
 * which each target's FP64 partial sums are added. */
sdot_status sdot_batch_set_shape(sdot_batch *batch, const int *shape);
sdot_status sdot_batch_get_shape(const sdot_batch *batch, int *shape);
/* Device milliseconds (CUDA events) of the batch's last batched evaluation. */
double sdot_batch_last_eval_ms(const sdot_batch *batch);
/* The batch's own autotuner: times `reps` batched evaluations at psi (host,
 * concatenated; gradient sweep in FP32 when fp32 != 0) for each candidate
 * of one shape entry at a time (slice target 4/8/16/32, then CTAs per SM
 * 4/8/12/16 for the value and the gradient sweep), keeps the fastest, and
 * leaves the batch on the result, written to shape_out[3].  The result is
 * remembered for the life of the process per bucket (dimension, log2 of the
 * batch's pairs, log2 of its problem count, fp32); a batch of a tuned
 * bucket takes the remembered shape without timing (*cached = 1). */
sdot_status sdot_batch_autotune(sdot_batch *batch, const double *psi, int fp32, int reps, int *shape_out,
                                int *cached);

/* ---- solve service (no reference counterpart: the reference runs one
 * SotSolver::solve per process at a time; this admits many) ----
 * n_slots worker threads each own one context (own CUDA stream); requests
 * wait in a FIFO queue and start when a slot is free and their device-memory
 * estimate fits in memory_budget (0 = no budget) beside the running ones, so
 * requests that arrive while others run are admitted as slots and memory
 * free up and their kernels overlap on the device.  Solves are deterministic:
 * a request gives the same potential alone or in any mix.  Inputs are copied
 * at submit. */
typedef enum { SDOT_METHOD_AUTO = 0, SDOT_METHOD_NEWTON = 1, SDOT_METHOD_LBFGS = 2 } sdot_method;
typedef struct {
    int dim;
    int64_t n_q;
    const double *x, *jxw, *density;     /* as sdot_set_source */
    int64_t n_cells;                     /* 0: points only (untruncated requests) */
    const int64_t *cell_offsets;
    const double *cell_centers;
    int64_t n_t;
    const double *y, *nu;
    const double *psi0;                  /* warm start (NULL: zeros) */
    sdot_solver_params params;
    int method;                          /* sdot_method; AUTO = Newton when untruncated, rho*JxW >= 0, n_t <= 46340 */
    int precision;                       /* sdot_precision of the evaluation sweeps (L-BFGS; Newton uses FP64) */
    int hessian_method;                  /* sdot_hessian_method for Newton */
    double epsilon_scaling_factor;       /* levels eps f^(s-1), ..., eps, warm started */
    int epsilon_scaling_steps;           /* 0 or 1: no scaling */
    double intermediate_tolerance;       /* tolerance of the levels before the last (<= 0: params.tolerance) */
} sdot_request;
typedef struct {
    sdot_status status;
    int converged;
    int method;                          /* method used */
    unsigned iterations;                 /* over all epsilon levels */
    int64_t n_evaluations;
    double last_value, last_check_value;
    double queue_ms, run_ms, latency_ms; /* host wall clock: submit -> start, start -> done, submit -> done */
    int slot;
    char message[160];                   /* error text when status != SDOT_OK */
} sdot_result;
typedef struct {
    int64_t completed, failed, queued;
    int running, peak_running;
    size_t in_use_bytes, peak_bytes;     /* admitted device-memory estimates */
    double p50_ms, p99_ms, mean_ms;      /* latency of completed requests */
} sdot_server_stats;
sdot_status sdot_server_create(sdot_server **server, int device, int n_slots, size_t memory_budget);
/* Finishes the queued and running requests, then stops the workers. */
void sdot_server_destroy(sdot_server *server);
const char *sdot_server_last_error(const sdot_server *server);
/* SDOT_EBUDGET when the request alone exceeds the budget. */
sdot_status sdot_server_submit(sdot_server *server, const sdot_request *request, int64_t *ticket);
/* 1 done, 0 pending, -1 unknown ticket. */
int sdot_server_poll(sdot_server *server, int64_t ticket);
/* Waits (timeout_s <= 0: forever; SDOT_ETIMEOUT on expiry) and returns the
 * request's status; psi receives n_t doubles.  The ticket is then released. */
sdot_status sdot_server_wait(sdot_server *server, int64_t ticket, double timeout_s, double *psi, sdot_result *result);
sdot_status sdot_server_get_stats(sdot_server *server, sdot_server_stats *stats);
sdot_status sdot_server_reset_stats(sdot_server *server);

/* Getters replacing SotSolver::get_last_functional_value, get_last_iteration_count,
 * get_convergence_status, get_last_distance_threshold, get_C_global
 * (SotSolver.h:233-255) and the setter set_distance_threshold (:261). */
double sdot_get_last_functional_value(const sdot_ctx *ctx);
unsigned sdot_get_last_iteration_count(const sdot_ctx *ctx);
int sdot_get_convergence_status(const sdot_ctx *ctx);
double sdot_get_last_distance_threshold(const sdot_ctx *ctx);
double sdot_get_C_global(const sdot_ctx *ctx);
sdot_status sdot_set_distance_threshold(sdot_ctx *ctx, double threshold);

/* Replaces SotSolver::compute_covering_radius (SotSolver.h:275; SotSolver.cc:431-473). */
sdot_status sdot_compute_covering_radius(sdot_ctx *ctx, double *radius);
/* Replaces SotSolver::compute_geometric_radius_bound (SotSolver.h:296-299;
 * SotSolver.cc:509-551). */
sdot_status sdot_compute_geometric_radius_bound(sdot_ctx *ctx, const double *psi, double epsilon,
                                                double tolerance, double *radius);
/* Replaces SotSolver::set_distance_function (SotSolver.h:305; SotSolver.cc:22-41):
 * "euclidean" (the default, the accelerated path) or "spherical" (the
 * great-circle distance acos(clamp(a.b / (|a| |b|))) of Distance.h, for
 * points on a sphere about the origin).  With "spherical", evaluations and
 * sdot_solve use it for the candidate predicate and the cost, through FP64
 * sweeps over every (point, target) pair and the pointwise threshold only;
 * the Hessian, Newton, the softmax refinement, the conditioned densities, the
 * euclidean barycenters and the no-allocation evaluation return SDOT_EINVAL.
 * Anything else is SDOT_EINVAL. */
sdot_status sdot_set_distance_function(sdot_ctx *ctx, const char *name);

/* Replaces SotSolver::evaluate_weighted_barycenters with the spherical
 * distance (SotSolver.cc:612-650, compute_weighted_barycenters_non_euclidean
 * :662-767): evaluates at psi (caller order), then iterates at most
 * max_iterations times: G_j = sum_q w_q pi_qj grad_b d^2(b_j, x_q)
 * (spherical_distance_gradient, Distance.h) over the candidates; stop when
 * ||G||_2 < tolerance, else b_j <- exp_{b_j}(-G_j) (spherical_distance_exp_map).
 * bary (n_targets * dim, caller order) holds the starting points and receives
 * the result; *iterations the gradient evaluations run, *grad_norm the last
 * ||G||_2.  At a zero distance d/sin(d) is taken as 1 and a zero step leaves
 * the point in place (the reference divides 0 by 0 there).  Needs
 * sdot_set_distance_function(ctx, "spherical"). */
sdot_status sdot_weighted_barycenters_spherical(sdot_ctx *ctx, const double *psi, double *bary,
                                                unsigned max_iterations, double tolerance, unsigned *iterations,
                                                double *grad_norm);

/* ---- multi-GPU sharding (no reference counterpart as one call: it replaces
 * the MPI sums of SotSolver.cc:316-319 by letting the caller all-reduce). ----
 * Evaluation of this context's source shard only: writes n_targets + 3
 * doubles to out_dev (device memory): [0, n) the source part of the gradient
 * sum_q w_q pi_qj (caller ordering, nu NOT subtracted), [n] the source part
 * of the functional (linear term NOT subtracted), [n+1] C_global part,
 * [n+2] candidate pairs.  Summing out_dev over the shards and then
 * subtracting nu_j and sum_j psi_j nu_j gives sdot_evaluate's results. */
sdot_status sdot_evaluate_partial_device(sdot_ctx *ctx, const double *psi_dev, double *out_dev,
                                         sdot_eval_info *info);
/* Sets the state the integral/geometric thresholds read (the reference's
 * members global_functional and C_global, SotSolver.cc:316-331) after a
 * sharded evaluation has been reduced. */
sdot_status sdot_set_state(sdot_ctx *ctx, double global_functional, double C_global);

/* ---- measurement ---- */
/* The CUDA stream (cudaStream_t) every kernel of this context is launched on. */
void *sdot_get_stream(const sdot_ctx *ctx);
/* Enable CUDA-event timing of each evaluation phase (0 = off). */
sdot_status sdot_set_profiling(sdot_ctx *ctx, int enable);
/* Cumulative device milliseconds and launch counts per phase since the last
 * reset: phases 0 threshold, 1 target prep, 2 value sweep, 3 gradient sweep,
 * 4 finalize.  ms and launches hold n entries; reset != 0 zeroes them after
 * reading. */
sdot_status sdot_get_kernel_times(sdot_ctx *ctx, double *ms, int64_t *launches, int n, int reset);
/* Microbenchmarks of the pipes the kernels are bound by, on device `device`:
 * out[0] FP64 FMA TFLOP/s, out[1] FP32 FMA TFLOP/s, out[2] MUFU ex2.approx.f32
 * Gop/s, out[3] SM clock (MHz) reported by the device. */
sdot_status sdot_measure_peaks(int device, double *out);

/* ---- failure injection for tests (no counterpart in the reference) ----
 * sdot_debug_fail_allocation(k): the library's device allocations (the
 * buffers of every context and batch of the process) count down from k, and
 * the allocation that finds the count at 0 fails as if the device were out
 * of memory, without calling cudaMalloc: the call making it returns
 * SDOT_ENOMEM.  k < 0 turns the injection off.  Returns the previous count
 * (-1: off).  sdot_debug_allocation_count: allocations made or failed so far
 * in the process.  After a failed set-up call the context holds no source
 * (or no target) and evaluations return SDOT_ESTATE until it is set again. */
int64_t sdot_debug_fail_allocation(int64_t after);
int64_t sdot_debug_allocation_count(void);

/* ---- no-allocation evaluation (no counterpart in the reference) ----
 * Same results as sdot_evaluate_device (same kernels, same launch shapes) for
 * an untruncated problem (pointwise threshold with tau <= 0), but the call
 * allocates no device memory: its scratch is one file-scope static device
 * array of SDOT_NOALLOC_SCRATCH_BYTES (8 MiB) per device, not the context's
 * evaluation buffers.  For callers that must not allocate while they run:
 * a loop whose device memory is already fully committed to a pool or an
 * admission budget, where a cudaMalloc could fail mid-request, or a
 * latency-bound loop that cannot absorb cudaMalloc / cudaFree and the
 * synchronisation they imply.  The set-up calls (sdot_create,
 * sdot_set_source, sdot_set_target) still allocate, as before.
 *   - Requests whose scratch exceeds the limit (about 8 * n_q * (1 + 2 * vs)
 *     + (10 + slices) * 8 * n_targets bytes, where vs <= 16 is the number of
 *     target slices of the value sweep when n_q < 75,776 and 0 otherwise, and
 *     slices <= 64 that of the gradient sweep) are rejected with SDOT_EINVAL and
 *     a message giving the need and the limit; truncated problems likewise.
 *   - Nothing in the scratch has to start at zero: every word a call reads is
 *     written earlier by the same call on the context's stream.
 *   - The scratch is shared by all contexts of the process on a device: calls
 *     whose executions overlap (other threads, streams or contexts on the same
 *     device) race and corrupt each other's results.  Serialise them.
 *   - The first call on a device does one-time set-up: it looks up the
 *     scratch address with cudaGetSymbolAddress, which may load the module,
 *     so make that first call before any stream capture.  The address is
 *     kept for the life of the process; a cudaDeviceReset invalidates it, so
 *     make no no-alloc call after one.
 *   - Every call ends by synchronising the context's stream and reading the
 *     scalars (J, C_global, norms) back to the host.
 * psi_dev, grad_dev: device arrays of n_targets doubles in caller order;
 * *value receives J.  Updates the same state as sdot_evaluate_device. */
#define SDOT_NOALLOC_SCRATCH_BYTES (8u << 20)
sdot_status sdot_evaluate_device_noalloc(sdot_ctx *ctx, const double *psi_dev, double *grad_dev,
                                         double *value);

#ifdef __cplusplus
}
#endif
#endif /* SDOT_H */
