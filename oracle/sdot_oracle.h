/*
 * sdot_oracle.h -- FP64 CPU restatement of SemiDiscreteOT's entropic
 * semi-discrete dual evaluation, used ONLY as test infrastructure.
 *
 * This oracle is the checker for the CUDA path: only tests/, the smoke test
 * in __graft_entry__.py and the cpu_baseline / reference legs of bench.py
 * may load it.  The product library never links or calls it.
 *
 * Parity status: UNPINNED.  The reference (deal.II 9.5 + Boost + MPI) cannot
 * be built or imported in this environment and it ships no golden vectors,
 * known-answer tests or fixtures for this path.  Every function below cites
 * the reference file:line it restates; correctness of the restatement is
 * established by first-principles known-answer tests (tests/test_oracle_*.py)
 * rather than by reference outputs.
 *
 * Third-party arithmetic restated here (absent from the reference tree):
 *   - deal.II 9.5.0 SolverBFGS + LineMinimization::line_search/poly_fit
 *     (called at src/solvers/SotSolver.cc:190-198); the readable copy in the
 *     reference is include/SemiDiscreteOT/core/wasserstein_solver_bfgs.h:302-492
 *     and include/SemiDiscreteOT/core/line_minimization.h:332-749.
 *   - deal.II SolverControl::check (success if value <= tol, failure if
 *     step >= max_steps or value is NaN).
 *   - deal.II QGauss<1> Gauss-Legendre nodes (Newton iteration on Legendre
 *     polynomials), FE_Q(1)/MappingQ1 on axis-aligned hexes/quads.
 */
#ifndef SDOT_ORACLE_H
#define SDOT_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Flattened source quadrature + discrete target measure.
 * Layout follows SemiDiscreteOT::save_discrete_measures
 * (src/core/SemiDiscreteOT.cc:2489-2558): quadrature points, JxW, density at
 * the quadrature points, all cell-major; plus the cell centres used by the
 * truncation query (SotSolver.cc:801). */
typedef struct {
    int dim;                       /* spacedim: 2 or 3 */
    int64_t n_q;                   /* quadrature points */
    int64_t n_cells;
    int64_t n_targets;
    const double *xq;              /* n_q * dim, row-major */
    const double *jxw;             /* n_q */
    const double *rho;             /* n_q, density value at x_q */
    const int64_t *cell_offsets;   /* n_cells + 1, q-range of each cell */
    const double *cell_centers;    /* n_cells * dim */
    const double *y;               /* n_targets * dim */
    const double *nu;              /* n_targets */
    int distance;                  /* ORC_DIST_*: the candidate predicate and cost of
                                      orc_evaluate / orc_solve / orc_candidates */
} orc_problem;

/* SotSolver::set_distance_function (SotSolver.cc:22-41): "euclidean" or
 * "spherical" (Distance.h). */
enum { ORC_DIST_EUCLIDEAN = 0, ORC_DIST_SPHERICAL = 1 };

enum { ORC_THRESH_POINTWISE = 0, ORC_THRESH_INTEGRAL = 1, ORC_THRESH_GEOMETRIC = 2 };
enum { ORC_CONTROL_L1 = 0, ORC_CONTROL_COMPONENTWISE = 1, ORC_CONTROL_LINF = 2 };
enum { ORC_LS_UPSTREAM = 0, ORC_LS_VENDORED = 1 };

/* SotParameterManager::SolverParameters (ParameterManager.h:56-72) subset. */
typedef struct {
    double epsilon;
    double tau;
    int use_log_sum_exp;       /* use_log_sum_exp_trick */
    int threshold_type;        /* distance_threshold_type */
    int control_type;          /* solver_control_type (+ linf extension) */
    double tolerance;
    unsigned max_iterations;
    int line_search_variant;   /* deal.II upstream (default) or the vendored copy */
} orc_params;

/* Members of SotSolver that persist across evaluations (SotSolver.h:503-512). */
typedef struct {
    double global_functional;
    double C_global;
    double covering_radius;
    double min_target_density;
    double current_distance_threshold;
} orc_state;

typedef struct {
    double threshold;          /* distance threshold used */
    int64_t n_pairs;           /* sum over q of |candidates(cell(q))| */
    int64_t n_active_cells;    /* cells with a non-empty candidate set */
    int64_t n_skipped_q;       /* q points skipped because S_q <= 0 */
} orc_eval_stats;

typedef struct {
    unsigned iterations;       /* last_step of the solver control */
    int converged;             /* last_check == success */
    int status;                /* 0 ok, 1 no convergence, 2 line search failure, 3 bracket failure */
    int64_t n_evaluations;
    double last_value;
    double last_check_value;
} orc_solve_info;

/* Gauss-Legendre rule with n points on [0,1]. */
void orc_gauss_legendre(int n, double *x, double *w);

/* Structured [lo,hi]^dim Q1 mesh with n cells per axis and QGauss(order).
 * nodal: (n+1)^dim vertex densities (lexicographic, x fastest) or NULL for 1.
 * normalize: divide the nodal density by sum_q |rho_q| JxW_q first
 * (SemiDiscreteOT::normalize_density, src/core/SemiDiscreteOT.cc:422-449).
 * Returns the number of quadrature points written. */
int64_t orc_structured_source(int dim, int n, double lo, double hi, int order,
                              const double *nodal, int normalize,
                              double *xq, double *jxw, double *rho,
                              int64_t *cell_offsets, double *cell_centers);

/* Distance thresholds (SotSolver.cc:379-551). */
double orc_covering_radius(const orc_problem *p);
double orc_integral_radius_bound(const orc_problem *p, const double *psi, double eps,
                                 double tol, double C_value, double J_value);
double orc_geometric_radius_bound(const orc_problem *p, const orc_state *s,
                                  const double *psi, double eps, double tol);
double orc_distance_threshold(const orc_problem *p, const orc_params *prm,
                              const orc_state *s, const double *psi);

/* Candidate query (SotSolver.cc:553-570): writes indices j with
 * ||y_j - c|| <= r in increasing j; returns the count. */
int64_t orc_candidates(const orc_problem *p, const double *c, double r, int64_t *out);

/* SotSolver::evaluate_functional (SotSolver.cc:217-377).  Updates the state
 * (threshold, global_functional, C_global) like the reference members.
 * faithful_overheads: reproduce WorkStream's per-cell O(N) CopyData zeroing
 * and the serialised per-cell dense merge (timing baseline).
 * n_threads <= 0: all cores. */
double orc_evaluate(const orc_problem *p, const orc_params *prm, orc_state *s,
                    const double *psi, double *grad, orc_eval_stats *stats,
                    int faithful_overheads, int n_threads);

/* Same per-cell work restricted to cells [c0, c1) with a fixed threshold r;
 * returns the partial functional (no linear term), accumulates the partial
 * gradient into grad (may be NULL) and the partial C into *C_out.  Used for
 * bounded CPU-baseline samples. */
double orc_evaluate_cells(const orc_problem *p, const orc_params *prm, double r,
                          const double *psi, int64_t c0, int64_t c1,
                          double *grad, double *C_out, int64_t *n_pairs,
                          int faithful_overheads, int n_threads);

/* SotSolver::solve (SotSolver.cc:105-215) with deal.II SolverBFGS. */
int orc_solve(const orc_problem *p, const orc_params *prm, orc_state *s,
              double *psi, orc_solve_info *info, double *trace, int64_t trace_cap,
              int n_threads);
/* The same solve; faithful_overheads != 0 evaluates with the reference's
 * per-cell O(N) CopyData zeroing and serialised merge (as orc_evaluate), for
 * timing the reference-faithful full solve. */
int orc_solve_ex(const orc_problem *p, const orc_params *prm, orc_state *s,
                 double *psi, orc_solve_info *info, double *trace, int64_t trace_cap,
                 int n_threads, int faithful_overheads);

/* SotSolver::evaluate_weighted_barycenters with the spherical distance
 * (SotSolver.cc:612-650) through compute_weighted_barycenters_non_euclidean
 * (:662-767): Riemannian gradient steps on the barycenters, bary (n_targets *
 * dim, in/out) the starting points.  Per iteration the accumulator
 * G_j = sum_q w_q pi_qj grad_b d^2(b_j, x_q) (spherical_distance_gradient,
 * Distance.h) over the candidates of each cell is formed; if ||G||_2 <
 * tolerance the iteration stops, else b_j = exp_map(b_j, -G_j).  Returns the
 * iterations run (gradient evaluations) and ||G||_2 of the last one.  At a
 * zero distance the factor dist/sin(dist) is taken as its limit 1, and a zero
 * step leaves the point where it is (the reference divides 0 by 0 there). */
int orc_spherical_barycenters(const orc_problem *p, const orc_params *prm, double r, const double *psi,
                              double *bary, unsigned max_iterations, double tolerance, double *grad_norm);

/* Dense Hessian of the dual functional (declared at SotSolver.h:343-344,
 * never defined in the reference):
 *   H = (1/eps) sum_q w_q (diag(pi_q) - pi_q pi_q^T),
 * with the same candidate truncation as the evaluation at threshold r. */
void orc_hessian(const orc_problem *p, const orc_params *prm, double r,
                 const double *psi, double *H, int n_threads);

/* SoftmaxRefinement::compute_refinement (src/solvers/SoftmaxRefinement.cc:61-280)
 * for one level: fine potentials from coarse ones.
 * child_offsets/child_indices: CSR children of each coarse point. */
void orc_softmax_refinement(const orc_problem *coarse, const double *psi_coarse,
                            double eps, double r, int use_lse,
                            int64_t n_fine, const double *y_fine,
                            const int64_t *child_offsets, const int64_t *child_indices,
                            double *psi_fine, int n_threads);

/* SotSolver::compute_weighted_barycenters_euclidean (SotSolver.cc:871-971):
 * bary (n_targets x dim) = sum_q rho JxW pi_qj x_q / nu_j at threshold r. */
void orc_weighted_barycenters(const orc_problem *p, const orc_params *prm, double r,
                              const double *psi, double *bary, int n_threads);

/* SotSolver::get_potential_conditioned_density (SotSolver.cc:973-1046):
 * out[k * n_points + pt] for the requested targets idx[k]. */
void orc_conditioned_densities(const orc_problem *p, const double *psi, double eps, double r,
                               int64_t n_points, const double *points, const double *density,
                               int64_t n_idx, const int64_t *idx, double *out);

/* EpsilonScalingHandler (src/solvers/EpsilonScalingHandler.cc:30-90). */
int orc_epsilon_sequence(double eps, double factor, unsigned steps, double *out);

#ifdef __cplusplus
}
#endif
#endif
