/*
 * sdot_oracle.c -- FP64 CPU restatement of SemiDiscreteOT's entropic
 * semi-discrete dual path.  TEST INFRASTRUCTURE ONLY (see sdot_oracle.h):
 * the product library never links this file.  Parity status: unpinned (the
 * reference cannot be built here and ships no golden vectors).
 *
 * Every routine cites the reference lines it restates.  Arithmetic order is
 * kept as in the reference where it is visible in the source:
 *   d2 = pow(|x - y|, 2) with |a-b| = sqrt(sum_i (a_i-b_i)^2)
 *     (include/SemiDiscreteOT/solvers/Distance.h:23-27, SotSolver.cc:830,838);
 *   exponent = (psi_j - 0.5*d2) * (1/eps)                     (SotSolver.cc:831);
 *   two passes (max, then shifted exp)                        (SotSolver.cc:826-842);
 *   value += rho*eps*(m + log S)*JxW; C += rho*JxW/S;
 *   grad[j] += (rho*JxW/S) * nu_j e^{t_j-m} if the term is > 0 (SotSolver.cc:267-296);
 *   J -= sum psi_j nu_j; g_j -= nu_j                           (SotSolver.cc:322-327).
 * Compile with -ffp-contract=off: the reference is built for baseline x86-64
 * (no FMA contraction), and the candidate predicate must be bit-exact.
 */
#include "sdot_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static int orc_threads(int n_threads)
{
#ifdef _OPENMP
    return n_threads > 0 ? n_threads : omp_get_max_threads();
#else
    (void)n_threads;
    return 1;
#endif
}

/* ------------------------------------------------------------------ */
/* Quadrature and structured Q1 source (utils.h:818-850, FE_Q(1),       */
/* MappingQ1, QGauss; SemiDiscreteOT.cc:422-449 normalize_density).     */
/* ------------------------------------------------------------------ */

void orc_gauss_legendre(int n, double *x, double *w)
{
    /* Newton iteration on P_n over [-1,1], then mapped to [0,1] (the way
     * deal.II's QGauss<1> builds its rule). */
    const int m = (n + 1) / 2;
    for (int i = 0; i < m; ++i) {
        double z = cos(M_PI * (i + 0.75) / (n + 0.5));
        double pp = 0.0;
        for (int it = 0; it < 100; ++it) {
            double p1 = 1.0, p2 = 0.0;
            for (int j = 1; j <= n; ++j) {
                double p3 = p2;
                p2 = p1;
                p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
            }
            pp = n * (z * p1 - p2) / (z * z - 1.0);
            double z1 = z;
            z = z1 - p1 / pp;
            if (fabs(z - z1) < 1e-16) {
                /* one more evaluation at the converged node for the weight */
                p1 = 1.0; p2 = 0.0;
                for (int j = 1; j <= n; ++j) {
                    double p3 = p2;
                    p2 = p1;
                    p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
                }
                pp = n * (z * p1 - p2) / (z * z - 1.0);
                break;
            }
        }
        const double wi = 2.0 / ((1.0 - z * z) * pp * pp);
        /* node -z (left) and +z (right) on [-1,1] -> [0,1] */
        x[i] = 0.5 - 0.5 * z;
        x[n - 1 - i] = 0.5 + 0.5 * z;
        w[i] = 0.5 * wi;
        w[n - 1 - i] = 0.5 * wi;
    }
    if (n % 2 == 1) x[n / 2] = 0.5;
}

/* Q1 shape function of vertex v (bit d of v selects xi_d or 1-xi_d). */
static double q1_shape(int dim, int v, const double *xi)
{
    double r = 1.0;
    for (int d = 0; d < dim; ++d)
        r *= ((v >> d) & 1) ? xi[d] : (1.0 - xi[d]);
    return r;
}

int64_t orc_structured_source(int dim, int n, double lo, double hi, int order,
                              const double *nodal, int normalize,
                              double *xq, double *jxw, double *rho,
                              int64_t *cell_offsets, double *cell_centers)
{
    double gx[16], gw[16];
    if (order < 1 || order > 16 || (dim != 2 && dim != 3) || n < 1) return -1;
    orc_gauss_legendre(order, gx, gw);
    const double h = (hi - lo) / n;
    const int nv = 1 << dim;
    const int64_t ncell = (dim == 2) ? (int64_t)n * n : (int64_t)n * n * n;
    const int qpc = (dim == 2) ? order * order : order * order * order;
    const int64_t nn = n + 1;
    double detJ = 1.0;
    for (int d = 0; d < dim; ++d) detJ *= h;

    double scale = 1.0;
    for (int pass = 0; pass < 2; ++pass) {
        double l1 = 0.0;
        for (int64_t c = 0; c < ncell; ++c) {
            int64_t ci[3];
            ci[0] = c % n;
            ci[1] = (c / n) % n;
            ci[2] = (dim == 3) ? c / ((int64_t)n * n) : 0;
            double X[8][3];
            double vnod[8];
            for (int v = 0; v < nv; ++v) {
                int64_t vi[3] = {0, 0, 0};
                for (int d = 0; d < dim; ++d) {
                    vi[d] = ci[d] + ((v >> d) & 1);
                    X[v][d] = lo + (double)vi[d] * h;
                }
                int64_t lin = vi[0] + nn * (vi[1] + nn * vi[2]);
                vnod[v] = nodal ? nodal[lin] : 1.0;
                vnod[v] = vnod[v] / scale;
            }
            if (pass == 1) {
                cell_offsets[c] = c * qpc;
                double ctr[3] = {0.0, 0.0, 0.0};
                for (int v = 0; v < nv; ++v)
                    for (int d = 0; d < dim; ++d) ctr[d] += X[v][d];
                for (int d = 0; d < dim; ++d) cell_centers[c * dim + d] = ctr[d] / nv;
            }
            for (int iq = 0; iq < qpc; ++iq) {
                int qi[3] = {iq % order, (iq / order) % order, iq / (order * order)};
                double xi[3] = {gx[qi[0]], gx[qi[1]], (dim == 3) ? gx[qi[2]] : 0.0};
                double wq = 1.0;
                for (int d = 0; d < dim; ++d) wq *= gw[qi[d]];
                double val = 0.0;
                double xx[3] = {0.0, 0.0, 0.0};
                for (int v = 0; v < nv; ++v) {
                    const double phi = q1_shape(dim, v, xi);
                    for (int d = 0; d < dim; ++d) xx[d] += phi * X[v][d];
                    if (vnod[v] != 0.0) val += vnod[v] * phi;
                }
                const double JxW = detJ * wq;
                if (pass == 0) {
                    l1 += fabs(val) * JxW;
                } else {
                    const int64_t q = c * qpc + iq;
                    for (int d = 0; d < dim; ++d) xq[q * dim + d] = xx[d];
                    jxw[q] = JxW;
                    rho[q] = val;
                }
            }
        }
        if (pass == 0) scale = (normalize && l1 > 0.0) ? l1 : 1.0;
    }
    cell_offsets[ncell] = ncell * qpc;
    return ncell * qpc;
}

/* ------------------------------------------------------------------ */
/* Distances, thresholds, candidates                                    */
/* ------------------------------------------------------------------ */

/* (a-b).norm(): sqrt(((a0-b0)^2 + (a1-b1)^2) + (a2-b2)^2)  (Distance.h:23-27) */
static inline double orc_dist(int dim, const double *a, const double *b)
{
    double s = 0.0;
    for (int d = 0; d < dim; ++d) {
        const double t = a[d] - b[d];
        s += t * t;
    }
    return sqrt(s);
}

/* spherical_distance (Distance.h): acos of the normalised dot product,
 * clamped to [-1, 1]; norms as Point::norm (sqrt of the ordered sum). */
static inline double orc_sph_dist(int dim, const double *a, const double *b)
{
    double dot = 0.0, na = 0.0, nb = 0.0;
    for (int d = 0; d < dim; ++d) dot += a[d] * b[d];
    for (int d = 0; d < dim; ++d) na += a[d] * a[d];
    for (int d = 0; d < dim; ++d) nb += b[d] * b[d];
    double c = dot / (sqrt(na) * sqrt(nb));
    c = c > 1.0 ? 1.0 : (c < -1.0 ? -1.0 : c);
    return acos(c);
}

/* The problem's distance_function (SotSolver.cc:22-41). */
static inline double orc_pdist(const orc_problem *p, const double *a, const double *b)
{
    return p->distance == ORC_DIST_SPHERICAL ? orc_sph_dist(p->dim, a, b) : orc_dist(p->dim, a, b);
}

static double vmax(const double *v, int64_t n)
{
    double m = v[0];
    for (int64_t i = 1; i < n; ++i) if (v[i] > m) m = v[i];
    return m;
}

static double vmin(const double *v, int64_t n)
{
    double m = v[0];
    for (int64_t i = 1; i < n; ++i) if (v[i] < m) m = v[i];
    return m;
}

/* SotSolver::compute_covering_radius (SotSolver.cc:431-473): max over cells
 * of the distance from the cell centre to its nearest target. */
double orc_covering_radius(const orc_problem *p)
{
    double best = 0.0;
    for (int64_t c = 0; c < p->n_cells; ++c) {
        const double *cc = p->cell_centers + c * p->dim;
        double dmin = DBL_MAX;
        for (int64_t j = 0; j < p->n_targets; ++j) {
            const double d = orc_dist(p->dim, p->y + j * p->dim, cc);
            if (d < dmin) dmin = d;
        }
        if (dmin > best) best = dmin;
    }
    return best;
}

/* SotSolver::compute_integral_radius_bound (SotSolver.cc:475-507). */
double orc_integral_radius_bound(const orc_problem *p, const double *psi, double eps,
                                 double tol, double C_value, double J_value)
{
    const double max_potential = vmax(psi, p->n_targets);
    double abs_J = fabs(J_value);
    if (abs_J < 1e-10) abs_J = 1e-10;
    const double num = eps * C_value;
    const double den = tol * abs_J;
    const double arg = num / den;
    const double r2 = 2.0 * max_potential + 2.0 * eps * log(arg);
    return sqrt(r2 > 0.0 ? r2 : 0.0);
}

/* SotSolver::compute_geometric_radius_bound (SotSolver.cc:509-551). */
double orc_geometric_radius_bound(const orc_problem *p, const orc_state *s,
                                  const double *psi, double eps, double tol)
{
    const double r0 = s->covering_radius > 0.0 ? s->covering_radius : orc_covering_radius(p);
    const double range = vmax(psi, p->n_targets) - vmin(psi, p->n_targets);
    const double min_density = s->min_target_density > 0.0 ? s->min_target_density
                                                            : vmin(p->nu, p->n_targets);
    double fv = fabs(s->global_functional);
    if (fv < 1e-10) fv = 1e-10;
    const double log_term = log(eps / (min_density * tol * fv));
    double r2 = r0 * r0 + 2.0 * range + 2.0 * eps * log_term;
    if (r2 < r0 * r0) r2 = r0 * r0;
    return sqrt(r2);
}

/* SotSolver::compute_distance_threshold (SotSolver.cc:379-429). */
double orc_distance_threshold(const orc_problem *p, const orc_params *prm,
                              const orc_state *s, const double *psi)
{
    if (psi == NULL) return DBL_MAX;
    if (prm->threshold_type == ORC_THRESH_INTEGRAL) {
        double r = orc_integral_radius_bound(p, psi, prm->epsilon, prm->tau,
                                             s->C_global, s->global_functional);
        return r > s->covering_radius ? r : s->covering_radius;
    }
    if (prm->threshold_type == ORC_THRESH_GEOMETRIC)
        return orc_geometric_radius_bound(p, s, psi, prm->epsilon, prm->tau);
    const double max_potential = vmax(psi, p->n_targets);
    const double nu_min = s->min_target_density > 0.0 ? s->min_target_density
                                                       : vmin(p->nu, p->n_targets);
    if (nu_min <= 0 || prm->tau <= 0) return DBL_MAX;
    const double r2 = -2.0 * prm->epsilon * log(prm->tau / nu_min) + 2.0 * max_potential;
    return sqrt(r2 > 0.0 ? r2 : 0.0);
}

/* find_nearest_target_points (SotSolver.cc:553-570): the R-tree query
 * carries only a satisfies() predicate, i.e. it is a scan of all targets. */
int64_t orc_candidates(const orc_problem *p, const double *c, double r, int64_t *out)
{
    int64_t k = 0;
    for (int64_t j = 0; j < p->n_targets; ++j)
        if (orc_pdist(p, p->y + j * p->dim, c) <= r) out[k++] = j;
    return k;
}

/* ------------------------------------------------------------------ */
/* local_assemble (SotSolver.cc:769-869) + value/grad lambda (:267-296) */
/* ------------------------------------------------------------------ */

typedef struct {
    int64_t *cand;
    double *ty, *tnu, *tpsi, *et;
} cell_scratch;

/* Contribution of one cell.  grad_dense != NULL: dense N-vector (reference
 * CopyData layout); otherwise the sparse contribution is written to
 * cand/gsp (parallel arrays, length returned through *ncand). */
static double cell_assemble(const orc_problem *p, const orc_params *prm, double r,
                            const double *psi, int64_t c, cell_scratch *sc,
                            double *grad_dense, double *gsp, int64_t *ncand,
                            double *C_cell, int64_t *n_pairs, int64_t *n_skip)
{
    const int dim = p->dim;
    const double eps = prm->epsilon;
    const double epsilon_inv = 1.0 / eps;
    double value = 0.0, Csum = 0.0;
    const int64_t nc = orc_candidates(p, p->cell_centers + c * dim, r, sc->cand);
    *ncand = nc;
    if (gsp) for (int64_t i = 0; i < nc; ++i) gsp[i] = 0.0;
    if (nc == 0) { *C_cell = 0.0; return 0.0; }
    for (int64_t i = 0; i < nc; ++i) {
        const int64_t j = sc->cand[i];
        for (int d = 0; d < dim; ++d) sc->ty[i * dim + d] = p->y[j * dim + d];
        sc->tnu[i] = p->nu[j];
        sc->tpsi[i] = psi[j];
    }
    for (int64_t q = p->cell_offsets[c]; q < p->cell_offsets[c + 1]; ++q) {
        const double *x = p->xq + q * dim;
        const double density_value = p->rho[q];
        const double JxW = p->jxw[q];
        double total = 0.0;
        double maxe = -DBL_MAX;
        *n_pairs += nc;
        if (prm->use_log_sum_exp) {
            for (int64_t i = 0; i < nc; ++i) {
                const double d2 = pow(orc_pdist(p, x, sc->ty + i * dim), 2);
                const double e = (sc->tpsi[i] - 0.5 * d2) * epsilon_inv;
                maxe = maxe > e ? maxe : e;
            }
            for (int64_t i = 0; i < nc; ++i) {
                const double d2 = pow(orc_pdist(p, x, sc->ty + i * dim), 2);
                const double se = exp((sc->tpsi[i] - 0.5 * d2) * epsilon_inv - maxe);
                sc->et[i] = sc->tnu[i] * se;
                total += sc->et[i];
            }
        } else {
            for (int64_t i = 0; i < nc; ++i) {
                const double d2 = pow(orc_pdist(p, x, sc->ty + i * dim), 2);
                sc->et[i] = sc->tnu[i] * exp((sc->tpsi[i] - 0.5 * d2) * epsilon_inv);
                total += sc->et[i];
            }
        }
        if (total <= 0.0) { (*n_skip)++; continue; }
        if (prm->use_log_sum_exp)
            value += density_value * eps * (maxe + log(total)) * JxW;
        else
            value += density_value * eps * log(total) * JxW;
        const double scale = density_value * JxW / total;
        Csum += scale;
        for (int64_t i = 0; i < nc; ++i) {
            if (sc->et[i] > 0.0) {
                if (grad_dense) grad_dense[sc->cand[i]] += scale * sc->et[i];
                else gsp[i] += scale * sc->et[i];
            }
        }
    }
    *C_cell = Csum;
    return value;
}

static void scratch_alloc(cell_scratch *sc, int64_t n, int dim)
{
    sc->cand = (int64_t *)malloc(sizeof(int64_t) * (n + 1));
    sc->ty = (double *)malloc(sizeof(double) * (n + 1) * dim);
    sc->tnu = (double *)malloc(sizeof(double) * (n + 1));
    sc->tpsi = (double *)malloc(sizeof(double) * (n + 1));
    sc->et = (double *)malloc(sizeof(double) * (n + 1));
}

static void scratch_free(cell_scratch *sc)
{
    free(sc->cand); free(sc->ty); free(sc->tnu); free(sc->tpsi); free(sc->et);
}

double orc_evaluate_cells(const orc_problem *p, const orc_params *prm, double r,
                          const double *psi, int64_t c0, int64_t c1,
                          double *grad, double *C_out, int64_t *n_pairs_out,
                          int faithful_overheads, int n_threads)
{
    const int64_t N = p->n_targets;
    const int dim = p->dim;
    const int nt = orc_threads(n_threads);
    double J = 0.0, C = 0.0;
    int64_t pairs = 0, skipped = 0;
    if (c1 > p->n_cells) c1 = p->n_cells;
    if (c0 < 0) c0 = 0;

    if (faithful_overheads) {
        /* WorkStream::run (SotSolver.cc:299-313): per-cell CopyData with
         * gradient_values[N] and barycenters_values[dim*N] zeroed for every
         * cell (:792-795), and a copier that adds the dense N-vector into the
         * process gradient serially, in cell order (:307-311). */
#pragma omp parallel num_threads(nt) reduction(+ : pairs, skipped)
        {
            cell_scratch sc;
            scratch_alloc(&sc, N, dim);
            double *gcell = (double *)malloc(sizeof(double) * N);
            double *bary = (double *)malloc(sizeof(double) * N * dim);
            int64_t ncand = 0;
#pragma omp for ordered schedule(static, 1)
            for (int64_t c = c0; c < c1; ++c) {
                memset(bary, 0, sizeof(double) * N * dim);
                memset(gcell, 0, sizeof(double) * N);
                double Cc = 0.0;
                const double v = cell_assemble(p, prm, r, psi, c, &sc, gcell, NULL, &ncand,
                                               &Cc, &pairs, &skipped);
#pragma omp ordered
                {
                    J += v;
                    C += Cc;
                    if (grad)
                        for (int64_t j = 0; j < N; ++j) grad[j] += gcell[j];
                }
            }
            free(gcell); free(bary);
            scratch_free(&sc);
        }
    } else {
        /* Same arithmetic per cell; contributions kept sparse and merged per
         * thread (static partition -> deterministic for a fixed thread count). */
        double *Jt = (double *)calloc(nt, sizeof(double));
        double *Ct = (double *)calloc(nt, sizeof(double));
        double *Gt = grad ? (double *)calloc((size_t)nt * N, sizeof(double)) : NULL;
#pragma omp parallel num_threads(nt) reduction(+ : pairs, skipped)
        {
#ifdef _OPENMP
            const int t = omp_get_thread_num();
#else
            const int t = 0;
#endif
            cell_scratch sc;
            scratch_alloc(&sc, N, dim);
            double *gsp = (double *)malloc(sizeof(double) * (N + 1));
            double *Gl = Gt ? Gt + (size_t)t * N : NULL;
            int64_t ncand = 0;
#pragma omp for schedule(static)
            for (int64_t c = c0; c < c1; ++c) {
                double Cc = 0.0;
                const double v = cell_assemble(p, prm, r, psi, c, &sc, NULL, gsp, &ncand,
                                               &Cc, &pairs, &skipped);
                Jt[t] += v;
                Ct[t] += Cc;
                if (Gl)
                    for (int64_t i = 0; i < ncand; ++i) Gl[sc.cand[i]] += gsp[i];
            }
            free(gsp);
            scratch_free(&sc);
        }
        for (int t = 0; t < nt; ++t) {
            J += Jt[t];
            C += Ct[t];
            if (Gt) for (int64_t j = 0; j < N; ++j) grad[j] += Gt[(size_t)t * N + j];
        }
        free(Jt); free(Ct); free(Gt);
    }
    if (C_out) *C_out = C;
    if (n_pairs_out) *n_pairs_out = pairs;
    (void)skipped;
    return J;
}

double orc_evaluate(const orc_problem *p, const orc_params *prm, orc_state *s,
                    const double *psi, double *grad, orc_eval_stats *stats,
                    int faithful_overheads, int n_threads)
{
    const int64_t N = p->n_targets;
    /* compute_distance_threshold() runs before the accumulators are reset,
     * so the integral/geometric variants see the previous J and C. */
    const double r = orc_distance_threshold(p, prm, s, psi);
    s->current_distance_threshold = r;
    for (int64_t j = 0; j < N; ++j) grad[j] = 0.0;
    double C = 0.0;
    int64_t pairs = 0;
    double J = orc_evaluate_cells(p, prm, r, psi, 0, p->n_cells, grad, &C, &pairs,
                                  faithful_overheads, n_threads);
    /* linear term, rank 0 (SotSolver.cc:322-327) */
    for (int64_t j = 0; j < N; ++j) {
        J -= psi[j] * p->nu[j];
        grad[j] -= p->nu[j];
    }
    s->global_functional = J;
    s->C_global = C;
    if (stats) {
        stats->threshold = r;
        stats->n_pairs = pairs;
        stats->n_active_cells = 0;
        stats->n_skipped_q = 0;
    }
    return J;
}

/* ------------------------------------------------------------------ */
/* deal.II SolverBFGS + LineMinimization (third-party; restated from the */
/* published algorithm, readable copy in core/wasserstein_solver_bfgs.h   */
/* :302-492 and core/line_minimization.h:332-749).                        */
/* ------------------------------------------------------------------ */

typedef struct {
    const orc_problem *p;
    const orc_params *prm;
    orc_state *s;
    int n_threads;
    int faithful;
    int64_t n_evals;
    double *x, *x0, *g, *pdir;
    int64_t N;
} bfgs_ctx;

static double dot(const double *a, const double *b, int64_t n)
{
    double s = 0.0;
    for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

static double compute_fg(bfgs_ctx *c)
{
    c->n_evals++;
    return orc_evaluate(c->p, c->prm, c->s, c->x, c->g, NULL, c->faithful, c->n_threads);
}

/* line_func of the default line search: x = x0 + a p; f = compute(x, g) */
static void line_func(bfgs_ctx *c, double a, double *f, double *gp)
{
    for (int64_t i = 0; i < c->N; ++i) c->x[i] = c->x0[i] + a * c->pdir[i];
    *f = compute_fg(c);
    *gp = dot(c->g, c->pdir, c->N);
}

static int cubic_fit(double x1, double f1, double g1, double x2, double f2, double g2, double *res)
{
    const double beta1 = g1 + g2 - 3. * (f1 - f2) / (x1 - x2);
    const double s = beta1 * beta1 - g1 * g2;
    if (s < 0) return 0;
    const double beta2 = sqrt(s);
    const double denom = x1 < x2 ? g2 - g1 + 2. * beta2 : g1 - g2 + 2. * beta2;
    if (denom == 0.) return 0;
    *res = x1 < x2 ? x2 - (x2 - x1) * (g2 + beta2 - beta1) / denom
                   : x1 - (x1 - x2) * (g1 + beta2 - beta1) / denom;
    return 1;
}

static int quadratic_fit(double x1, double f1, double g1, double x2, double f2, double *res)
{
    const double denom = (2. * g1 * x2 - 2. * g1 * x1 - 2. * f2 + 2. * f1);
    if (denom == 0) return 0;
    *res = (g1 * (x2 * x2 - x1 * x1) + 2. * (f1 - f2) * x1) / denom;
    return 1;
}

/* poly_fit (line_minimization.h:423-455): cubic, then quadratic, then bisection. */
static double poly_fit(double x1, double f1, double g1, double x2, double f2, double g2,
                       double b0, double b1)
{
    double r;
    if (cubic_fit(x1, f1, g1, x2, f2, g2, &r) && r >= b0 && r <= b1) return r;
    if (quadratic_fit(x1, f1, g1, x2, f2, &r) && r >= b0 && r <= b1) return r;
    return (b0 + b1) * 0.5;
}

/* LineMinimization::line_search (line_minimization.h:498-749).
 * Returns 0 on success (alpha in *alpha), 1 if no bracket was found within
 * max_evals (AssertThrow), 2 if the sectioning phase ran out of evaluations. */
static int line_search(bfgs_ctx *c, double f0, double g0, double a1, double eta,
                       double mu, double a_max, unsigned max_evals, double *alpha)
{
    const double tau1 = 9., tau2 = 0.1, tau3 = 0.5;
    const double g0_abs = fabs(g0);
    const double f_min = f0 + a_max * mu * g0;
#define W1(a, f) ((f) <= f0 + (a) * mu * g0)
#define W2(g) (fabs(g) <= eta * g0_abs)
    double a_lo = NAN, f_lo = NAN, g_lo = NAN, a_hi = NAN, f_hi = NAN, g_hi = NAN;
    double ai, fi, gi;
    unsigned i = 0;
    {
        double f_prev = f0, g_prev = g0, a_prev = 0;
        ai = a1;
        while (i < max_evals) {
            line_func(c, ai, &fi, &gi);
            ++i;
            if (fi <= f_min || ai == a_max) { *alpha = ai; return 0; }
            if (!W1(ai, fi) || (fi >= f_prev && i > 1)) {
                a_lo = a_prev; f_lo = f_prev; g_lo = g_prev;
                a_hi = ai; f_hi = fi; g_hi = gi;
                break;
            }
            if (W2(gi)) { *alpha = ai; return 0; }
            if (gi >= 0) {
                a_lo = ai; f_lo = fi; g_lo = gi;
                a_hi = a_prev; f_hi = f_prev; g_hi = g_prev;
                break;
            }
            const double ub = ai + tau1 * (ai - a_prev);
            a_prev = ai; f_prev = fi; g_prev = gi;
            ai = a_max < ub ? a_max : ub;
        }
    }
    if (!(i < max_evals)) return 1;
    while (i < max_evals) {
        const double lo_safe = a_lo + tau2 * (a_hi - a_lo);
        const double hi_safe = a_hi - tau3 * (a_hi - a_lo);
        const double b0 = hi_safe < lo_safe ? hi_safe : lo_safe;
        const double b1 = hi_safe < lo_safe ? lo_safe : hi_safe;
        ai = poly_fit(a_lo, f_lo, g_lo, a_hi, f_hi, g_hi, b0, b1);
        line_func(c, ai, &fi, &gi);
        ++i;
        if (!W1(ai, fi) || fi >= f_lo) {
            a_hi = ai; f_hi = fi; g_hi = gi;
        } else {
            if (W2(gi)) { *alpha = ai; return 0; }
            if (gi * (a_hi - a_lo) >= 0) { a_hi = a_lo; f_hi = f_lo; g_hi = g_lo; }
            a_lo = ai; f_lo = fi; g_lo = gi;
        }
    }
#undef W1
#undef W2
    *alpha = NAN;
    return 2;
}

/* VerboseSolverControl::check (SotSolver.h:382-446) + SolverControl::check. */
static int control_check(const orc_problem *p, const orc_params *prm, unsigned step,
                         const double *g, double *value_out)
{
    const int64_t N = p->n_targets;
    double v = 0.0, tol = prm->tolerance;
    if (prm->control_type == ORC_CONTROL_COMPONENTWISE) {
        double m = -INFINITY;
        for (int64_t j = 0; j < N; ++j) {
            const double sr = fabs(g[j]) - p->nu[j] * prm->tolerance;
            m = m > sr ? m : sr;
        }
        v = m;
        tol = DBL_MIN;
    } else if (prm->control_type == ORC_CONTROL_LINF) {
        for (int64_t j = 0; j < N; ++j) v = v > fabs(g[j]) ? v : fabs(g[j]);
    } else {
        for (int64_t j = 0; j < N; ++j) v += fabs(g[j]);
    }
    *value_out = v;
    if (v <= tol) return 1;                                    /* success */
    if (step >= prm->max_iterations || isnan(v)) return -1;    /* failure */
    return 0;                                                  /* iterate */
}

int orc_solve(const orc_problem *p, const orc_params *prm, orc_state *s,
              double *psi, orc_solve_info *info, double *trace, int64_t trace_cap,
              int n_threads)
{
    return orc_solve_ex(p, prm, s, psi, info, trace, trace_cap, n_threads, 0);
}

int orc_solve_ex(const orc_problem *p, const orc_params *prm, orc_state *s,
                 double *psi, orc_solve_info *info, double *trace, int64_t trace_cap,
                 int n_threads, int faithful_overheads)
{
    const int64_t N = p->n_targets;
    const int M = 5; /* SolverBFGS::AdditionalData::max_history_size */
    bfgs_ctx c;
    c.p = p; c.prm = prm; c.s = s; c.n_threads = n_threads; c.n_evals = 0; c.N = N;
    c.faithful = faithful_overheads;
    c.x = psi;
    c.x0 = (double *)calloc(N, sizeof(double));
    c.g = (double *)calloc(N, sizeof(double));
    c.pdir = (double *)calloc(N, sizeof(double));
    double *yk = (double *)calloc(N, sizeof(double));
    double *sk = (double *)calloc(N, sizeof(double));
    double *S = (double *)calloc((size_t)M * N, sizeof(double));
    double *Y = (double *)calloc((size_t)M * N, sizeof(double));
    double rho[5], c1[5];
    int head = 0, m = 0; /* ring buffer; newest at index (head-1) */

    /* SotSolver::solve prologue (SotSolver.cc:131-133). */
    s->covering_radius = orc_covering_radius(p) * 1.1;
    s->min_target_density = vmin(p->nu, N);

    int status = 0, conv;
    unsigned k = 0;
    double f, check_value = 0.0;
    int first_step = 1;
    double f_prev = 0.;

    f = compute_fg(&c);
    conv = control_check(p, prm, k, c.g, &check_value);
    int64_t ntr = 0;
    if (trace && ntr < trace_cap) { trace[3 * ntr] = f; trace[3 * ntr + 1] = check_value; trace[3 * ntr + 2] = 0.0; ntr++; }
    while (conv == 0) {
        /* two-loop recursion, history newest first */
        for (int64_t i = 0; i < N; ++i) c.pdir[i] = c.g[i];
        for (int i = 0; i < m; ++i) {
            const int slot = (head - 1 - i + 2 * M) % M;
            c1[i] = rho[slot] * dot(S + (size_t)slot * N, c.pdir, N);
            const double a = -c1[i];
            const double *yv = Y + (size_t)slot * N;
            for (int64_t t = 0; t < N; ++t) c.pdir[t] += a * yv[t];
        }
        for (int i = m - 1; i >= 0; --i) {
            const int slot = (head - 1 - i + 2 * M) % M;
            const double c2 = rho[slot] * dot(Y + (size_t)slot * N, c.pdir, N);
            const double a = c1[i] - c2;
            const double *sv = S + (size_t)slot * N;
            for (int64_t t = 0; t < N; ++t) c.pdir[t] += a * sv[t];
        }
        for (int64_t i = 0; i < N; ++i) c.pdir[i] *= -1.;

        for (int64_t i = 0; i < N; ++i) { sk[i] = c.x[i]; yk[i] = c.g[i]; }

        /* default line search lambda (wasserstein_solver_bfgs.h:316-389) */
        double alpha;
        {
            const double f0 = f;
            const double g0 = dot(c.g, c.pdir, N);
            for (int64_t i = 0; i < N; ++i) c.x0[i] = c.x[i];
            double df = f_prev - f;
            const double dmin = 100. * DBL_EPSILON;
            df = df > dmin ? df : dmin;
            double a1 = 1.;
            if (!first_step) {
                const double t = -1.01 * 2. * df / g0;
                a1 = t < 1. ? t : 1.;
            }
            f_prev = f;
            const int rc = line_search(&c, f0, g0, a1, 0.9, 0.001, DBL_MAX, 20, &alpha);
            f = c.s->global_functional;
            if (rc == 1) { status = 3; break; }
            if (rc == 2) {
                if (prm->line_search_variant != ORC_LS_VENDORED) { status = 2; break; }
                /* vendored NaN fallback (wasserstein_solver_bfgs.h:371-386) */
                alpha = 0.5;
                for (int it = 0; it < 5; ++it) {
                    for (int64_t i = 0; i < N; ++i) c.x[i] = c.x0[i] + alpha * c.pdir[i];
                    f = compute_fg(&c);
                    if (f < f_prev) break;
                    alpha *= 0.5;
                }
            } else if (first_step) {
                first_step = 0;
            }
        }
        for (int64_t i = 0; i < N; ++i) { sk[i] = c.x[i] - sk[i]; yk[i] = c.g[i] - yk[i]; }
        ++k;
        conv = control_check(p, prm, k, c.g, &check_value);
        if (trace && ntr < trace_cap) { trace[3 * ntr] = f; trace[3 * ntr + 1] = check_value; trace[3 * ntr + 2] = alpha; ntr++; }
        if (conv != 0) break;
        const double curvature = dot(sk, yk, N);
        if (curvature > 0.) {
            memcpy(S + (size_t)head * N, sk, sizeof(double) * N);
            memcpy(Y + (size_t)head * N, yk, sizeof(double) * N);
            rho[head] = 1. / curvature;
            head = (head + 1) % M;
            if (m < M) ++m;
        }
    }
    if (info) {
        info->iterations = k;
        info->converged = (conv == 1);
        info->status = status ? status : (conv == 1 ? 0 : 1);
        info->n_evaluations = c.n_evals;
        info->last_value = f;
        info->last_check_value = check_value;
    }
    free(c.x0); free(c.g); free(c.pdir); free(yk); free(sk); free(S); free(Y);
    return info ? info->status : 0;
}

/* ------------------------------------------------------------------ */
/* Hessian (declared at SotSolver.h:343-344; no definition exists)       */
/* ------------------------------------------------------------------ */

void orc_hessian(const orc_problem *p, const orc_params *prm, double r,
                 const double *psi, double *H, int n_threads)
{
    const int64_t N = p->n_targets;
    const int dim = p->dim;
    const double eps = prm->epsilon;
    const double einv = 1.0 / eps;
    const int nt = orc_threads(n_threads);
    memset(H, 0, sizeof(double) * (size_t)N * N);
    /* Row-partitioned accumulation: each thread owns rows j in its range and
     * walks all cells, so no two threads write the same entry. */
#pragma omp parallel num_threads(nt)
    {
        int64_t *cand = (int64_t *)malloc(sizeof(int64_t) * (N + 1));
        double *pi = (double *)malloc(sizeof(double) * (N + 1));
#ifdef _OPENMP
        const int t = omp_get_thread_num(), T = omp_get_num_threads();
#else
        const int t = 0, T = 1;
#endif
        const int64_t r0 = N * t / T, r1 = N * (t + 1) / T;
        for (int64_t c = 0; c < p->n_cells; ++c) {
            const int64_t nc = orc_candidates(p, p->cell_centers + c * dim, r, cand);
            if (nc == 0) continue;
            for (int64_t q = p->cell_offsets[c]; q < p->cell_offsets[c + 1]; ++q) {
                const double *x = p->xq + q * dim;
                double maxe = -DBL_MAX, total = 0.0;
                for (int64_t i = 0; i < nc; ++i) {
                    const int64_t j = cand[i];
                    const double d2 = pow(orc_dist(dim, x, p->y + j * dim), 2);
                    const double e = (psi[j] - 0.5 * d2) * einv;
                    maxe = maxe > e ? maxe : e;
                }
                for (int64_t i = 0; i < nc; ++i) {
                    const int64_t j = cand[i];
                    const double d2 = pow(orc_dist(dim, x, p->y + j * dim), 2);
                    pi[i] = p->nu[j] * exp((psi[j] - 0.5 * d2) * einv - maxe);
                    total += pi[i];
                }
                if (total <= 0.0) continue;
                const double w = p->rho[q] * p->jxw[q];
                for (int64_t i = 0; i < nc; ++i) pi[i] /= total;
                for (int64_t a = 0; a < nc; ++a) {
                    const int64_t ja = cand[a];
                    if (ja < r0 || ja >= r1) continue;
                    double *row = H + (size_t)ja * N;
                    const double wa = w * pi[a] * einv;
                    row[ja] += wa;
                    for (int64_t b = 0; b < nc; ++b) row[cand[b]] -= wa * pi[b];
                }
            }
        }
        free(cand); free(pi);
    }
}

/* ------------------------------------------------------------------ */
/* SoftmaxRefinement::local_assemble + compute_refinement                */
/* (src/solvers/SoftmaxRefinement.cc:61-280)                              */
/* ------------------------------------------------------------------ */

void orc_softmax_refinement(const orc_problem *cp, const double *psi_coarse,
                            double eps, double r, int use_lse,
                            int64_t n_fine, const double *y_fine,
                            const int64_t *child_offsets, const int64_t *child_indices,
                            double *psi_fine, int n_threads)
{
    const int dim = cp->dim;
    const int64_t Nc = cp->n_targets;
    const double lambda_inv = 1.0 / eps;
    const double threshold_sq = r * r;
    const int nt = orc_threads(n_threads);
    double *acc = (double *)calloc((size_t)nt * n_fine, sizeof(double));
#pragma omp parallel num_threads(nt)
    {
#ifdef _OPENMP
        const int t = omp_get_thread_num();
#else
        const int t = 0;
#endif
        double *pl = acc + (size_t)t * n_fine;
        int64_t *cand = (int64_t *)malloc(sizeof(int64_t) * (Nc + 1));
        double *et = (double *)malloc(sizeof(double) * (Nc + 1));
        int64_t *fine = (int64_t *)malloc(sizeof(int64_t) * (n_fine + 1));
#pragma omp for schedule(static)
        for (int64_t c = 0; c < cp->n_cells; ++c) {
            const int64_t nc = orc_candidates(cp, cp->cell_centers + c * dim, r, cand);
            if (nc == 0) continue;
            int64_t nf = 0;
            for (int64_t i = 0; i < nc; ++i)
                for (int64_t k = child_offsets[cand[i]]; k < child_offsets[cand[i] + 1]; ++k)
                    fine[nf++] = child_indices[k];
            if (nf == 0) continue;
            for (int64_t q = cp->cell_offsets[c]; q < cp->cell_offsets[c + 1]; ++q) {
                const double *x = cp->xq + q * dim;
                double total = 0.0, maxe = -DBL_MAX;
                for (int64_t i = 0; i < nc; ++i) et[i] = 0.0;
                if (use_lse) {
                    for (int64_t i = 0; i < nc; ++i) {
                        const int64_t j = cand[i];
                        const double d2 = pow(orc_dist(dim, x, cp->y + j * dim), 2);
                        if (d2 <= threshold_sq) {
                            const double e = (psi_coarse[j] - 0.5 * d2) * lambda_inv;
                            maxe = maxe > e ? maxe : e;
                        }
                    }
                    for (int64_t i = 0; i < nc; ++i) {
                        const int64_t j = cand[i];
                        const double d2 = pow(orc_dist(dim, x, cp->y + j * dim), 2);
                        if (d2 <= threshold_sq) {
                            et[i] = cp->nu[j] * exp((psi_coarse[j] - 0.5 * d2) * lambda_inv - maxe);
                            total += et[i];
                        }
                    }
                } else {
                    for (int64_t i = 0; i < nc; ++i) {
                        const int64_t j = cand[i];
                        const double d2 = pow(orc_dist(dim, x, cp->y + j * dim), 2);
                        if (d2 <= threshold_sq) {
                            et[i] = cp->nu[j] * exp((psi_coarse[j] - 0.5 * d2) * lambda_inv);
                            total += et[i];
                        }
                    }
                }
                if (total <= 0.0) continue;
                double scale = cp->rho[q] * cp->jxw[q] / total;
                if (use_lse) scale *= exp(-maxe);
                for (int64_t i = 0; i < nf; ++i) {
                    const int64_t f = fine[i];
                    const double d2 = pow(orc_dist(dim, x, y_fine + f * dim), 2);
                    if (d2 <= threshold_sq) pl[f] += scale * exp((-0.5 * d2) * lambda_inv);
                }
            }
        }
        free(cand); free(et); free(fine);
    }
    for (int64_t f = 0; f < n_fine; ++f) {
        double v = 0.0;
        for (int t = 0; t < nt; ++t) v += acc[(size_t)t * n_fine + f];
        psi_fine[f] = v > 0.0 ? -eps * log(v) : v;
    }
    free(acc);
}

/* ------------------------------------------------------------------ */
/* compute_weighted_barycenters_euclidean (SotSolver.cc:871-971) through */
/* local_assemble (:770-869): per point the candidate terms of cell(q),   */
/* scale = rho JxW / total, barycenter += scale * term * x where term > 0 */
/* ------------------------------------------------------------------ */

void orc_weighted_barycenters(const orc_problem *p, const orc_params *prm, double r,
                              const double *psi, double *bary, int n_threads)
{
    const int dim = p->dim;
    const int64_t N = p->n_targets;
    const double epsilon_inv = 1.0 / prm->epsilon;
    const int nt = orc_threads(n_threads);
    double *acc = (double *)calloc((size_t)nt * N * dim, sizeof(double));
#pragma omp parallel num_threads(nt)
    {
#ifdef _OPENMP
        const int t = omp_get_thread_num();
#else
        const int t = 0;
#endif
        double *pl = acc + (size_t)t * N * dim;
        int64_t *cand = (int64_t *)malloc(sizeof(int64_t) * (N + 1));
        double *et = (double *)malloc(sizeof(double) * (N + 1));
#pragma omp for schedule(static)
        for (int64_t c = 0; c < p->n_cells; ++c) {
            const int64_t nc = orc_candidates(p, p->cell_centers + c * dim, r, cand);
            if (nc == 0) continue;
            for (int64_t q = p->cell_offsets[c]; q < p->cell_offsets[c + 1]; ++q) {
                const double *x = p->xq + q * dim;
                double total = 0.0, maxe = -DBL_MAX;
                if (prm->use_log_sum_exp) {
                    for (int64_t i = 0; i < nc; ++i) {
                        const int64_t j = cand[i];
                        const double d2 = pow(orc_dist(dim, x, p->y + j * dim), 2);
                        const double e = (psi[j] - 0.5 * d2) * epsilon_inv;
                        maxe = maxe > e ? maxe : e;
                    }
                    for (int64_t i = 0; i < nc; ++i) {
                        const int64_t j = cand[i];
                        const double d2 = pow(orc_dist(dim, x, p->y + j * dim), 2);
                        et[i] = p->nu[j] * exp((psi[j] - 0.5 * d2) * epsilon_inv - maxe);
                        total += et[i];
                    }
                } else {
                    for (int64_t i = 0; i < nc; ++i) {
                        const int64_t j = cand[i];
                        const double d2 = pow(orc_dist(dim, x, p->y + j * dim), 2);
                        et[i] = p->nu[j] * exp((psi[j] - 0.5 * d2) * epsilon_inv);
                        total += et[i];
                    }
                }
                if (total <= 0.0) continue;
                const double scale = p->rho[q] * p->jxw[q] / total;
                for (int64_t i = 0; i < nc; ++i)
                    if (et[i] > 0.0)
                        for (int d = 0; d < dim; ++d) pl[cand[i] * dim + d] += scale * et[i] * x[d];
            }
        }
        free(cand); free(et);
    }
    for (int64_t k = 0; k < N * dim; ++k) {
        double v = 0.0;
        for (int t = 0; t < nt; ++t) v += acc[(size_t)t * N * dim + k];
        bary[k] = v / p->nu[k / dim];
    }
    free(acc);
}

/* spherical_distance_gradient(a, b) (Distance.h): -2 (d / sin d) (b - (a.b) a),
 * d the spherical distance, a.b the raw dot product; d / sin d -> 1 at d = 0. */
static void orc_sph_grad(int dim, const double *a, const double *b, double *g)
{
    const double dist = orc_sph_dist(dim, a, b);
    double dot = 0.0;
    for (int d = 0; d < dim; ++d) dot += a[d] * b[d];
    const double f = dist > 0.0 ? dist / sin(dist) : 1.0;
    for (int d = 0; d < dim; ++d) g[d] = -2 * f * (b[d] - dot * a[d]);
}

int orc_spherical_barycenters(const orc_problem *p, const orc_params *prm, double r, const double *psi,
                              double *bary, unsigned max_iterations, double tolerance, double *grad_norm)
{
    const int dim = p->dim;
    const int64_t N = p->n_targets;
    const double epsilon_inv = 1.0 / prm->epsilon;
    double *G = (double *)calloc((size_t)N * dim, sizeof(double));
    int64_t *cand = (int64_t *)malloc(sizeof(int64_t) * (N + 1));
    double *et = (double *)malloc(sizeof(double) * (N + 1));
    unsigned it = 0;
    double l2 = 0.0;
    for (it = 0; it < max_iterations; ++it) {
        for (int64_t k = 0; k < N * dim; ++k) G[k] = 0.0;
        for (int64_t c = 0; c < p->n_cells; ++c) {
            const int64_t nc = orc_candidates(p, p->cell_centers + c * dim, r, cand);
            if (nc == 0) continue;
            for (int64_t q = p->cell_offsets[c]; q < p->cell_offsets[c + 1]; ++q) {
                const double *x = p->xq + q * dim;
                double total = 0.0, maxe = -DBL_MAX;
                if (prm->use_log_sum_exp) {
                    for (int64_t i = 0; i < nc; ++i) {
                        const int64_t j = cand[i];
                        const double d2 = pow(orc_pdist(p, x, p->y + j * dim), 2);
                        const double e = (psi[j] - 0.5 * d2) * epsilon_inv;
                        maxe = maxe > e ? maxe : e;
                    }
                    for (int64_t i = 0; i < nc; ++i) {
                        const int64_t j = cand[i];
                        const double d2 = pow(orc_pdist(p, x, p->y + j * dim), 2);
                        et[i] = p->nu[j] * exp((psi[j] - 0.5 * d2) * epsilon_inv - maxe);
                        total += et[i];
                    }
                } else {
                    for (int64_t i = 0; i < nc; ++i) {
                        const int64_t j = cand[i];
                        const double d2 = pow(orc_pdist(p, x, p->y + j * dim), 2);
                        et[i] = p->nu[j] * exp((psi[j] - 0.5 * d2) * epsilon_inv);
                        total += et[i];
                    }
                }
                if (total <= 0.0) continue;
                const double scale = p->rho[q] * p->jxw[q] / total;
                for (int64_t i = 0; i < nc; ++i) {
                    if (!(et[i] > 0.0)) continue;
                    const int64_t j = cand[i];
                    double v[3];
                    orc_sph_grad(dim, bary + j * dim, x, v);
                    for (int d = 0; d < dim; ++d) G[j * dim + d] += scale * et[i] * v[d];
                }
            }
        }
        double s2 = 0.0;
        for (int64_t k = 0; k < N * dim; ++k) s2 += G[k] * G[k];
        l2 = sqrt(s2);
        if (l2 < tolerance) { ++it; break; }
        /* exp map at b_j of the step -G_j: cos|v| b + sin|v| v / |v| */
        for (int64_t j = 0; j < N; ++j) {
            double nv = 0.0;
            for (int d = 0; d < dim; ++d) nv += G[j * dim + d] * G[j * dim + d];
            nv = sqrt(nv);
            if (!(nv > 0.0)) continue;
            const double cs = cos(nv), sn = sin(nv);
            for (int d = 0; d < dim; ++d) bary[j * dim + d] = cs * bary[j * dim + d] + sn * (-G[j * dim + d] / nv);
        }
    }
    free(G); free(cand); free(et);
    if (grad_norm) *grad_norm = l2;
    return (int)it;
}

/* SotSolver::get_potential_conditioned_density (SotSolver.cc:973-1046) at
 * n_points support points with the source density there. */
void orc_conditioned_densities(const orc_problem *p, const double *psi, double eps, double r,
                               int64_t n_points, const double *points, const double *density,
                               int64_t n_idx, const int64_t *idx, double *out)
{
    const int dim = p->dim;
    const int64_t N = p->n_targets;
    const double epsilon_inv = 1.0 / eps;
    int64_t *cand = (int64_t *)malloc(sizeof(int64_t) * (N + 1));
    double *ex = (double *)malloc(sizeof(double) * (N + 1));
    char *in = (char *)malloc((size_t)N + 1);
    for (int64_t k = 0; k < n_idx * n_points; ++k) out[k] = 0.0;
    for (int64_t pt = 0; pt < n_points; ++pt) {
        const double *x = points + pt * dim;
        const int64_t nc = orc_candidates(p, x, r, cand);
        for (int64_t j = 0; j < N; ++j) { ex[j] = 0.0; in[j] = 0; }
        double total = 0.0, maxe = -DBL_MAX;
        for (int64_t i = 0; i < nc; ++i) {
            const int64_t j = cand[i];
            const double e = (psi[j] - 0.5 * pow(orc_dist(dim, x, p->y + j * dim), 2)) * epsilon_inv;
            maxe = maxe > e ? maxe : e;
        }
        for (int64_t i = 0; i < nc; ++i) {
            const int64_t j = cand[i];
            ex[j] = exp((psi[j] - 0.5 * pow(orc_dist(dim, x, p->y + j * dim), 2)) * epsilon_inv - maxe);
            in[j] = 1;
            total += p->nu[j] * ex[j];
        }
        if (total > 0.0)
            for (int64_t k = 0; k < n_idx; ++k)
                if (in[idx[k]]) out[k * n_points + pt] = density[pt] * (ex[idx[k]] / total);
    }
    free(cand); free(ex); free(in);
}

/* EpsilonScalingHandler (EpsilonScalingHandler.cc:6-42). */
int orc_epsilon_sequence(double eps, double factor, unsigned steps, double *out)
{
    if (factor <= 1.0) factor = 2.0;
    if (steps == 0) steps = 1;
    for (unsigned i = 0; i < steps; ++i) out[i] = eps * pow(factor, (double)(steps - 1 - i));
    return (int)steps;
}
