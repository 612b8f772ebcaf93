// sdot/SotSolver.hpp -- header-only C++ facade over libsdot_cuda (sdot.h).
//
// Mirrors the interface of SemiDiscreteOT's SotSolver<dim, spacedim>
// (include/SemiDiscreteOT/solvers/SotSolver.h:54-525) with standard types in
// place of deal.II ones: points are std::array<double, spacedim>, vectors are
// std::vector<double>, the source is the flattened quadrature data of
// SemiDiscreteOT::save_discrete_measures.  Error statuses raise
// std::runtime_error like the reference's exceptions; non-convergence of
// solve() does not (the reference swallows NoConvergence, SotSolver.cc:207-211)
// and is reported by get_convergence_status().
#ifndef SDOT_SOTSOLVER_HPP
#define SDOT_SOTSOLVER_HPP

#include <array>
#include <stdexcept>
#include <string>
#include <vector>

#include "../sdot.h"

namespace sdot {

// SotParameterManager::SolverParameters (ParameterManager.h:56-72), every
// field with the reference's default, plus the line-search variant.  Fields
// the solve itself does not read (solver_type, quadrature_order, nb_points,
// n_threads, the epsilon-scaling settings) are kept for the callers that
// read them, as in the reference.
struct SolverParameters {
    unsigned max_iterations = 1000;
    double tolerance = 1;
    std::string solver_control_type = "l1norm";  // l1norm | componentwise | linf
    double epsilon = 1e-3;
    double tau = 1e-8;
    std::string distance_threshold_type = "pointwise";  // pointwise | integral | geometric
    bool verbose_output = true;
    std::string solver_type = "BFGS";
    unsigned quadrature_order = 3;
    unsigned nb_points = 1000;
    unsigned n_threads = 0;
    bool use_epsilon_scaling = false;
    double epsilon_scaling_factor = 2.0;
    unsigned epsilon_scaling_steps = 5;
    bool use_log_sum_exp_trick = false;
    std::string line_search = "upstream";  // upstream | vendored

    sdot_solver_params c() const {
        sdot_solver_params p;
        sdot_default_params(&p);
        p.max_iterations = max_iterations;
        p.tolerance = tolerance;
        p.control_type = solver_control_type == "componentwise" ? SDOT_CONTROL_COMPONENTWISE
                         : solver_control_type == "linf"       ? SDOT_CONTROL_LINF
                                                                : SDOT_CONTROL_L1NORM;
        if (solver_control_type != "l1norm" && solver_control_type != "componentwise" && solver_control_type != "linf")
            throw std::invalid_argument("Unknown solver_control_type: " + solver_control_type);
        p.epsilon = epsilon;
        p.tau = tau;
        p.threshold_type = distance_threshold_type == "integral"    ? SDOT_THRESH_INTEGRAL
                           : distance_threshold_type == "geometric" ? SDOT_THRESH_GEOMETRIC
                                                                    : SDOT_THRESH_POINTWISE;
        p.use_log_sum_exp = use_log_sum_exp_trick ? 1 : 0;
        p.line_search = line_search == "vendored" ? SDOT_LS_VENDORED : SDOT_LS_UPSTREAM;
        return p;
    }
};

template <int dim, int spacedim = dim>
class SotSolver {
public:
    using Point = std::array<double, spacedim>;

    explicit SotSolver(int device = 0, sdot_precision precision = SDOT_PREC_HYBRID) {
        sdot_options o{};
        o.device = device;
        o.precision = precision;
        check(sdot_create(&ctx_, &o), "SotSolver");
    }
    ~SotSolver() { sdot_destroy(ctx_); }
    SotSolver(const SotSolver &) = delete;
    SotSolver &operator=(const SotSolver &) = delete;

    // setup_source on flattened quadrature data: x (n_q points), JxW, density
    // at the points, per-cell offsets (n_cells + 1) and cell centres.
    void setup_source(const std::vector<Point> &x, const std::vector<double> &jxw, const std::vector<double> &density,
                      const std::vector<int64_t> &cell_offsets, const std::vector<Point> &cell_centers) {
        if (x.size() != jxw.size() || x.size() != density.size() || cell_offsets.size() != cell_centers.size() + 1)
            throw std::runtime_error("setup_source: inconsistent sizes");
        check(sdot_set_source(ctx_, spacedim, (int64_t)x.size(), x.data()->data(), jxw.data(), density.data(),
                              (int64_t)cell_centers.size(), cell_offsets.data(), cell_centers.data()->data()),
              "setup_source");
    }
    void setup_target(const std::vector<Point> &points, const std::vector<double> &density) {
        if (points.size() != density.size()) throw std::runtime_error("Dimension mismatch");
        check(sdot_set_target(ctx_, (int64_t)points.size(), points.data()->data(), density.data()), "setup_target");
        n_ = points.size();
    }
    void configure(const SolverParameters &params) {
        current_params = params;
        const sdot_solver_params p = params.c();
        check(sdot_configure(ctx_, &p), "configure");
    }
    void solve(std::vector<double> &potential, const SolverParameters &params) {
        current_params = params;
        if (potential.size() != n_) potential.assign(n_, 0.0);
        const sdot_solver_params p = params.c();
        sdot_solve_info info{};
        check(sdot_solve(ctx_, potential.data(), &p, &info), "solve");
    }
    double evaluate_functional(const std::vector<double> &potential, std::vector<double> &gradient_out) {
        if (potential.size() != n_) throw std::runtime_error("evaluate_functional: potential size");
        gradient_out.resize(n_);
        double v = 0;
        check(sdot_evaluate(ctx_, potential.data(), gradient_out.data(), &v, nullptr), "evaluate_functional");
        return v;
    }
    // Dense row-major n x n Hessian (declared-only in the reference).
    void compute_hessian(const std::vector<double> &potential, std::vector<double> &hessian_out) {
        hessian_out.resize(n_ * n_);
        check(sdot_hessian(ctx_, potential.data(), hessian_out.data()), "compute_hessian");
    }
    // Newton with the tensor-core (or FP64) Hessian; same parameters and controls as solve.
    void solve_newton(std::vector<double> &potential, const SolverParameters &params,
                      int hessian_method = SDOT_HESS_AUTO) {
        current_params = params;
        if (potential.size() != n_) potential.assign(n_, 0.0);
        const sdot_solver_params p = params.c();
        sdot_newton_info info{};
        check(sdot_solve_newton(ctx_, potential.data(), &p, hessian_method, &info), "solve_newton");
    }
    // Lagged Hessians in solve_newton: keep the Hessian after a full step that reduced |g|_2 by `contraction`
    // (default 0.1; 0 recomputes it every step).
    void set_newton_hessian_reuse(double contraction) {
        check(sdot_set_newton_hessian_reuse(ctx_, contraction), "set_newton_hessian_reuse");
    }
    // SotSolver::evaluate_weighted_barycenters, euclidean distance (SotSolver.cc:584-660).
    void evaluate_weighted_barycenters(const std::vector<double> &potentials, std::vector<Point> &barycenters_out,
                                       const SolverParameters &params) {
        if (potentials.size() != n_) throw std::runtime_error("evaluate_weighted_barycenters: potential size");
        (void)params;  // like the reference, the current parameters' epsilon is used
        barycenters_out.resize(n_);
        check(sdot_weighted_barycenters(ctx_, potentials.data(), barycenters_out.data()->data()),
              "evaluate_weighted_barycenters");
    }
    // SotSolver::get_potential_conditioned_density (SotSolver.cc:973-1046) at given support
    // points and the source density there; one vector per requested potential index.
    void get_potential_conditioned_density(const std::vector<Point> &support_points,
                                           const std::vector<double> &density_at_points,
                                           const std::vector<double> &potential,
                                           const std::vector<unsigned int> &potential_indices,
                                           std::vector<std::vector<double>> &conditioned_densities) {
        if (support_points.size() != density_at_points.size() || potential.size() != n_)
            throw std::runtime_error("get_potential_conditioned_density: sizes");
        const int64_t np = (int64_t)support_points.size(), ni = (int64_t)potential_indices.size();
        std::vector<int64_t> idx(potential_indices.begin(), potential_indices.end());
        std::vector<double> out((size_t)(np * ni));
        check(sdot_conditioned_densities(ctx_, potential.data(), current_params.epsilon,
                                         get_last_distance_threshold(), np, support_points.data()->data(),
                                         density_at_points.data(), ni, idx.data(), out.data()),
              "get_potential_conditioned_density");
        conditioned_densities.assign((size_t)ni, std::vector<double>((size_t)np));
        for (int64_t k = 0; k < ni; ++k)
            std::copy(out.begin() + k * np, out.begin() + (k + 1) * np, conditioned_densities[k].begin());
    }
    // SoftmaxRefinement::compute_refinement (SoftmaxRefinement.cc:61-280): this solver's
    // targets are the coarse level; children CSR per coarse target.
    std::vector<double> softmax_refinement(const std::vector<double> &potential_coarse, double epsilon,
                                           double threshold, const std::vector<Point> &fine_points,
                                           const std::vector<int64_t> &child_offsets,
                                           const std::vector<int64_t> &child_indices) {
        std::vector<double> fine(fine_points.size(), 0.0);
        check(sdot_softmax_refinement(ctx_, potential_coarse.data(), epsilon, threshold,
                                      current_params.use_log_sum_exp_trick ? 1 : 0, (int64_t)fine_points.size(),
                                      fine_points.data()->data(), child_offsets.data(), child_indices.data(),
                                      fine.data()),
              "softmax_refinement");
        return fine;
    }
    double get_last_functional_value() const { return sdot_get_last_functional_value(ctx_); }
    unsigned get_last_iteration_count() const { return sdot_get_last_iteration_count(ctx_); }
    bool get_convergence_status() const { return sdot_get_convergence_status(ctx_) != 0; }
    double get_last_distance_threshold() const { return sdot_get_last_distance_threshold(ctx_); }
    double get_C_global() const { return sdot_get_C_global(ctx_); }
    void set_distance_threshold(double threshold) { check(sdot_set_distance_threshold(ctx_, threshold), "set"); }
    double compute_covering_radius() const {
        double r = 0;
        check(sdot_compute_covering_radius(ctx_, &r), "compute_covering_radius");
        return r;
    }
    double compute_geometric_radius_bound(const std::vector<double> &potentials, double epsilon, double tolerance) const {
        double r = 0;
        check(sdot_compute_geometric_radius_bound(ctx_, potentials.data(), epsilon, tolerance, &r),
              "compute_geometric_radius_bound");
        return r;
    }
    void set_distance_function(const std::string &name) {
        if (sdot_set_distance_function(ctx_, name.c_str()) != SDOT_OK)
            throw std::invalid_argument("Unknown distance function: " + name);
    }

    SolverParameters current_params;

private:
    void check(sdot_status s, const char *where) const {
        if (s != SDOT_OK && s != SDOT_EMAXITER)
            throw std::runtime_error(std::string(where) + ": " + sdot_last_error(ctx_));
    }
    sdot_ctx *ctx_ = nullptr;
    size_t n_ = 0;
};

}  // namespace sdot

#endif  // SDOT_SOTSOLVER_HPP
