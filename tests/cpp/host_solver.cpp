// A C++ host program on the library's C++ facade, as a C++ caller of the
// reference's SotSolver would write it: parameters from a parameter file
// (sdot/ParameterFile.hpp), the solver through sdot/SotSolver.hpp, linked
// against libsdot_cuda.so.
//
//   host_solver prm <file.prm>          print the parsed parameters, one
//                                       "key value" line each (no GPU)
//   host_solver solve <file.prm> <dir>  read the problem from <dir> (written by
//                                       the test), evaluate at psi = 0 and
//                                       solve; write the results back to <dir>
//
// Problem files in <dir> (raw little-endian): meta.txt "dim n_q n_cells n_t",
// x.bin, jxw.bin, density.bin, centers.bin, y.bin, nu.bin (doubles),
// offsets.bin (int64).  Results: eval.bin = {J, C_global, threshold,
// grad[n_t]}, solve.bin = {converged, iterations, J, psi[n_t]}.
#include <cstdio>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "sdot/ParameterFile.hpp"

template <class T>
static std::vector<T> read_bin(const std::string &path, size_t n) {
    std::vector<T> v(n);
    std::ifstream f(path, std::ios::binary);
    if (!f.read(reinterpret_cast<char *>(v.data()), (std::streamsize)(n * sizeof(T))))
        throw std::runtime_error("cannot read " + path);
    return v;
}

static void write_bin(const std::string &path, const std::vector<double> &v) {
    std::ofstream f(path, std::ios::binary);
    f.write(reinterpret_cast<const char *>(v.data()), (std::streamsize)(v.size() * sizeof(double)));
    if (!f) throw std::runtime_error("cannot write " + path);
}

static int print_prm(const std::string &file) {
    const sdot::PrmNode root = sdot::read_prm_file(file);
    const sdot::SolverParameters p = sdot::solver_parameters_from_prm(root);
    const sdot::MultilevelParameters m = sdot::multilevel_parameters_from_prm(root);
    const sdot::B200Options o = sdot::b200_options_from_prm(root);
    std::printf("max_iterations %u\ntolerance %.17g\nsolver_control_type %s\nepsilon %.17g\ntau %.17g\n",
                p.max_iterations, p.tolerance, p.solver_control_type.c_str(), p.epsilon, p.tau);
    std::printf("distance_threshold_type %s\nverbose_output %d\nsolver_type %s\nquadrature_order %u\n",
                p.distance_threshold_type.c_str(), (int)p.verbose_output, p.solver_type.c_str(), p.quadrature_order);
    std::printf("n_threads %u\nuse_epsilon_scaling %d\nepsilon_scaling_factor %.17g\nepsilon_scaling_steps %u\n",
                p.n_threads, (int)p.use_epsilon_scaling, p.epsilon_scaling_factor, p.epsilon_scaling_steps);
    std::printf("use_log_sum_exp_trick %d\nline_search %s\n", (int)p.use_log_sum_exp_trick, p.line_search.c_str());
    std::printf("source_enabled %d\nsource_min_vertices %d\nsource_max_vertices %d\nsource_hierarchy_dir %s\n",
                (int)m.source_enabled, m.source_min_vertices, m.source_max_vertices, m.source_hierarchy_dir.c_str());
    std::printf("target_enabled %d\ntarget_min_points %d\ntarget_max_points %d\ntarget_hierarchy_dir %s\n",
                (int)m.target_enabled, m.target_min_points, m.target_max_points, m.target_hierarchy_dir.c_str());
    std::printf("use_softmax_potential_transfer %d\nuse_python_clustering %d\npython_script_name %s\n",
                (int)m.use_softmax_potential_transfer, (int)m.use_python_clustering, m.python_script_name.c_str());
    std::printf("output_prefix %s\nprecision %s\ndevice %d\n", m.output_prefix.c_str(), o.precision.c_str(), o.device);
    const std::vector<double> eps =
        sdot::epsilon_sequence(p.epsilon, p.epsilon_scaling_factor, p.epsilon_scaling_steps);
    std::printf("epsilon_sequence");
    for (double e : eps) std::printf(" %.17g", e);
    std::printf("\n");
    return 0;
}

static int solve(const std::string &file, const std::string &dir) {
    const sdot::PrmNode root = sdot::read_prm_file(file);
    const sdot::SolverParameters prm = sdot::solver_parameters_from_prm(root);
    const sdot::B200Options opt = sdot::b200_options_from_prm(root);
    int dim = 0;
    long long nq = 0, ncells = 0, nt = 0;
    {
        std::ifstream meta(dir + "/meta.txt");
        if (!(meta >> dim >> nq >> ncells >> nt) || dim != 2) throw std::runtime_error("bad meta.txt (2D problems)");
    }
    using Solver = sdot::SotSolver<2>;
    using Point = Solver::Point;
    auto as_points = [](const std::vector<double> &v) {
        std::vector<Point> p(v.size() / 2);
        for (size_t i = 0; i < p.size(); ++i) p[i] = {v[2 * i], v[2 * i + 1]};
        return p;
    };
    const std::vector<Point> x = as_points(read_bin<double>(dir + "/x.bin", (size_t)(nq * 2)));
    const std::vector<double> jxw = read_bin<double>(dir + "/jxw.bin", (size_t)nq);
    const std::vector<double> density = read_bin<double>(dir + "/density.bin", (size_t)nq);
    const std::vector<int64_t> offsets = read_bin<int64_t>(dir + "/offsets.bin", (size_t)(ncells + 1));
    const std::vector<Point> centers = as_points(read_bin<double>(dir + "/centers.bin", (size_t)(ncells * 2)));
    const std::vector<Point> y = as_points(read_bin<double>(dir + "/y.bin", (size_t)(nt * 2)));
    const std::vector<double> nu = read_bin<double>(dir + "/nu.bin", (size_t)nt);

    Solver solver(opt.device, opt.c_precision());
    solver.setup_source(x, jxw, density, offsets, centers);
    solver.setup_target(y, nu);
    solver.configure(prm);
    std::vector<double> psi(nu.size(), 0.0), grad;
    const double J = solver.evaluate_functional(psi, grad);
    std::vector<double> ev{J, solver.get_C_global(), solver.get_last_distance_threshold()};
    ev.insert(ev.end(), grad.begin(), grad.end());
    write_bin(dir + "/eval.bin", ev);

    solver.solve(psi, prm);
    std::vector<double> so{solver.get_convergence_status() ? 1.0 : 0.0, (double)solver.get_last_iteration_count(),
                           solver.get_last_functional_value()};
    so.insert(so.end(), psi.begin(), psi.end());
    write_bin(dir + "/solve.bin", so);
    std::printf("solve: converged %d after %u iterations, J = %.17g\n", (int)solver.get_convergence_status(),
                solver.get_last_iteration_count(), solver.get_last_functional_value());
    return 0;
}

int main(int argc, char **argv) {
    try {
        const std::string mode = argc > 1 ? argv[1] : "";
        if (mode == "prm" && argc == 3) return print_prm(argv[2]);
        if (mode == "solve" && argc == 4) return solve(argv[2], argv[3]);
        std::cerr << "usage: host_solver prm <file.prm> | solve <file.prm> <dir>\n";
        return 2;
    } catch (const std::exception &e) {
        std::cerr << "host_solver: " << e.what() << "\n";
        return 1;
    }
}
