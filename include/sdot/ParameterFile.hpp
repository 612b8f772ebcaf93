// sdot/ParameterFile.hpp -- header-only reader of SemiDiscreteOT parameter files.
//
// The reference reads its run configuration with deal.II's ParameterHandler
// through SotParameterManager (src/utils/ParameterManager.cc:3-158): nested
// `subsection NAME` ... `end` blocks holding `set key = value` lines, `#`
// starting a comment, a trailing backslash continuing a line.  This header
// parses that grammar with the standard library only and maps the
// subsections the accelerated path uses onto plain structs:
//   SotParameterManager / rsot_solver            -> SolverParameters
//     (ParameterManager.cc:64-95, ParameterManager.h:56-72)
//   SotParameterManager / multilevel_parameters  -> MultilevelParameters
//     (ParameterManager.cc:97-131, ParameterManager.h:78-98)
//   SotParameterManager / b200                   -> B200Options
//     (keys of this implementation: precision, device, line_search)
// Other subsections (mesh_generation, power_diagram_parameters, ...) are
// parsed and kept in the tree but not interpreted.  Like ParameterHandler,
// an unknown key inside an interpreted subsection, a malformed value or an
// unbalanced `end` throws std::runtime_error naming the line.
#ifndef SDOT_PARAMETERFILE_HPP
#define SDOT_PARAMETERFILE_HPP

#include <cctype>
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "SotSolver.hpp"

namespace sdot {

struct PrmNode {
    std::map<std::string, std::string> values;      // key -> raw value text
    std::map<std::string, PrmNode> subsections;     // name -> subsection
    const PrmNode *find(const std::string &name) const {
        auto it = subsections.find(name);
        return it == subsections.end() ? nullptr : &it->second;
    }
};

namespace prm_detail {

inline std::string trim(const std::string &s) {
    const char *ws = " \t\r\n";
    const size_t b = s.find_first_not_of(ws);
    if (b == std::string::npos) return std::string();
    const size_t e = s.find_last_not_of(ws);
    return s.substr(b, e - b + 1);
}

inline std::string where(int line) { return "parameter file line " + std::to_string(line) + ": "; }

inline bool to_bool(const std::string &v, const std::string &key) {
    std::string t;
    for (char ch : trim(v)) t += (char)std::tolower((unsigned char)ch);
    if (t == "true" || t == "1" || t == "yes" || t == "on") return true;
    if (t == "false" || t == "0" || t == "no" || t == "off") return false;
    throw std::runtime_error("parameter '" + key + "': not a boolean: '" + v + "'");
}

inline double to_double(const std::string &v, const std::string &key) {
    const std::string t = trim(v);
    char *end = nullptr;
    const double d = std::strtod(t.c_str(), &end);
    if (t.empty() || end != t.c_str() + t.size())
        throw std::runtime_error("parameter '" + key + "': not a number: '" + v + "'");
    return d;
}

inline long long to_int(const std::string &v, const std::string &key) {
    const std::string t = trim(v);
    char *end = nullptr;
    const long long i = std::strtoll(t.c_str(), &end, 10);
    if (t.empty() || end != t.c_str() + t.size())
        throw std::runtime_error("parameter '" + key + "': not an integer: '" + v + "'");
    return i;
}

}  // namespace prm_detail

// Parses parameter-file text into a tree rooted at an unnamed node.
inline PrmNode read_prm_text(const std::string &text) {
    using namespace prm_detail;
    PrmNode root;
    std::vector<PrmNode *> stack{&root};
    std::istringstream in(text);
    std::string raw, line;
    int lineno = 0, start = 0;
    while (std::getline(in, raw)) {
        ++lineno;
        if (line.empty()) start = lineno;
        const size_t hash = raw.find('#');
        std::string part = hash == std::string::npos ? raw : raw.substr(0, hash);
        const std::string tp = trim(part);
        if (!tp.empty() && tp.back() == '\\' && hash == std::string::npos) {  // continuation
            line += tp.substr(0, tp.size() - 1) + " ";
            continue;
        }
        line += part;
        const std::string s = trim(line);
        line.clear();
        if (s.empty()) continue;
        if (s.compare(0, 11, "subsection ") == 0) {
            const std::string name = trim(s.substr(11));
            if (name.empty()) throw std::runtime_error(where(start) + "subsection without a name");
            stack.push_back(&stack.back()->subsections[name]);
        } else if (s == "end") {
            if (stack.size() == 1) throw std::runtime_error(where(start) + "'end' without subsection");
            stack.pop_back();
        } else if (s.compare(0, 4, "set ") == 0) {
            const std::string body = s.substr(4);
            const size_t eq = body.find('=');
            if (eq == std::string::npos) throw std::runtime_error(where(start) + "expected 'set key = value'");
            const std::string key = trim(body.substr(0, eq));
            if (key.empty()) throw std::runtime_error(where(start) + "empty key");
            stack.back()->values[key] = trim(body.substr(eq + 1));
        } else {
            throw std::runtime_error(where(start) + "cannot parse '" + s + "'");
        }
    }
    if (!line.empty()) throw std::runtime_error(where(start) + "line continuation at end of file");
    if (stack.size() != 1) throw std::runtime_error("parameter file: unterminated subsection");
    return root;
}

inline PrmNode read_prm_file(const std::string &path) {
    std::ifstream f(path);
    if (!f) throw std::runtime_error("cannot open parameter file " + path);
    std::stringstream ss;
    ss << f.rdbuf();
    return read_prm_text(ss.str());
}

// SotParameterManager::MultilevelParameters (ParameterManager.h:78-98), defaults as there.
struct MultilevelParameters {
    bool source_enabled = false;
    int source_min_vertices = 1000;
    int source_max_vertices = 10000;
    std::string source_hierarchy_dir = "output/data_multilevel/source_multilevel";
    bool target_enabled = false;
    int target_min_points = 100;
    int target_max_points = 1000;
    std::string target_hierarchy_dir = "output/data_multilevel/target_multilevel";
    bool use_softmax_potential_transfer = true;
    bool use_python_clustering = false;
    std::string python_script_name = "multilevel_clustering_scipy.py";
    std::string output_prefix = "output/multilevel/sot";
};

// Options of this implementation (subsection b200).
struct B200Options {
    std::string precision = "hybrid";  // fp64 | hybrid | mixed
    int device = 0;
    sdot_precision c_precision() const {
        if (precision == "fp64") return SDOT_PREC_FP64;
        if (precision == "hybrid") return SDOT_PREC_HYBRID;
        if (precision == "mixed") return SDOT_PREC_MIXED;
        throw std::runtime_error("b200.precision: unknown precision '" + precision + "'");
    }
};

// The solver node: SotParameterManager when present (the reference's root
// subsection), else the root itself.
inline const PrmNode &prm_manager_node(const PrmNode &root) {
    const PrmNode *m = root.find("SotParameterManager");
    return m ? *m : root;
}

inline SolverParameters solver_parameters_from_prm(const PrmNode &root) {
    using namespace prm_detail;
    SolverParameters p;
    const PrmNode &mgr = prm_manager_node(root);
    if (const PrmNode *rs = mgr.find("rsot_solver")) {
        for (const auto &kv : rs->values) {
            const std::string &k = kv.first, &v = kv.second;
            if (k == "max_iterations") p.max_iterations = (unsigned)to_int(v, k);
            else if (k == "tolerance") p.tolerance = to_double(v, k);
            else if (k == "solver_control_type") p.solver_control_type = trim(v);
            else if (k == "epsilon") p.epsilon = to_double(v, k);
            else if (k == "tau") p.tau = to_double(v, k);
            else if (k == "distance_threshold_type") p.distance_threshold_type = trim(v);
            else if (k == "verbose_output") p.verbose_output = to_bool(v, k);
            else if (k == "solver_type") p.solver_type = trim(v);
            else if (k == "quadrature_order") p.quadrature_order = (unsigned)to_int(v, k);
            else if (k == "number_of_threads") p.n_threads = (unsigned)to_int(v, k);
            else if (k == "use_epsilon_scaling") p.use_epsilon_scaling = to_bool(v, k);
            else if (k == "epsilon_scaling_factor") p.epsilon_scaling_factor = to_double(v, k);
            else if (k == "epsilon_scaling_steps") p.epsilon_scaling_steps = (unsigned)to_int(v, k);
            else if (k == "use_log_sum_exp_trick") p.use_log_sum_exp_trick = to_bool(v, k);
            else throw std::runtime_error("unknown rsot_solver key '" + k + "'");
        }
    }
    if (const PrmNode *b = mgr.find("b200")) {
        auto it = b->values.find("line_search");
        if (it != b->values.end()) p.line_search = trim(it->second);
    }
    return p;
}

inline MultilevelParameters multilevel_parameters_from_prm(const PrmNode &root) {
    using namespace prm_detail;
    MultilevelParameters m;
    if (const PrmNode *ml = prm_manager_node(root).find("multilevel_parameters")) {
        for (const auto &kv : ml->values) {
            const std::string &k = kv.first, &v = kv.second;
            if (k == "source_enabled") m.source_enabled = to_bool(v, k);
            else if (k == "source_min_vertices") m.source_min_vertices = (int)to_int(v, k);
            else if (k == "source_max_vertices") m.source_max_vertices = (int)to_int(v, k);
            else if (k == "source_hierarchy_dir") m.source_hierarchy_dir = trim(v);
            else if (k == "target_enabled") m.target_enabled = to_bool(v, k);
            else if (k == "target_min_points") m.target_min_points = (int)to_int(v, k);
            else if (k == "target_max_points") m.target_max_points = (int)to_int(v, k);
            else if (k == "target_hierarchy_dir") m.target_hierarchy_dir = trim(v);
            else if (k == "use_softmax_potential_transfer") m.use_softmax_potential_transfer = to_bool(v, k);
            else if (k == "use_python_clustering") m.use_python_clustering = to_bool(v, k);
            else if (k == "python_script_name") m.python_script_name = trim(v);
            else if (k == "output_prefix") m.output_prefix = trim(v);
            else throw std::runtime_error("unknown multilevel_parameters key '" + k + "'");
        }
    }
    return m;
}

inline B200Options b200_options_from_prm(const PrmNode &root) {
    using namespace prm_detail;
    B200Options o;
    if (const PrmNode *b = prm_manager_node(root).find("b200")) {
        for (const auto &kv : b->values) {
            const std::string &k = kv.first, &v = kv.second;
            if (k == "precision") o.precision = trim(v);
            else if (k == "device") o.device = (int)to_int(v, k);
            else if (k == "line_search") continue;  // read by solver_parameters_from_prm
            else throw std::runtime_error("unknown b200 key '" + k + "'");
        }
        o.c_precision();  // validates the name
    }
    return o;
}

// Epsilon sequence of EpsilonScalingHandler::generate_epsilon_sequence
// (src/solvers/EpsilonScalingHandler.cc:31-43): eps * pow(f, s-1-i), largest
// first; a factor <= 1 is replaced by 2 and zero steps by one (:19-27).
inline std::vector<double> epsilon_sequence(double epsilon, double factor, unsigned steps) {
    if (factor <= 1.0) factor = 2.0;
    if (steps == 0) steps = 1;
    std::vector<double> out;
    for (unsigned i = 0; i < steps; ++i) out.push_back(epsilon * std::pow(factor, (double)(steps - 1 - i)));
    return out;
}

}  // namespace sdot

#endif  // SDOT_PARAMETERFILE_HPP
