"""Solver parameters and a dependency-free reader of SemiDiscreteOT ``.prm`` files.

``SolverParameters`` mirrors ``SotParameterManager::SolverParameters``
(include/SemiDiscreteOT/utils/ParameterManager.h:56-72) with the same field
names and defaults; ``MultilevelParameters`` mirrors ``MultilevelParameters``
(:78-98).  ``read_prm`` understands the deal.II ParameterHandler grammar the
reference's parameter files use (``subsection NAME`` / ``set key = value`` /
``end``, ``#`` comments, a trailing backslash continuing a line;
src/utils/ParameterManager.cc:20-158, run/parameters.prm).  The C++ reader
``include/sdot/ParameterFile.hpp`` parses the same grammar the same way.
Keys of this implementation that the reference does not have live in a
separate ``subsection b200`` (precision, line_search).
"""
from __future__ import annotations

from dataclasses import dataclass, field, fields
from typing import Any, Dict


@dataclass
class SolverParameters:
    max_iterations: int = 1000
    tolerance: float = 1.0
    solver_control_type: str = "l1norm"        # l1norm | componentwise | linf (linf: extension)
    epsilon: float = 1e-3
    tau: float = 1e-8
    distance_threshold_type: str = "pointwise"  # pointwise | integral | geometric
    verbose_output: bool = True
    solver_type: str = "BFGS"
    quadrature_order: int = 3
    nb_points: int = 1000
    n_threads: int = 0
    use_epsilon_scaling: bool = False
    epsilon_scaling_factor: float = 2.0
    epsilon_scaling_steps: int = 5
    use_log_sum_exp_trick: bool = False
    line_search: str = "upstream"               # upstream (deal.II SolverBFGS) | vendored


@dataclass
class MultilevelParameters:
    source_enabled: bool = False
    source_min_vertices: int = 1000
    source_max_vertices: int = 10000
    source_hierarchy_dir: str = "output/data_multilevel/source_multilevel"
    target_enabled: bool = False
    target_min_points: int = 100
    target_max_points: int = 1000
    target_hierarchy_dir: str = "output/data_multilevel/target_multilevel"
    use_softmax_potential_transfer: bool = True
    use_python_clustering: bool = False
    python_script_name: str = "multilevel_clustering_scipy.py"
    output_prefix: str = "output/multilevel/sot"


# rsot_solver keys (ParameterManager.cc:64-95) -> SolverParameters fields
_RSOT_KEYS = {
    "max_iterations": "max_iterations", "tolerance": "tolerance", "solver_control_type": "solver_control_type",
    "epsilon": "epsilon", "tau": "tau", "distance_threshold_type": "distance_threshold_type",
    "verbose_output": "verbose_output", "solver_type": "solver_type", "quadrature_order": "quadrature_order",
    "number_of_threads": "n_threads", "use_epsilon_scaling": "use_epsilon_scaling",
    "epsilon_scaling_factor": "epsilon_scaling_factor", "epsilon_scaling_steps": "epsilon_scaling_steps",
    "use_log_sum_exp_trick": "use_log_sum_exp_trick",
}


def _convert(value: str, like: Any) -> Any:
    if isinstance(like, bool):
        v = value.strip().lower()
        if v in ("true", "1", "yes", "on"):
            return True
        if v in ("false", "0", "no", "off"):
            return False
        raise ValueError(f"not a boolean: {value!r}")
    if isinstance(like, int):
        return int(value)
    if isinstance(like, float):
        return float(value)
    return value.strip()


def read_prm(path_or_text: str, is_text: bool = False) -> Dict[str, Any]:
    """Parse a ``.prm`` file into nested dicts (subsection -> dict, key -> str)."""
    text = path_or_text if is_text else open(path_or_text).read()
    root: Dict[str, Any] = {}
    stack = [root]
    pending, start = "", 0
    for lineno, raw in enumerate(text.splitlines(), 1):
        if not pending:
            start = lineno
        part = raw.split("#", 1)[0]
        if "#" not in raw and part.strip().endswith("\\"):   # continued on the next line
            pending += part.strip()[:-1] + " "
            continue
        line = (pending + part).strip()
        pending = ""
        lineno = start
        if not line:
            continue
        if line.startswith("subsection "):
            name = line[len("subsection "):].strip()
            node = stack[-1].setdefault(name, {})
            stack.append(node)
        elif line == "end":
            if len(stack) == 1:
                raise ValueError(f"line {lineno}: 'end' without subsection")
            stack.pop()
        elif line.startswith("set "):
            body = line[4:]
            if "=" not in body:
                raise ValueError(f"line {lineno}: expected 'set key = value'")
            k, v = body.split("=", 1)
            stack[-1][k.strip()] = v.strip()
        else:
            raise ValueError(f"line {lineno}: cannot parse {raw!r}")
    if pending:
        raise ValueError(f"line {start}: line continuation at end of file")
    if len(stack) != 1:
        raise ValueError("unterminated subsection")
    return root


def solver_parameters_from_prm(tree: Dict[str, Any]) -> SolverParameters:
    """``SotParameterManager`` -> ``rsot_solver`` subsection as SolverParameters."""
    p = SolverParameters()
    node = tree.get("SotParameterManager", tree)
    rs = node.get("rsot_solver", {})
    defaults = {f.name: getattr(p, f.name) for f in fields(p)}
    for key, val in rs.items():
        if key not in _RSOT_KEYS:
            raise KeyError(f"unknown rsot_solver key {key!r}")
        fname = _RSOT_KEYS[key]
        setattr(p, fname, _convert(val, defaults[fname]))
    ext = node.get("b200", {})
    if "line_search" in ext:
        p.line_search = ext["line_search"].strip()
    return p


def multilevel_parameters_from_prm(tree: Dict[str, Any]) -> MultilevelParameters:
    m = MultilevelParameters()
    node = tree.get("SotParameterManager", tree).get("multilevel_parameters", {})
    defaults = {f.name: getattr(m, f.name) for f in fields(m)}
    for key, val in node.items():
        if key not in defaults:
            raise KeyError(f"unknown multilevel_parameters key {key!r}")
        setattr(m, key, _convert(val, defaults[key]))
    return m


def b200_options_from_prm(tree: Dict[str, Any]) -> Dict[str, Any]:
    node = tree.get("SotParameterManager", tree).get("b200", {})
    out: Dict[str, Any] = {}
    if "precision" in node:
        out["precision"] = node["precision"].strip()
        if out["precision"] not in ("fp64", "hybrid", "mixed"):
            raise ValueError(f"b200.precision: unknown precision {out['precision']!r}")
    if "device" in node:
        out["device"] = int(node["device"])
    return out


def epsilon_sequence(epsilon: float, factor: float, steps: int):
    """EpsilonScalingHandler::generate_epsilon_sequence (EpsilonScalingHandler.cc:6-42):
    eps * factor^(steps-1-i), largest first; factor <= 1 -> 2, steps == 0 -> 1."""
    if factor <= 1.0:
        factor = 2.0
    if steps == 0:
        steps = 1
    return [epsilon * factor ** (steps - 1 - i) for i in range(steps)]


def distribute_epsilon_values(seq, num_levels: int):
    """EpsilonScalingHandler::distribute_epsilon_values (EpsilonScalingHandler.cc:44-90)."""
    dist = [[] for _ in range(num_levels)]
    if num_levels == 0:
        return dist
    if len(seq) <= num_levels:
        for level in range(num_levels):
            dist[level].append(seq[level] if level < len(seq) else seq[-1])
    else:
        remaining_eps, remaining_lv, idx = len(seq), num_levels, 0
        for level in range(num_levels):
            n_here = (remaining_eps + remaining_lv - 1) // remaining_lv
            for _ in range(n_here):
                if idx < len(seq):
                    dist[level].append(seq[idx])
                    idx += 1
            remaining_eps -= n_here
            remaining_lv -= 1
    return dist
