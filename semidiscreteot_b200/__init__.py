"""semidiscreteot_b200 -- B200-native entropic semi-discrete OT dual evaluation.

A drop-in for the hot path of SemiDiscreteOT's ``SotSolver`` (functional,
gradient, Hessian and the L-BFGS solve), implemented as hand-written sm_100a
CUDA kernels behind the C ABI in ``include/sdot.h`` (``libsdot_cuda.so``).
"""
from .parameters import (MultilevelParameters, SolverParameters, distribute_epsilon_values, epsilon_sequence,
                         read_prm, solver_parameters_from_prm, multilevel_parameters_from_prm)
from . import io
from .batch import BatchSolver
from .lloyd import run_lloyd
from .multilevel import build_hierarchy, run_source_multilevel, run_target_multilevel
from .server import SolveServer
from .solver import SotSolver
from .simplex import simplex_source
from .source import sphere_source, structured_source

__all__ = [
    "SotSolver", "BatchSolver", "SolveServer", "SolverParameters", "build_hierarchy", "run_target_multilevel", "run_source_multilevel", "run_lloyd", "simplex_source", "io", "MultilevelParameters", "read_prm", "solver_parameters_from_prm",
    "multilevel_parameters_from_prm", "epsilon_sequence", "distribute_epsilon_values", "structured_source", "sphere_source",
]
