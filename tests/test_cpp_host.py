"""The C++ host side: the facade (include/sdot/SotSolver.hpp) and the parameter-file
reader (include/sdot/ParameterFile.hpp), compiled with g++ into a program
(tests/cpp/host_solver.cpp) linked against libsdot_cuda.so.

CPU tests compile and link the program and check the C++ reader against the
Python reader on the same parameter file, key by key, and its error
behaviour.  The GPU test runs the program's solve mode on the dense 2D
benchmark problem at full size (64 x 64 cells x 3 x 3 Gauss points = 36,864
points, 1,000 targets, eps = 1e-2, no truncation, FP64 sweeps, L-BFGS to
|g|_inf <= 1e-8) and compares its evaluation at psi = 0 with the oracle
(value 1e-10 relative, gradient 1e-12 absolute) and its converged potential
with the oracle's gradient (|g|_inf <= 1.5e-8 at the C++ potential).
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

from semidiscreteot_b200 import parameters as P
from semidiscreteot_b200 import workloads

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "semidiscreteot_b200")
FIXTURE = os.path.join(ROOT, "tests", "fixtures", "parameters.prm")


@pytest.fixture(scope="module")
def host_solver(tmp_path_factory):
    gxx = shutil.which("g++")
    if not gxx:
        pytest.skip("no g++")
    from semidiscreteot_b200 import _lib
    _lib.load()   # the library must exist (built in-tree)
    exe = str(tmp_path_factory.mktemp("cpp") / "host_solver")
    subprocess.run([gxx, "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "host_solver.cpp"), "-L", PKG, "-lsdot_cuda",
                    f"-Wl,-rpath,{PKG}", "-o", exe], check=True)
    return exe


def _cpp_prm(exe, path):
    out = subprocess.run([exe, "prm", path], check=True, capture_output=True, text=True).stdout
    return dict(line.split(" ", 1) for line in out.strip().splitlines())


def test_cpp_reader_matches_python_reader(host_solver):
    cpp = _cpp_prm(host_solver, FIXTURE)
    tree = P.read_prm(FIXTURE)
    p = P.solver_parameters_from_prm(tree)
    m = P.multilevel_parameters_from_prm(tree)
    o = P.b200_options_from_prm(tree)
    for f in ("max_iterations", "quadrature_order", "n_threads", "epsilon_scaling_steps"):
        assert int(cpp[f]) == getattr(p, f), f
    for f in ("tolerance", "epsilon", "tau", "epsilon_scaling_factor"):
        assert float(cpp[f]) == getattr(p, f), f
    for f in ("verbose_output", "use_epsilon_scaling", "use_log_sum_exp_trick"):
        assert bool(int(cpp[f])) == getattr(p, f), f
    for f in ("solver_control_type", "distance_threshold_type", "solver_type", "line_search"):
        assert cpp[f] == getattr(p, f), f
    for f in ("source_enabled", "target_enabled", "use_softmax_potential_transfer", "use_python_clustering"):
        assert bool(int(cpp[f])) == getattr(m, f), f
    for f in ("source_min_vertices", "source_max_vertices", "target_min_points", "target_max_points"):
        assert int(cpp[f]) == getattr(m, f), f
    for f in ("source_hierarchy_dir", "target_hierarchy_dir", "python_script_name", "output_prefix"):
        assert cpp[f] == getattr(m, f), f
    assert cpp["precision"] == o["precision"] and int(cpp["device"]) == o["device"]
    seq = [float(v) for v in cpp["epsilon_sequence"].split()]
    assert seq == P.epsilon_sequence(p.epsilon, p.epsilon_scaling_factor, p.epsilon_scaling_steps)
    # the values the fixture sets (a line continuation included)
    assert p.max_iterations == 5000 and p.epsilon == 1e-2 and p.tau == 0.0 and p.epsilon_scaling_steps == 3
    assert m.target_min_points == 250 and m.target_hierarchy_dir == "output/levels/targets"


@pytest.mark.parametrize("text,err", [
    ("subsection SotParameterManager\n subsection rsot_solver\n  set epsilonn = 1\n end\nend\n", "unknown rsot_solver key"),
    ("subsection SotParameterManager\n subsection rsot_solver\n  set epsilon = abc\n end\nend\n", "not a number"),
    ("subsection SotParameterManager\nend\nend\n", "'end' without subsection"),
    ("subsection SotParameterManager\n set a\nend\n", "expected 'set key = value'"),
    ("subsection SotParameterManager\n subsection rsot_solver\n", "unterminated subsection"),
    ("subsection SotParameterManager\n subsection b200\n  set precision = fp16\n end\nend\n", "unknown precision"),
])
def test_cpp_reader_rejects_bad_files(host_solver, tmp_path, text, err):
    f = tmp_path / "bad.prm"
    f.write_text(text)
    r = subprocess.run([host_solver, "prm", str(f)], capture_output=True, text=True)
    assert r.returncode == 1 and err in r.stderr, (r.returncode, r.stderr)
    # the Python reader rejects the same files
    with pytest.raises((ValueError, KeyError)):
        tree = P.read_prm(str(f))
        P.solver_parameters_from_prm(tree)
        P.b200_options_from_prm(tree)


def _write_problem(d, wl):
    src = wl["source"]
    dim = wl["dim"]
    nq = src["jxw"].size
    ncell = src["cell_offsets"].size - 1
    nt = wl["y"].shape[0]
    (d / "meta.txt").write_text(f"{dim} {nq} {ncell} {nt}\n")
    np.ascontiguousarray(src["x"], dtype=np.float64).tofile(d / "x.bin")
    np.ascontiguousarray(src["jxw"], dtype=np.float64).tofile(d / "jxw.bin")
    np.ascontiguousarray(src["density"], dtype=np.float64).tofile(d / "density.bin")
    np.ascontiguousarray(src["cell_offsets"], dtype=np.int64).tofile(d / "offsets.bin")
    np.ascontiguousarray(src["cell_centers"], dtype=np.float64).tofile(d / "centers.bin")
    np.ascontiguousarray(wl["y"], dtype=np.float64).tofile(d / "y.bin")
    np.ascontiguousarray(wl["nu"], dtype=np.float64).tofile(d / "nu.bin")


@pytest.mark.gpu
def test_cpp_host_solves_dense_2d(host_solver, tmp_path, oracle_mod):
    wl = workloads.dense_2d()
    _write_problem(tmp_path, wl)
    prm_text = open(FIXTURE).read().replace("set use_epsilon_scaling = true", "set use_epsilon_scaling = false")
    prm_file = tmp_path / "run.prm"
    prm_file.write_text(prm_text)
    r = subprocess.run([host_solver, "solve", str(prm_file), str(tmp_path)], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    N = wl["y"].shape[0]
    ev = np.fromfile(tmp_path / "eval.bin")
    so = np.fromfile(tmp_path / "solve.bin")
    J, C, thr, g = ev[0], ev[1], ev[2], ev[3:]
    converged, iters, Jstar, psi = so[0], so[1], so[2], so[3:]
    assert g.size == N and psi.size == N

    src = wl["source"]
    Po = oracle_mod.Problem(src["x"], src["jxw"], src["density"], src["cell_offsets"], src["cell_centers"],
                            wl["y"], wl["nu"])
    op = oracle_mod.Params(epsilon=1e-2, tau=0.0, use_log_sum_exp=True, tolerance=1e-8, solver_control_type="linf",
                           max_iterations=5000)
    Jo, go, st = Po.evaluate(np.zeros(N), op)
    assert abs(J - Jo) <= 1e-10 * abs(Jo)
    assert np.max(np.abs(g - go)) <= 1e-12
    assert abs(C - st["C_global"]) <= 1e-10 * abs(st["C_global"])
    assert converged == 1.0 and 0 < iters <= 5000
    Po.reset_state()
    _, gs, _ = Po.evaluate(psi, op)
    assert np.max(np.abs(gs)) <= 1.5e-8
