"""The C-ABI library loads without a GPU and exports every declared symbol."""
import ctypes as C
import os
import re

import pytest

from semidiscreteot_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "sdot.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sdot_[A-Za-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported():
    lib = _lib.load()
    decl = declared_symbols()
    assert len(decl) >= 25
    for name in decl:
        assert hasattr(lib, name), name
    assert sorted(_lib.EXPORTED) == decl


def test_identity():
    lib = _lib.load()
    assert lib.sdot_abi_version() == 1
    assert b"sm_100a" in lib.sdot_build_info()


def test_default_params_match_reference():
    lib = _lib.load()
    p = _lib.SolverParams()
    lib.sdot_default_params(C.byref(p))
    assert (p.max_iterations, p.tolerance, p.epsilon, p.tau) == (1000, 1.0, 1e-3, 1e-8)
    assert p.control_type == 0 and p.threshold_type == 0 and p.use_log_sum_exp == 0 and p.line_search == 0


def test_no_silent_cpu_fallback():
    """Without a GPU, creating a context fails with a status (no CPU path)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = _lib.load()
    h = C.c_void_p()
    opts = _lib.Options(0, 1, 0, 0)
    st = lib.sdot_create(C.byref(h), C.byref(opts))
    assert st != 0 and not h.value
    from semidiscreteot_b200 import SotSolver
    with pytest.raises(RuntimeError):
        SotSolver(dim=2)


def test_header_compiles_as_c_and_cpp(tmp_path):
    import shutil
    import subprocess
    gcc = shutil.which("gcc")
    if not gcc:
        pytest.skip("no gcc")
    src = tmp_path / "t.c"
    src.write_text('#include "sdot.h"\nint main(void){ sdot_solver_params p; sdot_default_params(&p); return 0; }\n')
    subprocess.run([gcc, "-std=c99", "-Wall", "-Werror", "-fsyntax-only", "-I", os.path.join(ROOT, "include"), str(src)],
                   check=True)
    facade = os.path.join(ROOT, "include", "sdot", "SotSolver.hpp")
    cpp = tmp_path / "t.cpp"
    cpp.write_text('#include "sdot/SotSolver.hpp"\ntemplate class sdot::SotSolver<2>;\n'
                   'template class sdot::SotSolver<3>;\nint main(){ return 0; }\n')
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-fsyntax-only", "-I", os.path.join(ROOT, "include"),
                    str(cpp)], check=True)
    assert os.path.exists(facade)
