"""The .prm reader and the parameter structures (no GPU)."""
import pytest

from semidiscreteot_b200.parameters import (MultilevelParameters, SolverParameters, distribute_epsilon_values,
                                            epsilon_sequence, multilevel_parameters_from_prm, read_prm,
                                            solver_parameters_from_prm, b200_options_from_prm)

PRM = """
# a parameter file in the grammar of the reference's run/parameters.prm
subsection SotParameterManager
  set selected_task = sot
  set io_coding = txt
  subsection rsot_solver
    set max_iterations = 10000
    set epsilon = 1e-2
    set tau = 1e-8  # truncation tolerance
    set tolerance = 1e-2
    set distance_threshold_type = pointwise
    set solver_control_type = l1norm
    set verbose_output = false
    set quadrature_order = 3
    set number_of_threads = 0
    set use_log_sum_exp_trick = true
    set use_epsilon_scaling = false
    set epsilon_scaling_factor = 10
    set epsilon_scaling_steps = 3
  end
  subsection multilevel_parameters
    set target_enabled = true
    set target_min_points = 100
    set use_softmax_potential_transfer = true
  end
  subsection b200
    set precision = fp64
    set line_search = vendored
  end
end
"""


def test_read_and_map():
    tree = read_prm(PRM, is_text=True)
    assert tree["SotParameterManager"]["selected_task"] == "sot"
    p = solver_parameters_from_prm(tree)
    assert p.max_iterations == 10000 and p.epsilon == 1e-2 and p.tau == 1e-8 and p.tolerance == 1e-2
    assert p.use_log_sum_exp_trick is True and p.verbose_output is False
    assert p.epsilon_scaling_factor == 10.0 and p.epsilon_scaling_steps == 3 and p.n_threads == 0
    assert p.line_search == "vendored"
    m = multilevel_parameters_from_prm(tree)
    assert m.target_enabled and m.target_min_points == 100 and not m.source_enabled
    assert b200_options_from_prm(tree) == {"precision": "fp64"}


def test_defaults_match_reference():
    # ParameterManager.h:56-72
    p = SolverParameters()
    assert (p.max_iterations, p.tolerance, p.solver_control_type, p.epsilon, p.tau) == (1000, 1.0, "l1norm", 1e-3, 1e-8)
    assert p.distance_threshold_type == "pointwise" and p.use_log_sum_exp_trick is False
    assert (p.epsilon_scaling_factor, p.epsilon_scaling_steps, p.quadrature_order) == (2.0, 5, 3)
    m = MultilevelParameters()
    assert m.use_softmax_potential_transfer and m.target_max_points == 1000


def test_errors():
    with pytest.raises(ValueError):
        read_prm("subsection A\n set x = 1\n", is_text=True)
    with pytest.raises(ValueError):
        read_prm("end\n", is_text=True)
    with pytest.raises(KeyError):
        solver_parameters_from_prm(read_prm("subsection rsot_solver\n set bogus = 1\nend\n", is_text=True))
    with pytest.raises(ValueError):
        solver_parameters_from_prm(read_prm("subsection rsot_solver\n set verbose_output = maybe\nend\n", is_text=True))


def test_epsilon_distribution():
    # EpsilonScalingHandler::distribute_epsilon_values (EpsilonScalingHandler.cc:44-90)
    seq = epsilon_sequence(1e-3, 10.0, 3)
    assert distribute_epsilon_values(seq, 3) == [[seq[0]], [seq[1]], [seq[2]]]
    assert distribute_epsilon_values(seq, 5)[3:] == [[seq[2]], [seq[2]]]
    d = distribute_epsilon_values(epsilon_sequence(1e-3, 2.0, 7), 3)
    assert [len(x) for x in d] == [3, 2, 2]
    assert distribute_epsilon_values(seq, 0) == []
