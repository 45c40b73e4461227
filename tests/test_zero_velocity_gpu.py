"""Step-count runs with a velocity whose time factor starts at zero (the
plume's 1 - exp(-t)): the substep falls back to the spatial CFL estimate
instead of becoming infinite."""
import numpy as np
import pytest

from felspa_b200 import abi, fields as F
from felspa_b200.level_set import AdvectSimulator, Mesh

pytestmark = pytest.mark.gpu


def test_plume_step_count_run_stays_finite():
    sim = AdvectSimulator(Mesh(3, (10, 10, 10)), 1, basis=abi.BASIS_Q, precision=abi.FP64, cfl_max=0.1)
    sim.initialize(F.sphere((0.5, 0.5, 0.5), 0.2), F.plume_3d())
    sim.advance_steps(5)
    t = sim.get_time()
    assert np.isfinite(t) and t > 0.0
    assert np.all(np.isfinite(sim.get_solution_vector()))


def test_plume_step_count_run_with_far_end_time():
    """a step-count run capped by a far end time (not an unbounded one)
    does not jump to that end time from a vanishing time factor: the first
    substep falls back to the spatial estimate, the next ones follow the
    CFL rule at the (growing) current velocity"""
    import ctypes as C
    from felspa_b200.lib import check, load
    sim = AdvectSimulator(Mesh(3, (10, 10, 10)), 2, basis=abi.BASIS_Q, precision=abi.FP32, cfl_max=0.1)
    sim.initialize(F.sphere((0.5, 0.5, 0.5), 0.2), F.plume_3d())
    check(load().flsp_advance_steps(sim.problem.h, 5, C.c_double(1e30)))
    t = sim.get_time()
    assert np.isfinite(t) and 0.0 < t < 10.0
    assert np.all(np.isfinite(sim.get_solution_vector()))
