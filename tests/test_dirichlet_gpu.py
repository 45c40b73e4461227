"""Dirichlet inflow boundaries (LevelSetSurface::append_boundary_condition
with constant values): the library against the oracle.

Boundary ids are given per boundary face (mixed within a side), with
conditions on some ids and none on others (zero-Neumann); velocities with
inflow through every side.  Bars as in tests/test_gpu_parity.py: 1e-12
relative for one operator evaluation (advection RHS through both stage
kernels, LDG left / right gradients), 1e-11 after short horizons (SSP-RK3
substeps, reinit pseudo-steps, the level-set driver)."""
import numpy as np
import pytest

from felspa_b200 import abi, fields as F
from felspa_b200.level_set import (AdvectSimulator, LevelSetSurface, Mesh, Problem, ReinitSimulatorLDG,
                                   boundary_face_count)
from felspa_b200.lib import FlspError

pytestmark = pytest.mark.gpu

ONE = (abi.F_ONE, 0.0, 0.0)


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def face_ids(dim, n, seed):
    """per-face ids drawn from {0, 3, 4, 5} (0 and 5 carry no condition)"""
    rng = np.random.default_rng(seed)
    return rng.choice(np.array([0, 3, 4, 5], dtype=np.int32), size=boundary_face_count(dim, n))


CONDITIONS = {3: 0.7, 4: -0.3}


def shear_2d():
    """u = y - 0.4, v = 0.7 (x - 0.6): inflow through parts of every side,
    tangential factors that change sign along x- and y- sides"""
    return F.VelocityField(2, [(0, 1.0, [ONE, (abi.F_LIN, 1.0, -0.4)]),
                               (1, 0.7, [(abi.F_LIN, 1.0, -0.6), ONE])], name="shear_2d")


def shear_3d():
    """one separable term per component, inflow through every side"""
    return F.VelocityField(3, [(0, 1.0, [ONE, (abi.F_LIN, 1.0, -0.4), ONE]),
                               (1, 0.7, [(abi.F_LIN, 1.0, -0.6), ONE, ONE]),
                               (2, -0.5, [ONE, ONE, (abi.F_LIN, 1.0, 0.2)])], name="shear_3d")


def multiterm(field):
    """the same field split into two terms per component (the point-wise
    quadrature stage kernel instead of the separable one)"""
    terms = []
    for comp, coeff, fs in field.terms:
        terms.append((comp, 0.25 * coeff, fs))
        terms.append((comp, 0.75 * coeff, fs))
    return F.VelocityField(field.dim, terms, name=field.name + "_split")


def pair(oracle, dim, n, p, basis, field, ic, seed, prec=abi.FP64, cfl=0.1):
    ids = face_ids(dim, n, seed)
    sim = AdvectSimulator(Mesh(dim, n, boundary_ids=ids), p, basis=basis, precision=prec, cfl_max=cfl)
    sim.initialize(ic, field)
    orc = oracle.Problem(dim, n, p, basis, boundary_ids=ids)
    orc.set_velocity(field)
    for k, v in CONDITIONS.items():
        sim.append_boundary_condition(k, v)
        orc.set_dirichlet(k, v)
    return sim, orc, orc.project(ic)


CASES_2D = [(1, abi.BASIS_P), (1, abi.BASIS_Q), (2, abi.BASIS_P), (2, abi.BASIS_Q), (3, abi.BASIS_Q),
            (3, abi.BASIS_P)]
CASES_3D = [(1, abi.BASIS_Q), (2, abi.BASIS_P), (2, abi.BASIS_Q)]
IC2 = F.sphere((0.4731, 0.5193), 0.3)
IC3 = F.sphere((0.45, 0.5, 0.55), 0.3)


@pytest.mark.parametrize("split", [False, True])
@pytest.mark.parametrize("p,basis", CASES_2D)
def test_rhs_2d(oracle, flsp, p, basis, split):
    field = multiterm(shear_2d()) if split else shear_2d()
    sim, orc, phi = pair(oracle, 2, (20, 17), p, basis, field, IC2, seed=p)
    for t in (0.0, 0.3):
        assert rel(sim.explicit_time_derivative(t), orc.advect_rhs(phi, t)) <= 1e-12


@pytest.mark.parametrize("split", [False, True])
@pytest.mark.parametrize("p,basis", CASES_3D)
def test_rhs_3d(oracle, flsp, p, basis, split):
    field = multiterm(shear_3d()) if split else shear_3d()
    sim, orc, phi = pair(oracle, 3, (9, 7, 10), p, basis, field, IC3, seed=10 + p)
    assert rel(sim.explicit_time_derivative(0.0), orc.advect_rhs(phi, 0.0)) <= 1e-12


@pytest.mark.parametrize("dim,p,basis", [(2, 1, abi.BASIS_P), (2, 2, abi.BASIS_Q), (2, 3, abi.BASIS_Q),
                                         (3, 1, abi.BASIS_Q), (3, 2, abi.BASIS_Q), (3, 2, abi.BASIS_P)])
def test_ldg_gradients(oracle, flsp, dim, p, basis):
    n = (14, 11) if dim == 2 else (7, 6, 8)
    field, ic = (shear_2d(), IC2) if dim == 2 else (shear_3d(), IC3)
    sim, orc, phi = pair(oracle, dim, n, p, basis, field, ic, seed=20 + p)
    gl, gr = ReinitSimulatorLDG(sim.problem).local_left_right_gradients()
    ol, orr = orc.hj_gradients(phi)
    assert rel(gl, ol) <= 1e-12 and rel(gr, orr) <= 1e-12


@pytest.mark.parametrize("dim,p,basis", [(2, 1, abi.BASIS_P), (2, 2, abi.BASIS_Q), (3, 2, abi.BASIS_Q)])
def test_reinit(oracle, flsp, dim, p, basis):
    n = (16, 14) if dim == 2 else (8, 7, 9)
    field, ic = (shear_2d(), IC2) if dim == 2 else (shear_3d(), IC3)
    sim, orc, phi = pair(oracle, dim, n, p, basis, field, ic, seed=30 + p)
    ro = abi.default_reinit_opts(mode=abi.REINIT_FIXED, n_pseudo_steps=3)
    ReinitSimulatorLDG(sim.problem).run_iteration(ro)
    st, _ = orc.reinit(phi, ro)
    assert st == 0
    assert rel(sim.get_solution_vector(), phi) <= 1e-11


@pytest.mark.parametrize("dim,p,basis", [(2, 1, abi.BASIS_Q), (2, 2, abi.BASIS_P), (3, 2, abi.BASIS_Q)])
def test_advance(oracle, flsp, dim, p, basis):
    n = (16, 14) if dim == 2 else (8, 7, 9)
    field, ic = (shear_2d(), IC2) if dim == 2 else (shear_3d(), IC3)
    sim, orc, phi = pair(oracle, dim, n, p, basis, field, ic, seed=40 + p)
    a = sim.advance_time(0.05)
    b = orc.advance(phi, 0.05, single_cycle=False, cfl_max=0.1)
    assert abs(a - b) <= 1e-15
    assert rel(sim.get_solution_vector(), phi) <= 1e-11


def test_level_set_driver_graph_periods(oracle, flsp):
    """graph-replayed periods (substeps + fixed reinit with the WENO
    limiter) with Dirichlet faces, against the oracle step by step"""
    n, p = (18, 16), 2
    ids = face_ids(2, n, 7)
    ctl = abi.default_ls_opts(reinit_frequency=5,
                              reinit=abi.default_reinit_opts(mode=abi.REINIT_FIXED, n_pseudo_steps=3))
    ls = LevelSetSurface(Mesh(2, n, boundary_ids=ids), p, basis=abi.BASIS_Q, precision=abi.FP64, cfl_max=0.1,
                         control=ctl)
    ls.initialize(IC2, shear_2d())
    orc = oracle.Problem(2, n, p, abi.BASIS_Q, boundary_ids=ids)
    orc.set_velocity(shear_2d())
    phi = orc.project(IC2)
    for k, v in CONDITIONS.items():
        ls.append_boundary_condition(k, v)
        orc.set_dirichlet(k, v)
    ls.run_steps(12)
    for _ in range(12):
        orc.ls_advance(phi, 1e30, ctl, single_step=True, cfl_max=0.1)
    assert abs(ls.get_time() - orc.clock.t) <= 1e-15
    assert rel(ls.get_solution_vector(), phi) <= 1e-11


def test_conditions_replace_and_clear(oracle, flsp):
    """changing a value replaces it (captured graphs are dropped), clearing
    restores the zero-Neumann operator bit for bit"""
    n = (12, 12)
    sim, orc, phi = pair(oracle, 2, n, 2, abi.BASIS_Q, shear_2d(), IC2, seed=3)
    sim.append_boundary_condition(3, 2.5)
    orc.set_dirichlet(3, 2.5)
    assert rel(sim.explicit_time_derivative(0.0), orc.advect_rhs(phi, 0.0)) <= 1e-12
    plain = AdvectSimulator(Mesh(2, n), 2, basis=abi.BASIS_Q, precision=abi.FP64)
    plain.initialize(IC2, shear_2d())
    sim.problem.clear_dirichlet()
    assert np.array_equal(sim.explicit_time_derivative(0.2), plain.explicit_time_derivative(0.2))


def test_fp32_close_to_fp64(flsp):
    n = (24, 24)
    ids = face_ids(2, n, 11)
    outs = []
    for prec in (abi.FP32, abi.FP64):
        s = AdvectSimulator(Mesh(2, n, boundary_ids=ids), 2, basis=abi.BASIS_Q, precision=prec, cfl_max=0.1)
        s.initialize(IC2, shear_2d())
        for k, v in CONDITIONS.items():
            s.append_boundary_condition(k, v)
        s.advance_steps(20)
        outs.append(s.get_solution_vector())
    assert rel(outs[0], outs[1]) <= 1e-4


def test_bad_conditions_rejected(flsp):
    pb = Problem(Mesh(2, (8, 8)), 1)
    for bid, v in ((0, 1.0), (-2, 1.0), (3, float("nan")), (3, float("inf"))):
        with pytest.raises(FlspError):
            pb.set_dirichlet(bid, v)
    with pytest.raises(FlspError, match="negative boundary id"):
        Problem(Mesh(2, (4, 4), boundary_ids=np.full(16, -1, dtype=np.int32)), 1)
    from felspa_b200.batch import make_batch, uneven_batch_instances
    b = make_batch(uneven_batch_instances(2, n_min=16, n_max=20), precision=abi.FP64)
    with pytest.raises(FlspError, match="batch member"):
        b.problems[0].set_dirichlet(3, 1.0)
    b.close()
