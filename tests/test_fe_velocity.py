"""Velocity from a coupled FE simulator (flsp_set_velocity_fe): the
continuous nodal field of degree 1..3 on the mesh's Gauss-Lobatto lattice,
evaluated at the advection's quadrature points from each cell's own nodes
(the assembler's simulator branch, advection.implement.h:472-477,891-905).

CPU: the oracle's restatement against known answers - a field that is a
polynomial of degree <= the lattice degree is reproduced exactly, so the
advection operator and the CFL estimate equal those of the same analytic
field; a field with zero normal velocity on the boundary conserves the
total mass (interior face fluxes cancel only if a face's velocity is the
same from both of its cells).

GPU: the library against the oracle.  Bars as in tests/test_gpu_parity.py:
1e-12 relative for one operator evaluation, 1e-11 after short horizons
(substeps, the level-set driver's graph-replayed periods)."""
import math

import numpy as np
import pytest

from felspa_b200 import abi, fields as F

IC2 = F.sphere((0.4731, 0.5193), 0.3)
IC3 = F.sphere((0.45, 0.5, 0.55), 0.3)


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def linear_field(dim):
    """rotation plus a shear: linear in x, so every lattice degree holds it exactly"""
    if dim == 2:
        return F.ccw_rotation()
    one = (abi.F_ONE, 0.0, 0.0)
    return F.VelocityField(3, [(0, -1.0, [one, (abi.F_LIN, 1.0, -0.5), one]),
                               (1, 1.0, [(abi.F_LIN, 1.0, -0.5), one, one]),
                               (2, 0.3, [(abi.F_LIN, 1.0, -0.4), one, one])], name="linear_3d")


def tangential_lattice(n, degree, seed):
    """random continuous field whose normal component is zero on the boundary"""
    u = F.random_fe_lattice(n, degree, seed)
    dim = len(n)
    for d in range(dim):
        ax = dim - 1 - d        # array axis of direction d (components, z, y, x)
        sl = [slice(None)] * dim
        sl[ax] = 0
        u[d][tuple(sl)] = 0.0
        sl[ax] = -1
        u[d][tuple(sl)] = 0.0
    return u


# ---------------------------------------------------------------- CPU: oracle
@pytest.mark.parametrize("dim,p,degree", [(2, 1, 1), (2, 2, 2), (2, 3, 3), (3, 1, 1), (3, 2, 2), (3, 2, 3)])
def test_oracle_polynomial_field_exact(oracle, dim, p, degree):
    n = (7, 6) if dim == 2 else (4, 3, 5)
    field = linear_field(dim)
    a = oracle.Problem(dim, n, p, abi.BASIS_Q)
    a.set_velocity(field)
    b = oracle.Problem(dim, n, p, abi.BASIS_Q)
    b.set_velocity_fe(degree, F.fe_lattice(field, n, degree))
    phi = a.project(IC2 if dim == 2 else IC3)
    assert rel(b.advect_rhs(phi, 0.0), a.advect_rhs(phi, 0.0)) <= 1e-13
    assert abs(b.advect_cfl(0.0) - a.advect_cfl(0.0)) <= 1e-14 * a.advect_cfl(0.0)


@pytest.mark.parametrize("dim,p,degree", [(2, 1, 2), (2, 2, 3), (3, 1, 2)])
def test_oracle_conserves_mass(oracle, dim, p, degree):
    n = (9, 8) if dim == 2 else (4, 5, 3)
    pr = oracle.Problem(dim, n, p, abi.BASIS_Q)
    pr.set_velocity_fe(degree, tangential_lattice(n, degree, seed=5))
    phi = pr.project(IC2 if dim == 2 else IC3)
    r = pr.advect_rhs(phi, 0.0).reshape(-1, pr.nb)
    # cell means: mode 0 of the orthonormal basis
    assert abs(r[:, 0].sum()) <= 1e-12 * np.abs(r[:, 0]).sum()


def test_oracle_cfl_is_largest_vertex_node(oracle):
    n, degree = (6, 5), 3
    u = F.random_fe_lattice(n, degree, seed=2)
    pr = oracle.Problem(2, n, 1, abi.BASIS_Q)
    pr.set_velocity_fe(degree, u)
    verts = u[:, ::degree, ::degree]
    want = np.sqrt((verts ** 2).sum(axis=0)).max() / math.hypot(1 / 6, 1 / 5)
    assert abs(pr.advect_cfl(0.0) - want) <= 1e-15 * want


def test_oracle_rejects_bad_lattice(oracle):
    pr = oracle.Problem(2, (4, 4), 1, abi.BASIS_Q)
    with pytest.raises(RuntimeError):
        pr.set_velocity_fe(2, np.zeros(10))
    with pytest.raises(RuntimeError):
        pr.set_velocity_fe(4, np.zeros(2 * 17 * 17))


# ------------------------------------------------------------ GPU: library
def pair(oracle, dim, n, p, basis, degree, values, prec=abi.FP64, cfl=0.1):
    from felspa_b200.level_set import AdvectSimulator, Mesh
    sim = AdvectSimulator(Mesh(dim, n), p, basis=basis, precision=prec, cfl_max=cfl)
    ic = IC2 if dim == 2 else IC3
    sim.initialize(ic, linear_field(dim))
    sim.problem.set_velocity_fe(degree, values)
    orc = oracle.Problem(dim, n, p, basis)
    orc.set_velocity_fe(degree, values)
    return sim, orc, orc.project(ic)


CASES = [(2, 1, abi.BASIS_Q, 1), (2, 1, abi.BASIS_P, 2), (2, 2, abi.BASIS_Q, 2), (2, 2, abi.BASIS_P, 3),
         (2, 3, abi.BASIS_Q, 2), (2, 3, abi.BASIS_P, 1), (3, 1, abi.BASIS_Q, 2), (3, 2, abi.BASIS_Q, 2),
         (3, 2, abi.BASIS_P, 1), (3, 2, abi.BASIS_Q, 3), (3, 1, abi.BASIS_P, 3)]


@pytest.mark.gpu
@pytest.mark.parametrize("dim,p,basis,degree", CASES)
def test_rhs_random_field(oracle, flsp, dim, p, basis, degree):
    """a random continuous field (every lattice is one), partial tiles"""
    n = (21, 18) if dim == 2 else (9, 7, 10)
    u = F.random_fe_lattice(n, degree, seed=100 * dim + 10 * p + degree)
    sim, orc, phi = pair(oracle, dim, n, p, basis, degree, u)
    sim.problem.set_state(phi)
    assert rel(sim.explicit_time_derivative(0.0), orc.advect_rhs(phi, 0.0)) <= 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("dim,p,degree", [(2, 2, 3), (3, 2, 2)])
def test_mass_conserved_on_device(oracle, flsp, dim, p, degree):
    n = (20, 17) if dim == 2 else (9, 8, 7)
    sim, orc, phi = pair(oracle, dim, n, p, abi.BASIS_Q, degree, tangential_lattice(n, degree, seed=9))
    sim.problem.set_state(phi)
    r = sim.explicit_time_derivative(0.0).reshape(-1, sim.problem.dofs_per_cell)
    assert abs(r[:, 0].sum()) <= 1e-12 * np.abs(r[:, 0]).sum()


@pytest.mark.gpu
@pytest.mark.parametrize("dim,p,degree", [(2, 1, 2), (2, 2, 2), (3, 2, 2)])
def test_advance_vs_oracle(oracle, flsp, dim, p, degree):
    """CFL-limited SSP-RK3 substeps with the FE field's CFL estimate"""
    n = (16, 14) if dim == 2 else (8, 7, 9)
    field = F.single_vortex(period=4.0) if dim == 2 else F.deformation_3d()
    u = F.fe_lattice(lambda x: field(x, 0.0), n, degree)
    sim, orc, phi = pair(oracle, dim, n, p, abi.BASIS_Q, degree, u)
    sim.problem.set_state(phi)
    a = sim.advance_time(0.05)
    b = orc.advance(phi, 0.05, single_cycle=False, cfl_max=0.1)
    assert abs(a - b) <= 1e-15
    assert sim.problem.get_step_count() == orc.clock.n_substeps
    assert rel(sim.get_solution_vector(), phi) <= 1e-11


@pytest.mark.gpu
def test_level_set_driver_update_in_place(oracle, flsp):
    """graph-replayed periods (substeps + fixed reinit); the field is
    rewritten between runs with the same degree (the captured graphs are
    kept and read the new values), then replaced by one of another degree"""
    from felspa_b200.level_set import LevelSetSurface, Mesh
    n = (18, 16)
    ctl = abi.default_ls_opts(reinit_frequency=5,
                              reinit=abi.default_reinit_opts(mode=abi.REINIT_FIXED, n_pseudo_steps=3))
    ls = LevelSetSurface(Mesh(2, n), 2, basis=abi.BASIS_Q, precision=abi.FP64, cfl_max=0.1, control=ctl)
    ls.initialize(IC2, linear_field(2))
    orc = oracle.Problem(2, n, 2, abi.BASIS_Q)
    phi = orc.project(IC2)
    fields = [(2, F.fe_lattice(lambda x: F.single_vortex(period=4.0)(x, 0.0), n, 2)),
              (2, F.random_fe_lattice(n, 2, seed=3, scale=0.5)),
              (3, F.random_fe_lattice(n, 3, seed=4, scale=0.5))]
    for degree, u in fields:
        ls.problem.set_velocity_fe(degree, u)
        orc.set_velocity_fe(degree, u)
        ls.run_steps(7)
        for _ in range(7):
            orc.ls_advance(phi, 1e30, ctl, single_step=True, cfl_max=0.1)
        assert abs(ls.get_time() - orc.clock.t) <= 1e-15
        assert rel(ls.get_solution_vector(), phi) <= 1e-11


@pytest.mark.gpu
def test_fp32_close_to_fp64(flsp):
    from felspa_b200.level_set import AdvectSimulator, Mesh
    n = (24, 24)
    u = F.fe_lattice(lambda x: F.single_vortex(period=4.0)(x, 0.0), n, 2)
    outs = []
    for prec in (abi.FP32, abi.FP64):
        s = AdvectSimulator(Mesh(2, n), 2, basis=abi.BASIS_Q, precision=prec, cfl_max=0.1)
        s.initialize(IC2, linear_field(2))
        s.problem.set_velocity_fe(2, u)
        s.advance_steps(20)
        outs.append(s.get_solution_vector())
    assert rel(outs[0], outs[1]) <= 1e-4


@pytest.mark.gpu
def test_bad_fields_rejected(flsp):
    from felspa_b200.batch import make_batch, uneven_batch_instances
    from felspa_b200.level_set import Mesh, Problem
    from felspa_b200.lib import FlspError
    pb = Problem(Mesh(2, (8, 8)), 1)
    good = F.random_fe_lattice((8, 8), 2, seed=1)
    for degree, vals, msg in ((0, good, "degree"), (4, good, "degree"), (3, good, "size"),
                              (2, good.ravel()[:-1], "size")):
        with pytest.raises(FlspError, match=msg):
            pb.set_velocity_fe(degree, vals)
    bad = good.copy()
    bad[1, 2, 3] = float("nan")
    with pytest.raises(FlspError, match="non-finite"):
        pb.set_velocity_fe(2, bad)
    pb.close()
    b = make_batch(uneven_batch_instances(2, n_min=16, n_max=20), precision=abi.FP64)
    with pytest.raises(FlspError, match="batch member"):
        b.problems[0].set_velocity_fe(1, np.zeros(10))
    b.close()
