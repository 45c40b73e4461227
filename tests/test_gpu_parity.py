"""GPU parity: libflsp_dg.so (FP64 mode) against the CPU FP64 oracle.

Bar: relative max-norm difference <= 1e-12 for single operator
evaluations and short horizons (the oracle restates the reference's
algorithms; see oracle/oracle.h for its pinning status).

Geometries that feed the minmod detector are placed off the lattice's
symmetry lines: on a 45-degree line through a disk centre a P1 cell has
equal x and y slopes, the detector's vertex and neighbour slopes are both
exactly zero, and its decision is decided by rounding noise (in the
reference as well), so no two implementations agree there bit for bit.
"""
import math

import numpy as np
import pytest

from felspa_b200 import abi, fields as F
from felspa_b200.level_set import (AdvectSimulator, LevelSetSurface, Mesh, Problem,
                                   ReinitSimulatorLDG, dealii_hypercube_order)

pytestmark = pytest.mark.gpu

TOL = 1e-12


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


CASES_2D = [(1, abi.BASIS_P), (1, abi.BASIS_Q), (2, abi.BASIS_P), (2, abi.BASIS_Q), (3, abi.BASIS_Q),
            (3, abi.BASIS_P)]
CASES_3D = [(1, abi.BASIS_P), (1, abi.BASIS_Q), (2, abi.BASIS_P), (2, abi.BASIS_Q)]


def make_pair(oracle, dim, n, p, basis, field, ic, lo=(0, 0, 0), hi=(1, 1, 1)):
    mesh = Mesh(dim, n, lo, hi)
    sim = AdvectSimulator(mesh, p, basis=basis, precision=abi.FP64)
    sim.initialize(ic, field)
    orc = oracle.Problem(dim, n, p, basis, lo, hi)
    orc.set_velocity(field)
    phi = orc.project(ic)
    return sim, orc, phi


@pytest.mark.parametrize("p,basis", CASES_2D)
def test_projection_2d(oracle, flsp, p, basis):
    sim, orc, phi = make_pair(oracle, 2, (24, 20), p, basis, F.ccw_rotation(), F.zalesak_disk())
    assert rel(sim.get_solution_vector(), phi) <= TOL


@pytest.mark.parametrize("p,basis", CASES_2D)
def test_advect_rhs_2d(oracle, flsp, p, basis):
    sim, orc, phi = make_pair(oracle, 2, (24, 20), p, basis, F.ccw_rotation(), F.zalesak_disk())
    for t in (0.0, 0.3):
        assert rel(sim.explicit_time_derivative(t), orc.advect_rhs(phi, t)) <= TOL


@pytest.mark.parametrize("p,basis", CASES_3D)
def test_advect_rhs_3d(oracle, flsp, p, basis):
    ic = F.sphere((0.35, 0.35, 0.35), 0.15)
    sim, orc, phi = make_pair(oracle, 3, (10, 9, 8), p, basis, F.deformation_3d(), ic)
    assert rel(sim.get_solution_vector(), phi) <= TOL
    for t in (0.0, 0.7):
        assert rel(sim.explicit_time_derivative(t), orc.advect_rhs(phi, t)) <= TOL


def drifting_deformation_3d():
    """3D deformation plus a uniform drift: two separable terms per
    component, so the stage runs the point-wise quadrature kernel."""
    base = F.deformation_3d()
    drift = F.constant((0.3, -0.2, 0.1))
    return F.VelocityField(3, base.terms + drift.terms, time_kind=base.time_kind, ta=base.ta,
                           tb=base.tb, name="drifting_deformation_3d")


@pytest.mark.parametrize("p,basis", CASES_2D)
def test_advect_rhs_2d_multiterm(oracle, flsp, p, basis):
    # 8-mode Fourier stream function: several terms per component
    field = F.fourier_stream_2d(seed=1007)
    sim, orc, phi = make_pair(oracle, 2, (22, 19), p, basis, field, F.zalesak_disk())
    for t in (0.0, 0.4):
        assert rel(sim.explicit_time_derivative(t), orc.advect_rhs(phi, t)) <= TOL


@pytest.mark.parametrize("p,basis", CASES_3D)
def test_advect_rhs_3d_multiterm(oracle, flsp, p, basis):
    ic = F.sphere((0.35, 0.35, 0.35), 0.15)
    sim, orc, phi = make_pair(oracle, 3, (9, 8, 10), p, basis, drifting_deformation_3d(), ic)
    for t in (0.0, 0.7):
        assert rel(sim.explicit_time_derivative(t), orc.advect_rhs(phi, t)) <= TOL


@pytest.mark.parametrize("p,basis", CASES_3D)
def test_advect_rhs_3d_missing_component(oracle, flsp, p, basis):
    # plume rolls: no y component (a zero term stands in for it)
    ic = F.perturbed_plane(seed=3)
    sim, orc, phi = make_pair(oracle, 3, (8, 9, 10), p, basis, F.plume_3d(), ic)
    for t in (0.0, 1.3):
        assert rel(sim.explicit_time_derivative(t), orc.advect_rhs(phi, t)) <= TOL


@pytest.mark.parametrize("rk", [1, 2, 3])
def test_advance_2d(oracle, flsp, rk):
    mesh = Mesh(2, (32, 32))
    sim = AdvectSimulator(mesh, 2, basis=abi.BASIS_Q, precision=abi.FP64, rk_order=rk, cfl_max=0.1)
    sim.initialize(F.zalesak_disk(), F.ccw_rotation())
    orc = oracle.Problem(2, (32, 32), 2, abi.BASIS_Q)
    orc.set_velocity(F.ccw_rotation())
    phi = orc.project(F.zalesak_disk())
    # 10 CFL-limited substeps one by one, then a multi-substep call
    for _ in range(10):
        a = sim.advance_time(0.05, compute_single_cycle=True)
        b = orc.advance(phi, 0.05, single_cycle=True, rk_order=rk, cfl_max=0.1)
        assert abs(a - b) <= 1e-15
    a = sim.advance_time(0.013, compute_single_cycle=False)
    b = orc.advance(phi, 0.013, single_cycle=False, rk_order=rk, cfl_max=0.1)
    assert abs(a - b) <= 1e-15
    assert abs(sim.get_time() - orc.clock.t) <= 1e-14
    assert rel(sim.get_solution_vector(), phi) <= 1e-11


def test_advance_3d_time_dependent(oracle, flsp):
    mesh = Mesh(3, (12, 12, 12))
    field = F.deformation_3d()
    ic = F.sphere((0.35, 0.35, 0.35), 0.15)
    sim = AdvectSimulator(mesh, 2, basis=abi.BASIS_Q, precision=abi.FP64, cfl_max=0.1)
    sim.initialize(ic, field)
    orc = oracle.Problem(3, (12, 12, 12), 2, abi.BASIS_Q)
    orc.set_velocity(field)
    phi = orc.project(ic)
    a = sim.advance_time(0.2, compute_single_cycle=False)
    b = orc.advance(phi, 0.2, single_cycle=False, cfl_max=0.1)
    assert abs(a - b) <= 1e-15
    assert orc.clock.n_substeps > 3
    assert rel(sim.get_solution_vector(), phi) <= 1e-11


@pytest.mark.parametrize("dim,p,basis", [(2, 1, abi.BASIS_P), (2, 2, abi.BASIS_Q), (2, 3, abi.BASIS_Q),
                                         (3, 1, abi.BASIS_Q), (3, 2, abi.BASIS_P), (3, 2, abi.BASIS_Q)])
def test_hj_gradients(oracle, flsp, dim, p, basis):
    n = (20, 18) if dim == 2 else (8, 7, 6)
    ic = F.zalesak_disk() if dim == 2 else F.sphere((0.4, 0.5, 0.45), 0.3)
    field = F.ccw_rotation() if dim == 2 else F.deformation_3d()
    sim, orc, phi = make_pair(oracle, dim, n, p, basis, field, ic)
    gl, gr = ReinitSimulatorLDG(sim.problem).local_left_right_gradients()
    ol, orr = orc.hj_gradients(phi)
    assert rel(gl, ol) <= TOL
    assert rel(gr, orr) <= TOL


@pytest.mark.parametrize("dim,p,basis,mode", [
    (2, 1, abi.BASIS_P, abi.REINIT_BAND), (2, 2, abi.BASIS_Q, abi.REINIT_FIXED),
    (3, 1, abi.BASIS_Q, abi.REINIT_BAND), (3, 2, abi.BASIS_Q, abi.REINIT_FIXED),
    (3, 2, abi.BASIS_P, abi.REINIT_FIXED)])
def test_reinit(oracle, flsp, dim, p, basis, mode):
    n = (24, 24) if dim == 2 else (10, 10, 10)
    if dim == 2:
        ic = F.sphere((0.5137, 0.4871), 0.3) + F.sphere((0.3071, 0.3529), 0.15)
    else:
        ic = F.sphere((0.4, 0.5, 0.45), 0.25) + F.sphere((0.7, 0.6, 0.5), 0.2)
    field = F.ccw_rotation() if dim == 2 else F.deformation_3d()
    sim, orc, phi = make_pair(oracle, dim, n, p, basis, field, ic)
    o = abi.default_reinit_opts(mode=mode, n_pseudo_steps=5)
    nit = ReinitSimulatorLDG(sim.problem).run_iteration(o)
    st, nit_o = orc.reinit(phi, o)
    assert st == 0 and nit == nit_o and nit > 0
    assert rel(sim.get_solution_vector(), phi) <= 1e-11


@pytest.mark.parametrize("p,basis", [(1, abi.BASIS_P), (2, abi.BASIS_Q), (3, abi.BASIS_Q)])
def test_weno(oracle, flsp, p, basis):
    disk = F.zalesak_disk(center=(0.4927, 0.7481))
    sim, orc, phi = make_pair(oracle, 2, (32, 32), p, basis, F.ccw_rotation(), disk)
    flags = orc.minmod_flags(phi)
    n_gpu = ReinitSimulatorLDG(sim.problem).apply_weno_limiter()
    n_orc = orc.weno(phi)
    assert n_gpu == n_orc == int(flags.sum()) and n_orc > 0
    assert rel(sim.get_solution_vector(), phi) <= 1e-11


def test_reductions(oracle, flsp):
    ic = F.zalesak_disk()
    ls = LevelSetSurface(Mesh(2, (40, 40)), 2, basis=abi.BASIS_Q, precision=abi.FP64)
    ls.initialize(ic, F.ccw_rotation())
    orc = oracle.Problem(2, (40, 40), 2, abi.BASIS_Q)
    phi = orc.project(ic)
    ls.problem.snapshot()
    for which, ref in [(abi.RED_MASS, None), (abi.RED_MASS_ERROR, ic), (abi.RED_GRAD_DEVIATION, None),
                       (abi.RED_MAX_ABS, None), (abi.RED_L2_ERROR_IC, ic), (abi.RED_L1_INTERFACE_IC, ic),
                       (abi.RED_MASS_SHARP, None)]:
        g = ls.problem.reduce(which, ref)
        o = orc.reduce(which, phi, None, ref)
        # the relative mass error is a difference of two O(1) masses
        scale = 1.0 if which == abi.RED_MASS_ERROR else max(abs(o), 1e-12)
        assert abs(g - o) <= 1e-12 * scale, (which, g, o)
    assert ls.problem.reduce(abi.RED_L1_INTERFACE) == 0.0
    assert ls.problem.reduce(abi.RED_MEAN_ABS_DIFF) == 0.0


def test_host_cell_order(oracle, flsp):
    order = dealii_hypercube_order(2, 2, 4)          # 32 x 32 cells, deal.II order
    mesh = Mesh(2, (32, 32), host_cell_order=order)
    sim = AdvectSimulator(mesh, 1, basis=abi.BASIS_P, precision=abi.FP64)
    sim.initialize(F.zalesak_disk(), F.ccw_rotation())
    orc = oracle.Problem(2, (32, 32), 1, abi.BASIS_P)
    orc.set_velocity(F.ccw_rotation())
    phi = orc.project(F.zalesak_disk())
    nb = 3
    host = phi.reshape(-1, nb)[order].reshape(-1)    # oracle (lexicographic) -> host order
    assert rel(sim.get_solution_vector(), host) <= TOL
    rhs = orc.advect_rhs(phi, 0.1).reshape(-1, nb)[order].reshape(-1)
    assert rel(sim.explicit_time_derivative(0.1), rhs) <= TOL
    # set_state in host order round-trips
    sim.problem.set_state(host * 2.0)
    assert rel(sim.get_solution_vector(), host * 2.0) == 0.0


def test_ls_advance(oracle, flsp):
    mesh = Mesh(2, (24, 24))
    ctl = abi.default_ls_opts(reinit_frequency=4,
                              reinit=abi.default_reinit_opts(mode=abi.REINIT_FIXED, n_pseudo_steps=3))
    ls = LevelSetSurface(mesh, 1, basis=abi.BASIS_Q, precision=abi.FP64, cfl_max=0.1, control=ctl)
    ls.initialize(F.zalesak_disk(), F.ccw_rotation())
    orc = oracle.Problem(2, (24, 24), 1, abi.BASIS_Q)
    orc.set_velocity(F.ccw_rotation())
    phi = orc.project(F.zalesak_disk())
    a = ls.advance_time(0.05)
    b = orc.ls_advance(phi, 0.05, ctl, cfl_max=0.1)
    assert abs(a - b) <= 1e-15
    assert rel(ls.get_solution_vector(), phi) <= 1e-11


def test_graph_run_matches_stepwise(flsp):
    """flsp_ls_run_steps (CUDA graph replay) == the same steps issued one by one."""
    ctl = abi.default_ls_opts(reinit_frequency=3,
                              reinit=abi.default_reinit_opts(mode=abi.REINIT_FIXED, n_pseudo_steps=2))
    outs = []
    for use_graph in (True, False):
        ls = LevelSetSurface(Mesh(2, (32, 32)), 2, basis=abi.BASIS_Q, precision=abi.FP64, cfl_max=0.1,
                             control=ctl)
        ls.initialize(F.zalesak_disk(), F.ccw_rotation())
        if use_graph:
            ls.run_steps(7)
        else:
            for _ in range(7):
                ls.advance_time(1.0, compute_single_step=True)
        outs.append(ls.get_solution_vector())
    assert rel(outs[0], outs[1]) == 0.0


def test_fp32_mode_close(oracle, flsp):
    ic = F.sphere((0.35, 0.35, 0.35), 0.15)
    sims = []
    for prec in (abi.FP32, abi.FP64):
        s = AdvectSimulator(Mesh(3, (16, 16, 16)), 2, basis=abi.BASIS_Q, precision=prec, cfl_max=0.1)
        s.initialize(ic, F.deformation_3d())
        s.advance_steps(20)
        sims.append(s.get_solution_vector())
    assert rel(sims[0], sims[1]) <= 1e-4


def test_fp32_mode_close_multiterm(oracle, flsp):
    ic = F.sphere((0.35, 0.35, 0.35), 0.15)
    sims = []
    for prec in (abi.FP32, abi.FP64):
        s = AdvectSimulator(Mesh(3, (12, 12, 12)), 2, basis=abi.BASIS_Q, precision=prec, cfl_max=0.1)
        s.initialize(ic, drifting_deformation_3d())
        s.advance_steps(20)
        sims.append(s.get_solution_vector())
    assert rel(sims[0], sims[1]) <= 1e-4


def test_nonfinite_rejected(flsp):
    from felspa_b200.lib import FlspError
    sim = AdvectSimulator(Mesh(2, (8, 8)), 1, basis=abi.BASIS_Q)
    bad = np.zeros(sim.n_dofs)
    bad[5] = np.nan
    with pytest.raises(FlspError) as e:
        sim.problem.set_state(bad)
    assert e.value.code == abi.FLSP_ERR_NONFINITE


@pytest.mark.parametrize("dim,p,basis,mode", [(2, 1, abi.BASIS_P, abi.REINIT_BAND), (2, 2, abi.BASIS_Q, abi.REINIT_FIXED),
                                              (3, 2, abi.BASIS_Q, abi.REINIT_FIXED)])
def test_reinit_viscosity(oracle, flsp, dim, p, basis, mode):
    """LDG artificial viscosity (the reference Zalesak test uses nu = 0.001)"""
    n = (20, 20) if dim == 2 else (8, 8, 8)
    if dim == 2:
        ic = F.sphere((0.5137, 0.4871), 0.3) + F.sphere((0.3071, 0.3529), 0.15)
    else:
        ic = F.sphere((0.4137, 0.5071, 0.4529), 0.25)
    field = F.ccw_rotation() if dim == 2 else F.deformation_3d()
    sim, orc, phi = make_pair(oracle, dim, n, p, basis, field, ic)
    o = abi.default_reinit_opts(mode=mode, n_pseudo_steps=4, viscosity=0.001, cfl_max=0.3)
    nit = ReinitSimulatorLDG(sim.problem).run_iteration(o)
    st, nit_o = orc.reinit(phi, o)
    assert st == 0 and nit == nit_o and nit > 0
    assert rel(sim.get_solution_vector(), phi) <= 1e-11


@pytest.mark.parametrize("name", ["zalesak_p1_rhs", "zalesak_q2_rk3", "circles_q2_reinit", "sphere_q2_3d_rhs",
                                  "sphere_p2_3d_grad", "circles_q2_curvature"])
def test_golden_fixtures(flsp, name):
    """the library against the committed oracle fixtures (tests/golden/)"""
    import importlib.util
    import os
    golden = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(golden, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    dim, n, p, basis, field, ic, what = mg.cases()[name]
    ref = np.load(os.path.join(golden, name + ".npz"))
    sim = AdvectSimulator(Mesh(dim, n), p, basis=basis, precision=abi.FP64, cfl_max=0.1)
    sim.initialize(ic, field)
    assert rel(sim.get_solution_vector(), ref["phi0"]) <= TOL
    if what == "rhs":
        got = sim.explicit_time_derivative(0.2)
    elif what == "advance":
        sim.advance_time(0.05)
        got = sim.get_solution_vector()
        assert abs(sim.get_time() - ref["t"][0]) <= 1e-15
    elif what == "reinit":
        ReinitSimulatorLDG(sim.problem).run_iteration(abi.default_reinit_opts(mode=abi.REINIT_FIXED,
                                                                              n_pseudo_steps=3))
        got = sim.get_solution_vector()
    elif what == "curvature":
        got = sim.problem.curvature(abi.CURV_REFERENCE)
        assert rel(sim.problem.curvature(abi.CURV_NEIGHBOUR), ref["result_neighbour"]) <= 1e-11
    else:
        gl, gr = ReinitSimulatorLDG(sim.problem).local_left_right_gradients()
        got = np.concatenate([gl.ravel(), gr.ravel()])
    assert rel(got, ref["result"]) <= 1e-11


def test_cpp_driver_matches_python(flsp):
    """the C++ facade (include/flsp_dg.hpp) driving the Zalesak test, against
    the same run through the Python host mirror"""
    import os
    import re
    import subprocess
    import math
    exe = os.path.join(os.path.dirname(flsp.LIB_PATH), "examples", "zalesak_disk.bin")
    out = subprocess.run([exe, "6", "0.001"], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    vals = dict(re.findall(r"^(mean \|coeff - initial\|) (\S+)$", out.stdout, re.M))
    mesh = Mesh(2, (64, 64), (-50, -50), (50, 50), host_cell_order=dealii_hypercube_order(2, 2, 5))
    ctl = abi.default_ls_opts(reinit_frequency=40, reinit=abi.default_reinit_opts(cfl_max=0.3, viscosity=0.001))
    ls = LevelSetSurface(mesh, 1, basis=abi.BASIS_P, precision=abi.FP64, control=ctl)
    disk = F.zalesak_reference()
    ls.initialize(disk, F.rigid_rotation((0.0, 0.0), math.pi / 314.0))
    init = ls.get_solution_vector()
    for _ in range(6):
        ls.advance_time(1.0)
    mine = ls.compute_error(init)
    assert abs(float(vals["mean |coeff - initial|"]) - mine) <= 1e-6 * mine
