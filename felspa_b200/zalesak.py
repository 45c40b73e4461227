"""The Zalesak slotted-disk run of the 2D workload on the GPU path, as the
reference's only level-set driver runs it (ZalesakDiskTest::run,
tests/test_zalesak_disk.cc:136-174: advance the level set for one full
revolution with periodic reinitialisation, then report the errors,
:177-213), on the unit square: 128^2 cells, degree 1 (Q or P basis), disk
r = 0.15 at (0.5, 0.75) with a 0.05 x 0.25 slot, counter-clockwise rotation
u = 2 pi (0.5 - y, x - 0.5) (period 1), SSP-RK3 at CFL 0.1, a fixed
5-pseudo-step reinitialisation every 10 substeps.

Reported: the L1 interface error against the initial shape (sharp
Heaviside at QGauss(p+2) points) and the area change (smoothed Heaviside,
LevelSetSurface::compute_mass_error's integrand, level_set.implement.h:
215-256), both FP64 device reductions.
"""
import time

from . import abi, fields as F
from .level_set import LevelSetSurface, Mesh


def revolution_control(viscosity=0.0, n_pseudo_steps=5, reinit_every=10):
    ro = abi.default_reinit_opts(mode=abi.REINIT_FIXED, n_pseudo_steps=n_pseudo_steps, band_width_coeff=6.0,
                                 viscosity=viscosity)
    return abi.default_ls_opts(reinit_frequency=reinit_every, reinit=ro)


def revolution(basis=abi.BASIS_Q, viscosity=0.0, precision=abi.FP64, n=128, degree=1, t_end=1.0, device=0):
    """One run of LevelSetSurface::advance_time(t_end) from the projected
    slotted disk; returns the run's outputs and its wall time."""
    ic = F.zalesak_disk()
    ls = LevelSetSurface(Mesh(2, (n, n)), degree, basis=basis, precision=precision, cfl_max=0.1,
                         device=device, control=revolution_control(viscosity))
    ls.initialize(ic, F.ccw_rotation())
    area0 = ls.integrate_mass()
    ls.problem.sync()
    t0 = time.perf_counter()
    ls.advance_time(t_end)
    ls.problem.sync()
    wall = time.perf_counter() - t0
    steps = ls.problem.get_step_count()
    area1 = ls.integrate_mass()
    out = {"n_dofs": ls.n_dofs, "t_end": ls.get_time(), "substeps": steps,
           "l1_interface_error": ls.interface_error_l1(ic), "area_initial": area0,
           "area_change_rel": (area1 - area0) / area0, "wall_s": wall,
           "dof_steps_per_s": ls.n_dofs * steps / wall, "state": ls.get_solution_vector()}
    ls.problem.close()
    return out
