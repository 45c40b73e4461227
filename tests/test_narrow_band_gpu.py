"""Compute-restricted narrow band of the reinitialisation (not in the
reference, whose sweep covers every cell): only tiles within two cells of
the band |mean phi0| <= band_cells * min_diam are swept, cells outside the
band keep phi0."""
import ctypes as C

import numpy as np
import pytest

from felspa_b200 import abi, fields as F
from felspa_b200.level_set import LevelSetSurface, Mesh, Problem
from felspa_b200.lib import check, load

pytestmark = pytest.mark.gpu


def reinit(pb, **kw):
    o = abi.default_reinit_opts(mode=abi.REINIT_FIXED, n_pseudo_steps=8)
    for k, v in kw.items():
        setattr(o, k, v)
    nit = C.c_int(0)
    check(load().flsp_reinit(pb.h, C.byref(o), C.byref(nit)))
    return pb.get_state()


def problem(dim, n, p, basis, prec=abi.FP64):
    pb = Problem(Mesh(dim, n), p, basis=basis, precision=prec, cfl_max=0.1)
    if dim == 2:
        pb.set_velocity(F.ccw_rotation())
        pb.project(F.zalesak_disk(center=(0.4927, 0.7481)))
    else:
        pb.set_velocity(F.deformation_3d())
        pb.project(F.sphere((0.35, 0.35, 0.35), 0.15))
    check(load().flsp_advance_steps(pb.h, 15, 1e30))
    return pb


@pytest.mark.parametrize("dim,n,p,basis,visc", [
    (2, (40, 36), 2, abi.BASIS_Q, 0.0), (2, (40, 36), 1, abi.BASIS_P, 0.0), (2, (32, 32), 2, abi.BASIS_Q, 1e-3),
    (3, (12, 12, 12), 2, abi.BASIS_Q, 0.0)])
def test_band_covering_everything_equals_full_sweep(dim, n, p, basis, visc):
    pb = problem(dim, n, p, basis)
    pre = pb.get_state()
    full = reinit(pb, viscosity=visc)
    pb.set_state(pre)
    nb = reinit(pb, viscosity=visc, narrow_band=1, band_cells=1e9)
    assert np.array_equal(full, nb)
    pb.close()


@pytest.mark.parametrize("dim,n,p,basis,visc", [
    (2, (64, 64), 2, abi.BASIS_Q, 0.0), (2, (64, 64), 2, abi.BASIS_Q, 1e-3), (3, (24, 24, 24), 2, abi.BASIS_Q, 0.0)])
def test_band_keeps_outside_and_tracks_full_sweep(dim, n, p, basis, visc):
    pb = problem(dim, n, p, basis)
    pre = pb.get_state()
    nbp = pre.size // int(np.prod(n))
    full = reinit(pb, viscosity=visc).reshape(-1, nbp)
    pb.set_state(pre)
    band = 4.0
    got = reinit(pb, viscosity=visc, narrow_band=1, band_cells=band).reshape(-1, nbp)
    p0 = pre.reshape(-1, nbp)
    diam = np.sqrt(dim) / n[0]
    inside = np.abs(p0[:, 0]) <= band * diam
    assert inside.sum() > 0 and (~inside).sum() > 0
    assert np.array_equal(got[~inside], p0[~inside])
    # inside the band: the sweep's own change, up to the band-limited CFL
    # estimate and the frozen outside, within 5 % of the full sweep's change
    ch_full = np.abs(full[inside] - p0[inside]).max()
    assert np.abs(got[inside] - full[inside]).max() <= 0.05 * ch_full + 1e-12
    pb.close()


def test_graph_run_matches_stepwise_narrow_band():
    ctl = abi.default_ls_opts(reinit_frequency=3,
                              reinit=abi.default_reinit_opts(mode=abi.REINIT_FIXED, n_pseudo_steps=2))
    ctl.reinit.narrow_band = 1
    ctl.reinit.band_cells = 3.0
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
    assert np.array_equal(outs[0], outs[1])
