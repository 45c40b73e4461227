"""Groups: the reinit periods of several independent problems (2D and 3D,
different sizes and degrees) replayed from one CUDA graph give every
problem exactly the state it gets alone (the same kernels with the same
arguments on a different stream: bit-identical), and a group of one
problem reproduces flsp_ls_run_steps."""
import ctypes as C

import numpy as np
import pytest

from felspa_b200 import abi, fields as F
from felspa_b200.batch import Group
from felspa_b200.level_set import Mesh, Problem
from felspa_b200.lib import check, load

pytestmark = pytest.mark.gpu

MEMBERS = [
    (Mesh(3, (12, 12, 12)), 2, F.deformation_3d(), F.sphere((0.35, 0.35, 0.35), 0.15)),
    (Mesh(3, (10, 10, 10)), 1, F.plume_3d(), F.perturbed_plane(seed=5)),
    (Mesh(2, (24, 24)), 2, F.ccw_rotation(), F.zalesak_disk()),
]


def control(narrow_band=0):
    return abi.default_ls_opts(reinit_frequency=4,
                               reinit=abi.default_reinit_opts(mode=abi.REINIT_FIXED, n_pseudo_steps=3,
                                                              narrow_band=narrow_band))


def make(prec):
    out = []
    for mesh, p, vel, ic in MEMBERS:
        pb = Problem(mesh, p, basis=abi.BASIS_Q, precision=prec, cfl_max=0.1)
        pb.set_velocity(vel)
        pb.project(ic)
        out.append(pb)
    return out


@pytest.mark.parametrize("prec,narrow_band", [(abi.FP64, 0), (abi.FP32, 0), (abi.FP64, 1)])
def test_group_matches_each_problem_alone(prec, narrow_band):
    ctl = control(narrow_band)
    grouped, alone = make(prec), make(prec)
    g = Group(grouped)
    g.run_periods(3, ctl)
    for pb in alone:
        check(load().flsp_ls_run_steps(pb.h, C.byref(ctl), 3 * 4))
        pb.sync()
    for a, b in zip(grouped, alone):
        sa, sb = a.get_state(), b.get_state()
        assert np.all(np.isfinite(sa))
        assert np.array_equal(sa, sb)
        assert a.get_time() == b.get_time() > 0.0
    g.close()
    for pb in grouped + alone:
        pb.close()


def test_group_orders_member_work():
    """work the caller enqueues on a member's stream after the group's
    periods sees their result, and a member inside a period is refused"""
    ctl = control()
    pbs = make(abi.FP64)
    g = Group(pbs[:2])
    g.run_periods(1, ctl, sync=False)
    s0 = pbs[0].get_state()          # ordered after the group's work
    g.sync()
    assert np.array_equal(s0, pbs[0].get_state())
    # a member one substep into a period cannot join a period replay
    ls = abi.default_ls_opts(reinit_frequency=4, reinit=abi.default_reinit_opts(mode=abi.REINIT_FIXED))
    check(load().flsp_ls_run_steps(pbs[1].h, C.byref(ls), 1))
    with pytest.raises(Exception):
        g.run_periods(1, ctl)
    g.close()
    for pb in pbs:
        pb.close()


def test_group_learned_periods_match_each_problem_alone():
    """learned periods of a group (the members' network passes one after
    another on the network's stream) equal each member's own graph-replayed
    learned periods"""
    from felspa_b200.learned import MLP, default_learned_opts
    net = MLP(device=0, seed=4, dim=3)
    lo = default_learned_opts()

    def members():
        out = []
        for n, seed in ((12, 5), (10, 6)):
            pb = Problem(Mesh(3, (n, n, n)), 2, basis=abi.BASIS_Q, precision=abi.FP32, cfl_max=0.1)
            pb.set_velocity(F.deformation_3d())
            pb.project(F.sphere((0.4, 0.5, 0.5), 0.2))
            out.append(pb)
        return out

    grouped, alone = members(), members()
    g = Group(grouped)
    g.run_periods_learned(net, lo, 4, 3)
    for pb in alone:
        check(load().flsp_ls_run_steps_learned(pb.h, net.h, C.byref(lo), 4, 12))
        pb.sync()
    for a, b in zip(grouped, alone):
        sa, sb = a.get_state(), b.get_state()
        assert np.all(np.isfinite(sa))
        assert np.array_equal(sa, sb)
    g.close()
    for pb in grouped + alone:
        pb.close()
    net.close()
