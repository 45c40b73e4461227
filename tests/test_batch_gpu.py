"""Batched problems: the persistent batched launches (one per RK stage /
reinit pseudo-step for every problem) give each problem the result it gets
alone.  The batch's tile shapes may differ from a single problem's, which
moves a face's flux to the other cell of the face for some faces (a
rounding-level difference), so the bar is 1e-12 relative in FP64."""
import numpy as np
import pytest

from felspa_b200 import abi
from felspa_b200.batch import uneven_batch_instances, make_batch
from felspa_b200.level_set import Mesh, Problem

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def control(limiter=-1):
    return abi.default_ls_opts(reinit_frequency=10,
                               reinit=abi.default_reinit_opts(mode=abi.REINIT_FIXED, n_pseudo_steps=3,
                                                              limiter=limiter))


@pytest.mark.parametrize("limiter", [-1, 0])
def test_batch_matches_single_problems(limiter):
    inst = uneven_batch_instances(6, n_min=16, n_max=40)
    b = make_batch(inst, precision=abi.FP64)
    tune = b.autotune()
    b.run_steps(25, control(limiter))
    for d, pb in zip(inst, b.problems):
        single = Problem(Mesh(2, (d["n"], d["n"])), d["degree"], basis=abi.BASIS_Q, precision=abi.FP64,
                         cfl_max=0.1)
        single.set_velocity(d["velocity"])
        single.project(d["ic"])
        from felspa_b200.lib import check, load
        import ctypes as C
        ctl = control(limiter)
        check(load().flsp_ls_run_steps(single.h, C.byref(ctl), 25))
        single.sync()
        ref = single.get_state()
        got = pb.get_state()
        assert abs(pb.get_time() - single.get_time()) <= 1e-14
        assert rel(got, ref) <= 1e-12, (d["n"], d["degree"], rel(got, ref))
        single.close()
    assert tune["adv_tile"] in [(32, 8), (16, 16), (16, 8), (8, 8)]
    assert all(v > 0 for v in tune["adv_ms"].values())
    b.close()


def test_batch_fp32_close_to_fp64():
    inst = uneven_batch_instances(5, n_min=16, n_max=48)
    outs = []
    for prec in (abi.FP32, abi.FP64):
        b = make_batch(inst, precision=prec)
        b.run_steps(20, control())
        outs.append([p.get_state() for p in b.problems])
        b.close()
    for a, r in zip(*outs):
        assert rel(a, r) <= 1e-4
