"""GPU: the stage-kernel tile autotuner (flsp_autotune).  It keeps the
state and the clock, picks one of the shapes it timed, and a run with the
picked tile gives the run with the default tile's result (the per-cell
arithmetic does not depend on the tile: interior and tile-boundary faces go
through the same flux routine with the same operands)."""
import math

import numpy as np
import pytest

from felspa_b200 import abi, fields as F
from felspa_b200.level_set import LevelSetSurface, Mesh

pytestmark = pytest.mark.gpu


def make(dim, n, p, prec):
    ctl = abi.default_ls_opts(reinit_frequency=5,
                              reinit=abi.default_reinit_opts(mode=abi.REINIT_FIXED, n_pseudo_steps=2))
    ls = LevelSetSurface(Mesh(dim, (n,) * dim), p, basis=abi.BASIS_Q, precision=prec, cfl_max=0.1,
                         control=ctl)
    if dim == 3:
        ls.initialize(F.sphere((0.35, 0.35, 0.35), 0.15), F.deformation_3d())
    else:
        ls.initialize(F.zalesak_disk(), F.ccw_rotation())
    return ls


@pytest.mark.parametrize("dim,n,p,prec", [(3, 16, 2, abi.FP64), (3, 24, 2, abi.FP32), (2, 64, 2, abi.FP32),
                                          (2, 48, 3, abi.FP64)])
def test_autotune_keeps_results(flsp, dim, n, p, prec):
    a, b = make(dim, n, p, prec), make(dim, n, p, prec)
    s0, t0 = a.problem.get_state(), a.get_time()
    tile, cands = a.problem.autotune(reps=3)
    assert tile in cands and math.isfinite(cands[tile])
    assert cands[tile] == min(v for v in cands.values() if math.isfinite(v))
    assert a.problem.stage_tile() == tile
    np.testing.assert_array_equal(a.problem.get_state(), s0)
    assert a.get_time() == t0
    a.run_steps(10)
    b.run_steps(10)
    assert a.get_time() == b.get_time()
    np.testing.assert_array_equal(a.problem.get_state(), b.problem.get_state())
    a.problem.close()
    b.problem.close()
