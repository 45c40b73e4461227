"""MaterialStack mixing on the device (flsp_material_mix) against the
oracle: level sets of different degrees, bases and precisions on one mesh,
every Heaviside smoothing, lexicographic and deal.II cell orders.  The
arithmetic is the same FP64 expression on the same inputs, summed in the
same order, so the bar is 1e-13 of the largest material value."""
import numpy as np
import pytest

from felspa_b200 import abi, fields as F
from felspa_b200.level_set import MaterialStack, Mesh, Problem, dealii_hypercube_order
from felspa_b200.lib import FlspError

pytestmark = pytest.mark.gpu


def make(dim, n, p, basis, prec, ic, order=None):
    pb = Problem(Mesh(dim, (n,) * dim, host_cell_order=order), p, basis=basis, precision=prec)
    pb.set_velocity(F.ccw_rotation() if dim == 2 else F.deformation_3d())
    pb.project(ic)
    return pb


@pytest.mark.parametrize("smoothing", [abi.HEAVISIDE_NONE, abi.HEAVISIDE_LINEAR, abi.HEAVISIDE_SINE])
@pytest.mark.parametrize("dim", [2, 3])
def test_mix_matches_oracle(oracle, flsp, dim, smoothing):
    n = 16 if dim == 2 else 8
    order = dealii_hypercube_order(dim, 2, 3 if dim == 2 else 2)
    if dim == 2:
        ics = [F.zalesak_disk(), F.sphere((0.3, 0.4), 0.2), F.sphere((0.6, 0.55), 0.25)]
        specs = [(2, abi.BASIS_Q, abi.FP64), (1, abi.BASIS_P, abi.FP32), (3, abi.BASIS_Q, abi.FP64)]
    else:
        ics = [F.sphere((0.35, 0.4, 0.45), 0.25), F.sphere((0.6, 0.55, 0.5), 0.3)]
        specs = [(2, abi.BASIS_Q, abi.FP32), (1, abi.BASIS_P, abi.FP64)]
    pbs = [make(dim, n, p, b, pr, ic, order) for (p, b, pr), ic in zip(specs, ics)]
    values = [4.0, -1.5, 2.25, 0.75][:len(pbs)] + [10.0]
    ms = MaterialStack()
    ms.set_background_material(values[-1])
    for v, pb in zip(values, pbs):
        ms.push(v, pb)
    for nq in (2, 4):
        got = ms.eval_scalars(nq, smoothing)
        prs, phis = [], []
        for (p, b, _), pb in zip(specs, pbs):
            pr = oracle.Problem(dim, (n,) * dim, p, b)
            # the device states, through the host cell order, back to lexicographic
            host = pb.get_state().reshape(-1, pb.dofs_per_cell)
            lex = np.empty_like(host)
            lex[order] = host
            prs.append(pr)
            phis.append(lex.ravel())
        want = oracle.material_mix(prs, phis, values, nq, smoothing, order=order)
        assert np.max(np.abs(got - want)) <= 1e-13 * 10.0
        # the materials are mixed: the value varies over the points
        assert np.ptp(got) > 1.0
    for pb in pbs:
        pb.close()


def test_mix_rejects_bad_arguments(flsp):
    a = make(2, 8, 1, abi.BASIS_Q, abi.FP64, F.sphere((0.5, 0.5), 0.2))
    b = make(2, 9, 1, abi.BASIS_Q, abi.FP64, F.sphere((0.5, 0.5), 0.2))
    ms = MaterialStack(1.0)
    ms.push(2.0, a)
    ms.push(3.0, b)
    with pytest.raises(FlspError, match="share mesh"):
        ms.eval_scalars(2)
    ms = MaterialStack(1.0)
    ms.push(2.0, a)
    for nq in (0, abi.MAX_MIX_QPTS + 1):
        with pytest.raises(FlspError, match="n_qpts_1d"):
            ms.eval_scalars(nq)
    with pytest.raises(FlspError, match="smoothing"):
        ms.eval_scalars(2, smoothing=7)
    no_background = MaterialStack()
    no_background.push(1.0, a)
    with pytest.raises(ValueError, match="background"):
        no_background.eval_scalars(2)
    a.close()
    b.close()
