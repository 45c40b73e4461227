"""GPU curvature estimate (flsp_curvature) against the CPU oracle's
restatement of LevelSetSurface::CurvatureEstimator::estimate
(include/felspa/level_set/src/level_set.implement.h:600-812), in both
face-term modes, with and without a deal.II cell order (the CellId order
decides which cell owns a face in the reference mode).

Bar: relative max-norm difference <= 1e-11 (FP64 arithmetic on both sides;
FP32 states are compared on the same FP32-rounded coefficients).
"""
import numpy as np
import pytest

from felspa_b200 import abi, fields as F
from felspa_b200.level_set import LevelSetSurface, Mesh, Problem, dealii_hypercube_order

pytestmark = pytest.mark.gpu

TOL = 1e-11


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def to_lex(x_host, order, nb):
    lex = np.empty_like(x_host).reshape(-1, nb)
    lex[order] = x_host.reshape(-1, nb)
    return lex.ravel()


CASES = [
    (2, (16, 16), 1, abi.BASIS_P, abi.FP64, False),
    (2, (16, 16), 2, abi.BASIS_Q, abi.FP64, True),
    (2, (16, 16), 3, abi.BASIS_Q, abi.FP64, True),
    (2, (16, 16), 3, abi.BASIS_P, abi.FP64, False),
    (2, (16, 16), 2, abi.BASIS_Q, abi.FP32, True),
    (3, (8, 8, 8), 1, abi.BASIS_Q, abi.FP64, True),
    (3, (8, 8, 8), 2, abi.BASIS_Q, abi.FP64, False),
    (3, (8, 8, 8), 2, abi.BASIS_P, abi.FP64, True),
    (3, (8, 8, 8), 2, abi.BASIS_Q, abi.FP32, False),
]


@pytest.mark.parametrize("dim,n,p,basis,prec,dealii", CASES)
@pytest.mark.parametrize("mode", [abi.CURV_REFERENCE, abi.CURV_NEIGHBOUR])
@pytest.mark.parametrize("field", ["sdf", "random"])
def test_curvature_vs_oracle(flsp, oracle, dim, n, p, basis, prec, dealii, mode, field):
    order = dealii_hypercube_order(dim, 2, int(np.log2(n[0] // 2))) if dealii else None
    pr = Problem(Mesh(dim, n, host_cell_order=order), p, basis=basis, precision=prec)
    orc = oracle.Problem(dim, n, p, basis)
    if field == "sdf":
        centre = (0.47, 0.53, 0.51)[:dim]
        lex = orc.project(F.sphere(centre, 0.3))
    else:
        lex = np.random.default_rng(7 + dim + p).standard_normal(orc.n_dofs)
    if prec == abi.FP32:
        lex = lex.astype(np.float32).astype(np.float64)
    host = lex.reshape(-1, orc.nb)[order].ravel() if dealii else lex
    pr.set_state(host)
    got = pr.curvature(mode)
    got_lex = to_lex(got, order, orc.nb) if dealii else got
    want = orc.curvature(lex, order=order, to_neighbour=(mode == abi.CURV_NEIGHBOUR))
    assert rel(got_lex, want) <= TOL
    pr.close()


def test_curvature_of_a_circle_through_the_mirror(flsp):
    """LevelSetSurface.estimate_curvature: the neighbour mode's cell means
    near the interface approach 1/r; the reference mode's vanish"""
    n = 64
    ls = LevelSetSurface(Mesh(2, (n, n)), 2, basis=abi.BASIS_Q, precision=abi.FP64)
    ls.initialize(F.sphere((0.5, 0.5), 0.25), F.ccw_rotation())
    idx = np.arange(n * n)
    d = np.hypot((idx % n + 0.5) / n - 0.5, (idx // n + 0.5) / n - 0.5)
    band = np.abs(d - 0.25) < 0.5 / n
    kn = ls.estimate_curvature(abi.CURV_NEIGHBOUR).reshape(-1, 9)[:, 0]
    kr = ls.estimate_curvature(abi.CURV_REFERENCE).reshape(-1, 9)[:, 0]
    assert abs(np.mean(kn[band]) - 4.0) < 0.035
    inner = (idx % n > 0) & (idx % n < n - 1) & (idx // n > 0) & (idx // n < n - 1)
    assert np.max(kr[inner]) < 1e-11
    ls.problem.close()


def test_curvature_rejects_bad_arguments(flsp):
    from felspa_b200.lib import FlspError
    pr = Problem(Mesh(2, (4, 4)), 1)
    with pytest.raises(FlspError):
        pr.curvature(2)
    pr.close()
