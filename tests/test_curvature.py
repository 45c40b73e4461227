"""CPU oracle of the curvature estimate (LevelSetSurface::CurvatureEstimator,
include/felspa/level_set/src/level_set.implement.h:600-812): known answers
for both face-term modes.

FLSP_CURV_REFERENCE restates the reference, whose face loop binds the
exterior face term to the face's owner (copy_ex.reinit(cell), :731): the
owner's two face terms cancel on the constant mode, so the cell means vanish
away from the boundary.  FLSP_CURV_NEIGHBOUR hands that term to the
neighbour, a standard DG divergence of grad phi / |grad phi|: its cell means
approach the mean curvature (1/r in 2D, 2/r in 3D for a sphere).
"""
import math

import numpy as np
import pytest

from felspa_b200 import abi, fields as F


def band_means(orc, kappa, dim, n, centre, r):
    """cell means of kappa over the cells whose centre lies within half a
    cell of the sphere |x - centre| = r"""
    k = kappa.reshape(-1, orc.nb)[:, 0]
    h = 1.0 / n
    idx = np.arange(n ** dim)
    X = [(idx % n + 0.5) * h, (idx // n % n + 0.5) * h]
    if dim == 3:
        X.append((idx // (n * n) + 0.5) * h)
    d = np.sqrt(sum((X[e] - centre[e]) ** 2 for e in range(dim)))
    return k[np.abs(d - r) < 0.5 * h]


@pytest.mark.parametrize("n", [32, 64])
def test_neighbour_mode_circle_curvature(oracle, n):
    orc = oracle.Problem(2, (n, n), 2, abi.BASIS_Q)
    phi = orc.project(F.sphere((0.5, 0.5), 0.25))
    m = band_means(orc, orc.curvature(phi, to_neighbour=True), 2, n, (0.5, 0.5), 0.25)
    assert abs(np.mean(m) - 4.0) < (0.1 if n == 32 else 0.035)   # 0.087 / 0.027 / 0.012 at 32 / 64 / 128


def test_neighbour_mode_sphere_curvature(oracle):
    n = 24
    orc = oracle.Problem(3, (n, n, n), 2, abi.BASIS_Q)
    phi = orc.project(F.sphere((0.5, 0.5, 0.5), 0.3))
    m = band_means(orc, orc.curvature(phi, to_neighbour=True), 3, n, (0.5, 0.5, 0.5), 0.3)
    assert abs(np.mean(m) - 2.0 / 0.3) < 0.1


def test_equal_normals_carry_no_face_flux(oracle):
    """an exactly represented linear field has the same normal on both sides
    of every face: the reference's shock speed is 0 (or 0/0) there, so the
    face flux is 0 and only the cell term -int grad psi . n remains; for
    phi = y - 0.37 that is 2 sqrt(3) / h on the L_1(y) mode, in both modes"""
    n = 16
    orc = oracle.Problem(2, (n, n), 1, abi.BASIS_Q)
    phi = orc.project(F.height_function(1, 0.37, []))
    for tn in (False, True):
        k = orc.curvature(phi, to_neighbour=tn).reshape(n, n, orc.nb)
        inner = k[1:-1, 1:-1]
        np.testing.assert_allclose(inner[..., 2], 2 * math.sqrt(3) * n, rtol=1e-12)
        assert np.max(np.abs(inner[..., [0, 1, 3]])) < 1e-12


def test_reference_mode_cell_means_vanish_inside(oracle):
    n = 32
    orc = oracle.Problem(2, (n, n), 2, abi.BASIS_Q)
    phi = orc.project(F.sphere((0.5, 0.5), 0.25))
    k = orc.curvature(phi).reshape(n, n, orc.nb)
    assert np.max(np.abs(k[1:-1, 1:-1, 0])) < 1e-12
    assert np.max(np.abs(k[1:-1, 1:-1, 1:])) > 1e-3   # the higher modes carry the face terms


def test_reference_mode_depends_on_cell_order(oracle):
    """which cell owns a face follows the CellId order; the neighbour mode
    does not depend on it"""
    n = 8
    orc = oracle.Problem(2, (n, n), 2, abi.BASIS_Q)
    phi = np.random.default_rng(3).standard_normal(orc.n_dofs)
    rev = np.arange(n * n, dtype=np.int64)[::-1].copy()
    a, b = orc.curvature(phi), orc.curvature(phi, order=rev)
    assert np.max(np.abs(a - b)) > 1e-3
    c, d = orc.curvature(phi, to_neighbour=True), orc.curvature(phi, order=rev, to_neighbour=True)
    np.testing.assert_array_equal(c, d)


def test_neighbour_mode_boundary_rows_of_a_plane(oracle):
    """phi = y: n = (0, 1); interior faces carry no flux (equal normals),
    the boundary rows y = 0 and y = 1 get n . normal = -1 / +1 over a face
    of length h, so their cell means are 1 / h and the others 0"""
    n = 8
    orc = oracle.Problem(2, (n, n), 1, abi.BASIS_Q)
    ic = F.height_function(1, 0.0, [])
    phi = orc.project(ic)
    k = orc.curvature(phi, to_neighbour=True).reshape(n, n, orc.nb)
    h = 1.0 / n
    np.testing.assert_allclose(k[0, :, 0], 1.0 / h, rtol=1e-12)
    np.testing.assert_allclose(k[-1, :, 0], 1.0 / h, rtol=1e-12)
    assert np.max(np.abs(k[1:-1, :, 0])) < 1e-12
