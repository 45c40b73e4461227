"""Known-answer tests of the CPU FP64 oracle (no GPU).

The reference holds no golden vectors for this path, so the oracle is
pinned by analytic properties of the DG scheme it restates (exact
quadrature and basis, free-stream preservation, exact transport of linear
fields by SSP-RK3, conservation, O(h^{p+1}) convergence, stationarity of an
exact signed distance under reinitialisation, conservation of the WENO
limiter, an FD-checked MLP gradient) and by the regression fixtures of
tests/golden/.
"""
import math
import os

import numpy as np
import pytest

from felspa_b200 import abi, fields as F

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_gauss_exactness(oracle):
    for n in range(1, 6):
        x, w = oracle.gauss(n)
        assert np.all(np.diff(x) > 0) and abs(w.sum() - 1.0) < 1e-15
        for k in range(2 * n):
            assert abs(np.dot(w, x ** k) - 1.0 / (k + 1)) < 1e-14


def test_legendre_orthonormal(oracle):
    n = 4
    x, w = oracle.gauss(6)
    V = np.array([oracle.legendre(n, xi)[0] for xi in x])       # (pts, n)
    G = V.T @ (w[:, None] * V)
    assert np.max(np.abs(G - np.eye(n))) < 1e-14
    # derivative of L_1 = sqrt(3)(2x-1) is 2 sqrt(3)
    assert abs(oracle.legendre(2, 0.3)[1][1] - 2 * math.sqrt(3)) < 1e-14


@pytest.mark.parametrize("basis,nb", [(abi.BASIS_P, 6), (abi.BASIS_Q, 9)])
def test_dof_order(oracle, basis, nb):
    pr = oracle.Problem(2, (2, 2), 2, basis)
    assert pr.nb == nb
    # deal.II order: x fastest; P (PolynomialSpace): (0,0),(1,0),(2,0),(0,1),(1,1),(0,2)
    val, grad = pr.shape([[0.25, 0.6, 0.0]])
    L = lambda k, t: oracle.legendre(3, t)[0][k]  # noqa: E731
    if basis == abi.BASIS_P:
        modes = [(0, 0), (1, 0), (2, 0), (0, 1), (1, 1), (0, 2)]
    else:
        modes = [(a, b) for b in range(3) for a in range(3)]
    for i, (a, b) in enumerate(modes):
        assert abs(val[i, 0] - L(a, 0.25) * L(b, 0.6)) < 1e-14


def linear_ic(axis, c):
    """phi = x_axis - c (exact signed distance of a plane)"""
    return F.height_function(axis, c, [])


@pytest.mark.parametrize("p,basis", [(1, abi.BASIS_P), (2, abi.BASIS_Q), (3, abi.BASIS_Q)])
def test_projection_reproduces_linear(oracle, p, basis):
    pr = oracle.Problem(2, (5, 4), p, basis)
    phi = pr.project(linear_ic(1, 0.3))
    nb = pr.nb
    c = phi.reshape(-1, nb)
    h = 0.25
    # cell average (mode 0) = y_centre - 0.3, y-slope mode = h / (2 sqrt 3)
    j = np.arange(20) // 5
    assert np.max(np.abs(c[:, 0] - ((j + 0.5) * h - 0.3))) < 1e-14
    iy = p + 1   # mode (a, b) = (0, 1) in both orders
    assert np.max(np.abs(c[:, iy] - h / (2 * math.sqrt(3)))) < 1e-14
    others = [k for k in range(nb) if k not in (0, iy)]
    assert np.max(np.abs(c[:, others])) < 1e-14


def test_free_stream(oracle):
    """a constant field under a divergence-free (linear) rotation stays constant"""
    pr = oracle.Problem(2, (12, 12), 2, abi.BASIS_Q)
    pr.set_velocity(F.ccw_rotation())
    phi = np.zeros(pr.n_dofs)
    phi[:: pr.nb] = 0.7
    assert np.max(np.abs(pr.advect_rhs(phi, 0.0))) < 1e-12


@pytest.mark.parametrize("dim,p,basis", [(2, 1, abi.BASIS_P), (2, 2, abi.BASIS_Q), (3, 1, abi.BASIS_Q),
                                         (3, 2, abi.BASIS_P)])
def test_linear_transport_rhs(oracle, dim, p, basis):
    """phi = x - 0.3, u constant: phi_t = -u_x exactly, boundaries included"""
    n = (6,) * dim
    pr = oracle.Problem(dim, n, p, basis)
    u = (0.7, -0.2, 0.4)[:dim]
    pr.set_velocity(F.constant(u))
    phi = pr.project(linear_ic(0, 0.3))
    rhs = pr.advect_rhs(phi, 0.0).reshape(-1, pr.nb)
    assert np.max(np.abs(rhs[:, 0] + 0.7)) < 1e-12
    assert np.max(np.abs(rhs[:, 1:])) < 1e-12


def test_rk3_exact_for_linear_in_time(oracle):
    pr = oracle.Problem(2, (8, 8), 2, abi.BASIS_Q)
    pr.set_velocity(F.constant((0.7, -0.2)))
    phi = pr.project(linear_ic(0, 0.3))
    adv = pr.advance(phi, 0.05, single_cycle=False, cfl_max=0.3)
    assert abs(adv - 0.05) < 1e-15 and pr.clock.n_substeps > 1
    exact = pr.project(linear_ic(0, 0.3 + 0.7 * 0.05))
    assert np.max(np.abs(phi - exact)) < 1e-13


def test_conservation_closed_flow(oracle):
    """zero normal flux on the box: sum of cell means times |K| is conserved"""
    pr = oracle.Problem(2, (16, 16), 2, abi.BASIS_Q)
    pr.set_velocity(F.fourier_stream_2d(seed=1000, sample=256))
    phi = pr.project(F.sphere((0.45, 0.55), 0.2))
    m0 = phi[:: pr.nb].sum()
    pr.advance(phi, 0.05, single_cycle=False, cfl_max=0.3)
    assert abs(phi[:: pr.nb].sum() - m0) < 1e-12 * max(1.0, abs(m0))


def _l2_error_interior(oracle, pr, phi, n, fexact, xmin):
    """L2 error over the cells with x >= xmin (QGauss(p+3) points)"""
    x, w = oracle.gauss(pr.degree + 3)
    X, Y = np.meshgrid(x, x, indexing="ij")
    pts = np.stack([X.ravel(), Y.ravel(), np.zeros(X.size)], -1)
    W = np.outer(w, w).ravel()
    val, _ = pr.shape(pts)                        # (nb, npts)
    c = phi.reshape(n, n, pr.nb)                  # [j][i][k]
    h = 1.0 / n
    err = 0.0
    for j in range(n):
        for i in range(n):
            if i * h < xmin:
                continue
            uh = c[j, i] @ val
            xe = (i + pts[:, 0]) * h
            ye = (j + pts[:, 1]) * h
            err += np.sum(W * (uh - fexact(xe, ye)) ** 2) * h * h
    return math.sqrt(err)


@pytest.mark.parametrize("p", [1, 2])
def test_convergence_order(oracle, p):
    """translated smooth profile: the L2 error away from the inflow boundary
    (whose zero-Neumann condition cannot carry the moving profile in)
    decreases like h^(p+1)"""
    a, u, T = 0.05, 0.5, 0.04
    errs = []
    for n in (8, 16):
        pr = oracle.Problem(2, (n, n), p, abi.BASIS_Q)
        pr.set_velocity(F.constant((u, 0.0)))
        phi = pr.project(F.height_function(1, 0.5, [(a, 1.0, 0.0, 0.0)]))
        pr.advance(phi, T, single_cycle=False, cfl_max=0.2)
        exact = lambda x, y: y - 0.5 - a * np.cos(2 * np.pi * (x - u * T))  # noqa: E731
        errs.append(_l2_error_interior(oracle, pr, phi, n, exact, 0.25))
    rate = math.log2(errs[0] / errs[1])
    assert rate > p + 0.6, (errs, rate)


def test_ldg_gradients_of_linear_field(oracle):
    pr = oracle.Problem(3, (5, 4, 3), 2, abi.BASIS_Q)
    phi = pr.project(linear_ic(1, 0.3))
    gl, gr = pr.hj_gradients(phi)
    for g in (gl, gr):
        g = g.reshape(3, -1, pr.nb)
        assert np.max(np.abs(g[1, :, 0] - 1.0)) < 1e-12
        assert np.max(np.abs(g[1, :, 1:])) < 1e-12
        assert np.max(np.abs(g[0])) < 1e-12 and np.max(np.abs(g[2])) < 1e-12


@pytest.mark.parametrize("dim", [2, 3])
def test_reinit_keeps_exact_sdf(oracle, dim):
    pr = oracle.Problem(dim, (8,) * dim, 2, abi.BASIS_Q)
    phi = pr.project(linear_ic(0, 0.43))
    ref = phi.copy()
    st, nit = pr.reinit(phi)
    assert st == 0 and nit > 0
    assert np.max(np.abs(phi - ref)) < 1e-12


def test_weno_conserves_cell_means(oracle):
    pr = oracle.Problem(2, (24, 24), 2, abi.BASIS_Q)
    phi = pr.project(F.zalesak_disk(center=(0.4927, 0.7481)))
    flags = pr.minmod_flags(phi)
    before = phi.copy()
    n = pr.weno(phi)
    assert n == flags.sum() > 0
    assert np.max(np.abs(phi[:: pr.nb] - before[:: pr.nb])) < 1e-14
    changed = np.any(phi.reshape(-1, pr.nb) != before.reshape(-1, pr.nb), axis=1)
    assert np.all(changed <= flags.astype(bool))


def test_linear_field_not_troubled(oracle):
    pr = oracle.Problem(2, (10, 10), 1, abi.BASIS_P)
    phi = pr.project(linear_ic(0, 0.37))
    assert pr.minmod_flags(phi).sum() == 0


def test_reductions_disk(oracle):
    pr = oracle.Problem(2, (64, 64), 2, abi.BASIS_Q)
    ic = F.sphere((0.5, 0.5), 0.25)
    phi = pr.project(ic)
    area = pr.reduce(abi.RED_MASS_SHARP, phi)
    assert abs(area - math.pi * 0.25 ** 2) < 2e-4
    assert abs(pr.reduce(abi.RED_MASS_ERROR, phi, ic=ic)) < 1e-6
    assert pr.reduce(abi.RED_L1_INTERFACE, phi, phi_ref=phi) == 0.0
    assert pr.reduce(abi.RED_L1_INTERFACE_IC, phi, ic=ic) < 1e-3
    plane = pr.project(linear_ic(0, 0.4))
    assert pr.reduce(abi.RED_GRAD_DEVIATION, plane) < 1e-13


def test_cfl_running_max(oracle):
    """the advection CFL estimate is a running maximum (CFLEstimator keeps velo_diam)"""
    pr = oracle.Problem(3, (4, 4, 4), 1, abi.BASIS_Q)
    pr.set_velocity(F.deformation_3d())
    phi = pr.project(F.sphere((0.35, 0.35, 0.35), 0.15))
    pr.clock.t = 1.4                       # cos(pi t / 3) smaller than at t = 0
    v14 = pr.advect_cfl(1.4)
    pr.clock.vd_run = pr.advect_cfl(0.0)
    pr.advance(phi, 1e-3, single_cycle=True, cfl_max=0.1)
    assert pr.clock.vd_run == pr.advect_cfl(0.0) > v14


def test_mlp_gradient_fd(oracle):
    rng = np.random.default_rng(0)
    widths = [5, 7, 6, 3]
    Ws = [rng.standard_normal((widths[i + 1], widths[i])) * 0.5 for i in range(3)]
    bs = [rng.standard_normal(widths[i + 1]) * 0.1 for i in range(3)]
    x = rng.standard_normal((4, 5))
    dy = rng.standard_normal((4, 3))
    dW, db = oracle.mlp_backward(Ws, bs, x, dy)
    eps = 1e-6
    for l in range(3):
        for (i, j) in [(0, 0), (1, 2), (widths[l + 1] - 1, widths[l] - 1)]:
            Wp = [W.copy() for W in Ws]
            Wm = [W.copy() for W in Ws]
            Wp[l][i, j] += eps
            Wm[l][i, j] -= eps
            fd = (np.sum(oracle.mlp_forward(Wp, bs, x) * dy) - np.sum(oracle.mlp_forward(Wm, bs, x) * dy)) / (2 * eps)
            assert abs(fd - dW[l][i, j]) < 1e-6 * max(1.0, abs(fd))
        bp = [b.copy() for b in bs]
        bp[l][0] += eps
        bm = [b.copy() for b in bs]
        bm[l][0] -= eps
        fd = (np.sum(oracle.mlp_forward(Ws, bp, x) * dy) - np.sum(oracle.mlp_forward(Ws, bm, x) * dy)) / (2 * eps)
        assert abs(fd - db[l][0]) < 1e-6 * max(1.0, abs(fd))


@pytest.mark.parametrize("name", ["zalesak_p1_rhs", "zalesak_q2_rk3", "circles_q2_reinit", "sphere_q2_3d_rhs",
                                  "sphere_p2_3d_grad", "circles_q2_curvature"])
def test_golden(oracle, name):
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    ref = np.load(os.path.join(GOLDEN, name + ".npz"))
    out = mg.compute(name, mg.cases()[name])
    for k in ref.files:
        scale = max(np.max(np.abs(ref[k])), 1e-300)
        assert np.max(np.abs(out[k] - ref[k])) <= 1e-13 * scale, k


# ----------------------------------------------------------------------
# Dirichlet boundary conditions
# ----------------------------------------------------------------------
def dof_modes(dim, p, basis):
    """(a, b, c) Legendre degrees of the in-cell DoFs in deal.II order:
    FE_DGQLegendre lexicographic, FE_DGP PolynomialSpace (c, b outer)"""
    cz = p if dim == 3 else 0
    out = []
    for c in range(cz + 1):
        for b in range(p + 1):
            for a in range(p + 1):
                if basis == abi.BASIS_P and a + b + c > p:
                    continue
                out.append((a, b, c))
    return out


def side_ids(dim, n, per_side):
    """boundary ids in flsp_mesh_desc's face order from one id per side"""
    from felspa_b200.level_set import colorized_boundary_ids
    col = colorized_boundary_ids(dim, n)
    return np.asarray([per_side[s] for s in col], dtype=np.int32)


@pytest.mark.parametrize("p,basis", [(1, abi.BASIS_Q), (2, abi.BASIS_P), (3, abi.BASIS_Q)])
def test_dirichlet_inflow_rhs_known_answer(oracle, p, basis):
    """phi = 0, u = (1, 0), Dirichlet g on the inflow side x-: the inflow
    flux -v_n psi_i g (advection.implement.h:719-741) is the only term, so
    phidot of the cells at x = 0 is g L_a(0) / h on the modes constant in
    y, L_a(0) = sqrt(2a+1) (-1)^a, and zero everywhere else; a Dirichlet
    value on the outflow side x+ changes nothing."""
    n, g = 8, 0.75
    h = 1.0 / n
    pr = oracle.Problem(2, (n, n), p, basis, boundary_ids=side_ids(2, (n, n), [7, 9, 0, 0]))
    pr.set_velocity(F.constant((1.0, 0.0)))
    pr.set_dirichlet(7, g)
    pr.set_dirichlet(9, -3.0)
    rhs = pr.advect_rhs(np.zeros(pr.n_dofs), 0.0).reshape(n, n, -1)   # [iy][ix][dof]
    want = np.zeros_like(rhs)
    for k, (a, b, c) in enumerate(dof_modes(2, p, basis)):
        if b == 0:
            want[:, 0, k] = g * math.sqrt(2 * a + 1) * (-1) ** a / h
    assert np.max(np.abs(rhs - want)) < 1e-12 * max(1.0, np.abs(want).max())


def test_dirichlet_ldg_gradients_known_answer(oracle):
    """phi = 0 with Dirichlet values on x- (g0) and x+ (g1): the left
    gradient takes the value on faces with n_x < 0 (ldg.cc:574-601), the
    right gradient on faces with n_x >= 0 (:711-735): left_x = -g0 L_a(0)/h
    at x = 0, right_x = g1 L_a(1)/h at x = 1, every other entry zero."""
    n, p, g0, g1 = 6, 2, 0.4, -1.1
    h = 1.0 / n
    pr = oracle.Problem(2, (n, n), p, abi.BASIS_Q, boundary_ids=side_ids(2, (n, n), [1, 2, 0, 0]))
    pr.set_velocity(F.constant((1.0, 0.0)))
    pr.set_dirichlet(1, g0)
    pr.set_dirichlet(2, g1)
    gl, gr = pr.hj_gradients(np.zeros(pr.n_dofs))
    wl, wr = np.zeros((2, n, n, 9)), np.zeros((2, n, n, 9))
    for k, (a, b, c) in enumerate(dof_modes(2, p, abi.BASIS_Q)):
        if b == 0:
            wl[0, :, 0, k] = -g0 * math.sqrt(2 * a + 1) * (-1) ** a / h
            wr[0, :, n - 1, k] = g1 * math.sqrt(2 * a + 1) / h
    assert np.max(np.abs(gl.reshape(2, n, n, 9) - wl)) < 1e-12 / h
    assert np.max(np.abs(gr.reshape(2, n, n, 9) - wr)) < 1e-12 / h


@pytest.mark.parametrize("dim", [2, 3])
def test_dirichlet_free_stream(oracle, dim):
    """a constant field with the same constant as Dirichlet value on every
    face stays constant under any velocity: RHS and LDG gradients vanish"""
    n = (6,) * dim
    pr = oracle.Problem(dim, n, 2, abi.BASIS_Q, boundary_ids=side_ids(dim, n, [1] * (2 * dim)))
    pr.set_velocity(F.constant((0.8, -0.6, 0.3)[:dim]))
    pr.set_dirichlet(1, 0.35)
    phi = np.zeros(pr.n_dofs)
    phi[::pr.nb] = 0.35
    assert np.max(np.abs(pr.advect_rhs(phi, 0.0))) < 1e-12
    gl, gr = pr.hj_gradients(phi)
    assert np.max(np.abs(gl)) < 1e-11 and np.max(np.abs(gr)) < 1e-11
    # without the condition the inflow is zero-Neumann: still constant
    pr.clear_dirichlet()
    assert np.max(np.abs(pr.advect_rhs(phi, 0.0))) < 1e-12


def test_dirichlet_id_zero_and_unset_ids_are_neumann(oracle):
    """faces of id 0 never take a condition (advection.implement.h:723),
    and ids without a condition stay zero-Neumann: setting conditions on
    other ids leaves the RHS unchanged"""
    n = (8, 8)
    ic, vel = F.zalesak_disk(), F.ccw_rotation()
    ref = oracle.Problem(2, n, 1, abi.BASIS_Q)
    ref.set_velocity(vel)
    phi = ref.project(ic)
    pr = oracle.Problem(2, n, 1, abi.BASIS_Q, boundary_ids=side_ids(2, n, [0, 0, 4, 4]))
    pr.set_velocity(vel)
    pr.set_dirichlet(5, 1.0)
    assert np.array_equal(pr.advect_rhs(phi, 0.1), ref.advect_rhs(phi, 0.1))
    with pytest.raises(RuntimeError):
        pr.set_dirichlet(0, 1.0)


# ----------------------------------------------------------------------
# MaterialStack mixing
# ----------------------------------------------------------------------
def _gauss_points(oracle, dim, n, nq):
    """physical coordinates (n_cells, nq^dim, dim) of QGauss(nq) on a
    lexicographic n^dim mesh of the unit box, points x fastest"""
    xg, _ = oracle.gauss(nq)
    h = 1.0 / n
    pts = []
    for c in range(n ** dim):
        I = [c % n, (c // n) % n, c // (n * n)][:dim]
        cell = []
        for j in range(nq ** dim):
            q = [j % nq, (j // nq) % nq, j // (nq * nq)][:dim]
            cell.append([(I[d] + xg[q[d]]) * h for d in range(dim)])
        pts.append(cell)
    return np.asarray(pts)


def _hsine(y, eps):
    return np.where(y > eps, 1.0, np.where(y < -eps, 0.0, 0.5 * (1 + y / eps + np.sin(np.pi * y / eps) / np.pi)))


@pytest.mark.parametrize("smoothing", [abi.HEAVISIDE_NONE, abi.HEAVISIDE_LINEAR, abi.HEAVISIDE_SINE])
def test_material_mix_known_answer(oracle, smoothing):
    """two planes (exact in the degree-1 space) stacked over a background:
    material 0 takes H0 = H(-(x - 0.45)), material 1 (1 - H0) H1 with
    H1 = H(-(y - 0.55)), the background the rest"""
    n, nq = 8, 3
    pr0 = oracle.Problem(2, (n, n), 1, abi.BASIS_Q)
    pr1 = oracle.Problem(2, (n, n), 2, abi.BASIS_P)
    phi0 = pr0.project(F.height_function(0, 0.45, []))
    phi1 = pr1.project(F.height_function(1, 0.55, []))
    got = oracle.material_mix([pr0, pr1], [phi0, phi1], [3.0, -2.0, 0.5], nq, smoothing)
    X = _gauss_points(oracle, 2, n, nq)
    eps = 1.5 * math.sqrt(2.0) / n

    def H(y):
        if smoothing == abi.HEAVISIDE_NONE:
            return np.where(y > 0, 1.0, np.where(y < 0, 0.0, 0.5))
        if smoothing == abi.HEAVISIDE_LINEAR:
            return np.clip(0.5 * (y / eps + 1), 0.0, 1.0)
        return _hsine(y, eps)

    h0 = H(-(X[..., 0] - 0.45))
    h1 = H(-(X[..., 1] - 0.55))
    want = 3.0 * h0 + (-2.0) * (1 - h0) * h1 + 0.5 * (1 - h0) * (1 - h1)
    assert np.max(np.abs(got - want)) < 1e-12


def test_material_mix_partition_of_unity(oracle):
    """equal values everywhere: the shares sum to one at every point"""
    n = 10
    prs = [oracle.Problem(2, (n, n), 2, abi.BASIS_Q) for _ in range(3)]
    phis = [prs[0].project(F.zalesak_disk()), prs[1].project(F.sphere((0.3, 0.4), 0.2)),
            prs[2].project(F.sphere((0.6, 0.6), 0.25))]
    got = oracle.material_mix(prs, phis, [1.0, 1.0, 1.0, 1.0], 4)
    assert np.max(np.abs(got - 1.0)) < 1e-14
