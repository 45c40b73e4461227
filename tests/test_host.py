"""Host-side pieces without a GPU: deal.II cell order, field and IC
descriptors against the reference formulas, bench helpers."""
import math

import numpy as np
import pytest

from felspa_b200 import abi, fields as F
from felspa_b200.level_set import Mesh, dealii_hypercube_order


def test_dealii_order():
    o = dealii_hypercube_order(2, 2, 1)      # 4x4 cells, 4 coarse cells of 2x2 children
    assert list(o[:8]) == [0, 1, 4, 5, 2, 3, 6, 7]
    o3 = dealii_hypercube_order(3, 2, 2)
    assert sorted(o3) == list(range(8 ** 3))
    assert o3[1] == 1 and o3[2] == 8 and o3[4] == 64


def test_rigid_rotation_matches_reference_formula(oracle):
    """RigidBodyRotation<2>: u = w (y - cy), v = -w (x - cx) (velocity_field.cc:38-47)"""
    w, c = math.pi / 314.0, (0.0, 0.0)
    f = F.rigid_rotation(c, w)
    pr = oracle.Problem(2, (4, 4), 1, abi.BASIS_P, lo=(-50, -50), hi=(50, 50))
    pr.set_velocity(f)
    for x in [(-12.5, 31.0), (40.0, -3.0)]:
        u = pr.eval_velocity(x)
        assert abs(u[0] - w * (x[1] - c[1])) < 1e-15 and abs(u[1] + w * (x[0] - c[0])) < 1e-15
        assert np.allclose(f(np.array(x)), u, atol=1e-15)


def test_single_vortex_formula(oracle):
    f = F.single_vortex(period=2.0, scaling=math.pi)
    pr = oracle.Problem(2, (4, 4), 1, abi.BASIS_P)
    pr.set_velocity(f)
    x, t = (0.3, 0.7), 0.4
    s = math.pi
    ref = (-2 * math.sin(s * x[0]) ** 2 * math.cos(s * x[1]) * math.cos(s * t / 2.0),
           2 * math.sin(s * x[1]) ** 2 * math.cos(s * x[0]) * math.cos(s * t / 2.0))
    assert np.allclose(pr.eval_velocity(x, t), ref, atol=1e-15)


def test_deformation_3d_formula(oracle):
    f = F.deformation_3d()
    pr = oracle.Problem(3, (2, 2, 2), 1, abi.BASIS_Q)
    pr.set_velocity(f)
    x, t = (0.2, 0.45, 0.8), 1.1
    c = math.cos(math.pi * t / 3)
    sp = math.sin
    ref = (2 * sp(math.pi * x[0]) ** 2 * sp(2 * math.pi * x[1]) * sp(2 * math.pi * x[2]) * c,
           -sp(2 * math.pi * x[0]) * sp(math.pi * x[1]) ** 2 * sp(2 * math.pi * x[2]) * c,
           -sp(2 * math.pi * x[0]) * sp(2 * math.pi * x[1]) * sp(math.pi * x[2]) ** 2 * c)
    assert np.allclose(pr.eval_velocity(x, t), ref, atol=1e-14)


def test_fourier_stream_divergence_free():
    f = F.fourier_stream_2d(seed=1003, sample=256)
    g = (np.arange(64) + 0.5) / 64
    X, Y = np.meshgrid(g, g, indexing="ij")
    eps = 1e-6
    P = np.stack([X, Y], -1)
    du = (f(P + [eps, 0]) - f(P - [eps, 0]))[..., 0] / (2 * eps)
    dv = (f(P + [0, eps]) - f(P - [0, eps]))[..., 1] / (2 * eps)
    assert np.max(np.abs(du + dv)) < 1e-6
    # zero normal velocity on the walls, |u| <= 1 on the sample grid
    assert np.max(np.abs(f(np.stack([np.zeros(50), np.linspace(0, 1, 50)], -1))[:, 0])) < 1e-12
    gs = (np.arange(256) + 0.5) / 256
    Xs, Ys = np.meshgrid(gs, gs, indexing="ij")
    assert abs(np.sqrt((f(np.stack([Xs, Ys], -1)) ** 2).sum(-1)).max() - 1.0) < 1e-12


def test_zalesak_geometry(oracle):
    ic = F.zalesak_disk()
    v = lambda x: oracle.eval_ic(ic, 2, [x[0], x[1], 0.0])  # noqa: E731
    assert abs(v((0.5, 0.75 - 0.15)) - 0.0) < 1e-15           # bottom of the disk
    assert v((0.5, 0.8)) > 0                                   # inside the slot
    assert abs(v((0.5, 0.65)) - 0.0) < 1e-15                   # slot floor
    assert v((0.4, 0.75)) < 0                                  # solid part
    assert abs(v((0.9, 0.75)) - 0.25) < 1e-15                  # outside: distance to the circle
    ref = F.zalesak_reference()                                # the reference's own geometry
    assert abs(oracle.eval_ic(ref, 2, [0.0, 10.0, 0.0])) < 1e-14
    assert abs(oracle.eval_ic(ref, 2, [0.0, 30.0, 0.0]) - 2.499999) < 1e-12


def test_csg_semantics(oracle):
    a, b = F.sphere((0.3, 0.5), 0.2), F.sphere((0.6, 0.5), 0.2)
    x = [0.45, 0.5, 0.0]
    va, vb = oracle.eval_ic(a, 2, x), oracle.eval_ic(b, 2, x)
    assert oracle.eval_ic(a + b, 2, x) == min(va, vb)
    assert oracle.eval_ic(a - b, 2, x) == max(va, -vb)
    assert oracle.eval_ic(a * b, 2, x) == max(va, vb)


def test_mesh_desc_and_diameter():
    m = Mesh(3, (64, 64, 64))
    assert m.n_cells == 64 ** 3
    assert abs(m.min_diameter - math.sqrt(3) / 64) < 1e-16
    d = m.desc()
    assert (d.dim, d.n[2], d.hi[2]) == (3, 64, 1.0)


def test_bench_clock_parser(tmp_path):
    import bench
    s = bench.ClockSampler(0)
    s.path = str(tmp_path / "c.csv")
    with open(s.path, "w") as f:
        f.write("0, 1965, 1965, 500.0, 0x0, Not Active, Not Active, Not Active, Not Active\n")
        f.write("0, 1800, 1965, 900.0, 0x4, Not Active, Not Active, Not Active, Active\n")

    class P:
        def terminate(self):
            pass

        def wait(self, timeout=None):
            return 0
    s.proc = P()
    r = s.stop()
    assert r["sm_mhz"] == 1882.5 and r["reasons"] == ["sw_power_cap"] and r["sm_max_mhz"] == 1965.0


def test_fe_lattice_layout():
    """the FE velocity lattice: Gauss-Lobatto nodes per cell, shared faces,
    components then z, y, x with x fastest"""
    import math
    import numpy as np
    from felspa_b200 import fields as F
    x3 = F.gauss_lobatto01(3)
    assert np.allclose(x3, [0.0, 0.5 - 0.5 / math.sqrt(5.0), 0.5 + 0.5 / math.sqrt(5.0), 1.0])
    cs = F.fe_lattice_coords((3, 2), 2, lo=(0.0, 1.0), hi=(3.0, 2.0))
    assert np.allclose(cs[0], [0, 0.5, 1, 1.5, 2, 2.5, 3])
    assert np.allclose(cs[1], [1.0, 1.25, 1.5, 1.75, 2.0])
    u = F.fe_lattice(lambda x: np.stack([x[..., 0], 10.0 * x[..., 1]], axis=-1), (3, 2), 2,
                     lo=(0.0, 1.0), hi=(3.0, 2.0))
    assert u.shape == (2, 5, 7)
    assert np.allclose(u[0][0], cs[0]) and np.allclose(u[1][:, 0], 10.0 * cs[1])
    r = F.random_fe_lattice((4, 3, 2), 3, seed=1)
    assert r.shape == (3, 7, 10, 13)
