"""Velocity fields and initial conditions of the level-set path.

Velocity fields are sums of separable terms (flsp_velocity_desc); initial
conditions are small CSG trees of signed-distance primitives
(flsp_ic_desc).  Reference counterparts:

* ``rigid_rotation``  — ls::RigidBodyRotation<2> (src/level_set/velocity_field.cc:38-47),
  which rotates clockwise: u = w (y - cy), v = -w (x - cx).
* ``single_vortex``   — ls::SingleVortex<2> (velocity_field.cc:62-77).
* ``sphere``, ``rectangle``, ``union``, ``diff``, ``intersect`` — ls::HyperSphere,
  ls::HyperRectangle, ICUnion/ICDiff/ICIntersect (src/level_set/geometry.cc:17-235,
  include/felspa/level_set/geometry.h:80-160).

Fields the benchmark configurations need and the reference does not have
(counter-clockwise rotation, 3D deformation, random Fourier stream
function, plume rolls, perturbed plane, union of circles) are built from
the same primitives.
"""
import math

import numpy as np

from . import abi


def _factor(kind, a=0.0, b=0.0):
    return abi.Factor(kind, float(a), float(b))


ONE = (abi.F_ONE, 0.0, 0.0)


class VelocityField:
    """Python view of flsp_velocity_desc: u_comp += coeff * prod_a f_a(x_a) * c(t)."""

    def __init__(self, dim, terms, time_kind=abi.T_ONE, ta=0.0, tb=0.0, name="field"):
        self.dim = dim
        self.terms = list(terms)   # (comp, coeff, [(kind, a, b)] * dim)
        self.time_kind = time_kind
        self.ta = ta
        self.tb = tb
        self.name = name
        if len(self.terms) > abi.MAX_VEL_TERMS:
            raise ValueError("too many velocity terms")

    def desc(self):
        d = abi.VelocityDesc()
        d.n_terms = len(self.terms)
        for k, (comp, coeff, fs) in enumerate(self.terms):
            t = d.terms[k]
            t.comp = comp
            t.coeff = float(coeff)
            fs = list(fs) + [ONE] * (3 - len(fs))
            for a in range(3):
                t.f[a] = _factor(*fs[a])
        d.time_kind = self.time_kind
        d.ta = float(self.ta)
        d.tb = float(self.tb)
        return d

    # numpy evaluation (host-side checks and plots only)
    def __call__(self, x, t=0.0):
        x = np.asarray(x, dtype=np.float64)
        u = np.zeros(x.shape[:-1] + (self.dim,))
        for comp, coeff, fs in self.terms:
            v = np.full(x.shape[:-1], float(coeff))
            for a in range(self.dim):
                kind, fa, fb = fs[a] if a < len(fs) else ONE
                v = v * _eval_factor(kind, fa, fb, x[..., a])
            u[..., comp] += v
        return u * _eval_time(self.time_kind, self.ta, self.tb, t)


def _eval_factor(kind, a, b, x):
    if kind == abi.F_ONE:
        return np.ones_like(x)
    if kind == abi.F_LIN:
        return a * x + b
    if kind == abi.F_SIN:
        return np.sin(a * x + b)
    if kind == abi.F_COS:
        return np.cos(a * x + b)
    if kind == abi.F_SINSQ:
        return np.sin(a * x + b) ** 2
    if kind == abi.F_SINPI:
        return np.sin(np.pi * (a * x + b))
    if kind == abi.F_COSPI:
        return np.cos(np.pi * (a * x + b))
    if kind == abi.F_SINPISQ:
        return np.sin(np.pi * (a * x + b)) ** 2
    raise ValueError(kind)


def _eval_time(kind, a, b, t):
    if kind == abi.T_ONE:
        return 1.0
    if kind == abi.T_COS:
        return math.cos(a * t + b)
    if kind == abi.T_COSPI:
        return math.cos(math.pi * (a * t + b))
    if kind == abi.T_ONE_MINUS_EXP:
        return 1.0 - math.exp(-a * t)
    raise ValueError(kind)


# ----------------------------------------------------------------------
# velocity fields
# ----------------------------------------------------------------------
def rigid_rotation(center=(0.0, 0.0), angular_velocity=1.0):
    """ls::RigidBodyRotation<2>: u = w (y - cy), v = -w (x - cx) (clockwise for w > 0)."""
    cx, cy = center
    w = float(angular_velocity)
    return VelocityField(2, [
        (0, w, [ONE, (abi.F_LIN, 1.0, -cy)]),
        (1, -w, [(abi.F_LIN, 1.0, -cx), ONE]),
    ], name="rigid_rotation")


def ccw_rotation(center=(0.5, 0.5), omega=2.0 * math.pi):
    """u = omega (cy - y, x - cx): counter-clockwise solid-body rotation (period 2 pi / omega)."""
    return rigid_rotation(center, -omega)


def single_vortex(period=1.0, scaling=math.pi):
    """ls::SingleVortex<2>: u = -2 sin^2(s x) cos(s y) cos(s t / T), v = 2 sin^2(s y) cos(s x) cos(s t / T)."""
    s = float(scaling)
    return VelocityField(2, [
        (0, -2.0, [(abi.F_SINSQ, s, 0.0), (abi.F_COS, s, 0.0)]),
        (1, 2.0, [(abi.F_COS, s, 0.0), (abi.F_SINSQ, s, 0.0)]),
    ], time_kind=abi.T_COS, ta=s / period, tb=0.0, name="single_vortex")


def deformation_3d(period=3.0):
    """u = 2 sin^2(pi x) sin(2 pi y) sin(2 pi z) c, v = -sin(2 pi x) sin^2(pi y) sin(2 pi z) c,
    w = -sin(2 pi x) sin(2 pi y) sin^2(pi z) c, with c = cos(pi t / T)."""
    S2 = (abi.F_SINPI, 2.0, 0.0)
    return VelocityField(3, [
        (0, 2.0, [(abi.F_SINPISQ, 1.0, 0.0), S2, S2]),
        (1, -1.0, [S2, (abi.F_SINPISQ, 1.0, 0.0), S2]),
        (2, -1.0, [S2, S2, (abi.F_SINPISQ, 1.0, 0.0)]),
    ], time_kind=abi.T_COSPI, ta=1.0 / period, tb=0.0, name="deformation_3d")


def fourier_stream_2d(seed, n_modes=8, kmax=4, sample=1024):
    """Divergence-free field from psi = sum_m a_m sin(k_m pi x) sin(l_m pi y),
    a_m ~ N(0,1) |k|^-2, k_m, l_m in {1..kmax}; u = d psi/dy, v = -d psi/dx,
    scaled so max |u| = 1 on a sample x sample grid.  Zero normal flux on
    the unit square."""
    rng = np.random.default_rng(seed)
    ks = rng.integers(1, kmax + 1, size=n_modes)
    ls = rng.integers(1, kmax + 1, size=n_modes)
    a = rng.standard_normal(n_modes) / (ks.astype(float) ** 2 + ls.astype(float) ** 2)
    terms = []
    for m in range(n_modes):
        k, l, am = int(ks[m]), int(ls[m]), float(a[m])
        terms.append((0, am * l * math.pi, [(abi.F_SINPI, k, 0.0), (abi.F_COSPI, l, 0.0)]))
        terms.append((1, -am * k * math.pi, [(abi.F_COSPI, k, 0.0), (abi.F_SINPI, l, 0.0)]))
    f = VelocityField(2, terms, name="fourier_stream")
    g = (np.arange(sample) + 0.5) / sample
    X, Y = np.meshgrid(g, g, indexing="ij")
    u = f(np.stack([X, Y], -1))
    umax = float(np.sqrt((u ** 2).sum(-1)).max())
    f.terms = [(c, coeff / umax, fs) for c, coeff, fs in f.terms]
    return f


def plume_3d(amplitude=0.5):
    """Rising/sinking rolls: u = curl(0, psi, 0) = (-d psi/dz, 0, d psi/dx) with
    psi = A sin(pi x) sin(pi y) sin(pi z) (1 - exp(-t)); divergence-free, zero
    normal flux on the unit cube."""
    A = float(amplitude)
    return VelocityField(3, [
        (0, -A * math.pi, [(abi.F_SINPI, 1.0, 0.0), (abi.F_SINPI, 1.0, 0.0), (abi.F_COSPI, 1.0, 0.0)]),
        (2, A * math.pi, [(abi.F_COSPI, 1.0, 0.0), (abi.F_SINPI, 1.0, 0.0), (abi.F_SINPI, 1.0, 0.0)]),
    ], time_kind=abi.T_ONE_MINUS_EXP, ta=1.0, tb=0.0, name="plume_3d")


def constant(u):
    dim = len(u)
    ones = [ONE] * dim
    return VelocityField(dim, [(d, float(u[d]), ones) for d in range(dim)], name="constant")


# ----------------------------------------------------------------------
# velocity of a coupled FE simulator: nodal lattice (flsp_set_velocity_fe)
# ----------------------------------------------------------------------
def gauss_lobatto01(degree):
    """the degree+1 Gauss-Lobatto points on [0, 1] (FE_Q support points)"""
    if degree == 1:
        return np.array([0.0, 1.0])
    if degree == 2:
        return np.array([0.0, 0.5, 1.0])
    if degree == 3:
        r = 0.5 / math.sqrt(5.0)
        return np.array([0.0, 0.5 - r, 0.5 + r, 1.0])
    raise ValueError("FE velocity degree must be 1..3")


def fe_lattice_coords(n, degree, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0)):
    """per-axis node coordinates of the lattice: node I of axis e at
    lo + h (I // degree + x_{I % degree})"""
    x = gauss_lobatto01(degree)
    out = []
    for e, ne in enumerate(n):
        h = (hi[e] - lo[e]) / ne
        idx = np.arange(degree * ne + 1)
        cell = np.minimum(idx // degree, ne - 1)
        out.append(lo[e] + h * (cell + x[idx - degree * cell]))
    return out


def fe_lattice(fn, n, degree, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0)):
    """sample fn(x[..., dim]) -> u[..., dim] at the lattice nodes; returns
    the flsp_set_velocity_fe array (components, then z, y, x)"""
    dim = len(n)
    cs = fe_lattice_coords(n, degree, lo, hi)
    grid = np.meshgrid(*cs[::-1], indexing="ij")[::-1]     # x fastest in memory
    x = np.stack(grid, axis=-1)
    u = np.asarray(fn(x), dtype=np.float64)
    return np.ascontiguousarray(np.moveaxis(u, -1, 0)).reshape((dim,) + x.shape[:-1])


def random_fe_lattice(n, degree, seed, scale=1.0):
    """a continuous field of random node values (any lattice is one)"""
    rng = np.random.default_rng(seed)
    shape = (len(n),) + tuple(degree * ne + 1 for ne in n[::-1])
    return scale * rng.uniform(-1.0, 1.0, size=shape)


# ----------------------------------------------------------------------
# initial conditions
# ----------------------------------------------------------------------
class IC:
    """CSG tree of signed-distance primitives (negative inside)."""

    def __init__(self, nodes, root, exact=True, waves=()):
        self.nodes = list(nodes)   # (kind, a, b, p[6])
        self.root = root
        self.exact = exact
        self.waves = list(waves)

    def desc(self):
        d = abi.ICDesc()
        if len(self.nodes) > abi.MAX_IC_NODES or len(self.waves) > abi.MAX_IC_WAVES:
            raise ValueError("IC too large")
        d.n_nodes = len(self.nodes)
        d.root = self.root
        d.exact = 1 if self.exact else 0
        for k, (kind, a, b, p) in enumerate(self.nodes):
            nd = d.nodes[k]
            nd.kind, nd.a, nd.b = kind, a, b
            p = list(p) + [0.0] * (6 - len(p))
            for i in range(6):
                nd.p[i] = float(p[i])
        d.n_waves = len(self.waves)
        for m, w in enumerate(self.waves):
            for i in range(4):
                d.waves[m][i] = float(w[i])
        return d

    def _merge(self, other, kind):
        off = len(self.nodes)
        nodes = list(self.nodes)
        for (k, a, b, p) in other.nodes:
            if k in (abi.IC_UNION, abi.IC_DIFF, abi.IC_INTERSECT):
                nodes.append((k, a + off, b + off, p))
            else:
                nodes.append((k, a, b, p))
        if self.waves and other.waves:
            raise ValueError("only one height-function family per IC")
        nodes.append((kind, self.root, other.root + off, [0.0] * 6))
        return IC(nodes, len(nodes) - 1, self.exact and other.exact, self.waves or other.waves)

    def __add__(self, other):   # union (geometry.h:139-143)
        return self._merge(other, abi.IC_UNION)

    def __sub__(self, other):   # difference (geometry.h:146-150)
        return self._merge(other, abi.IC_DIFF)

    def __mul__(self, other):   # intersection (geometry.h:153-157)
        return self._merge(other, abi.IC_INTERSECT)


def sphere(center, radius):
    c = list(center) + [0.0] * (3 - len(center))
    return IC([(abi.IC_SPHERE, 0, 0, c[:3] + [radius, 0.0, 0.0])], 0, True)


def rectangle(lower, upper):
    lo = list(lower) + [0.0] * (3 - len(lower))
    hi = list(upper) + [0.0] * (3 - len(upper))
    return IC([(abi.IC_RECT, 0, 0, lo[:3] + hi[:3])], 0, True)


def height_function(axis, base, waves):
    """phi = x_axis - (base + sum_m w0 cos(2 pi (w1 x_u + w2 x_v) + w3)); not an exact SDF."""
    return IC([(abi.IC_HEIGHT, 0, 0, [float(axis), float(base), 0, 0, 0, 0])], 0, False, waves)


def zalesak_disk(center=(0.5, 0.75), radius=0.15, slot_width=0.05, slot_depth=0.25):
    """Slotted disk = HyperSphere - HyperRectangle (tests/test_zalesak_disk.cc:109-111,146),
    scaled to the unit square: the slot |x - cx| < w/2 is cut from the top of the
    disk (y = cy + r) down to depth `slot_depth`, as the reference's rectangle
    (-2.5, 15)-(2.5, 40) cuts its r = 15 disk centred at (0, 25)."""
    cx, cy = center
    y1 = cy + radius
    return sphere(center, radius) - rectangle((cx - slot_width / 2, y1 - slot_depth), (cx + slot_width / 2, y1))


def zalesak_reference():
    """The reference test's own geometry on [-50, 50]^2 (test_zalesak_disk.cc:107-111)."""
    return sphere((0.0, 25.0), 15.0) - rectangle((-2.499999, 15.0), (2.499999, 40.0))


def circles_union(seed, kmin=1, kmax=4, cmin=0.2, cmax=0.8, rmin=0.05, rmax=0.2):
    rng = np.random.default_rng(seed)
    k = int(rng.integers(kmin, kmax + 1))
    ic = None
    for _ in range(k):
        c = rng.uniform(cmin, cmax, size=2)
        r = float(rng.uniform(rmin, rmax))
        s = sphere((float(c[0]), float(c[1])), r)
        ic = s if ic is None else ic + s
    return ic


def perturbed_plane(seed, n_modes=16, kmax=8, base=0.5, amp=0.02):
    """z = base + amp * sum_m a_m cos(2 pi (kx x + ky y)), 1 <= |k| <= kmax, a_m ~ N(0,1)/|k|."""
    rng = np.random.default_rng(seed)
    waves = []
    while len(waves) < n_modes:
        kx, ky = (int(v) for v in rng.integers(-kmax, kmax + 1, size=2))
        kn = math.hypot(kx, ky)
        if kn < 1 or kn > kmax:
            continue
        waves.append((amp * float(rng.standard_normal()) / kn, kx, ky, 0.0))
    return height_function(2, base, waves)
