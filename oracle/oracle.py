"""ctypes binding of the CPU FP64 oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline / reference arm as the checker and the CPU
baseline.  Parity status: UNPINNED (see oracle.h).
"""
import ctypes as C
import os
import subprocess

import numpy as np

from felspa_b200 import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class Clock(C.Structure):
    _fields_ = [("t", C.c_double), ("vd_run", C.c_double),
                ("n_since_reinit", C.c_int), ("n_substeps", C.c_int)]


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.orc_create.argtypes = [C.POINTER(abi.MeshDesc), C.c_int, C.c_int, C.POINTER(C.c_void_p)]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_set_dirichlet.argtypes = [C.c_void_p, C.c_int, C.c_double]
        L.orc_clear_dirichlet.argtypes = [C.c_void_p]
        L.orc_n_dofs.argtypes = [C.c_void_p]
        L.orc_n_dofs.restype = C.c_long
        L.orc_dofs_per_cell.argtypes = [C.c_void_p]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_gauss.argtypes = [C.c_int, _dp, _dp]
        L.orc_legendre.argtypes = [C.c_int, C.c_double, _dp, _dp, _dp]
        L.orc_shape.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _dp]
        L.orc_set_velocity.argtypes = [C.c_void_p, C.POINTER(abi.VelocityDesc)]
        L.orc_set_velocity_fe.argtypes = [C.c_void_p, C.c_int, _dp, C.c_long]
        L.orc_eval_velocity.argtypes = [C.c_void_p, _dp, C.c_double, _dp]
        L.orc_eval_ic.argtypes = [C.POINTER(abi.ICDesc), C.c_int, _dp]
        L.orc_eval_ic.restype = C.c_double
        L.orc_project_ic.argtypes = [C.c_void_p, C.POINTER(abi.ICDesc), _dp]
        L.orc_advect_rhs.argtypes = [C.c_void_p, _dp, C.c_double, _dp]
        L.orc_advect_cfl.argtypes = [C.c_void_p, C.c_double]
        L.orc_advect_cfl.restype = C.c_double
        L.orc_advance.argtypes = [C.c_void_p, _dp, C.POINTER(Clock), C.c_int, C.c_double,
                                  C.c_double, C.c_int, _dp]
        L.orc_hj_gradients.argtypes = [C.c_void_p, _dp, _dp, _dp]
        L.orc_hj_rhs.argtypes = [C.c_void_p, _dp, _dp, C.c_double, _dp]
        L.orc_hj_cfl.argtypes = [C.c_void_p, _dp, _dp]
        L.orc_hj_cfl.restype = C.c_double
        L.orc_reinit.argtypes = [C.c_void_p, _dp, C.POINTER(abi.ReinitOpts), _ip]
        L.orc_weno.argtypes = [C.c_void_p, _dp, _ip]
        L.orc_minmod_flags.argtypes = [C.c_void_p, _dp, _ip]
        L.orc_curvature.argtypes = [C.c_void_p, _dp, C.c_void_p, C.c_int, _dp]
        L.orc_ls_advance.argtypes = [C.c_void_p, _dp, C.POINTER(Clock), C.c_int, C.c_double,
                                     C.POINTER(abi.LSOpts), C.c_double, C.c_int, _dp]
        L.orc_reduce.argtypes = [C.c_void_p, C.c_int, _dp, _dp, C.POINTER(abi.ICDesc), _dp]
        L.orc_material_mix.argtypes = [C.c_int, C.POINTER(C.c_void_p), C.POINTER(_dp), _dp, C.c_int, C.c_int,
                                       C.c_void_p, _dp]
        L.orc_mlp_forward.argtypes = [C.c_int, _ip, C.POINTER(_dp), C.POINTER(_dp), C.c_int, _dp, _dp]
        L.orc_mlp_backward.argtypes = [C.c_int, _ip, C.POINTER(_dp), C.POINTER(_dp), C.c_int, _dp,
                                       _dp, C.POINTER(_dp), C.POINTER(_dp)]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(_dp)


def _check(st, what):
    if st != 0:
        raise RuntimeError(f"oracle {what} failed: {abi.STATUS_NAMES.get(st, st)}")


def set_threads(n):
    lib().orc_set_threads(int(n))


def gauss(n):
    x = np.zeros(n)
    w = np.zeros(n)
    lib().orc_gauss(n, _p(x), _p(w))
    return x, w


def legendre(n, x):
    v, d, dd = np.zeros(n), np.zeros(n), np.zeros(n)
    lib().orc_legendre(n, float(x), _p(v), _p(d), _p(dd))
    return v, d, dd


def eval_ic(ic, dim, x):
    d = ic.desc() if hasattr(ic, "desc") else ic
    xx = np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(3) if len(x) == 3
                              else np.array(list(x) + [0.0] * (3 - len(x))))
    return lib().orc_eval_ic(C.byref(d), dim, _p(xx))


class Problem:
    """One level-set problem on the CPU: mesh, DG space, velocity."""

    def __init__(self, dim, n, degree, basis=abi.BASIS_Q, lo=(0, 0, 0), hi=(1, 1, 1), boundary_ids=None):
        self.dim = dim
        self.degree = degree
        self.basis = basis
        self._bids = None
        if boundary_ids is not None:
            self._bids = np.ascontiguousarray(boundary_ids, dtype=np.int32)
        self.mesh = abi.mesh_desc(dim, n, lo, hi, None,
                                  self._bids.ctypes.data_as(C.POINTER(C.c_int32)) if self._bids is not None else None)
        h = C.c_void_p()
        _check(lib().orc_create(C.byref(self.mesh), degree, basis, C.byref(h)), "create")
        self.h = h
        self.n_dofs = lib().orc_n_dofs(h)
        self.nb = lib().orc_dofs_per_cell(h)
        self.clock = Clock(0.0, 0.0, 0, 0)
        self.velocity = None

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_destroy(self.h)
            self.h = None

    def set_dirichlet(self, boundary_id, value):
        _check(lib().orc_set_dirichlet(self.h, int(boundary_id), float(value)), "set_dirichlet")

    def clear_dirichlet(self):
        lib().orc_clear_dirichlet(self.h)

    def set_velocity(self, field):
        self.velocity = field
        self._vdesc = field.desc()
        _check(lib().orc_set_velocity(self.h, C.byref(self._vdesc)), "set_velocity")

    def set_velocity_fe(self, degree, values):
        """velocity of a coupled FE simulator: the nodal lattice of
        flsp_set_velocity_fe (components, then z, y, x)"""
        self.velocity = None
        self._fe_values = np.ascontiguousarray(values, dtype=np.float64).ravel()
        _check(lib().orc_set_velocity_fe(self.h, int(degree), _p(self._fe_values), self._fe_values.size),
               "set_velocity_fe")

    def eval_velocity(self, x, t=0.0):
        xx = np.zeros(3)
        xx[: len(x)] = x
        u = np.zeros(3)
        lib().orc_eval_velocity(self.h, _p(xx), float(t), _p(u))
        return u[: self.dim]

    def shape(self, xi):
        xi = np.ascontiguousarray(np.asarray(xi, dtype=np.float64).reshape(-1, 3))
        npts = xi.shape[0]
        val = np.zeros(self.nb * npts)
        grad = np.zeros(self.nb * npts * self.dim)
        lib().orc_shape(self.h, npts, _p(xi), _p(val), _p(grad))
        return val.reshape(self.nb, npts), grad.reshape(self.nb, npts, self.dim)

    def project(self, ic):
        self._icdesc = ic.desc()
        phi = np.zeros(self.n_dofs)
        _check(lib().orc_project_ic(self.h, C.byref(self._icdesc), _p(phi)), "project_ic")
        return phi

    def advect_rhs(self, phi, t):
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        out = np.zeros(self.n_dofs)
        _check(lib().orc_advect_rhs(self.h, _p(phi), float(t), _p(out)), "advect_rhs")
        return out

    def advect_cfl(self, t):
        return lib().orc_advect_cfl(self.h, float(t))

    def advance(self, phi, time_step, single_cycle=True, rk_order=3, cfl_max=0.9):
        adv = C.c_double(0.0)
        _check(lib().orc_advance(self.h, _p(phi), C.byref(self.clock), rk_order, cfl_max,
                                 float(time_step), 1 if single_cycle else 0, C.byref(adv)), "advance")
        return adv.value

    def hj_gradients(self, phi):
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        gl = np.zeros(self.dim * self.n_dofs)
        gr = np.zeros(self.dim * self.n_dofs)
        _check(lib().orc_hj_gradients(self.h, _p(phi), _p(gl), _p(gr)), "hj_gradients")
        return gl.reshape(self.dim, -1), gr.reshape(self.dim, -1)

    def hj_rhs(self, phi, phi0, viscosity=0.0):
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        phi0 = np.ascontiguousarray(phi0, dtype=np.float64)
        out = np.zeros(self.n_dofs)
        _check(lib().orc_hj_rhs(self.h, _p(phi), _p(phi0), float(viscosity), _p(out)), "hj_rhs")
        return out

    def hj_cfl(self, phi, phi0):
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        phi0 = np.ascontiguousarray(phi0, dtype=np.float64)
        return lib().orc_hj_cfl(self.h, _p(phi), _p(phi0))

    def reinit(self, phi, opts=None):
        o = opts if opts is not None else abi.default_reinit_opts()
        nit = C.c_int(0)
        st = lib().orc_reinit(self.h, _p(phi), C.byref(o), C.byref(nit))
        return st, nit.value

    def weno(self, phi):
        n = C.c_int(0)
        _check(lib().orc_weno(self.h, _p(phi), C.byref(n)), "weno")
        return n.value

    def minmod_flags(self, phi):
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        f = np.zeros(self.n_dofs // self.nb, dtype=np.int32)
        _check(lib().orc_minmod_flags(self.h, _p(phi), f.ctypes.data_as(_ip)), "minmod")
        return f

    def curvature(self, phi, order=None, to_neighbour=False):
        """CurvatureEstimator::estimate on lexicographic cells; `order` =
        the cells' CellId order (host_cell_order), None = lexicographic;
        to_neighbour: exterior face terms to the neighbour (False: to the
        face's owner, as the reference)"""
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        out = np.zeros(self.n_dofs)
        o = np.ascontiguousarray(order, dtype=np.int64) if order is not None else None
        _check(lib().orc_curvature(self.h, _p(phi), o.ctypes.data_as(C.c_void_p) if o is not None else None,
                                   1 if to_neighbour else 0, _p(out)), "curvature")
        return out

    def ls_advance(self, phi, time_step, opts=None, single_step=False, rk_order=3, cfl_max=0.9):
        o = opts if opts is not None else abi.default_ls_opts()
        adv = C.c_double(0.0)
        _check(lib().orc_ls_advance(self.h, _p(phi), C.byref(self.clock), rk_order, cfl_max,
                                    C.byref(o), float(time_step), 1 if single_step else 0,
                                    C.byref(adv)), "ls_advance")
        return adv.value

    def reduce(self, which, phi, phi_ref=None, ic=None):
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        out = C.c_double(0.0)
        ref = _p(np.ascontiguousarray(phi_ref, dtype=np.float64)) if phi_ref is not None else None
        icd = C.byref(ic.desc()) if ic is not None else None
        _check(lib().orc_reduce(self.h, which, _p(phi), ref, icd, C.byref(out)), "reduce")
        return out.value


def material_mix(problems, phis, values, nq, smoothing=abi.HEAVISIDE_SINE, order=None):
    """MaterialStack mixing of constant scalars (stack order; values[-1] is
    the background) at QGauss(nq) points: (n_cells, nq^dim)"""
    n = len(problems)
    prs = (C.c_void_p * n)(*[pr.h for pr in problems])
    ph = [np.ascontiguousarray(p, dtype=np.float64) for p in phis]
    php = (_dp * n)(*[_p(p) for p in ph])
    vals = np.ascontiguousarray(values, dtype=np.float64)
    o = np.ascontiguousarray(order, dtype=np.int64) if order is not None else None
    npt = nq ** problems[0].dim
    ncell = problems[0].n_dofs // problems[0].nb
    out = np.zeros(ncell * npt)
    _check(lib().orc_material_mix(n, prs, php, _p(vals), int(nq), int(smoothing),
                                  o.ctypes.data_as(C.c_void_p) if o is not None else None, _p(out)), "material_mix")
    return out.reshape(ncell, npt)


def mlp_forward(Ws, bs, x):
    widths = [Ws[0].shape[1]] + [W.shape[0] for W in Ws]
    L = len(Ws)
    Wc = [np.ascontiguousarray(W, dtype=np.float64) for W in Ws]
    bc = [np.ascontiguousarray(b, dtype=np.float64) for b in bs]
    Wp = (_dp * L)(*[_p(W) for W in Wc])
    bp = (_dp * L)(*[_p(b) for b in bc])
    w = (C.c_int * (L + 1))(*widths)
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.zeros((x.shape[0], widths[-1]))
    lib().orc_mlp_forward(L, w, Wp, bp, x.shape[0], _p(x), _p(y))
    return y


def mlp_backward(Ws, bs, x, dy):
    widths = [Ws[0].shape[1]] + [W.shape[0] for W in Ws]
    L = len(Ws)
    Wc = [np.ascontiguousarray(W, dtype=np.float64) for W in Ws]
    bc = [np.ascontiguousarray(b, dtype=np.float64) for b in bs]
    dW = [np.zeros_like(W) for W in Wc]
    db = [np.zeros_like(b) for b in bc]
    Wp = (_dp * L)(*[_p(W) for W in Wc])
    bp = (_dp * L)(*[_p(b) for b in bc])
    dWp = (_dp * L)(*[_p(W) for W in dW])
    dbp = (_dp * L)(*[_p(b) for b in db])
    w = (C.c_int * (L + 1))(*widths)
    x = np.ascontiguousarray(x, dtype=np.float64)
    dy = np.ascontiguousarray(dy, dtype=np.float64)
    lib().orc_mlp_backward(L, w, Wp, bp, x.shape[0], _p(x), _p(dy), dWp, dbp)
    return dW, db
