"""Host-side mirror of FELSPA's level-set simulator interface, on top of the
C ABI of libflsp_dg.so.

Class and method names follow the reference so that a driver written
against it reads the same:

* ``AdvectSimulator``   — dg::AdvectSimulator (include/felspa/pde/advection.h:91-381)
* ``ReinitSimulatorLDG`` — dg::ReinitSimulatorLDG (include/felspa/level_set/reinit.h:154-268)
* ``LevelSetSurface``   — ls::LevelSetSurface (include/felspa/level_set/level_set.h:176-413)

All three drive one device-resident problem (``Problem``): the reference's
reinit simulator shares the advection solution vector, and so do these.
Errors from the library surface as ``FlspError`` (the reference throws
EXCEPT_MSG exceptions, base/exceptions.h:227-245).
"""
import ctypes as C

import numpy as np

from . import abi
from .lib import check, dp, load

# ----------------------------------------------------------------------
# mesh helpers
# ----------------------------------------------------------------------


def dealii_hypercube_order(dim, n_subdiv, n_refine):
    """Active-cell order of deal.II's subdivided_hyper_cube(n_subdiv) refined
    n_refine times globally: coarse cells lexicographic, the children of
    every cell in lexicographic (x fastest) order, depth first.  Returns, for
    each cell of that order, its lexicographic lattice index (the
    permutation flsp_create takes as host_cell_order)."""
    N = n_subdiv * 2 ** n_refine
    order = []

    def rec(ix, iy, iz, level):
        if level == n_refine:
            order.append(ix + N * (iy + N * iz))
            return
        for cz in range(2 if dim == 3 else 1):
            for cy in range(2):
                for cx in range(2):
                    rec(2 * ix + cx, 2 * iy + cy, 2 * iz + cz, level + 1)

    for kz in range(n_subdiv if dim == 3 else 1):
        for ky in range(n_subdiv):
            for kx in range(n_subdiv):
                rec(kx, ky, kz, 0)
    return np.asarray(order, dtype=np.int64)


def boundary_face_count(dim, n):
    """domain-boundary faces of an n[0] x .. box: 2 sum_d prod_{e != d} n[e]"""
    return int(sum(2 * np.prod([n[e] for e in range(dim) if e != d]) for d in range(dim)))


def colorized_boundary_ids(dim, n):
    """boundary ids of deal.II's colorized hyper_rectangle: side s (x-, x+,
    y-, y+, z-, z+) has id s, in flsp_mesh_desc's face order"""
    ids = []
    for d in range(dim):
        side = int(np.prod([n[e] for e in range(dim) if e != d]))
        ids += [2 * d] * side + [2 * d + 1] * side
    return np.asarray(ids, dtype=np.int32)


class Mesh:
    """Uniform Cartesian mesh of a box (the part of dealii::Triangulation the
    hot path needs): cells per axis, corners, optional host cell order and
    boundary ids of the boundary faces (flsp_mesh_desc's order)."""

    def __init__(self, dim, n, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), host_cell_order=None,
                 boundary_ids=None):
        self.dim = dim
        self.n = tuple(int(v) for v in n[:dim])
        self.lo = tuple(float(v) for v in lo[:dim])
        self.hi = tuple(float(v) for v in hi[:dim])
        self.host_cell_order = None if host_cell_order is None else np.ascontiguousarray(
            host_cell_order, dtype=np.int64)
        self.boundary_ids = None
        if boundary_ids is not None:
            self.boundary_ids = np.ascontiguousarray(boundary_ids, dtype=np.int32)
            if self.boundary_ids.size != boundary_face_count(dim, self.n):
                raise ValueError("boundary_ids must hold one id per boundary face")

    @property
    def n_cells(self):
        return int(np.prod(self.n))

    @property
    def min_diameter(self):
        h = [(self.hi[d] - self.lo[d]) / self.n[d] for d in range(self.dim)]
        return float(np.sqrt(sum(x * x for x in h)))

    def desc(self):
        order = None
        if self.host_cell_order is not None:
            order = self.host_cell_order.ctypes.data_as(C.POINTER(C.c_int64))
        bids = None
        if self.boundary_ids is not None:
            bids = self.boundary_ids.ctypes.data_as(C.POINTER(C.c_int32))
        return abi.mesh_desc(self.dim, self.n, self.lo, self.hi, order, bids)


# ----------------------------------------------------------------------
# one device-resident problem
# ----------------------------------------------------------------------
class Problem:
    def __init__(self, mesh, fe_degree, basis=abi.BASIS_Q, precision=abi.FP64, rk_order=3,
                 cfl_max=0.9, device=0):
        L = load()
        self.mesh = mesh
        self.fe_degree = fe_degree
        self.basis = basis
        self.precision = precision
        self._mdesc = mesh.desc()
        o = abi.DGOpts()
        L.flsp_default_dg_opts(C.byref(o))
        o.degree = fe_degree
        o.basis = basis
        o.precision = precision
        o.rk_order = rk_order
        o.cfl_max = cfl_max
        o.device = device
        h = C.c_void_p()
        check(L.flsp_create(C.byref(self._mdesc), C.byref(o), C.byref(h)))
        self.h = h
        n = C.c_int64(0)
        check(L.flsp_n_dofs(h, C.byref(n)))
        self.n_dofs = n.value
        nb = C.c_int(0)
        check(L.flsp_dofs_per_cell(h, C.byref(nb)))
        self.dofs_per_cell = nb.value

    @classmethod
    def wrap(cls, handle, mesh, fe_degree, basis, precision):
        """A Problem view of a handle owned elsewhere (a batch member)."""
        self = cls.__new__(cls)
        self.mesh = mesh
        self.fe_degree = fe_degree
        self.basis = basis
        self.precision = precision
        self._mdesc = mesh.desc()
        self.h = handle
        self._owned = False
        n = C.c_int64(0)
        check(load().flsp_n_dofs(handle, C.byref(n)))
        self.n_dofs = n.value
        nb = C.c_int(0)
        check(load().flsp_dofs_per_cell(handle, C.byref(nb)))
        self.dofs_per_cell = nb.value
        return self

    def close(self):
        if getattr(self, "h", None):
            if getattr(self, "_owned", True):
                load().flsp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # state ------------------------------------------------------------
    def set_velocity(self, field):
        self._vdesc = field.desc()
        check(load().flsp_set_velocity(self.h, C.byref(self._vdesc)))

    def set_velocity_fe(self, degree, values):
        """velocity of a coupled FE simulator (flsp_set_velocity_fe): the
        continuous nodal field of degree 1..3 on the mesh's Gauss-Lobatto
        lattice, components then z, y, x (fields.fe_lattice samples one)"""
        v = np.ascontiguousarray(values, dtype=np.float64).ravel()
        check(load().flsp_set_velocity_fe(self.h, int(degree), v.ctypes.data_as(C.POINTER(C.c_double)), v.size))

    def project(self, ic):
        self._icdesc = ic.desc()
        check(load().flsp_project_ic(self.h, C.byref(self._icdesc)))

    def set_state(self, coeffs):
        a = np.ascontiguousarray(coeffs, dtype=np.float64)
        check(load().flsp_set_state(self.h, dp(a), a.size))

    def get_state(self, out=None):
        """solution coefficients in host DoF order (into `out` when given,
        e.g. a pinned buffer)"""
        if out is None:
            out = np.empty(self.n_dofs)
        if out.dtype != np.float64 or out.size != self.n_dofs or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous float64 array of n_dofs")
        check(load().flsp_get_state(self.h, dp(out), out.size))
        return out

    def get_time(self):
        t = C.c_double(0.0)
        check(load().flsp_get_time(self.h, C.byref(t)))
        return t.value

    def get_step_count(self):
        """advection substeps executed so far"""
        n = C.c_int64(0)
        check(load().flsp_get_step_count(self.h, C.byref(n)))
        return n.value

    def set_time(self, t):
        check(load().flsp_set_time(self.h, float(t)))

    def snapshot(self):
        check(load().flsp_snapshot(self.h))

    def learned_totals(self, reset=False):
        """(band cells, fallback cells) summed over the learned reinitialisations"""
        nb, nf = C.c_int64(0), C.c_int64(0)
        check(load().flsp_learned_totals(self.h, C.byref(nb), C.byref(nf), 1 if reset else 0))
        return nb.value, nf.value

    def set_dirichlet(self, boundary_id, value):
        """a Dirichlet condition of constant value on the faces of id boundary_id (> 0)"""
        check(load().flsp_set_dirichlet(self.h, int(boundary_id), float(value)))

    def clear_dirichlet(self):
        check(load().flsp_clear_dirichlet(self.h))

    def sync(self):
        check(load().flsp_sync(self.h))

    def stream(self):
        s = C.c_void_p()
        check(load().flsp_stream(self.h, C.byref(s)))
        return s.value

    def time_kernel(self, which, reps=20):
        """average ms per launch of a hot kernel (0: advection stage, 1: reinit step)."""
        ms = C.c_double(0.0)
        check(load().flsp_time_kernel(self.h, int(which), int(reps), C.byref(ms)))
        return ms.value

    def reduce(self, which, ic=None):
        out = C.c_double(0.0)
        icd = C.byref(ic.desc()) if ic is not None else None
        check(load().flsp_reduce(self.h, which, icd, C.byref(out)))
        return out.value

    def autotune(self, reps=10):
        """time every stage-kernel tile on this problem and keep the
        fastest; returns (tile, {tile: ms per stage launch})"""
        t = (C.c_int * 3)()
        ct = (C.c_int * (3 * 8))()
        cm = (C.c_double * 8)()
        n = C.c_int(0)
        check(load().flsp_autotune(self.h, int(reps), t, ct, cm, C.byref(n)))
        return tuple(t), {tuple(ct[3 * i:3 * i + 3]): cm[i] for i in range(n.value)}

    def stage_tile(self):
        t = (C.c_int * 3)()
        check(load().flsp_stage_tile(self.h, t))
        return tuple(t)

    def curvature(self, mode=abi.CURV_REFERENCE):
        """curvature coefficients of the state (host DoF order, FP64)"""
        out = np.empty(self.n_dofs)
        check(load().flsp_curvature(self.h, int(mode), dp(out), out.size))
        return out

    def eval_patches(self, n_sub=1):
        """values at the (n_sub+1)^dim equispaced vertices of every cell
        (DataOut::build_patches(n_sub)); shape (n_cells, (n_sub+1)^dim),
        cells in host order, vertices x fastest"""
        npt = (n_sub + 1) ** self.mesh.dim
        out = np.empty(self.mesh.n_cells * npt)
        check(load().flsp_eval_patches(self.h, int(n_sub), dp(out), out.size))
        return out.reshape(self.mesh.n_cells, npt)

    def export_solutions(self, path, label):
        """<path><label>_<count>.vtu plus <path><label>.pvd (pde_base.cc:93-115)"""
        check(load().flsp_export_solutions(self.h, str(path).encode(), str(label).encode()))


def write_vtu(mesh, values, label, filename, n_sub=1):
    """host-side VTU writer (no GPU): `values` as Problem.eval_patches returns them"""
    md = mesh.desc()
    v = np.ascontiguousarray(values, dtype=np.float64).ravel()
    if v.size != mesh.n_cells * (n_sub + 1) ** mesh.dim:
        raise ValueError("values must hold (n_sub+1)^dim values per cell")
    check(load().flsp_write_vtu(C.byref(md), int(n_sub), dp(v), str(label).encode(), str(filename).encode()))


def write_pvd(filename, records):
    """host-side PVD writer (no GPU): records = [(time, vtu file name), ...]"""
    times = np.ascontiguousarray([float(t) for t, _ in records], dtype=np.float64)
    names = (C.c_char_p * max(len(records), 1))(*[str(f).encode() for _, f in records])
    check(load().flsp_write_pvd(str(filename).encode(), len(records), dp(times), names))


def reduce_noalloc(mesh, fe_degree, basis, precision, state_ptr, which, result_ptr, ref_ptr=None,
                   ic=None, stream=None):
    """Enqueue flsp_reduce_noalloc: the reduction `which` of a caller-owned
    device state (lexicographic cells) into the caller's device double at
    `result_ptr`, on `stream` (a cudaStream_t handle, None = default stream),
    without allocating device memory.  Pointers are integer device addresses."""
    md = mesh.desc()
    icd = C.byref(ic.desc()) if ic is not None else None
    check(load().flsp_reduce_noalloc(C.byref(md), int(fe_degree), int(basis), int(precision),
                                     C.c_void_p(state_ptr), C.c_void_p(ref_ptr) if ref_ptr else None,
                                     int(which), icd, C.c_void_p(result_ptr),
                                     C.c_void_p(stream) if stream else None))


# ----------------------------------------------------------------------
# reference-named simulators
# ----------------------------------------------------------------------
class AdvectSimulator:
    """dg::AdvectSimulator: DG advection with CFL-limited SSP-RK substeps."""

    label = "Advect"   # default label string (include/felspa/pde/advection.h:132)

    def __init__(self, mesh, fe_degree, basis=abi.BASIS_Q, precision=abi.FP64, rk_order=3,
                 cfl_max=0.9, device=0, problem=None):
        self.problem = problem or Problem(mesh, fe_degree, basis, precision, rk_order, cfl_max, device)

    @property
    def n_dofs(self):
        return self.problem.n_dofs

    def initialize(self, initial_condition, velocity_field):
        """AdvectSimulator::initialize(ScalarFunction | vector, ptr_velocity_field)."""
        self.problem.set_velocity(velocity_field)
        if isinstance(initial_condition, np.ndarray):
            self.problem.set_state(initial_condition)
        else:
            self.problem.project(initial_condition)

    def explicit_time_derivative(self, current_time):
        """phidot = M^-1 R(phi, t) of the current solution (advection.cc:269-296)."""
        out = np.empty(self.n_dofs)
        check(load().flsp_advect_rhs(self.problem.h, float(current_time), dp(out), out.size))
        return out

    def advance_time(self, time_step, compute_single_cycle=False):
        """AdvectSimulator::advance_time(time_step, compute_single_cycle) (advection.cc:359-426)."""
        adv = C.c_double(0.0)
        check(load().flsp_advance(self.problem.h, float(time_step), 1 if compute_single_cycle else 0,
                                  C.byref(adv)))
        return adv.value

    def advance_steps(self, n_steps, t_end=float("inf")):
        """n CFL-limited substeps with the time step kept on the device."""
        check(load().flsp_advance_steps(self.problem.h, int(n_steps), float(t_end)))

    def get_solution_vector(self):
        return self.problem.get_state()

    def append_boundary_condition(self, boundary_id, dirichlet_value):
        """append_boundary_condition(bc) for a Dirichlet condition of
        constant value on the faces of id boundary_id (> 0); the level set's
        advection and reinitialisation share it (level_set.implement.h:384-392)"""
        self.problem.set_dirichlet(boundary_id, dirichlet_value)

    def export_solutions(self, path, label=None):
        """SimulatorBase::export_solutions(path): the solution's cell-corner
        values as <path><label>_<9-digit count>.vtu, and <path><label>.pvd
        listing every export of this simulator with its time."""
        self.problem.export_solutions(path, label or self.label)

    def get_time(self):
        return self.problem.get_time()

    def compute_error(self, reference):
        """compute_error(vector): mean |coefficient difference| (advection.cc:471-484);
        compute_error(ic): L2 error against an analytic IC with QGauss(p+1) (:452-468)."""
        if isinstance(reference, np.ndarray):
            return float(np.abs(self.get_solution_vector() - reference).mean())
        return self.problem.reduce(abi.RED_L2_ERROR_IC, reference)


class ReinitSimulatorLDG:
    """dg::ReinitSimulatorLDG acting on the advection solution in place."""

    def __init__(self, problem, control=None):
        self.problem = problem
        self.control = control if control is not None else abi.default_reinit_opts()

    def run_iteration(self, control=None):
        """initialize(solution) + run_iteration(); returns the iteration count."""
        o = control if control is not None else self.control
        nit = C.c_int(0)
        check(load().flsp_reinit(self.problem.h, C.byref(o), C.byref(nit)))
        return nit.value

    def local_left_right_gradients(self):
        """(left, right) LDG gradients, each of shape (dim, n_dofs)."""
        d = self.problem.mesh.dim
        out = np.empty(2 * d * self.problem.n_dofs)
        check(load().flsp_hj_gradients(self.problem.h, dp(out), out.size))
        g = out.reshape(2 * d, -1)
        return g[:d], g[d:]

    def apply_weno_limiter(self):
        n = C.c_int(0)
        check(load().flsp_weno_limit(self.problem.h, C.byref(n)))
        return n.value


class LevelSetSurface(AdvectSimulator):
    """ls::LevelSetSurface<AdvectSimulator, ReinitSimulatorLDG>."""

    label = "LevelSet"   # default label string (include/felspa/level_set/level_set.h:201)

    def __init__(self, mesh, fe_degree, basis=abi.BASIS_Q, precision=abi.FP64, rk_order=3,
                 cfl_max=0.9, device=0, control=None):
        super().__init__(mesh, fe_degree, basis, precision, rk_order, cfl_max, device)
        self.control = control if control is not None else abi.default_ls_opts()
        self.reinit_simulator = ReinitSimulatorLDG(self.problem, self.control.reinit)

    def initialize(self, initial_condition, velocity_field):
        """level_set.implement.h:119-142: project the IC; a non-exact IC gets a
        global reinit."""
        super().initialize(initial_condition, velocity_field)
        if not isinstance(initial_condition, np.ndarray) and not initial_condition.exact:
            o = abi.ReinitOpts.from_buffer_copy(self.control.reinit)
            o.mode = abi.REINIT_GLOBAL
            self.reinit_simulator.run_iteration(o)

    def advance_time(self, time_step, compute_single_step=False):
        """LevelSetSurface::advance_time(time_step, compute_single_step) (level_set.implement.h:180-205)."""
        adv = C.c_double(0.0)
        check(load().flsp_ls_advance(self.problem.h, C.byref(self.control), float(time_step),
                                     1 if compute_single_step else 0, C.byref(adv)))
        return adv.value

    def run_steps(self, n_steps, sync=True):
        """n advection substeps with a fixed-count reinit every reinit_frequency
        steps, replayed from captured CUDA graphs (enqueued asynchronously;
        sync=True waits for completion)."""
        check(load().flsp_ls_run_steps(self.problem.h, C.byref(self.control), int(n_steps)))
        if sync:
            self.problem.sync()

    # diagnostics (FP64 device reductions)
    def estimate_curvature(self, mode=abi.CURV_REFERENCE):
        """CurvatureEstimator::estimate (level_set.implement.h:600-620):
        |M^-1 RHS| of the weak divergence of grad phi / |grad phi|, per
        coefficient.  CURV_REFERENCE keeps the reference's face loop, whose
        exterior face term lands in the face owner's DoFs; CURV_NEIGHBOUR
        gives it to the neighbour (cell means approach the mean curvature)."""
        return self.problem.curvature(mode)

    def integrate_mass(self):
        return self.problem.reduce(abi.RED_MASS)

    def compute_mass_error(self, analytical_soln):
        return self.problem.reduce(abi.RED_MASS_ERROR, analytical_soln)

    def interface_error_l1(self, analytical_soln=None):
        if analytical_soln is None:
            return self.problem.reduce(abi.RED_L1_INTERFACE)
        return self.problem.reduce(abi.RED_L1_INTERFACE_IC, analytical_soln)

    def gradient_deviation(self):
        return self.problem.reduce(abi.RED_GRAD_DEVIATION)


class MaterialStack:
    """ls::MaterialStack (include/felspa/level_set/material_stack.h:22) for
    materials with one constant scalar each: materials pushed with their
    level sets (LevelSetSurface or Problem, all on one mesh), a background
    material, and the mixed scalar at the Gauss points of every cell
    (MaterialAccessor<MaterialStack>::reinit + eval_scalars,
    material_stack.implement.h:320-470), evaluated on the device."""

    def __init__(self, background_value=None):
        self.background = background_value
        self.entries = []

    def set_background_material(self, value):
        self.background = float(value)

    def push(self, value, level_set):
        if len(self.entries) >= abi.MAX_MATERIALS:
            raise ValueError("at most %d level sets" % abi.MAX_MATERIALS)
        self.entries.append((float(value), getattr(level_set, "problem", level_set)))

    def n_materials(self):
        return len(self.entries)

    def eval_scalars(self, n_qpts_1d, smoothing=abi.HEAVISIDE_SINE):
        """mixed scalar, shape (n_cells, n_qpts_1d^dim): host cell order of
        the first level set, QGauss(n_qpts_1d) points x fastest"""
        if self.background is None:
            raise ValueError("the background material must be set first (ExcBackgroundMaterialUndefined)")
        if not self.entries:
            raise ValueError("no material pushed")
        pb0 = self.entries[0][1]
        n = len(self.entries)
        hs = (C.c_void_p * n)(*[pb.h for _, pb in self.entries])
        vals = np.ascontiguousarray([v for v, _ in self.entries] + [self.background], dtype=np.float64)
        npt = n_qpts_1d ** pb0.mesh.dim
        out = np.empty(pb0.mesh.n_cells * npt)
        check(load().flsp_material_mix(hs, n, dp(vals), int(n_qpts_1d), int(smoothing), dp(out), out.size))
        return out.reshape(pb0.mesh.n_cells, npt)
