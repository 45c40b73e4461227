"""Learned reinitialisation: the tensor-core MLP of libflsp_dg.so.

No counterpart in the reference, whose ReinitSimulatorLDG
(src/level_set/reinit.cc:386-637) only has the HJ sweep; that sweep stays
as the source of the training targets and as the fallback where the
network's result is not distance-like enough (the cell mean of
||grad phi| - 1| above a threshold).

The network maps the 3 x 3 patch of a 2D degree-2 (Q basis) cell, 9
Legendre coefficients per cell divided by the cell size h, plus 64 h, to
the change of the centre cell's coefficients under the HJ sweep, divided
by h: 82 -> 256 x 4 (GELU) -> 9, BF16 weights on the tensor cores, FP32
accumulation, FP32 master weights and Adam.  The 3D variant takes the
3 x 3 x 3 patch of a 3D degree-2 cell (27 coefficients each) plus 64 h:
730 -> 256 x 4 -> 27.
"""
import ctypes as C

import numpy as np

from . import abi
from .lib import check, dp, fp, load

IN, HIDDEN, OUT = abi.MLP_IN, abi.MLP_HIDDEN, abi.MLP_OUT
WIDTHS = (IN, HIDDEN, HIDDEN, HIDDEN, HIDDEN, OUT)


def widths(dim=2):
    """layer widths of the 2D or 3D patch network"""
    if dim == 3:
        return (abi.MLP3_IN, HIDDEN, HIDDEN, HIDDEN, HIDDEN, abi.MLP3_OUT)
    return WIDTHS


def param_layout(dim=2):
    """[(name, offset, shape)] of the flat parameter vector (W_l row-major [out][in])."""
    out, off = [], 0
    W = widths(dim)
    for l in range(5):
        ni, no = W[l], W[l + 1]
        out.append((f"W{l + 1}", off, (no, ni)))
        off += ni * no
        out.append((f"b{l + 1}", off, (no,)))
        off += no
    return out


def split_params(p, dim=2):
    """W1, b1, ..., W5, b5 views of a flat parameter vector."""
    return {name: p[off:off + int(np.prod(shape))].reshape(shape) for name, off, shape in param_layout(dim)}


def default_train_opts(**kw):
    o = abi.TrainOpts()
    load().flsp_default_train_opts(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def default_learned_opts(**kw):
    o = abi.LearnedOpts()
    load().flsp_default_learned_opts(C.byref(o))
    for k, v in kw.items():
        if k == "fallback_pseudo_steps":
            o.fallback.n_pseudo_steps = v
        else:
            setattr(o, k, v)
    return o


class MLP:
    """dim = 2: the 3 x 3 patch network; dim = 3: the 3 x 3 x 3 patch network"""

    def __init__(self, device=0, seed=0, dim=2):
        L = load()
        h = C.c_void_p()
        patch = abi.PATCH_3D_Q2 if dim == 3 else abi.PATCH_2D_Q2
        check(L.flsp_mlp_create_patch(patch, int(device), C.c_uint64(seed), C.byref(h)))
        self.h = h
        self.dim = dim
        ni, no, n = C.c_int(0), C.c_int(0), C.c_int64(0)
        check(L.flsp_mlp_info(h, C.byref(ni), C.byref(no), C.byref(n)))
        self.n_in, self.n_out, self.n_params = ni.value, no.value, n.value

    def close(self):
        if getattr(self, "h", None):
            load().flsp_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def get_params(self):
        p = np.empty(self.n_params, dtype=np.float32)
        check(load().flsp_mlp_get_params(self.h, fp(p), p.size))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        check(load().flsp_mlp_set_params(self.h, fp(p), p.size))

    def forward(self, x):
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, self.n_in)
        y = np.empty((x.shape[0], self.n_out), dtype=np.float32)
        check(load().flsp_mlp_forward(self.h, fp(x), x.shape[0], fp(y)))
        return y

    def backward(self, x, dy):
        """gradient of sum(dy * net(x)) w.r.t. the parameters, summed over the batch"""
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, self.n_in)
        dy = np.ascontiguousarray(dy, dtype=np.float32).reshape(-1, self.n_out)
        g = np.empty(self.n_params, dtype=np.float32)
        check(load().flsp_mlp_backward(self.h, fp(x), fp(dy), x.shape[0], fp(g)))
        return g

    def collect(self, problem, band_cells=6.0, target=None):
        """training pairs from a Problem (its state is reinitialised by `target`)"""
        if target is None:
            target = abi.ReinitOpts()
            load().flsp_default_reinit_opts(C.byref(target))
            target.mode = abi.REINIT_FIXED
            target.n_pseudo_steps = 20
        n = C.c_int64(0)
        check(load().flsp_mlp_collect(self.h, problem.h, float(band_cells), C.byref(target), C.byref(n)))
        return n.value

    @property
    def n_pairs(self):
        n = C.c_int64(0)
        check(load().flsp_mlp_n_pairs(self.h, C.byref(n)))
        return n.value

    def clear_pairs(self):
        check(load().flsp_mlp_clear_pairs(self.h))

    def train(self, steps, batch=8192, lr=1e-3, seed=1):
        o = default_train_opts(steps=int(steps), batch=int(batch), lr=float(lr), seed=int(seed))
        loss = C.c_double(0.0)
        check(load().flsp_mlp_train(self.h, C.byref(o), C.byref(loss)))
        return loss.value

    def eval(self):
        loss = C.c_double(0.0)
        check(load().flsp_mlp_eval(self.h, C.byref(loss)))
        return loss.value

    def reinit(self, problem, opts=None):
        """learned reinitialisation of a Problem's state; returns the stats"""
        o = opts if opts is not None else default_learned_opts()
        st = abi.LearnedStats()
        check(load().flsp_reinit_learned(problem.h, self.h, C.byref(o), C.byref(st)))
        return {"n_band": st.n_band, "n_fallback": st.n_fallback, "hj_ran": bool(st.hj_ran)}


# ----------------------------------------------------------------------
# learned vs plain HJ reinitialisation (the comparison of the benchmark)
# ----------------------------------------------------------------------
def plain_reinit_opts(n_pseudo_steps=5, viscosity=1e-3, cfl_max=0.1):
    """The plain HJ sweep of the comparison: the reference's Lax-Friedrichs
    scheme in fixed-count mode with the artificial viscosity of its own
    Zalesak test and the lower of that test's two reinit CFL numbers
    (tests/test_zalesak_disk.cc:252-257).  Under repeated reinitialisation
    the scheme diverges without the viscosity, and at 256^2 and finer also
    with CFL 0.3."""
    return abi.default_reinit_opts(mode=abi.REINIT_FIXED, n_pseudo_steps=n_pseudo_steps, viscosity=viscosity,
                                   cfl_max=cfl_max)


def slotted_disk(seed):
    r = np.random.default_rng(seed)
    from . import fields as F
    cx, cy = r.uniform(0.3, 0.7, 2)
    rad = r.uniform(0.1, 0.2)
    return F.zalesak_disk(center=(float(cx), float(cy)), radius=float(rad), slot_width=float(r.uniform(0.03, 0.08)),
                          slot_depth=float(r.uniform(0.5, 1.6) * rad))


def collect_training_pairs(net, n=128, instances=24, periods=10, every=40, target=None, band_cells=6.0,
                           first=0):
    """Pairs from random instances i = first .. first + instances - 1
    (unions of circles and slotted disks; the velocity alternates between an
    8-mode Fourier stream function, which distorts the level set, and a
    rigid rotation about a random centre, which keeps it distance-like;
    seeds 1000 + i): advance `every` steps, record the band patches,
    reinitialise with `target`."""
    from . import fields as F
    from .level_set import Mesh, Problem
    target = target if target is not None else plain_reinit_opts()
    for i in range(first, first + instances):
        pb = Problem(Mesh(2, (n, n)), 2, basis=abi.BASIS_Q, precision=abi.FP32, cfl_max=0.1)
        if (i // 2) % 2 == 0:
            pb.set_velocity(F.fourier_stream_2d(seed=1000 + i))
        else:
            r = np.random.default_rng(3000 + i)
            c = r.uniform(0.4, 0.6, 2)
            pb.set_velocity(F.ccw_rotation(center=(float(c[0]), float(c[1])),
                                           omega=float(2 * np.pi * r.uniform(0.5, 1.5))))
        pb.project(F.circles_union(1000 + i) if i % 2 == 0 else slotted_disk(2000 + i))
        for _ in range(periods):
            check(load().flsp_advance_steps(pb.h, int(every), 1e30))
            net.collect(pb, band_cells, target)
        pb.close()
    return net.n_pairs


def zalesak_run(method, net=None, n=128, every=40, T=1.0, plain=None, max_residual=0.05, use_graph=False):
    """One revolution of the slotted disk (centre (0.5, 0.75), r 0.15, slot
    0.05 x 0.25) under the counter-clockwise rotation, degree-2 Q basis,
    FP32, CFL 0.1, reinitialised every `every` steps by `method` ("none",
    "plain" or "learned").  Wall-clock time of the whole run (every
    reinitialisation included); L1 interface error and area change against
    the initial shape (FP64 device reductions)."""
    import time
    from . import fields as F
    from .level_set import Mesh, Problem
    L = load()
    plain = plain if plain is not None else plain_reinit_opts()
    pb = Problem(Mesh(2, (n, n)), 2, basis=abi.BASIS_Q, precision=abi.FP32, cfl_max=0.1)
    pb.set_velocity(F.ccw_rotation())
    ic = F.zalesak_disk()
    pb.project(ic)
    area0 = pb.reduce(abi.RED_MASS_SHARP)
    lo = default_learned_opts(max_residual=max_residual)
    lo.fallback = abi.ReinitOpts.from_buffer_copy(plain)
    lo.fallback.narrow_band = 1
    lo.fallback.band_cells = lo.band_cells
    nit = C.c_int(0)
    steps = reinits = n_band = n_fb = 0
    check(L.flsp_sync(pb.h))
    t0 = time.perf_counter()
    if method == "learned" and use_graph:
        # learned periods replayed from captured CUDA graphs (the network's
        # result everywhere in the band: no residual fallback)
        nsteps = zalesak_run.steps_to_T.get((n, T))
        check(L.flsp_ls_run_steps_learned(pb.h, net.h, C.byref(lo), int(every), int(nsteps)))
        check(L.flsp_sync(pb.h))
        steps, reinits = nsteps, nsteps // every
    elif method == "plain" and use_graph:
        # fixed-count reinit replayed from captured CUDA graphs; the step
        # count is that of the host-driven run to T (CFL-limited, same for all)
        nsteps = zalesak_run.steps_to_T.get((n, T))
        ctl = abi.default_ls_opts(reinit_frequency=every, reinit=plain)
        check(L.flsp_ls_run_steps(pb.h, C.byref(ctl), int(nsteps)))
        check(L.flsp_sync(pb.h))
        steps, reinits = nsteps, nsteps // every
    else:
        while pb.get_time() < T - 1e-12:
            check(L.flsp_advance_steps(pb.h, int(every), float(T)))
            steps += every
            if method == "plain":
                check(L.flsp_reinit(pb.h, C.byref(plain), C.byref(nit)))
            elif method == "learned":
                st = net.reinit(pb, lo)
                n_band += st["n_band"]
                n_fb += st["n_fallback"]
            reinits += 1
        check(L.flsp_sync(pb.h))
        zalesak_run.steps_to_T[(n, T)] = steps
    wall = time.perf_counter() - t0
    out = {"method": method, "mesh": f"{n}x{n}", "steps": steps, "reinits": reinits, "wall_s": wall,
           "dof_steps_per_s": pb.n_dofs * steps / wall,
           "l1_interface_error": pb.reduce(abi.RED_L1_INTERFACE_IC, ic),
           "area_change": (pb.reduce(abi.RED_MASS_SHARP) - area0) / area0,
           "grad_deviation": pb.reduce(abi.RED_GRAD_DEVIATION)}
    if method == "learned":
        out["fallback_fraction"] = n_fb / n_band if n_band else 0.0
        out["max_residual"] = None if use_graph else max_residual   # None: no residual test
    if method in ("plain", "learned"):
        out["graph_replay"] = bool(use_graph)
    pb.close()
    return out


zalesak_run.steps_to_T = {}


def interface_run(method, net=None, velocity=None, ic=None, t_end=1.0, n=256, every=40, plain=None,
                  max_residual=0.05, steps=None, precision=abi.FP32):
    """One run of a 2D degree-2 Q level set (FP32, CFL 0.1) from the
    projected `ic` under `velocity` to `t_end` (or for `steps` substeps),
    reinitialised every `every` substeps by `method`: "none", "plain" (the
    fixed-count sweep `plain`, periods replayed from CUDA graphs) or
    "learned" (the network over the 6-cell band with the residual test and
    the narrow-band fallback sweep decided on the device; max_residual =
    inf: no fallback; periods replayed from CUDA graphs).  Device time of
    the whole run; L1 interface error against the exact solution `ic`
    (the shape returns at t_end for the periodic and time-reversed flows
    used here) and area change."""
    import torch
    from .level_set import Mesh, Problem
    L = load()
    plain = plain if plain is not None else plain_reinit_opts()
    pb = Problem(Mesh(2, (n, n)), 2, basis=abi.BASIS_Q, precision=precision, cfl_max=0.1)
    pb.set_velocity(velocity)
    pb.project(ic)
    area0 = pb.reduce(abi.RED_MASS_SHARP)
    if steps is None:
        # substep count to t_end: the CFL-limited step sequence depends on
        # the velocity alone (running-maximum estimate), so a run without
        # reinitialisation counts it
        probe = Problem(Mesh(2, (n, n)), 2, basis=abi.BASIS_Q, precision=precision, cfl_max=0.1)
        probe.set_velocity(velocity)
        probe.project(ic)
        while probe.get_time() < t_end - 1e-12:
            check(L.flsp_advance_steps(probe.h, 200, float(t_end)))
        steps = probe.get_step_count()
        probe.close()
    lo = default_learned_opts(max_residual=max_residual)
    lo.fallback = abi.ReinitOpts.from_buffer_copy(plain)
    lo.fallback.narrow_band = 1
    lo.fallback.band_cells = lo.band_cells
    s = torch.cuda.ExternalStream(pb.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    check(L.flsp_sync(pb.h))
    e0.record(s)
    if method == "none":
        check(L.flsp_advance_steps(pb.h, int(steps), float(t_end)))
    elif method == "plain":
        ctl = abi.default_ls_opts(reinit_frequency=every, reinit=plain)
        check(L.flsp_ls_run_steps(pb.h, C.byref(ctl), int(steps)))
    elif method == "learned":
        check(L.flsp_ls_run_steps_learned(pb.h, net.h, C.byref(lo), int(every), int(steps)))
    else:
        raise ValueError(method)
    e1.record(s)
    check(L.flsp_sync(pb.h))
    ms = e0.elapsed_time(e1)
    out = {"method": method, "every": every, "steps": int(steps), "t": pb.get_time(), "device_s": ms * 1e-3,
           "dof_steps_per_s": pb.n_dofs * steps / (ms * 1e-3),
           "l1_interface_error": pb.reduce(abi.RED_L1_INTERFACE_IC, ic),
           "area_change": (pb.reduce(abi.RED_MASS_SHARP) - area0) / area0,
           "grad_deviation": pb.reduce(abi.RED_GRAD_DEVIATION)}
    if method == "learned":
        out["max_residual"] = max_residual if np.isfinite(max_residual) else None
        nb, nf = C.c_int64(0), C.c_int64(0)
        check(L.flsp_learned_totals(pb.h, C.byref(nb), C.byref(nf), 0))
        out["band_cells_total"] = nb.value
        if np.isfinite(max_residual):
            out["fallback_fraction"] = nf.value / nb.value if nb.value else 0.0
    pb.close()
    return out


def learned_vs_plain(n=128, instances=24, train_steps=8000, seed=7):
    """Train the network on the plain sweep's pairs (on the GPU), then run
    the slotted-disk revolution with no reinit, the plain sweep (host loop
    and graph replay) and the learned reinit with and without the residual
    fallback."""
    import time
    net = MLP(device=0, seed=seed)
    t0 = time.perf_counter()
    n_pairs = collect_training_pairs(net, n=n, instances=instances)
    t1 = time.perf_counter()
    loss0 = net.eval()
    last = net.train(steps=train_steps, batch=8192, lr=1e-3, seed=1)
    t2 = time.perf_counter()
    loss1 = net.eval()
    runs = [zalesak_run("none", n=n), zalesak_run("plain", n=n), zalesak_run("plain", n=n, use_graph=True),
            zalesak_run("learned", net, n=n), zalesak_run("learned", net, n=n, max_residual=1e9),
            zalesak_run("learned", net, n=n, use_graph=True)]
    net.close()
    return {"training": {"pairs": n_pairs, "collect_s": t1 - t0, "steps": train_steps, "batch": 8192,
                         "train_s": t2 - t1, "mse_before": loss0, "mse_after": loss1, "last_batch_mse": last},
            "runs": runs}


# ----------------------------------------------------------------------
# the 3D patch network (learned reinitialisation of large 3D runs)
# ----------------------------------------------------------------------
def collect_training_pairs_3d(net, n=24, instances=8, periods=6, every=10, target=None, band_cells=6.0):
    """3D pairs: spheres (random centres and radii, seeds 4000 + i) under
    the deformation field and perturbed planes (seeds 100 + i) under the
    plume rolls; before each collection the state is scaled by a random
    factor in [0.5, 2] (the same interface, a level set that is not a
    distance function), then the band patches are recorded and the sweep
    `target` gives the targets."""
    from . import fields as F
    from .level_set import Mesh, Problem
    target = target if target is not None else plain_reinit_opts()
    for i in range(instances):
        r = np.random.default_rng(4000 + i)
        pb = Problem(Mesh(3, (n, n, n)), 2, basis=abi.BASIS_Q, precision=abi.FP32, cfl_max=0.1)
        if i % 2 == 0:
            pb.set_velocity(F.deformation_3d())
            c = r.uniform(0.35, 0.65, 3)
            pb.project(F.sphere(tuple(float(v) for v in c), float(r.uniform(0.12, 0.25))))
        else:
            # the plume's time factor 1 - exp(-t) vanishes at t = 0; start
            # where the rolls are established
            pb.set_velocity(F.plume_3d())
            pb.project(F.perturbed_plane(seed=100 + i))
            pb.set_time(1.0)
        for _ in range(periods):
            check(load().flsp_advance_steps(pb.h, int(every), 1e30))
            pb.set_state(pb.get_state() * float(r.uniform(0.5, 2.0)))
            net.collect(pb, band_cells, target)
        pb.close()
    return net.n_pairs


def deformation_run_3d(method, net=None, n=48, every=10, T=3.0, plain=None, max_residual=0.05):
    """The 3D deformation of the sphere r = 0.15 at (0.35, 0.35, 0.35) over
    one period (T = 3: the flow reverses and the shape returns), degree-2 Q,
    FP32, CFL 0.1, reinitialised every `every` steps by `method` ("none",
    "plain" or "learned").  Wall-clock time of the whole run; L1 interface
    error and volume change against the initial shape (FP64 reductions)."""
    import time
    from . import fields as F
    from .level_set import Mesh, Problem
    L = load()
    plain = plain if plain is not None else plain_reinit_opts()
    pb = Problem(Mesh(3, (n, n, n)), 2, basis=abi.BASIS_Q, precision=abi.FP32, cfl_max=0.1)
    pb.set_velocity(F.deformation_3d())
    ic = F.sphere((0.35, 0.35, 0.35), 0.15)
    pb.project(ic)
    vol0 = pb.reduce(abi.RED_MASS_SHARP)
    lo = default_learned_opts(max_residual=max_residual)
    lo.fallback = abi.ReinitOpts.from_buffer_copy(plain)
    lo.fallback.narrow_band = 1
    lo.fallback.band_cells = lo.band_cells
    nit = C.c_int(0)
    steps = reinits = n_band = n_fb = 0
    check(L.flsp_sync(pb.h))
    t0 = time.perf_counter()
    while pb.get_time() < T - 1e-12:
        check(L.flsp_advance_steps(pb.h, int(every), float(T)))
        steps += every
        if method == "plain":
            check(L.flsp_reinit(pb.h, C.byref(plain), C.byref(nit)))
        elif method == "learned":
            st = net.reinit(pb, lo)
            n_band += st["n_band"]
            n_fb += st["n_fallback"]
        reinits += 1
    check(L.flsp_sync(pb.h))
    wall = time.perf_counter() - t0
    out = {"method": method, "mesh": f"{n}^3", "steps": steps, "reinits": reinits, "wall_s": wall,
           "dof_steps_per_s": pb.n_dofs * steps / wall,
           "l1_interface_error": pb.reduce(abi.RED_L1_INTERFACE_IC, ic),
           "volume_change": (pb.reduce(abi.RED_MASS_SHARP) - vol0) / vol0,
           "grad_deviation": pb.reduce(abi.RED_GRAD_DEVIATION)}
    if method == "learned":
        out["fallback_fraction"] = n_fb / n_band if n_band else 0.0
        out["max_residual"] = max_residual
    pb.close()
    return out


def learned_vs_plain_3d(n=48, train_n=24, instances=8, train_steps=3000, seed=7, every=40):
    """Train the 3D patch network on the plain sweep's pairs (on the GPU),
    then run the sphere's deformation period with no reinit, the plain
    sweep and the learned reinit with and without the residual fallback."""
    import time
    net = MLP(device=0, seed=seed, dim=3)
    t0 = time.perf_counter()
    n_pairs = collect_training_pairs_3d(net, n=train_n, instances=instances)
    t1 = time.perf_counter()
    loss0 = net.eval()
    last = net.train(steps=train_steps, batch=8192, lr=1e-3, seed=1)
    t2 = time.perf_counter()
    loss1 = net.eval()
    runs = [deformation_run_3d("none", n=n, every=every), deformation_run_3d("plain", n=n, every=every),
            deformation_run_3d("learned", net, n=n, every=every),
            deformation_run_3d("learned", net, n=n, every=every, max_residual=1e9)]
    net.close()
    return {"training": {"pairs": n_pairs, "collect_s": t1 - t0, "steps": train_steps, "batch": 8192,
                         "train_s": t2 - t1, "mse_before": loss0, "mse_after": loss1, "last_batch_mse": last},
            "runs": runs}


def _rate_at_l1(points, target):
    """rate of a method at L1 interface error `target`, by linear
    interpolation in log L1 along its (L1, rate) points ordered by reinit
    interval; None when the target lies outside the points' L1 range"""
    pts = sorted(points, key=lambda p: p[0])
    for (l0, r0), (l1, r1) in zip(pts, pts[1:]):
        if l0 <= target <= l1:
            if l1 == l0:
                return max(r0, r1)
            w = (np.log(target) - np.log(l0)) / (np.log(l1) - np.log(l0))
            return float(r0 + w * (r1 - r0))
    return None


def equal_l1_study(net, workloads, n=256, intervals=(20, 40, 80, 160), plain=None, max_residual=0.05):
    """Learned against plain HJ reinitialisation at equal L1 interface error.
    For every workload (name -> (velocity, ic, t_end)): a run without
    reinitialisation, then for every reinit interval the plain sweep (the
    reference's algorithm over every cell), the learned reinit with its
    residual fallback decided on the device, and the learned reinit
    without fallback; every run replayed from CUDA graphs, device time.
    Each method's runs give an (L1, DoF-steps/s) front over the intervals;
    at the L1 of every plain run the learned methods' rates are read off
    their fronts (interpolated in log L1), and their ratio to the plain
    rate is the speed-up at equal L1."""
    out = {}
    for name, (vel, ic, t_end) in workloads.items():
        none = interface_run("none", velocity=vel, ic=ic, t_end=t_end, n=n, plain=plain)
        steps = none["steps"]
        runs = {"none": none, "plain": [], "learned": [], "learned_no_fallback": []}
        for every in intervals:
            runs["plain"].append(interface_run("plain", velocity=vel, ic=ic, t_end=t_end, n=n, every=every,
                                               plain=plain, steps=steps))
            runs["learned"].append(interface_run("learned", net=net, velocity=vel, ic=ic, t_end=t_end, n=n,
                                                 every=every, plain=plain, max_residual=max_residual,
                                                 steps=steps))
            runs["learned_no_fallback"].append(interface_run("learned", net=net, velocity=vel, ic=ic, t_end=t_end,
                                                             n=n, every=every, plain=plain,
                                                             max_residual=float("inf"), steps=steps))
        fronts = {k: [(r["l1_interface_error"], r["dof_steps_per_s"]) for r in runs[k]]
                  for k in ("plain", "learned", "learned_no_fallback")}
        equal = []
        for r in runs["plain"]:
            row = {"plain_every": r["every"], "l1": r["l1_interface_error"], "plain_rate": r["dof_steps_per_s"]}
            for k in ("learned", "learned_no_fallback"):
                rate = _rate_at_l1(fronts[k], r["l1_interface_error"])
                row[k + "_rate"] = rate
                row[k + "_speedup"] = rate / r["dof_steps_per_s"] if rate else None
            equal.append(row)
        out[name] = {"steps": steps, "runs": runs, "equal_l1": equal}
    return out
