"""Batched problems: many independent 2D level-set problems advanced by one
persistent launch per RK stage / reinit pseudo-step, periods replayed from
captured CUDA graphs, tile shapes from the batch autotuner
(flsp_batch_* in include/flsp_dg.h).  Not in the reference, where a
simulator object holds one problem."""
import ctypes as C

import numpy as np

from . import abi, fields as F
from .level_set import Mesh, Problem
from .lib import check, load


class Batch:
    def __init__(self, meshes, degrees, precision=abi.FP32, cfl_max=0.1, rk_order=3, device=0):
        L = load()
        n = len(meshes)
        md = (abi.MeshDesc * n)(*[m.desc() for m in meshes])
        od = (abi.DGOpts * n)()
        for i, p in enumerate(degrees):
            L.flsp_default_dg_opts(C.byref(od[i]))
            od[i].degree = int(p)
            od[i].basis = abi.BASIS_Q
            od[i].precision = precision
            od[i].rk_order = rk_order
            od[i].cfl_max = cfl_max
            od[i].device = device
        self._md, self._od = md, od
        b = C.c_void_p()
        check(L.flsp_batch_create(n, md, od, C.byref(b)))
        self.h = b
        self.problems = []
        for i in range(n):
            ph = C.c_void_p()
            check(L.flsp_batch_problem(b, i, C.byref(ph)))
            self.problems.append(Problem.wrap(ph, meshes[i], int(degrees[i]), abi.BASIS_Q, precision))
        self.n_dofs = sum(p.n_dofs for p in self.problems)

    def close(self):
        if getattr(self, "h", None):
            for p in self.problems:
                p.h = None
            load().flsp_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def autotune(self):
        t = abi.BatchTuning()
        check(load().flsp_batch_autotune(self.h, C.byref(t)))
        return {"adv_tile": tuple(t.adv_tile), "hj_tile": tuple(t.hj_tile),
                "adv_ms": {f"{t.adv_cand[i][0]}x{t.adv_cand[i][1]}": t.adv_ms[i] for i in range(t.n_adv)},
                "hj_ms": {f"{t.hj_cand[i][0]}x{t.hj_cand[i][1]}": t.hj_ms[i] for i in range(t.n_hj)}}

    def run_steps(self, n_steps, control=None, sync=True):
        ctl = control if control is not None else abi.default_ls_opts(
            reinit=abi.default_reinit_opts(mode=abi.REINIT_FIXED, n_pseudo_steps=5))
        check(load().flsp_batch_run_steps(self.h, C.byref(ctl), int(n_steps)))
        if sync:
            self.sync()

    def sync(self):
        check(load().flsp_batch_sync(self.h))

    def stream(self):
        s = C.c_void_p()
        check(load().flsp_batch_stream(self.h, C.byref(s)))
        return s.value


def uneven_batch_instances(n_problems=256, seed_base=1000, n_min=32, n_max=256):
    """The batched configuration: problem i draws from default_rng(seed_base + i)
    a mesh size N = round(32 * 8^U) (log-uniform 32..256), a degree in {1,2,3};
    its IC is a union of 1-4 circles (centres U[0.2,0.8]^2, radii U[0.05,0.2])
    and its velocity the 8-mode Fourier stream-function field scaled to
    max|u| = 1, both seeded with seed_base + i."""
    out = []
    for i in range(n_problems):
        rng = np.random.default_rng(seed_base + i)
        n = int(round(n_min * (n_max / n_min) ** rng.uniform()))
        p = int(rng.integers(1, 4))
        out.append({"n": n, "degree": p, "ic": F.circles_union(seed_base + i),
                    "velocity": F.fourier_stream_2d(seed=seed_base + i)})
    return out


def make_batch(instances, precision=abi.FP32, cfl_max=0.1):
    b = Batch([Mesh(2, (d["n"], d["n"])) for d in instances], [d["degree"] for d in instances],
              precision=precision, cfl_max=cfl_max)
    for pb, d in zip(b.problems, instances):
        pb.set_velocity(d["velocity"])
        pb.project(d["ic"])
    return b


def uneven_batch_benchmark(n_problems=256, steps=500, reinit_every=10, n_pseudo=5, compare_problems=256,
                           compare_steps=100):
    """Batched configuration: DoF-steps/s of the whole batch (device time of
    `steps` steps with a reinit every `reinit_every`, CUDA events on the batch
    stream) and the autotuner's report; for comparison, on `compare_problems`
    of the problems (all of them by default), the same problems issued one
    after the other, each in its own graph-replayed run on its own stream (so
    that they overlap on the GPU), and as one group (one graph per period, a
    branch per problem), against the batched launches, all by wall clock
    over `compare_steps` steps."""
    import time
    import torch
    from .lib import check, load
    ctl = abi.default_ls_opts(reinit_frequency=reinit_every,
                              reinit=abi.default_reinit_opts(mode=abi.REINIT_FIXED, n_pseudo_steps=n_pseudo))
    inst = uneven_batch_instances(n_problems)
    b = make_batch(inst, precision=abi.FP32)
    t0 = time.perf_counter()
    tune = b.autotune()
    t_tune = time.perf_counter() - t0
    b.run_steps(reinit_every, ctl)          # warm-up period (captures the graph)
    s = torch.cuda.ExternalStream(b.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(s)
    b.run_steps(steps, ctl, sync=False)
    e1.record(s)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    b.sync()
    finite = all(np.all(np.isfinite(p.get_state())) for p in b.problems[:16])
    n_dofs = b.n_dofs
    # the FP32 run against the same batch in FP64 after the same steps: per
    # problem the L1 interface difference and the relative area difference
    # (FP64 device reductions of the FP64 problem)
    s32 = [p.get_state() for p in b.problems]
    b.close()
    b64 = make_batch(inst, precision=abi.FP64)
    b64.run_steps(reinit_every + steps, ctl)
    l1, darea = [], []
    for pb, st in zip(b64.problems, s32):
        s64 = pb.get_state()
        a64 = pb.reduce(abi.RED_MASS)
        pb.set_state(st)
        a32 = pb.reduce(abi.RED_MASS)
        pb.snapshot()
        pb.set_state(s64)
        l1.append(pb.reduce(abi.RED_L1_INTERFACE))
        darea.append(abs(a32 - a64) / abs(a64))
    b64.close()
    fp32_vs_fp64 = {"steps": reinit_every + steps, "l1_interface_max": float(max(l1)),
                    "l1_interface_mean": float(np.mean(l1)), "area_rel_max": float(max(darea))}
    # the same problems one by one, each its own graph-replayed run on its own stream
    sub = inst[:compare_problems]
    singles = []
    for d in sub:
        pb = Problem(Mesh(2, (d["n"], d["n"])), d["degree"], basis=abi.BASIS_Q, precision=abi.FP32, cfl_max=0.1)
        pb.set_velocity(d["velocity"])
        pb.project(d["ic"])
        check(load().flsp_ls_run_steps(pb.h, C.byref(ctl), reinit_every))
        pb.sync()
        singles.append(pb)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for pb in singles:
        check(load().flsp_ls_run_steps(pb.h, C.byref(ctl), compare_steps))
    for pb in singles:
        pb.sync()
    t_single = time.perf_counter() - t0
    sub_dofs = sum(pb.n_dofs for pb in singles)
    # the same problems as one group: one graph per period, a branch per problem
    g = Group(singles)
    g.run_periods(1, ctl)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    g.run_periods(compare_steps // reinit_every, ctl)
    t_group = time.perf_counter() - t0
    g.close()
    for pb in singles:
        pb.close()
    bs = make_batch(sub, precision=abi.FP32)
    bs.run_steps(reinit_every, ctl)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    bs.run_steps(compare_steps, ctl)
    t_batch_sub = time.perf_counter() - t0
    bs.close()
    return {"problems": n_problems, "n_dofs": n_dofs, "steps": steps, "reinit_every": reinit_every,
            "pseudo_steps": n_pseudo, "device_ms": ms, "dof_steps_per_s": n_dofs * steps / (ms * 1e-3),
            "autotune": tune, "autotune_s": t_tune, "finite": bool(finite), "fp32_vs_fp64": fp32_vs_fp64,
            "streams_vs_batched": {"problems": compare_problems, "steps": compare_steps,
                                  "one_by_one_s": t_single, "batched_s": t_batch_sub,
                                  "one_by_one_dof_steps_per_s": sub_dofs * compare_steps / t_single,
                                  "batched_dof_steps_per_s": sub_dofs * compare_steps / t_batch_sub,
                                  "group_s": t_group,
                                  "group_dof_steps_per_s": sub_dofs * (compare_steps // reinit_every) * reinit_every
                                  / t_group}}


class Group:
    """Several independent problems (any dimension, size or degree) whose
    reinit periods run from ONE captured CUDA graph, one branch per problem
    (flsp_group_* in include/flsp_dg.h).  The problems stay the caller's:
    the group only orders and replays their periods."""

    def __init__(self, problems):
        L = load()
        self.problems = list(problems)
        hs = (C.c_void_p * len(self.problems))(*[p.h for p in self.problems])
        g = C.c_void_p()
        check(L.flsp_group_create(hs, len(self.problems), C.byref(g)))
        self.h = g
        self.n_dofs = sum(p.n_dofs for p in self.problems)

    def close(self):
        if getattr(self, "h", None):
            load().flsp_group_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run_periods(self, n_periods, control, sync=True):
        check(load().flsp_group_run_periods(self.h, C.byref(control), int(n_periods)))
        if sync:
            self.sync()

    def run_periods_learned(self, net, opts, reinit_frequency, n_periods, sync=True):
        """periods with the learned reinitialisation (no fallback)"""
        check(load().flsp_group_run_periods_learned(self.h, net.h, C.byref(opts), int(reinit_frequency),
                                                    int(n_periods)))
        if sync:
            self.sync()

    def sync(self):
        check(load().flsp_group_sync(self.h))

    def stream(self):
        s = C.c_void_p()
        check(load().flsp_group_stream(self.h, C.byref(s)))
        return s.value


def plume_group(n_main=128, n_side=64, n_sides=8, periods=4, reinit_every=5, n_pseudo=5, degree=2, net=None,
                fallback=True, precision=abi.FP32, timed=True, states=False):
    """The large 3D configuration's structure: a main n_main^3 Q2 problem and
    n_sides n_side^3 side problems (plume rolls u = curl(0, psi, 0),
    perturbed-plane ICs with seeds 5, 6, ...), one graph per reinit period
    (reinit_every SSP-RK3 substeps + a fixed n_pseudo-step reinit) covering
    every problem.  Returns DoF-steps/s over all problems (device time, CUDA
    events on the group's stream) and, for the plain reinit, the same
    periods with each problem replayed alone, one after the other.  With
    `net` (the 3D patch network) the reinit is the learned one, with its
    residual fallback decided on the device unless fallback=False.  The
    largest volume change over the problems is reported; states=True also
    returns every problem's final state (host order, FP64)."""
    import torch
    from .learned import default_learned_opts, plain_reinit_opts
    ctl = abi.default_ls_opts(reinit_frequency=reinit_every,
                              reinit=abi.default_reinit_opts(mode=abi.REINIT_FIXED, n_pseudo_steps=n_pseudo))
    lo = default_learned_opts(max_residual=0.05 if fallback else float("inf"))
    lo.fallback = abi.ReinitOpts.from_buffer_copy(plain_reinit_opts())
    lo.fallback.narrow_band = 1
    lo.fallback.band_cells = lo.band_cells
    sizes = [n_main] + [n_side] * n_sides
    probs, vol0 = [], []
    for i, n in enumerate(sizes):
        pb = Problem(Mesh(3, (n, n, n)), degree, basis=abi.BASIS_Q, precision=precision, cfl_max=0.1)
        pb.set_velocity(F.plume_3d())
        pb.project(F.perturbed_plane(seed=5 + i))
        vol0.append(pb.reduce(abi.RED_MASS_SHARP))
        probs.append(pb)
    g = Group(probs)

    def run(n_periods, sync=True):
        if net is None:
            g.run_periods(n_periods, ctl, sync=sync)
        else:
            g.run_periods_learned(net, lo, reinit_every, n_periods, sync=sync)

    run(1)                           # first period (captures the graph)
    s = torch.cuda.ExternalStream(g.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(s)
    run(periods - 1, sync=False)
    e1.record(s)
    e1.synchronize()
    ms_group = e0.elapsed_time(e1)
    g.sync()
    finite = all(bool(np.all(np.isfinite(p.get_state()))) for p in probs)
    dvol = [abs(p.reduce(abi.RED_MASS_SHARP) - v) / v for p, v in zip(probs, vol0)]
    n_dofs = g.n_dofs
    g.close()
    steps = (periods - 1) * reinit_every
    out = {"n_dofs": n_dofs, "problems": len(sizes), "periods": periods, "steps": periods * reinit_every,
           "timed_steps": steps, "device_ms": ms_group,
           "dof_steps_per_s": n_dofs * steps / (ms_group * 1e-3), "finite": finite,
           "max_volume_change": max(dvol), "volume_change": dvol,
           "reinit": ("learned" + (" with the device-side fallback" if fallback else " (no fallback)"))
           if net is not None else "plain"}
    if net is not None:
        tot = [p.learned_totals() for p in probs]
        nb, nf = sum(t[0] for t in tot), sum(t[1] for t in tot)
        out["fallback_fraction"] = nf / nb if (nb and fallback) else None
    if net is None and timed:
        # the same periods, each problem alone (its own graph), one after the other
        ms_alone = 0.0
        for pb in probs:
            check(load().flsp_ls_run_steps(pb.h, C.byref(ctl), reinit_every))   # warm-up / capture
            pb.sync()
            st = torch.cuda.ExternalStream(pb.stream())
            torch.cuda.synchronize()
            e0.record(st)
            check(load().flsp_ls_run_steps(pb.h, C.byref(ctl), steps))
            e1.record(st)
            e1.synchronize()
            ms_alone += e0.elapsed_time(e1)
        out["one_after_another_dof_steps_per_s"] = n_dofs * steps / (ms_alone * 1e-3)
    if states:
        out["states"] = [p.get_state() for p in probs]
    for pb in probs:
        pb.close()
    return out
