"""Benchmark of the level-set hot path: DG advection + HJ reinitialisation.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (the 3D configuration the headline metric is quoted on): degree-2
discontinuous Q (Legendre) elements on a uniform 64^3 hex mesh of the unit
cube (7,077,888 DoFs), sphere r = 0.15 at (0.35, 0.35, 0.35), periodic 3D
deformation field with period T = 3, SSP-RK3 at CFL 0.1, HJ reinit every 10
steps (5 RK1 pseudo-steps, fixed count), FP32 stencil arithmetic.

One bench step = one reinit period: 10 CFL-limited SSP-RK3 substeps plus one
reinitialisation, replayed from a captured CUDA graph.  value = DoF-steps/s
(DoFs x advection substeps / device time), L2 flushed (256 MiB write)
between timed steps.  Under torchrun every rank runs an independent replica
(weak scaling); the time is the max over ranks.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "DG level-set DoF-steps/s, learned vs plain HJ reinit at equal interface error"
WORKLOAD = "3D DG advection + HJ reinit, Q2 Legendre, 64^3 hex mesh, FP32"
N_CELLS = 64
DEGREE = 2
REINIT_EVERY = 10
N_PSEUDO = 5
CFL = 0.1


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--profile", action="store_true",
                    help="short run for ncu: set-up, 2 reinit periods, no timing loops")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64-check", action="store_true",
                    help="skip the FP64 run of the same periods (accuracy of the FP32 mode)")
    ap.add_argument("--no-variants", action="store_true",
                    help="skip the narrow-band and 128^3 variants of the 3D workload")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the batched configuration (256 2D problems, ~30 s)")
    ap.add_argument("--no-learned", action="store_true",
                    help="skip the learned-vs-plain reinitialisation comparison (2D, ~1 min)")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def read_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def read_traffic():
    p = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax = float(parts[2])
                except ValueError:
                    continue
                for nm, v in zip(names, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ----------------------------------------------------------------------
# CPU side: the oracle (CPU FP64 restatement of the reference path)
# ----------------------------------------------------------------------
def cpu_rate(n_slab_z=16, repeats=1):
    """DoF-steps/s of the CPU FP64 restatement on a bounded sample: a
    64 x 64 x n_slab_z slab of the same 64^3 mesh (same cell size), one
    SSP-RK3 step and one reinit pseudo-step, amortised to the workload's
    10 steps + 5 pseudo-steps per period."""
    from oracle import oracle as O
    from felspa_b200 import abi, fields as F
    h = 1.0 / N_CELLS
    pr = O.Problem(3, (N_CELLS, N_CELLS, n_slab_z), DEGREE, abi.BASIS_Q,
                   lo=(0.0, 0.0, 0.3), hi=(1.0, 1.0, 0.3 + n_slab_z * h))
    pr.set_velocity(F.deformation_3d())
    phi = pr.project(F.sphere((0.35, 0.35, 0.35), 0.15))
    t_step, t_pseudo = [], []
    ro = abi.default_reinit_opts(mode=abi.REINIT_FIXED, n_pseudo_steps=1)
    for _ in range(repeats):
        t0 = time.perf_counter()
        pr.advance(phi, 1.0, single_cycle=True, cfl_max=CFL)
        t1 = time.perf_counter()
        pr.reinit(phi, ro)
        t2 = time.perf_counter()
        t_step.append(t1 - t0)
        t_pseudo.append(t2 - t1)
    ts, tp = min(t_step), min(t_pseudo)
    rate = pr.n_dofs * REINIT_EVERY / (REINIT_EVERY * ts + N_PSEUDO * tp)
    return rate, {"step_s": ts, "pseudo_step_s": tp, "n_dofs": pr.n_dofs}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    rates = []
    for _ in range(args.warmup):
        cpu_rate()
    for _ in range(args.steps):
        r, info = cpu_rate()
        rates.append(r)
    value = statistics.median(rates)
    sample = (f"64x64x16 slab of the 64^3 Q2 mesh (same h, {info['n_dofs']} DoFs): 1 SSP-RK3 step + "
              f"1 reinit pseudo-step per bench step, amortised to 10 steps + 5 pseudo-steps")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "DoF-steps/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * info["n_dofs"] * REINIT_EVERY / value,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": {"workload": WORKLOAD.replace("FP32", "FP64 CPU restatement"),
                                        "mesh": "64^3", "degree": 2, "basis": "Q", "reinit_every": 10,
                                        "pseudo_steps": 5, "cfl": CFL},
        "cpu_baseline": {"value": value, "unit": "DoF-steps/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "DoF-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------
# GPU side
# ----------------------------------------------------------------------
def make_problem(precision, device):
    from felspa_b200 import abi, fields as F
    from felspa_b200.level_set import LevelSetSurface, Mesh
    ctl = abi.default_ls_opts(reinit_frequency=REINIT_EVERY,
                              reinit=abi.default_reinit_opts(mode=abi.REINIT_FIXED,
                                                             n_pseudo_steps=N_PSEUDO))
    ls = LevelSetSurface(Mesh(3, (N_CELLS,) * 3), DEGREE, basis=abi.BASIS_Q, precision=precision,
                         cfl_max=CFL, device=device, control=ctl)
    ls.initialize(F.sphere((0.35, 0.35, 0.35), 0.15), F.deformation_3d())
    return ls


def run_ours(args):
    import torch
    from felspa_b200 import abi, build
    from felspa_b200.lib import load

    rank, world, local = dist_env()
    build.build()
    load()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))

    ls = make_problem(abi.FP32, local)
    pb = ls.problem
    n_dofs = pb.n_dofs
    if args.profile:
        ls.run_steps(2 * REINIT_EVERY)
        print(json.dumps({"profile_run": True, "n_dofs": n_dofs}), flush=True)
        return 0

    # stage-kernel tile from the autotuner (timed on this problem; state kept)
    tile, tile_ms = pb.autotune(reps=10)
    stream = torch.cuda.ExternalStream(pb.stream(), device=local)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")
    area0 = ls.integrate_mass()
    pb.snapshot()

    # warm-up (also captures the CUDA graph of one reinit period)
    for _ in range(args.warmup):
        ls.run_steps(REINIT_EVERY)

    sampler = ClockSampler(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    times = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ls.run_steps(REINIT_EVERY, sync=False)
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    torch.cuda.synchronize()
    clocks = sampler.stop()
    total_ms = sum(times)

    # end to end through the C ABI: pinned host state in, period, state out
    host = torch.empty(n_dofs, dtype=torch.float64, pin_memory=True).numpy()
    pb.get_state(out=host)
    e2e_ms = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        pb.set_state(host)
        ls.run_steps(REINIT_EVERY, sync=False)
        pb.get_state(out=host)
        e1.record(stream)
        e1.synchronize()
        e2e_ms.append(e0.elapsed_time(e1))
    torch.cuda.synchronize()

    # FP32 production mode against FP64 on the same periods: L1 interface
    # difference and area (FP64 device reductions of the FP64 handle)
    acc64 = None
    if not args.no_fp64_check:
        periods = args.warmup + 2 * args.steps
        s32 = pb.get_state()
        mass32 = ls.integrate_mass()
        ls64 = make_problem(abi.FP64, local)
        ls64.run_steps(periods * REINIT_EVERY)
        s64 = ls64.problem.get_state()
        mass64 = ls64.integrate_mass()
        ls64.problem.set_state(s32)
        ls64.problem.snapshot()
        ls64.problem.set_state(s64)
        acc64 = {"periods": periods, "l1_interface_fp32_vs_fp64": ls64.problem.reduce(abi.RED_L1_INTERFACE),
                 "area_fp32_vs_fp64_rel": (mass32 - mass64) / mass64,
                 "max_coeff_diff_rel": float(abs(s32 - s64).max() / abs(s64).max())}
        ls64.problem.close()

    # roofline of the dominant kernel (advection stage), events on the library stream
    ms_stage = pb.time_kernel(0, reps=20)
    ms_hj = pb.time_kernel(1, reps=10)
    area1 = ls.integrate_mass()

    if dist:
        t = torch.tensor([total_ms, sum(e2e_ms)], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms, e2e_total = float(t[0]), float(t[1])
    else:
        e2e_total = sum(e2e_ms)

    dof_steps = n_dofs * REINIT_EVERY * args.steps * world
    value = dof_steps / (total_ms * 1e-3)
    e2e_value = dof_steps / (e2e_total * 1e-3)

    s = 4  # bytes per FP32 coefficient
    alg_bytes_per_launch = (8.0 / 3.0) * s * n_dofs   # SSP-RK3: 8 s per DoF-step over 3 stages
    achieved = alg_bytes_per_launch / (ms_stage * 1e-3) / 1e9
    peak, peak_kind = read_peaks()
    tr = read_traffic()
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": (tr or {}).get("adv_stage_bytes_per_launch"),
                "kernel": "adv_sep_kernel<3,2,float>", "ms_per_launch": ms_stage,
                "algorithmic_bytes_per_launch": alg_bytes_per_launch, "peak_source": peak_kind,
                "hj_ms_per_launch": ms_hj}

    per_step_launches = REINIT_EVERY * 5 + 2 + 3 * N_PSEUDO
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return 0

    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        rate, info = cpu_rate()
        cpu = {"value": rate, "unit": "DoF-steps/s", "cores": os.cpu_count() or 1, "kind": "port",
               "sample": (f"CPU FP64 restatement, 64x64x16 slab of the 64^3 Q2 mesh ({info['n_dofs']} DoFs): "
                          f"1 SSP-RK3 step {info['step_s']:.3f}s + 1 pseudo-step {info['pseudo_step_s']:.3f}s, "
                          f"amortised to 10 steps + 5 pseudo-steps")}

    line = {
        "metric": METRIC, "value": value, "unit": "DoF-steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "mesh": "64^3", "degree": 2, "basis": "Q", "n_dofs": n_dofs,
                   "velocity": "3D deformation, T=3", "ic": "sphere r=0.15 at (0.35,0.35,0.35)",
                   "rk": "SSP-RK3", "cfl": CFL, "reinit_every": REINIT_EVERY, "pseudo_steps": N_PSEUDO,
                   "step": "10 SSP-RK3 substeps + 1 reinit, one CUDA graph",
                   "l2": "flushed between steps (256 MiB write)", "parallelism": f"replicas x{world}",
                   "stage_tile": list(tile),
                   "stage_tile_ms": {"x".join(map(str, k)): v for k, v in tile_ms.items()}},
        "roofline": roofline,
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": "DoF-steps/s", "h2d_bytes_per_step": 8 * n_dofs,
                "d2h_bytes_per_step": 8 * n_dofs, "ms_per_step": e2e_total / args.steps},
        "gpu_launches": per_step_launches * args.steps,
        "clocks": clocks,
        "accuracy": {"area_rel_change": (area1 - area0) / area0, "fp32_vs_fp64": acc64},
    }
    if world == 1 and not args.no_learned:
        line["learned_vs_plain"] = learned_comparison()
        line["learned_vs_plain_3d"] = learned_comparison_3d()
    if world == 1 and not args.no_variants:
        from felspa_b200 import fields as F
        line["variants"] = {
            "narrow_band_64cubed": {
                "what": "the headline workload with the compute-restricted narrow band (6 cells) in the reinit",
                **variant_rate(abi.FP32, local, N_CELLS, F.deformation_3d(), F.sphere((0.35, 0.35, 0.35), 0.15), 10,
                               narrow_band=1)},
            "large_128cubed": {
                "what": "large 3D run: 128^3 Q2 FP32 (56.6 M DoFs), plume rolls u = curl(0, psi, 0), "
                        "psi = 0.5 sin(pi x) sin(pi y) sin(pi z)(1 - exp(-t)), perturbed plane z = 0.5 + 0.02 sum of "
                        "16 cosine modes; plain full-sweep reinit",
                **variant_rate(abi.FP32, local, 128, F.plume_3d(), F.perturbed_plane(seed=5), 4)},
        }
        from felspa_b200.batch import plume_group
        line["variants"]["plume_group"] = {
            "what": "a large 3D run with side problems: the 128^3 Q2 FP32 plume problem and 8 side 64^3 problems (perturbed "
                    "planes, seeds 5..13) advanced together, each reinit period (5 SSP-RK3 substeps + a fixed "
                    "5-pseudo-step plain reinit) of all 9 problems replayed from ONE CUDA graph (one branch per "
                    "problem); compared with the same periods replayed problem by problem",
            **plume_group(periods=4)}
        if not args.no_learned:
            # the same group with the learned reinit every 5 steps (the 3D patch network)
            from felspa_b200.learned import MLP, collect_training_pairs_3d
            net3 = MLP(device=0, seed=7, dim=3)
            collect_training_pairs_3d(net3, n=24, instances=8)
            net3.train(steps=3000, batch=8192, lr=1e-3, seed=1)
            line["variants"]["plume_group_learned"] = {
                "what": "the plume group with the learned reinit every 5 steps (the 3x3x3-patch network, "
                        "trained here on 24^3 sphere / plume pairs; no fallback), all 9 problems in one graph per "
                        "period",
                **plume_group(periods=4, net=net3)}
            net3.close()
    if world == 1 and not args.no_batched:
        from felspa_b200.batch import uneven_batch_benchmark
        r = uneven_batch_benchmark()
        line["batched"] = {
            "workload": "256 independent 2D Q problems, meshes log-uniform 32^2..256^2, degree U{1,2,3}, union of 1-4 "
                        "circles, 8-mode Fourier stream-function velocity (seeds default_rng(1000+i)), 500 SSP-RK3 "
                        "steps, fixed 5-pseudo-step reinit every 10, FP32; one persistent launch per RK stage / "
                        "pseudo-step, periods replayed from CUDA graphs, tiles from the autotuner",
            **{k: (round(v, 6) if isinstance(v, float) else v) for k, v in r.items()}}
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()
    return 0


def variant_rate(precision, device, n_cells, velocity, ic, periods, narrow_band=0, band_cells=6.0):
    """DoF-steps/s (device time, CUDA events on the library stream) of `periods`
    reinit periods (10 SSP-RK3 steps + 5 fixed pseudo-steps) of a 3D Q2 problem."""
    import torch
    from felspa_b200 import abi
    from felspa_b200.level_set import LevelSetSurface, Mesh
    ro = abi.default_reinit_opts(mode=abi.REINIT_FIXED, n_pseudo_steps=N_PSEUDO, narrow_band=narrow_band,
                                 band_cells=band_cells)
    ctl = abi.default_ls_opts(reinit_frequency=REINIT_EVERY, reinit=ro)
    ls = LevelSetSurface(Mesh(3, (n_cells,) * 3), DEGREE, basis=abi.BASIS_Q, precision=precision, cfl_max=CFL,
                         device=device, control=ctl)
    # projection only: the reference's initial global sweep (for ICs that are
    # not exact distance functions) diverges on fine 3D meshes without
    # artificial viscosity
    ls.problem.set_velocity(velocity)
    ls.problem.project(ic)
    a0 = ls.integrate_mass()
    ls.run_steps(REINIT_EVERY)   # warm-up, graph capture
    s = torch.cuda.ExternalStream(ls.problem.stream(), device=device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(s)
    ls.run_steps(periods * REINIT_EVERY, sync=False)
    e1.record(s)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    out = {"n_dofs": ls.problem.n_dofs, "periods": periods, "device_ms": ms,
           "dof_steps_per_s": ls.problem.n_dofs * periods * REINIT_EVERY / (ms * 1e-3),
           "area_rel_change": (ls.integrate_mass() - a0) / a0}
    ls.problem.close()
    return out


def learned_comparison():
    """Learned (tensor-core MLP) vs plain HJ reinitialisation on the 2D
    degree-2 slotted-disk revolution; the network is trained here, on the
    GPU, on pairs produced by the plain sweep."""
    from felspa_b200.learned import learned_vs_plain
    r = learned_vs_plain(n=256, instances=32, train_steps=12000)
    runs = {}
    for x in r["runs"]:
        key = x["method"]
        if key == "plain" and x.get("graph_replay"):
            key = "plain_graph"
        elif key == "learned" and x.get("graph_replay"):
            key = "learned_graph_no_fallback"
        elif key == "learned" and x.get("max_residual", 0) > 1e6:
            key = "learned_no_fallback"
        runs[key] = {k: (round(v, 6) if isinstance(v, float) else v) for k, v in x.items()
                     if k not in ("method", "mesh", "graph_replay")}
    best_plain = max(runs["plain"]["dof_steps_per_s"], runs["plain_graph"]["dof_steps_per_s"])
    return {
        "workload": "2D degree-2 Q slotted disk (centre (0.5,0.75), r 0.15, slot 0.05x0.25), 256^2, one CCW "
                    "revolution, CFL 0.1, FP32, reinit every 40 steps; L1 interface error and area change vs "
                    "the initial shape; wall clock of the whole run",
        "plain_reinit": "reference LF HJ sweep, 5 fixed pseudo-steps, LDG viscosity 1e-3, CFL 0.1",
        "learned_reinit": "MLP 82-256x4-9 (BF16 tcgen05) over the 6-cell band; fallback = the plain sweep "
                          "restricted to the band, for cells with mean ||grad phi|-1| > 0.05",
        "training": {k: (round(v, 8) if isinstance(v, float) else v) for k, v in r["training"].items()},
        "runs": runs,
        "learned_vs_best_plain_speed": runs["learned"]["dof_steps_per_s"] / best_plain,
        "learned_no_fallback_vs_best_plain_speed": runs["learned_no_fallback"]["dof_steps_per_s"] / best_plain,
        "learned_graph_no_fallback_vs_best_plain_speed":
            runs["learned_graph_no_fallback"]["dof_steps_per_s"] / best_plain,
    }


def learned_comparison_3d():
    """The 3D patch network (learned reinitialisation of large 3D runs) against the
    plain HJ sweep on the 3D deformation of a sphere over one period."""
    from felspa_b200.learned import learned_vs_plain_3d
    r = learned_vs_plain_3d(n=48, train_n=24, instances=8, train_steps=3000, every=40)
    runs = {}
    for x in r["runs"]:
        key = x["method"]
        if key == "learned" and x.get("max_residual", 0) > 1e6:
            key = "learned_no_fallback"
        runs[key] = {k: (round(v, 6) if isinstance(v, float) else v) for k, v in x.items()
                     if k not in ("method", "mesh")}
    return {
        "workload": "3D degree-2 Q sphere r 0.15 at (0.35,0.35,0.35), 48^3, deformation field over one period "
                    "(T = 3, the shape returns), CFL 0.1, FP32, reinit every 40 steps; plain = 5 fixed "
                    "pseudo-steps (LDG viscosity 1e-3, CFL 0.1: without it the repeated sweep diverges); learned = the 3x3x3-patch network (730 -> 256x4 -> 27) over "
                    "the 6-cell band, fallback to the narrow-band sweep where the cell residual exceeds 0.05; L1 "
                    "interface error and volume change vs the initial sphere; wall-clock DoF-steps/s",
        "training": {k: (round(v, 6) if isinstance(v, float) else v) for k, v in r["training"].items()},
        "runs": runs,
        "learned_vs_plain_speed": runs["learned"]["dof_steps_per_s"] / runs["plain"]["dof_steps_per_s"],
        "learned_no_fallback_vs_plain_speed": runs["learned_no_fallback"]["dof_steps_per_s"]
        / runs["plain"]["dof_steps_per_s"],
    }


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
