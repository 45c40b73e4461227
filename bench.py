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
    ap.add_argument("--profile", nargs="?", const="headline", default=None,
                    choices=["headline", "fe", "batched"],
                    help="short run for ncu, no timing loops: headline = the 64^3 workload's set-up and 2 reinit "
                         "periods; fe = the same with the deformation field at t = 0 as a degree-2 FE velocity "
                         "lattice; batched = the 256-problem batch, autotuned, 2 reinit periods")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64-check", action="store_true",
                    help="skip the FP64 run of the same periods (accuracy of the FP32 mode)")
    ap.add_argument("--no-oracle-checks", action="store_true",
                    help="skip the FP64/FP32 GPU runs against the oracle (64^3 first period, Zalesak revolutions)")
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
def workload_config():
    """the workload, identical on both arms' lines"""
    return {"workload": WORKLOAD, "mesh": "64^3", "degree": DEGREE, "basis": "Q", "n_dofs": 7077888,
            "velocity": "3D deformation, T=3", "ic": "sphere r=0.15 at (0.35,0.35,0.35)", "rk": "SSP-RK3",
            "cfl": CFL, "reinit_every": REINIT_EVERY, "pseudo_steps": N_PSEUDO,
            "step": "one reinit period: 10 SSP-RK3 substeps + a 5-pseudo-step reinit",
            "l2": "GPU: flushed between steps (256 MiB write); CPU: every state vector (57 MB) exceeds its caches"}


class CpuSample:
    """The CPU FP64 restatement on the full 64^3 mesh of the workload.  A
    bench step times one SSP-RK3 substep and one 5-pseudo-step reinit (the
    whole reinitialisation of a period: set-up, CFL pass, 5 pseudo-steps);
    the period's rate amortises them as the GPU does, 10 substeps per
    reinit: rate = n_dofs * 10 / (10 t_substep + t_reinit)."""

    def __init__(self):
        from oracle import oracle as O
        from felspa_b200 import abi, fields as F
        self.abi = abi
        self.pr = O.Problem(3, (N_CELLS,) * 3, DEGREE, abi.BASIS_Q)
        self.pr.set_velocity(F.deformation_3d())
        self.phi = self.pr.project(F.sphere((0.35, 0.35, 0.35), 0.15))
        self.ro = abi.default_reinit_opts(mode=abi.REINIT_FIXED, n_pseudo_steps=N_PSEUDO)
        self.n_dofs = self.pr.n_dofs

    def step(self):
        t0 = time.perf_counter()
        self.pr.advance(self.phi, 1e30, single_cycle=True, cfl_max=CFL)
        t1 = time.perf_counter()
        st, _ = self.pr.reinit(self.phi, self.ro)
        t2 = time.perf_counter()
        if st != 0:
            raise RuntimeError(f"oracle reinit failed ({st})")
        ts, tr = t1 - t0, t2 - t1
        return self.n_dofs * REINIT_EVERY / (REINIT_EVERY * ts + tr), ts, tr


def cpu_sample_text(ts, tr):
    return (f"CPU FP64 restatement (OpenMP, {os.cpu_count() or 1} threads) on the full 64^3 Q2 mesh "
            f"(7,077,888 DoFs): per bench step one SSP-RK3 substep ({ts:.3f} s) and one 5-pseudo-step reinit "
            f"({tr:.3f} s), amortised to the period (10 substeps per reinit)")


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    cs = CpuSample()
    for _ in range(args.warmup):
        cs.step()
    rates, walls, tss, trs = [], [], [], []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        r, ts, tr = cs.step()
        walls.append(time.perf_counter() - t0)
        rates.append(r)
        tss.append(ts)
        trs.append(tr)
    value = statistics.median(rates)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "DoF-steps/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        # wall time of one bench step as run (the timed sample), not the
        # amortised period it stands for
        "ms_per_step": 1e3 * sum(walls) / len(walls),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": workload_config(),
        "cpu_baseline": {"value": value, "unit": "DoF-steps/s", "cores": threads, "kind": "port",
                         "sample": cpu_sample_text(statistics.median(tss), statistics.median(trs)),
                         "period_s_amortised": cs.n_dofs * REINIT_EVERY / value},
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

    if args.profile == "batched":
        from felspa_b200.batch import make_batch, uneven_batch_instances
        b = make_batch(uneven_batch_instances(256), precision=abi.FP32)
        b.autotune()
        ctl = abi.default_ls_opts(reinit_frequency=REINIT_EVERY,
                                  reinit=abi.default_reinit_opts(mode=abi.REINIT_FIXED, n_pseudo_steps=N_PSEUDO))
        b.run_steps(2 * REINIT_EVERY, ctl)
        print(json.dumps({"profile_run": "batched", "n_dofs": b.n_dofs}), flush=True)
        b.close()
        return 0
    ls = make_problem(abi.FP32, local)
    pb = ls.problem
    n_dofs = pb.n_dofs
    if args.profile:
        if args.profile == "fe":
            from felspa_b200 import fields as F
            pb.set_velocity_fe(2, F.fe_lattice(lambda x: F.deformation_3d()(x, 0.0), (N_CELLS,) * 3, 2))
        ls.run_steps(2 * REINIT_EVERY)
        print(json.dumps({"profile_run": args.profile, "n_dofs": n_dofs}), flush=True)
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

    # FP64 mode on the same workload: timed like the FP32 headline, then the
    # FP32 state against the FP64 state after the same periods (L1
    # interface difference and area, FP64 device reductions)
    fp64 = None
    if not args.no_fp64_check:
        s32 = pb.get_state()
        mass32 = ls.integrate_mass()
        ls64 = make_problem(abi.FP64, local)
        p64 = ls64.problem
        st64 = torch.cuda.ExternalStream(p64.stream(), device=local)
        for _ in range(args.warmup):
            ls64.run_steps(REINIT_EVERY)
        t64 = []
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(st64)
            ls64.run_steps(REINIT_EVERY, sync=False)
            e1.record(st64)
            e1.synchronize()
            t64.append(e0.elapsed_time(e1))
        # the FP32 problem also ran the e2e periods
        ls64.run_steps(args.steps * REINIT_EVERY)
        periods = args.warmup + 2 * args.steps
        s64 = p64.get_state()
        mass64 = ls64.integrate_mass()
        p64.set_state(s32)
        p64.snapshot()
        p64.set_state(s64)
        fp64 = {"value": n_dofs * REINIT_EVERY * args.steps / (sum(t64) * 1e-3), "unit": "DoF-steps/s",
                "ms_per_step": sum(t64) / args.steps, "dtype": "f64",
                "what": "the same workload and timing in the FP64 (parity) mode",
                "fp32_vs_fp64": {"periods": periods,
                                 "l1_interface_fp32_vs_fp64": p64.reduce(abi.RED_L1_INTERFACE),
                                 "area_fp32_vs_fp64_rel": (mass32 - mass64) / mass64,
                                 "max_coeff_diff_rel": float(abs(s32 - s64).max() / abs(s64).max())}}
        p64.close()

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
                "hj_ms_per_launch": ms_hj, "hj_algorithmic_bytes_per_launch": 3.0 * s * n_dofs,
                "hj_frac": 3.0 * s * n_dofs / (ms_hj * 1e-3) / 1e9 / peak,
                "stage_tile": list(tile),
                "stage_tile_ms": {"x".join(map(str, k)): v for k, v in tile_ms.items()}}

    per_step_launches = REINIT_EVERY * 5 + 2 + 3 * N_PSEUDO
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return 0

    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        cs = CpuSample()
        rate, t_sub, t_re = cs.step()
        cpu = {"value": rate, "unit": "DoF-steps/s", "cores": os.cpu_count() or 1, "kind": "port",
               "sample": cpu_sample_text(t_sub, t_re)}
        del cs

    line = {
        "metric": METRIC, "value": value, "unit": "DoF-steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(), "parallelism": f"replicas x{world}",
        "roofline": roofline,
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": "DoF-steps/s", "h2d_bytes_per_step": 8 * n_dofs,
                "d2h_bytes_per_step": 8 * n_dofs, "ms_per_step": e2e_total / args.steps},
        "gpu_launches": per_step_launches * args.steps,
        "clocks": clocks,
        "fp64": fp64,
        "accuracy": {"area_rel_change": (area1 - area0) / area0,
                     "fp32_vs_fp64": (fp64 or {}).get("fp32_vs_fp64")},
    }
    if world == 1 and not args.no_oracle_checks:
        line["accuracy"]["sphere_64cubed_vs_oracle"] = sphere_vs_oracle(local)
        line["accuracy"]["zalesak_128"] = zalesak_accuracy(local)
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
        line["variants"]["fe_velocity_64cubed"] = {
            "what": "the headline workload with the velocity of a coupled FE simulator: the deformation field at "
                    "t = 0 as a continuous Q2 nodal field on the Gauss-Lobatto lattice (flsp_set_velocity_fe, "
                    "constant in time), evaluated per cell at the quadrature points by the point-wise stage kernel",
            **variant_rate(abi.FP32, local, N_CELLS, F.deformation_3d(), F.sphere((0.35, 0.35, 0.35), 0.15), 10,
                           fe_degree=2)}
        from felspa_b200.batch import plume_group
        line["variants"]["plume_group"] = {
            "what": "a large 3D run with side problems: the 128^3 Q2 FP32 plume problem and 8 side 64^3 problems (perturbed "
                    "planes, seeds 5..13) advanced together, each reinit period (5 SSP-RK3 substeps + a fixed "
                    "5-pseudo-step plain reinit) of all 9 problems replayed from ONE CUDA graph (one branch per "
                    "problem); compared with the same periods replayed problem by problem",
            **plume_group(periods=40)}
        if not args.no_learned:
            line["variants"]["plume_group_learned"] = plume_group_learned()
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


def sphere_vs_oracle(device):
    """The 3D workload's first reinit period from the projected sphere, FP64
    and FP32 GPU modes against the oracle (CPU FP64, all host cores) on the
    full 64^3 mesh."""
    from oracle import oracle as O
    from felspa_b200 import abi, fields as F
    ic = F.sphere((0.35, 0.35, 0.35), 0.15)
    orc = O.Problem(3, (N_CELLS,) * 3, DEGREE, abi.BASIS_Q)
    orc.set_velocity(F.deformation_3d())
    phi = orc.project(ic)
    ctl = abi.default_ls_opts(reinit_frequency=REINIT_EVERY,
                              reinit=abi.default_reinit_opts(mode=abi.REINIT_FIXED, n_pseudo_steps=N_PSEUDO))
    t0 = time.perf_counter()
    for _ in range(REINIT_EVERY):
        orc.ls_advance(phi, 1e30, ctl, single_step=True, cfl_max=CFL)
    cpu_s = time.perf_counter() - t0
    ref_l1 = orc.reduce(abi.RED_L1_INTERFACE_IC, phi, ic=ic)
    ref_mass = orc.reduce(abi.RED_MASS, phi)
    out = {"what": "64^3 Q2, one reinit period (10 SSP-RK3 substeps + 5 pseudo-steps) from the projected sphere; "
                   "GPU state against the oracle's",
           "oracle_cpu_s": cpu_s, "oracle_threads": os.cpu_count() or 1,
           "oracle_l1_interface_vs_ic": ref_l1}
    for prec, name in ((abi.FP64, "fp64"), (abi.FP32, "fp32")):
        ls = make_problem(prec, device)
        ls.run_steps(REINIT_EVERY)
        got = ls.problem.get_state()
        # L1 interface difference GPU vs oracle: the oracle's state as the snapshot
        ls.problem.set_state(phi)
        ls.problem.snapshot()
        ls.problem.set_state(got)
        out[name] = {"time_diff": ls.get_time() - orc.clock.t,
                     "max_coeff_diff_rel": float(np.abs(got - phi).max() / np.abs(phi).max()),
                     "l1_interface_vs_oracle": ls.problem.reduce(abi.RED_L1_INTERFACE),
                     "area_vs_oracle_rel": (ls.integrate_mass() - ref_mass) / ref_mass}
        ls.problem.close()
    return out


def zalesak_accuracy(device):
    """The 2D Zalesak workload (128^2, degree 1, Q and P bases, one full
    revolution, reinit every 10 substeps with 5 pseudo-steps): FP64 and
    FP32 GPU runs, each with its L1 interface error against the initial
    shape and its area change; beside them the oracle's full-revolution
    run of the FP64 mode (frozen in tests/golden, with the CPU time and
    thread count of the machine that ran it)."""
    from felspa_b200 import abi
    from felspa_b200.zalesak import revolution
    out = {"what": "128^2 degree-1 slotted disk, one CCW revolution (T = 1), SSP-RK3 at CFL 0.1, fixed "
                   "5-pseudo-step reinit every 10 substeps over every cell; L1 interface error vs the initial "
                   "shape, area change; LDG viscosity 0 (as the configuration), 6.28e-5 (the reference test's 1e-3 "
                   "on its [-50,50]^2 domain with period 628, rescaled to the unit square with period 1) and 1e-3"}
    for basis, bname in ((abi.BASIS_Q, "q1"), (abi.BASIS_P, "p1")):
        for nu, nname in ((0.0, "nu0"), (6.28e-5, "nu6.28e-5"), (1e-3, "nu1e-3")):
            key = f"zalesak128_{bname}_{nname}"
            r64 = revolution(basis, nu, abi.FP64, device=device)
            r32 = revolution(basis, nu, abi.FP32, device=device)
            row = {"n_dofs": r64["n_dofs"], "substeps": r64["substeps"], "t_end": r64["t_end"]}
            for r, nm in ((r64, "gpu_fp64"), (r32, "gpu_fp32")):
                row[nm] = {k: r[k] for k in ("l1_interface_error", "area_change_rel", "wall_s", "dof_steps_per_s")}
            row["fp32_vs_fp64_max_coeff_diff_rel"] = float(np.abs(r32["state"] - r64["state"]).max()
                                                           / np.abs(r64["state"]).max())
            gpath = os.path.join(ROOT, "tests", "golden", key + ".npz")
            if os.path.exists(gpath):
                g = np.load(gpath)
                row["oracle_fp64"] = {"l1_interface_error": float(g["l1_ic"]),
                                      "area_change_rel": float((g["area1"] - g["area0"]) / g["area0"]),
                                      "substeps": int(g["n_substeps"]), "cpu_s": float(g["cpu_s"]),
                                      "threads": int(g["threads"]),
                                      "dof_steps_per_s": r64["n_dofs"] * int(g["n_substeps"]) / float(g["cpu_s"])}
                if "result" in g:
                    row["gpu_fp64_vs_oracle_max_coeff_diff_rel"] = float(
                        np.abs(r64["state"] - g["result"]).max() / np.abs(g["result"]).max())
                else:
                    nb = 4 if basis == abi.BASIS_Q else 3
                    row["gpu_fp64_vs_oracle_cell_mean_diff_rel"] = float(
                        np.abs(r64["state"].reshape(-1, nb)[:, 0] - g["cell_means"]).max()
                        / np.abs(g["cell_means"]).max())
            out[key] = row
    return out


def plume_group_learned():
    """The large 3D production configuration as specified: the 128^3 Q2
    plume problem with 8 side 64^3 problems in one graph per period, 2000
    SSP-RK3 steps, the learned reinit (3x3x3-patch network, trained here)
    every 5 steps with its residual fallback decided on the device; FP32,
    and the same run in FP64 for its accuracy (L1 interface difference and
    volume of every problem)."""
    from felspa_b200 import abi
    from felspa_b200.batch import plume_group
    from felspa_b200.learned import MLP, collect_training_pairs_3d
    from felspa_b200.level_set import Mesh, Problem
    net3 = MLP(device=0, seed=7, dim=3)
    collect_training_pairs_3d(net3, n=24, instances=8)
    net3.train(steps=3000, batch=8192, lr=1e-3, seed=1)
    r32 = plume_group(periods=400, net=net3, states=True)
    r64 = plume_group(periods=400, net=net3, precision=abi.FP64, timed=False, states=True)
    nofb = plume_group(periods=40, net=net3, fallback=False)
    net3.close()
    s32, s64 = r32.pop("states"), r64.pop("states")
    l1, dmax = [], []
    for i, (a, b) in enumerate(zip(s32, s64)):
        n = 128 if i == 0 else 64
        pb = Problem(Mesh(3, (n, n, n)), 2, basis=abi.BASIS_Q, precision=abi.FP64)
        pb.set_state(b)
        pb.snapshot()
        pb.set_state(a)
        l1.append(pb.reduce(abi.RED_L1_INTERFACE))
        pb.close()
        dmax.append(float(np.abs(a - b).max() / np.abs(b).max()))
    return {"what": "the large 3D production configuration: 128^3 Q2 FP32 plume problem + 8 x 64^3 side problems in "
                    "one graph per period, 2000 SSP-RK3 steps, learned reinit every 5 steps (3x3x3-patch network "
                    "trained here on 24^3 sphere / plume pairs) with its residual fallback decided on the device",
            **r32,
            "no_fallback_200_steps": {k: nofb[k] for k in ("dof_steps_per_s", "max_volume_change", "steps")},
            "fp64": {"dof_steps_per_s": r64["dof_steps_per_s"], "max_volume_change": r64["max_volume_change"],
                     "fallback_fraction": r64.get("fallback_fraction")},
            "fp32_vs_fp64": {"l1_interface_diff": l1, "max_coeff_diff_rel": dmax,
                             "volume_change_fp32_minus_fp64": [x - y for x, y in zip(r32["volume_change"],
                                                                                      r64["volume_change"])]}}


def variant_rate(precision, device, n_cells, velocity, ic, periods, narrow_band=0, band_cells=6.0, fe_degree=0):
    """DoF-steps/s (device time, CUDA events on the library stream) of `periods`
    reinit periods (10 SSP-RK3 steps + 5 fixed pseudo-steps) of a 3D Q2 problem.
    fe_degree > 0: the velocity is the field at t = 0 sampled on the FE lattice
    of that degree (flsp_set_velocity_fe), constant in time."""
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
    if fe_degree:
        from felspa_b200 import fields as F
        ls.problem.set_velocity_fe(fe_degree, F.fe_lattice(lambda x: velocity(x, 0.0), (n_cells,) * 3, fe_degree))
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
    if fe_degree:
        ms_stage = ls.problem.time_kernel(0, reps=20)
        s_b = 4 if precision == abi.FP32 else 8
        out["stage_ms_per_launch"] = ms_stage
        out["stage_algorithmic_bytes_per_launch"] = (8.0 / 3.0) * s_b * ls.problem.n_dofs
        out["velocity_bytes_per_launch"] = 3 * (fe_degree * n_cells + 1) ** 3 * s_b
    ls.problem.close()
    return out


def learned_comparison():
    """Learned (tensor-core MLP) vs plain HJ reinitialisation at equal L1
    interface error (2D degree-2): the network is trained here, on the GPU,
    on pairs produced by the plain sweep; then for each workload and reinit
    interval the plain sweep, the learned reinit with its residual fallback
    (decided on the device) and without, every run replayed from CUDA
    graphs; speed-ups read off the (L1, rate) fronts at the plain runs' L1."""
    import time
    from felspa_b200 import fields as F
    from felspa_b200.learned import MLP, collect_training_pairs, equal_l1_study
    t0 = time.perf_counter()
    net = MLP(device=0, seed=7)
    n_pairs = collect_training_pairs(net, n=256, instances=32)
    t1 = time.perf_counter()
    loss0 = net.eval()
    last = net.train(steps=12000, batch=8192, lr=1e-3, seed=1)
    t2 = time.perf_counter()
    loss1 = net.eval()
    workloads = {
        "zalesak_rotation": (F.ccw_rotation(), F.zalesak_disk(), 1.0),
        "zalesak_vortex_T2": (F.single_vortex(period=2.0), F.zalesak_disk(), 2.0),
    }
    study = equal_l1_study(net, workloads, n=256)
    net.close()

    def slim(r):
        return {k: (round(v, 6) if isinstance(v, float) else v) for k, v in r.items()
                if k not in ("method", "t", "device_s", "steps")}

    out = {
        "workload": "2D degree-2 Q, 256^2, FP32, CFL 0.1: the slotted disk (centre (0.5,0.75), r 0.15, slot "
                    "0.05x0.25) over one CCW rotation (T = 1) and through the time-reversed single vortex "
                    "(period 2, t = 2); L1 interface error and area change vs the initial shape; device time",
        "plain_reinit": "reference LF HJ sweep over every cell, 5 fixed pseudo-steps, LDG viscosity 1e-3, CFL 0.1",
        "learned_reinit": "MLP 82-256x4-9 (BF16 tcgen05) over the 6-cell band; fallback (max_residual 0.05): cells "
                          "with mean ||grad phi|-1| > 0.05 take the plain sweep run over them, decided on the device",
        "training": {"pairs": n_pairs, "collect_s": round(t1 - t0, 3), "steps": 12000, "batch": 8192,
                     "train_s": round(t2 - t1, 3), "mse_before": loss0, "mse_after": loss1, "last_batch_mse": last},
    }
    for name, r in study.items():
        out[name] = {"steps": r["steps"], "none": slim(r["runs"]["none"]),
                     "plain": [slim(x) for x in r["runs"]["plain"]],
                     "learned": [slim(x) for x in r["runs"]["learned"]],
                     "learned_no_fallback": [slim(x) for x in r["runs"]["learned_no_fallback"]],
                     "equal_l1": r["equal_l1"]}
    return out


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
