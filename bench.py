"""Benchmark of the PIC-MCC timestep: particle-pushes/s on one or more B200s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl b200|reference]

One step = one full timestep of DigitalTwinSimulator (injection, deposit, Picard field
solve on even steps, sub-stepped push with absorption and tallies, compaction, CEX, thermal
and diagnostics) over the workload's particles.  particle-pushes = sum over species of
particles pushed x sub-steps, as the reference counts push calls.

The headline workload is long_erosion_3grid: 513 x 2049 nodes, 48M Xe+ and 16M electrons,
the largest configuration that one GPU holds.  large_aperture_3grid (257 x 1025 nodes, 8M
particles) is reported beside it under "workloads".

value: K steps enqueued back to back with the state resident in HBM, timed with CUDA
       events on the simulator's stream, max over ranks (replicas, weak scaling).
e2e:   K calls of the public DigitalTwinSimulator.step(params) (per-step parameters copied
       in, the step report copied out), wall clock after a device synchronize, on a fresh
       simulator that repeats the timed steps exactly.
roofline: the fused particle kernels, algorithmic bytes 41 B per particle and launch
       (20 B state read + 20 B written + 1 B flag) over each kernel's event-timed duration,
       against the measured HBM copy bandwidth; push + deposit together at 49 B per
       particle-step.  DRAM traffic per particle comes from the committed ncu summary and is
       reported only while the kernel sources still hash to the value recorded there.
sweep: C3-scale perveance sweep (64 points, 0.2M-4M particles, three grid sizes) plain
       against batched, and a C4-scale served run (Poisson arrivals, 1M-6M particles,
       retirement at < 0.5% change over 500 steps).
cpu_baseline: the CPU oracle (a NumPy restatement of the reference step, pinned bit for bit
       to the reference's own outputs) on one core.  A bounded particle sample runs on the
       full grid; its particle time is scaled linearly to the workload's particle count and
       the measured full-grid field-solve time is added once per step.
--impl reference: the same measurement on all host cores, one full-workload replica per
       core (forked after one shared domain build), rank 0 only.
"""
import argparse
import hashlib
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
# The batched sweep enqueues its members' kernels on one stream each; with the default 8
# hardware queues, streams share queues and the host blocks on full ones.  32 queues (the
# most CUDA allows, for this process only, read when the context is created) measured 1.5%
# less device time for the 64-point batch and half the host enqueue time.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

import numpy as np  # noqa: E402

DEFAULT_WORKLOAD = "long_erosion_3grid"
SECOND_WORKLOAD = "large_aperture_3grid"
ALG_BYTES_PUSH = 41     # per particle and fused step-kernel launch
ALG_BYTES_DEPOSIT = 8   # per particle deposited (x, y)
# ncu summaries of the DRAM bytes per particle of the step kernels, one per workload: the
# 513 x 2049 particle state exceeds L2 and moves more bytes per particle than 257 x 1025's
TRAFFIC_PROFILES = {name: os.path.join(ROOT, "profiles", f"dram_traffic_{name}.md")
                    for name in ("long_erosion_3grid", "large_aperture_3grid")}
KERNEL_SOURCES = ("pb_particles.cu", "pb_common.cuh", "pb_kernels.cuh")
# fine phases of pb_sim_phase_times
PHASES = ("inject_deposit", "field_solve", "corners_substeps", "ion_step", "sputter_break", "electron_step",
          "see_spawn", "thermal_grid_sums", "diagnostics_sort")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-sweep", action="store_true")
    ap.add_argument("--no-second", action="store_true", help="skip the large_aperture_3grid line")
    ap.add_argument("--sweep-points", type=int, default=64)
    ap.add_argument("--no-served", action="store_true", help="skip the served section of the sweep")
    ap.add_argument("--serve-requests", type=int, default=16)
    ap.add_argument("--serve-max-steps", type=int, default=20000)
    ap.add_argument("--kernel-options", type=int, default=None,
                    help="PB_OPT_* bits for the step kernels (default: the library's)")
    ap.add_argument("--smoother-sweeps", type=int, default=2,
                    help="damped-Jacobi sweeps on the fine multigrid level (1 or 2)")
    ap.add_argument("--batch-max-coarse", type=int, default=1536,
                    help="coarsest multigrid level of the batched sweep points")
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if p[5 + k].lower() in ("active", "1"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def reduce_over_ranks(t, pushes, device):
    """(max over ranks of the time t, sum over ranks of the pushes), every rank the same."""
    import torch
    import torch.distributed as dist
    a = torch.tensor([float(t)], device=device, dtype=torch.float64)
    dist.all_reduce(a, op=dist.ReduceOp.MAX)
    b = torch.tensor([float(pushes)], device=device, dtype=torch.float64)
    dist.all_reduce(b, op=dist.ReduceOp.SUM)
    return float(a.item()), float(b.item())


def measured_peak_gbs():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def kernel_source_sha():
    h = hashlib.sha256()
    for name in KERNEL_SOURCES:
        with open(os.path.join(ROOT, "thruster_cx_code_b200", "csrc", name), "rb") as f:
            h.update(f.read())
    return h.hexdigest()[:16]


def traffic_table(workload):
    """DRAM bytes per particle of each step kernel from the committed ncu summary of the
    workload: ({kernel: bytes per particle}, note).  Empty when there is none, or when it was
    taken on kernel sources other than the current ones (its 'kernel_source_sha:' line)."""
    path = TRAFFIC_PROFILES.get(workload)
    try:
        with open(path) as f:
            lines = f.read().splitlines()
    except (OSError, TypeError):
        return {}, f"no ncu traffic summary for {workload}"
    sha, table = None, {}
    for ln in lines:
        s = ln.strip()
        if s.startswith("kernel_source_sha:"):
            sha = s.split(":", 1)[1].strip()
        elif s.startswith("dram_bytes_per_particle:"):
            parts = s.split(":", 1)[1].split()
            if len(parts) >= 2:
                table[parts[0]] = float(parts[1])
    cur = kernel_source_sha()
    if sha != cur:
        return {}, f"stale: ncu summary taken on kernel sources {sha}, current {cur}"
    return table, f"ncu summary {os.path.basename(path)} on kernel sources {cur}"


# ----------------------------------------------------------------------------- GPU arm
KERNEL_OPTIONS = None
SMOOTHER_SWEEPS = 2


def make_gpu_sim(name, device, seed):
    from thruster_cx_code_b200 import physics_engine as PE
    from thruster_cx_code_b200 import workloads as W
    from thruster_cx_code_b200 import _lib
    sim = PE.DigitalTwinSimulator(device=device, seed=seed, sort_every=20, solver={"nu": SMOOTHER_SWEEPS})
    if KERNEL_OPTIONS is not None:
        _lib.check(sim._libh.pb_sim_set_kernel_options(sim._h, KERNEL_OPTIONS), "set_kernel_options")
    params = W.configure(sim, name)
    sim.build_domain(params)
    w = W.WORKLOADS[name]
    v_b, v_ti, v_te = W.thermal_speeds(sim, params)
    ions, eles = W.preload(sim.isBound, sim.dx, sim.dy, sim.Lx, sim.Ly, w["n_ions"], w["n_e"], v_b, 4 * v_ti, v_te,
                           seed=seed, x_max_ions=W.plume_boundary(sim, params))
    sim.set_particles("ions", *ions)
    sim.set_particles("electrons", *eles)
    return sim, params


def pushes_of(reports, n_p0, n_e0):
    tot = 0
    np_prev, ne_prev = n_p0, n_e0
    for r in reports:
        tot += (np_prev + r.injected) * r.n_sub_ion + (ne_prev + r.rf_injected + r.neut_injected) * r.n_sub_e
        np_prev, ne_prev = r.num_p, r.num_e
    return tot


def timed_run(sim, params, K, profile=True):
    """K steps through pb_sim_run.  Returns a dict: device ms, reports, fine phase sums
    (ms over the K steps), launches, pushes and the mean particles per step-kernel launch."""
    import ctypes as C
    from thruster_cx_code_b200 import _lib
    lib = _lib.load()
    it0 = sim.iteration
    plist = []
    for k in range(K):
        sim.iteration = it0 + k
        plist.append(sim.step_params(params))
    sim.iteration = it0
    P = (_lib.StepParams * K)(*plist)
    R = (_lib.StepReport * K)()
    n_p0, n_e0 = sim.num_p, sim.num_e
    stats_before = list(sim.last_report.poisson_stats) if sim.last_report is not None else None
    lib.pb_sim_set_profiling(sim._h, 1 if profile else 0)
    mg0 = (C.c_int64 * 8)()
    _lib.check(lib.pb_sim_mg_stats(sim._h, mg0), "pb_sim_mg_stats")
    _lib.check(lib.pb_sim_run(sim._h, P, K, R), "pb_sim_run")
    mg1 = (C.c_int64 * 8)()
    _lib.check(lib.pb_sim_mg_stats(sim._h, mg1), "pb_sim_mg_stats")
    tm = (C.c_double * 9)()
    lib.pb_sim_timing(sim._h, tm)
    ph = (C.c_double * 10)()
    lib.pb_sim_phase_times(sim._h, ph)
    lib.pb_sim_set_profiling(sim._h, 0)
    sim.iteration = it0 + K
    sim._invalidate()
    for r in R:
        sim._apply_report(r, params)
    ions = [(n_p0 if k == 0 else R[k - 1].num_p) + R[k].injected for k in range(K)]
    eles = [(n_e0 if k == 0 else R[k - 1].num_e) + R[k].rf_injected + R[k].neut_injected for k in range(K)]
    return {"ms": float(tm[0]), "reports": R, "phases": {k: float(ph[i]) for i, k in enumerate(PHASES)},
            "launches": int(tm[8]), "pushes": pushes_of(R, n_p0, n_e0), "n_p0": n_p0, "n_e0": n_e0,
            "ions_per_launch": float(np.mean(ions)), "eles_per_launch": float(np.mean(eles)),
            "stats_before": stats_before, "cells_broken": int(sum(r.broken for r in R)),
            "mg_rebuilds": {"device": int(mg1[0] - mg0[0]), "left_to_host": int(mg1[1] - mg0[1]),
                            "host": int(mg1[2] - mg0[2]),
                            "device_ms": {k: (mg1[4 + j] - mg0[4 + j]) / 1e3 for j, k in
                                          enumerate(("levels", "cholesky", "inverse", "transfer"))}}}


def kernel_rooflines(run, K, peak, traffic):
    """Roofline entries of the fused particle kernels and of push + deposit together."""
    ph = run["phases"]
    out = {}
    for kern, phase, n in (("k_ion_step", "ion_step", run["ions_per_launch"]),
                           ("k_ele_step", "electron_step", run["eles_per_launch"])):
        t = ph[phase] / K * 1e-3
        ach = ALG_BYTES_PUSH * n / t / 1e9 if t > 0 else None
        tb = traffic.get(kern)
        out[kern] = {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
                     "frac": ach / peak if ach else None, "launch_ms": t * 1e3, "particles_per_launch": n,
                     "algorithmic_bytes_per_launch": ALG_BYTES_PUSH * n,
                     "traffic": tb * n if tb else None}
    n_all = run["ions_per_launch"] + run["eles_per_launch"]
    t_pd = (ph["ion_step"] + ph["electron_step"] + ph["inject_deposit"]) / K * 1e-3
    ach = (ALG_BYTES_PUSH + ALG_BYTES_DEPOSIT) * n_all / t_pd / 1e9 if t_pd > 0 else None
    out["push_deposit"] = {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
                           "frac": ach / peak if ach else None, "bytes_per_particle_step": 49,
                           "time": "ion step + electron step + injection/deposit phase per step",
                           "ms_per_step": t_pd * 1e3}
    return out


def gpu_arm(args):
    import ctypes as C
    import torch
    from thruster_cx_code_b200 import _lib
    rank, local, world = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    _lib.load()
    sim, params = make_gpu_sim(args.workload, local, seed=1000 + rank)
    for _ in range(args.warmup):
        sim.step(params)
    K = args.steps
    clocks = ClockSampler(local)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clocks.start()
    run = timed_run(sim, params, K)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms, pushes = run["ms"], run["pushes"]
    if world > 1:
        ms_max, pushes_all = reduce_over_ranks(ms, pushes, "cuda")
    else:
        ms_max, pushes_all = ms, float(pushes)
    value = pushes_all / (ms_max * 1e-3)
    ny, nx = sim.ny, sim.nx
    # ---- end to end through the public API, on the same steps: a fresh simulator with
    # the same seed and warm-up reproduces the timed region's workload exactly
    e2e = None
    if not args.no_e2e:
        sim.close()
        del sim
        sim, params = make_gpu_sim(args.workload, local, seed=1000 + rank)
        for _ in range(args.warmup):
            sim.step(params)
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        n_p1, n_e1 = sim.num_p, sim.num_e
        reps = []
        t0 = time.perf_counter()
        for _ in range(K):
            sim.step(params)
            reps.append(sim.last_report)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        pe2e = pushes_of(reps, n_p1, n_e1)
        if world > 1:
            wall, pe2e = reduce_over_ranks(wall, pe2e, "cuda")
        e2e = {"value": pe2e / wall, "unit": "particle-pushes/s", "h2d_bytes_per_step": C.sizeof(_lib.StepParams),
               "d2h_bytes_per_step": C.sizeof(_lib.StepReport), "same_steps_as_value": pe2e == pushes_all}
    peak, peak_kind = measured_peak_gbs()
    traffic, traffic_note = traffic_table(args.workload)
    kr = kernel_rooflines(run, K, peak, traffic)
    # the dominant kernel of the step: the electron step (many sub-steps per launch)
    dom = "k_ele_step" if kr["k_ele_step"]["launch_ms"] >= kr["k_ion_step"]["launch_ms"] else "k_ion_step"
    roof = dict(kr[dom])
    roof.update({"kernel": dom, "peak_source": peak_kind, "traffic_source": traffic_note,
                 "limiter": "instruction issue (float64 weights and conversions per sub-step), not DRAM",
                 "kernels": kr,
                 "phase_ms_per_step": {k: v / K for k, v in run["phases"].items()}})
    line = {"metric": "particle-pushes/s", "value": value, "unit": "particle-pushes/s", "n_gpus": world,
            "steps": K, "warmup": args.warmup, "ms_per_step": ms_max / K, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 weights, field solve and damage)",
            "data": "synthetic (seeded pre-load, Philox injection)",
            "config": {"workload": args.workload, "grid_nodes": [ny, nx], "ions": run["n_p0"],
                       "electrons": run["n_e0"], "parallelism": f"replicas x{world}",
                       "l2": "particle state > L2 (126 MB); no flush needed", "sort_every": 20,
                       "picard": "5 solves every 2nd step, FP32 MG-PCG + FP64 refinement"},
            "cells_broken": run["cells_broken"], "mg_rebuilds": run["mg_rebuilds"],
            "e2e": e2e, "roofline": roof, "clocks": clk, "gpu_launches": run["launches"],
            "kernel_options": kernel_options_of(local)}
    if rank == 0 and world == 1 and run["stats_before"] is not None:
        line["poisson"] = poisson_section(sim, run["stats_before"], run["reports"], run["phases"]["field_solve"],
                                          peak)
    sim.close()
    del sim
    if rank == 0 and world == 1 and not args.no_second and args.workload != SECOND_WORKLOAD:
        line["workloads"] = {SECOND_WORKLOAD: second_workload(args, local, peak, traffic_table(SECOND_WORKLOAD)[0])}
    if rank == 0 and world == 1 and not args.no_sweep:
        line["sweep"] = sweep_section(local, args)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_port(args.workload, args.warmup)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


def kernel_options_of(device):
    """The PB_OPT_* bits the step kernels ran with (a fresh simulator's, or the override)."""
    import ctypes as C
    from thruster_cx_code_b200 import physics_engine as PE
    if KERNEL_OPTIONS is not None:
        return KERNEL_OPTIONS
    s = PE.DigitalTwinSimulator(device=device)
    v = C.c_uint32()
    s._libh.pb_sim_get_kernel_options(s._h, C.byref(v))
    s.close()
    return int(v.value)


def second_workload(args, device, peak, traffic):
    sim, params = make_gpu_sim(SECOND_WORKLOAD, device, seed=1000)
    for _ in range(args.warmup):
        sim.step(params)
    K = args.steps
    run = timed_run(sim, params, K)
    out = {"value": run["pushes"] / (run["ms"] * 1e-3), "unit": "particle-pushes/s", "ms_per_step": run["ms"] / K,
           "grid_nodes": [sim.ny, sim.nx], "ions": run["n_p0"], "electrons": run["n_e0"],
           "roofline": kernel_rooflines(run, K, peak, traffic),
           "phase_ms_per_step": {k: v / K for k, v in run["phases"].items()},
           "cells_broken": run["cells_broken"], "mg_rebuilds": run["mg_rebuilds"]}
    if run["stats_before"] is not None:
        out["poisson"] = poisson_section(sim, run["stats_before"], run["reports"], run["phases"]["field_solve"], peak)
    sim.close()
    return out


# ----------------------------------------------------------------------------- field solve
POISSON_BYTES_LB = 9     # per unknown and linear solve: right-hand side read, phi written, class
POISSON_BYTES_ITER = 72  # per unknown and PCG iteration: ~40 B of Krylov vectors + ~32 B of V-cycle


def poisson_section(sim, stats_before, reports, field_ms, peak):
    """Linear solves/s of the field solve inside the timed steps (recalc_poisson(5) every
    second step, solving for the charge the particles just deposited): solves and PCG
    iterations from the step reports' cumulative solver statistics, time from the
    field-solve phase (CUDA events).  The solve is L2-resident and latency-bound (about 11
    grid-wide phases per PCG iteration), so its bytes are reported against HBM for scale
    only: the lower bound of 9 B per unknown and solve, and a model of 72 B per unknown
    and PCG iteration."""
    import ctypes as C
    from thruster_cx_code_b200 import _lib
    lib = _lib.load()
    cls = np.empty((sim.ny, sim.nx), np.uint8)
    _lib.check(lib.pb_sim_get_field(sim._h, 12, cls.ctypes.data_as(C.c_void_p), cls.nbytes), "get_field")
    unknowns = int(np.count_nonzero(cls == 0))
    last = reports[-1].poisson_stats
    solves = last[3] - stats_before[3]
    if solves <= 0 or field_ms <= 0:
        return {"metric": "linear solves/s", "value": None}
    its = (last[1] - stats_before[1]) / solves
    passes = (last[0] - stats_before[0]) / solves
    s_per_solve = field_ms * 1e-3 / solves
    lb = POISSON_BYTES_LB * unknowns / s_per_solve / 1e9
    model = POISSON_BYTES_ITER * unknowns * its / s_per_solve / 1e9
    return {"metric": "linear solves/s", "value": 1.0 / s_per_solve, "unknowns": unknowns,
            "solves_timed": solves, "ms_per_solve": s_per_solve * 1e3, "pcg_iterations_per_solve": its,
            "refinement_passes_per_solve": passes, "tolerance": sim.solver["tol"],
            "bound": "latency (L2-resident grid)", "peak_hbm_gbs": peak,
            "lower_bound_bytes_per_solve": POISSON_BYTES_LB * unknowns, "lower_bound_gbs": lb,
            "lower_bound_frac": lb / peak if peak else None,
            "model_bytes_per_solve": POISSON_BYTES_ITER * unknowns * its, "model_gbs": model,
            "model_frac": model / peak if peak else None,
            "note": "time is the field-solve phase of the timed steps (Picard right-hand sides, FP64 "
                    "refinement and E included)"}


# ----------------------------------------------------------------------------- sweeps
SWEEP_STEPS, SWEEP_REF_STEPS = 40, 3000
# Each form (plain, batched on streams, batched as step graphs) runs its own copy of the same
# points, built from the same seeds, and times the same steps: two warm-up runs of 20 and 40
# steps, then 40 timed steps (steps 61-100 of every point).  The first warm-up run measures
# each point's field-solve cost for the batch's block plan; the second grows the particle
# buffers to what 40-step runs reserve and, as graphs, captures every step shape (field solve
# or not, buffer parity, the sort step) under that plan.  A point's results are the same bits
# in every form, so the three timed regions do the same work.
SWEEP_WARMUP_RUNS = (20, 40)
# a request retires when the 500-step means of its saddle potential and beamlet current
# change by less than 0.5% from one 500 steps to the next
SERVE_RATE_HZ, SERVE_WINDOW, SERVE_TOL, SERVE_CHUNK = 20.0, 1000, 5e-3, 50
# Served requests live for a few thousand steps at most, so their host set-up weighs on
# the latency: a coarsest multigrid level of <= 256 nodes builds its dense inverse in
# milliseconds instead of about 0.1-0.2 s (17 x 65 nodes), for one more level per V-cycle.
SERVE_SOLVER = {"max_coarse": 256}


def _run_plain(sim, params, K, pushes_out=None, solve_out=None):
    """K steps of one simulator through pb_sim_run; returns the device time (ms) and, if
    ``pushes_out`` / ``solve_out`` are lists, appends the particle-pushes and the field-solve
    time (ms) of those steps."""
    run = timed_run(sim, params, K, profile=solve_out is not None)
    if pushes_out is not None:
        pushes_out.append(run["pushes"])
    if solve_out is not None:
        solve_out.append(run["phases"]["field_solve"])
    return run["ms"]


def _build_all(specs, device, solver=None, workers=8):
    from concurrent.futures import ThreadPoolExecutor
    from thruster_cx_code_b200 import workloads as W
    with ThreadPoolExecutor(max_workers=workers) as pool:
        return list(pool.map(lambda sp: W.make_sweep_sim(sp, device, solver=solver), specs))


def sweep_section(device, args):
    """Sweep points per hour, plain against batched, on C3 perveance-sweep points: screen
    600-1800 V, accel -300..-100 V, plasma density log-uniform 3e16-3e17 m^-3, grids drawn
    from {64x256, 128x512, 256x1024} cells and 0.2M-4M macro-particles log-uniform.  Plain:
    each point alone through pb_sim_run.  Batched: all points together through pb_batch_run,
    with every member's kernels enqueued on its own stream, and with each batch step shape
    captured as one CUDA graph and replayed; the faster form is the one reported as batched,
    both are listed.  Each form runs its own copy of the same points and times the same steps
    (SWEEP_WARMUP_RUNS), so the three timed regions do the same work (``same_work`` checks
    the pushes).  Rates use device time, scaled to 3000 steps per point; setup is excluded.
    Then the C4 served run."""
    from thruster_cx_code_b200 import serving as SV
    from thruster_cx_code_b200 import workloads as W
    rng = np.random.default_rng(7)
    npts = args.sweep_points
    specs = [W.sweep_point(rng, i, n_range=(2e5, 4e6)) for i in range(npts)]
    t_setup = time.perf_counter()
    built = _build_all(specs, device)
    t_setup = time.perf_counter() - t_setup
    for s, p in built:
        for k in SWEEP_WARMUP_RUNS:
            _run_plain(s, p, k)
    plain_pushes, plain_solve = [], []
    plain_ms = sum(_run_plain(s, p, SWEEP_STEPS, plain_pushes, plain_solve) for s, p in built)
    for s, _ in built:
        s.close()

    batch = SV.SweepBatch(device)

    def batched(graphs):
        """One batched form on a fresh copy of the points; returns device ms, host enqueue ms,
        pushes, field-solve ms and the graph captures that fell in the timed steps."""
        sb = _build_all(specs, device)
        sims, prm = [s for s, _ in sb], [p for _, p in sb]
        # the batched points' coarsest level (default: the plain points' own; 256 measured slower)
        if args.batch_max_coarse != 1536:
            from thruster_cx_code_b200 import autotune as AT
            for s in sims:
                AT.apply(s, {"max_coarse": args.batch_max_coarse})
        batch.set_graphs(graphs)
        for k in SWEEP_WARMUP_RUNS:
            batch.run(sims, prm, k)
        n0 = [(s.num_p, s.num_e) for s in sims]
        g0 = batch.graph_stats()
        res = batch.run(sims, prm, SWEEP_STEPS)
        captures = batch.graph_stats()[0] - g0[0]
        pushes = sum(SV.pushes_of([rep for _, rep in r], a, b) for r, (a, b) in zip(res, n0))
        out = (batch.last_ms, batch.last_host_ms, pushes, batch.last_solve_ms, captures)
        batch.set_graphs(False)
        for s in sims:
            s.close()
        return out

    streams_ms, streams_host_ms, streams_pushes, streams_solve_ms, _ = batched(False)
    graph_ms, graph_host_ms, graph_pushes, graph_solve_ms, graph_timed_captures = batched(True)
    g_stats = batch.graph_stats()
    # the batched form reported: the faster of the two (graphs only when no capture failed)
    use_graphs = not g_stats[2] and graph_ms < streams_ms
    if use_graphs:
        batched_ms, batched_host_ms, batched_pushes = graph_ms, graph_host_ms, graph_pushes
    else:
        batched_ms, batched_host_ms, batched_pushes = streams_ms, streams_host_ms, streams_pushes
    per_point_plain_s = plain_ms / SWEEP_STEPS * SWEEP_REF_STEPS / 1e3 / npts
    per_point_batched_s = batched_ms / SWEEP_STEPS * SWEEP_REF_STEPS / 1e3 / npts
    peak, _ = measured_peak_gbs()
    out = {"points": npts, "steps_timed": SWEEP_STEPS, "steps_per_point": SWEEP_REF_STEPS,
           "grids": sorted({sp["grid"] for sp in specs}),
           "particles": [int(min(sp["n_ions"] + sp["n_e"] for sp in specs)),
                         int(max(sp["n_ions"] + sp["n_e"] for sp in specs))],
           "plain_points_per_hr": 3600.0 / per_point_plain_s,
           "batched_points_per_hr": 3600.0 / per_point_batched_s,
           "batched_over_plain": plain_ms / batched_ms,
           "plain_device_ms": plain_ms, "plain_field_solve_ms": float(sum(plain_solve)),
           "batched_device_ms": batched_ms, "batched_host_enqueue_ms": batched_host_ms,
           "batched_form": "graphs" if use_graphs else "streams",
           "solver": {"plain_max_coarse": 1536, "batched_max_coarse": args.batch_max_coarse,
                      "smoother_sweeps": SMOOTHER_SWEEPS},
           "graph_captures_replays_failed": list(g_stats),
           "graph_captures_in_timed_steps": graph_timed_captures,
           "streams": {"points_per_hr": 3600.0 / (streams_ms / SWEEP_STEPS * SWEEP_REF_STEPS / 1e3 / npts),
                       "device_ms": streams_ms, "host_enqueue_ms": streams_host_ms,
                       "field_solve_ms": streams_solve_ms,
                       "over_plain": plain_ms / streams_ms},
           "graphs": {"points_per_hr": 3600.0 / (graph_ms / SWEEP_STEPS * SWEEP_REF_STEPS / 1e3 / npts),
                      "device_ms": graph_ms, "host_enqueue_ms": graph_host_ms,
                      "field_solve_ms": graph_solve_ms if graph_solve_ms >= 0 else None,
                      "over_plain": plain_ms / graph_ms},
           "steps": f"each form on its own copy of the points: warm-up runs of {SWEEP_WARMUP_RUNS} steps, "
                    f"then steps {sum(SWEEP_WARMUP_RUNS) + 1}-{sum(SWEEP_WARMUP_RUNS) + SWEEP_STEPS} timed",
           "same_work": float(sum(plain_pushes)) == float(streams_pushes) == float(graph_pushes),
           "setup": f"excluded ({t_setup:.1f} s per copy of host geometry, multigrid build and pre-load on 8 threads)"}
    for name, pushes, ms in (("plain", float(sum(plain_pushes)), plain_ms),
                             ("batched", float(batched_pushes), batched_ms)):
        rate = pushes / (ms * 1e-3)
        out[f"{name}_pushes"] = pushes
        out[f"{name}_pushes_per_s"] = rate
        out[f"{name}_hbm_frac"] = rate * ALG_BYTES_PUSH / 1e9 / peak if peak else None
    out["served"] = None if args.no_served else served_section(device, batch, args)
    batch.close()
    return out


def served_section(device, batch, args):
    """C4 served backstreaming-limit sweep: requests arrive as a Poisson stream (20/s);
    each draws accel voltage -300..-50 V, neutralizer electron injection 0.1-1 A/m^2 at
    2 eV, a grid of 128x512 or 256x1024 cells and 1M-6M macro-particles.  Admission is
    gated at 150 GB of device memory, set-up runs on host threads while the GPU steps the
    admitted requests in chunks of 50, and a request retires once the 500-step means of its
    centreline saddle potential and beamlet current change by less than 0.5% from one 500
    steps to the next (or at the step cap).  Latencies include set-up."""
    from thruster_cx_code_b200 import serving as SV
    from thruster_cx_code_b200 import workloads as W
    rs = np.random.default_rng(11)
    arrivals = []
    t = 0.0
    for i in range(args.serve_requests):
        t += rs.exponential(1.0 / SERVE_RATE_HZ)
        sp = W.served_point(rs, 100 + i)
        # beamlet current (A) = ions crossing per step x q w / dt
        cell_vol = (sp["dx"] * 1e-3) ** 2 * 1e-3
        w = max(sp["params"]["n0_plasma"] * cell_vol / 80.0, 1e3)
        per_crossing = 1.602e-19 * w / sp["dt"]
        req = SV.Request(i, (lambda sp=sp: W.make_sweep_sim(sp, device, solver=SERVE_SOLVER)),
                         W.sweep_point_bytes(sp), args.serve_max_steps,
                         SV.Convergence(window=SERVE_WINDOW, tol=SERVE_TOL, keys=("current", "saddle"),
                                        counts={"current": per_crossing}))
        req.dt_over_qw = 1.0 / per_crossing
        arrivals.append((t, req))
    srv = SV.SweepServer(device, hbm_budget_bytes=150e9, max_active=64, chunk=SERVE_CHUNK, batch=batch,
                         setup_workers=max(2, min(8, (os.cpu_count() or 2) // 2)))
    srv.serve(arrivals)
    st = srv.stats()
    st.update({"requests": args.serve_requests, "arrival_rate_hz": SERVE_RATE_HZ, "max_steps": args.serve_max_steps,
               "retire_rule": f"{SERVE_WINDOW // 2}-step means of saddle and current change < {SERVE_TOL:g} "
                              f"over {SERVE_WINDOW // 2} steps (the current: or within twice the Poisson noise "
                              f"of its crossing counts)",
               "current_noise": [round(r.conv.noise("current"), 5) for r in srv.done],
               "steps": [r.steps for r in srv.done], "particle_pushes": srv.pushes, "gpu_ms": srv.gpu_ms,
               "final_changes": [{k: round(v, 5) for k, v in r.conv.changes().items()} for r in srv.done],
               "mean_crossings_per_step": [float(np.mean(r.conv.hist["current"][-SERVE_WINDOW:])) * r.dt_over_qw
                                           for r in srv.done]})
    srv.active = []
    return st


# ----------------------------------------------------------------------------- CPU oracle
def _oracle_domain(name):
    from oracle.pic_oracle import OracleSimulator
    from thruster_cx_code_b200.domain import build_domain_geometry
    from thruster_cx_code_b200 import workloads as W
    o = OracleSimulator(build_domain_geometry)
    params = W.configure(o, name)
    o.build_domain(params)
    return o, params


def _oracle_load(o, params, name, n_ions, n_e, seed):
    from thruster_cx_code_b200 import workloads as W
    v_b, v_ti, v_te = W.thermal_speeds(o, params)
    ions, eles = W.preload(o.isBound, o.dx, o.dy, o.Lx, o.Ly, n_ions, n_e, v_b, 4 * v_ti, v_te, seed=seed,
                           x_max_ions=W.plume_boundary(o, params))
    o._add_ions(*ions, np.zeros(n_ions, bool), o.new_ion_ids(n_ions))
    o._add_electrons(*eles, o.new_e_ids(n_e))


def _oracle_steps(o, params, k, seed):
    """k oracle steps: (pushes, particle-phase seconds, field-solve seconds)."""
    from oracle.pic_oracle import PhiloxDraws
    draws = PhiloxDraws(seed)
    solve = o.recalc_poisson
    t_field = [0.0]

    def timed_solve(*a, **kw):
        t0 = time.perf_counter()
        r = solve(*a, **kw)
        t_field[0] += time.perf_counter() - t0
        return r

    o.recalc_poisson = timed_solve
    pushes = 0
    t0 = time.perf_counter()
    for _ in range(k):
        n_p, n_e = o.num_p, o.num_e
        o.step(params, draws)
        inj = o.injected_ions_step
        pushes += (n_p + inj) * o.n_sub_ion + (n_e + int(params.get("neut_rate", 30))) * o.n_sub_e
    total = time.perf_counter() - t0
    o.recalc_poisson = solve
    return pushes, total - t_field[0], t_field[0]


def _extrapolate(name, frac, pushes, t_part, t_field, k):
    """Full-workload step of one instance from a sample of ``frac`` of its particles on
    the full grid: particle work scales with the particle count, the field solve does not.
    Returns (pushes per full step, seconds per full step)."""
    return pushes / k / frac, t_part / k / frac + t_field / k


def cpu_baseline_port(name, warmup, frac=1 / 1000, steps=4):
    from thruster_cx_code_b200 import workloads as W
    w = W.WORKLOADS[name]
    ni, ne = max(1, int(w["n_ions"] * frac)), max(1, int(w["n_e"] * frac))
    o, params = _oracle_domain(name)
    _oracle_load(o, params, name, ni, ne, seed=5)
    if warmup:
        _oracle_steps(o, params, warmup, seed=5)
    pushes, t_part, t_field = _oracle_steps(o, params, steps, seed=5)
    ps, ts = _extrapolate(name, frac, pushes, t_part, t_field, steps)
    return {"value": ps / ts, "unit": "particle-pushes/s", "cores": 1, "kind": "port",
            "sample": f"{name}: {ni} ions + {ne} electrons ({frac:.4g} of the workload) on the full "
                      f"{o.ny} x {o.nx} grid, {warmup} warm-up + {steps} timed steps of the NumPy/SciPy oracle of "
                      f"the reference step; particle time x {1 / frac:.0f} plus the measured SuperLU Picard "
                      f"time per step ({t_field / steps:.3f} s)",
            "sample_pushes_per_s": pushes / (t_part + t_field)}


def _ref_worker(args):
    name, ni, ne, seed, warm, k, frac = args
    o, params = _REF_DOMAIN
    _oracle_load(o, params, name, ni, ne, seed)
    if warm:
        _oracle_steps(o, params, warm, seed)
    return _oracle_steps(o, params, k, seed)


_REF_DOMAIN = None


def reference_arm(args):
    """The reference's CPU path (the oracle port: the reference's own source tree is not on
    the bench host) on all host cores.  One domain build, then one forked worker per core, each a
    replica of the workload run on a particle sample; each replica's step time is its
    particle time scaled to the workload's particle count plus its full-grid field-solve
    time.  value = replicas x pushes per full step / the slowest replica's step time."""
    global _REF_DOMAIN
    rank, _, world = dist_env()
    if rank != 0:
        return
    os.environ["OMP_NUM_THREADS"] = "1"
    import multiprocessing as mp
    from thruster_cx_code_b200 import workloads as W
    w = W.WORKLOADS[args.workload]
    P = max(1, min(os.cpu_count() or 1, 64))
    frac = 1 / 1000 if w["n_ions"] + w["n_e"] > 20_000_000 else 1 / 200
    ni, ne = max(1, int(w["n_ions"] * frac)), max(1, int(w["n_e"] * frac))
    t0 = time.perf_counter()
    _REF_DOMAIN = _oracle_domain(args.workload)
    t_build = time.perf_counter() - t0
    ctx = mp.get_context("fork")  # no GPU is touched in this process
    with ctx.Pool(P) as pool:
        res = pool.map(_ref_worker, [(args.workload, ni, ne, 11 + i, args.warmup, args.steps, frac)
                                     for i in range(P)])
    full = [_extrapolate(args.workload, frac, *r, args.steps) for r in res]
    step_s = max(t for _, t in full)
    pushes_step = sum(p for p, _ in full)
    value = pushes_step / step_s
    o = _REF_DOMAIN[0]
    sample = (f"{P} forked processes, each a replica of {args.workload} ({o.ny} x {o.nx} grid) run on "
              f"{ni} ions + {ne} electrons ({frac:.4g} of the workload's particles) for {args.warmup} warm-up + "
              f"{args.steps} timed steps; each replica's particle time x {1 / frac:.0f} plus its full-grid "
              f"SuperLU Picard time ({statistics.mean(r[2] for r in res) / args.steps:.3f} s per step) is its "
              f"full-workload step; domain build {t_build:.1f} s, once, not timed")
    line = {"impl": "reference", "metric": "particle-pushes/s", "value": value, "unit": "particle-pushes/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_s * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 (NumPy, f64 potential)",
            "data": "synthetic (seeded pre-load)",
            "config": {"workload": args.workload, "grid_nodes": [o.ny, o.nx], "ions": w["n_ions"],
                       "electrons": w["n_e"], "replicas": P},
            "cpu_baseline": {"value": value, "unit": "particle-pushes/s", "cores": P, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "particle-pushes/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


if __name__ == "__main__":
    a = parse()
    KERNEL_OPTIONS = a.kernel_options
    SMOOTHER_SWEEPS = a.smoother_sweeps
    if a.impl == "reference":
        reference_arm(a)
    else:
        gpu_arm(a)
