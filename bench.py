"""Benchmark of the PIC-MCC timestep: particle-pushes/s on one or more B200s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl b200|reference]

One step = one full timestep of DigitalTwinSimulator (injection, deposit, Picard field
solve on even steps, sub-stepped push with absorption and tallies, compaction, CEX, thermal
and diagnostics) over the workload's particles.  particle-pushes = sum over species of
particles pushed x sub-steps, as the reference counts push calls.

value: K steps enqueued back to back with the state resident in HBM, timed with CUDA
       events on the simulator's stream, max over ranks (replicas, weak scaling).
e2e:   K calls of the public DigitalTwinSimulator.step(params) (per-step parameters copied
       in, the step report copied out), wall clock after a device synchronize.
roofline: the fused ion-step kernel, algorithmic bytes 41 B per ion per launch
       (20 B state read + 20 B written + 1 B flag) over its event-timed duration, against
       the measured HBM copy bandwidth.
cpu_baseline: the CPU oracle (a NumPy restatement of the reference step, numerically the
       reference's own path) on one core, on a bounded sample of the same workload.
--impl reference: the same oracle on all host cores (one process per core, each stepping
       the workload's grid with an equal share of the particles), rank 0 only.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

DEFAULT_WORKLOAD = "large_aperture_3grid"
ALG_BYTES_PER_ION = 41


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


def ion_step_traffic_per_ion():
    """DRAM bytes per ion of one k_ion_step launch, from the 'dram_bytes_per_ion:' line of
    the committed ncu summary, if present."""
    try:
        with open(os.path.join(ROOT, "profiles", "k_ion_step_large_aperture_3grid.md")) as f:
            for line in f:
                if line.strip().startswith("dram_bytes_per_ion:"):
                    return float(line.split(":", 1)[1].split()[0])
    except Exception:
        pass
    return None


# ----------------------------------------------------------------------------- GPU arm
def make_gpu_sim(name, device, seed):
    from thruster_cx_code_b200 import physics_engine as PE
    from thruster_cx_code_b200 import workloads as W
    sim = PE.DigitalTwinSimulator(device=device, seed=seed, sort_every=20)
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
    lib = _lib.load()
    sim, params = make_gpu_sim(args.workload, local, seed=1000 + rank)
    for _ in range(args.warmup):
        sim.step(params)
    # ---- device-timed region: K steps enqueued back to back
    K = args.steps
    plist = []
    it0 = sim.iteration
    for k in range(K):
        sim.iteration = it0 + k
        plist.append(sim.step_params(params))
    sim.iteration = it0
    P = (_lib.StepParams * K)(*plist)
    R = (_lib.StepReport * K)()
    n_p0, n_e0 = sim.num_p, sim.num_e
    stats_before = list(sim.last_report.poisson_stats) if sim.last_report is not None else None
    lib.pb_sim_set_profiling(sim._h, 1)
    clocks = ClockSampler(local)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clocks.start()
    _lib.check(lib.pb_sim_run(sim._h, P, K, R), "pb_sim_run")
    torch.cuda.synchronize()
    clk = clocks.stop()
    tm = (C.c_double * 9)()
    lib.pb_sim_timing(sim._h, tm)
    lib.pb_sim_set_profiling(sim._h, 0)
    ms = float(tm[0])
    sim.iteration = it0 + K
    sim._invalidate()
    for r in R:
        sim._apply_report(r, params)
    pushes = pushes_of(R, n_p0, n_e0)
    ion_ms_total = float(tm[4])
    ions_per_launch = float(np.mean([n_p0 if k == 0 else R[k - 1].num_p for k in range(K)]) +
                        np.mean([r.injected for r in R]))
    if world > 1:
        ms_max, pushes_all = reduce_over_ranks(ms, pushes, "cuda")
    else:
        ms_max, pushes_all = ms, float(pushes)
    value = pushes_all / (ms_max * 1e-3)
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
    ion_launch_s = ion_ms_total / K * 1e-3
    achieved = ALG_BYTES_PER_ION * ions_per_launch / ion_launch_s / 1e9 if ion_launch_s > 0 else None
    tpi = ion_step_traffic_per_ion()
    roof = {"kernel": "k_ion_step", "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak if achieved else None, "peak_source": peak_kind,
            "traffic": tpi * ions_per_launch if tpi else None,
            "algorithmic_bytes_per_launch": ALG_BYTES_PER_ION * ions_per_launch,
            "launch_ms": ion_launch_s * 1e3,
            "phase_ms_per_step": {k: float(tm[i + 1]) / K for i, k in enumerate(
                ["inject_deposit", "field_solve", "substep_reduce", "ion_step", "electron_step", "thermal_diag_sort"])}}
    line = {"metric": "particle-pushes/s", "value": value, "unit": "particle-pushes/s", "n_gpus": world,
            "steps": K, "warmup": args.warmup, "ms_per_step": ms_max / K, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 weights, field solve and damage)",
            "data": "synthetic (seeded pre-load, Philox injection)",
            "config": {"workload": args.workload, "grid_nodes": [sim.ny, sim.nx], "ions": n_p0, "electrons": n_e0,
                       "parallelism": f"replicas x{world}", "l2": "particle state 8M x 25 B x 2 > L2 (126 MB)",
                       "sort_every": 20, "picard": "5 solves every 2nd step, FP32 MG-PCG + FP64 refinement"},
            "e2e": e2e, "roofline": roof, "clocks": clk, "gpu_launches": int(tm[8])}
    if rank == 0 and world == 1 and stats_before is not None:
        line["poisson"] = poisson_section(sim, stats_before, R, float(tm[2]), peak)
    if rank == 0 and world == 1 and not args.no_sweep:
        sim.close()
        line["sweep"] = sweep_section(local)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_port(args.workload)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    sim.close()
    if rank == 0:
        print(json.dumps(line))


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
SWEEP_POINTS, SWEEP_WARMUP, SWEEP_STEPS, SWEEP_REF_STEPS = 16, 2, 40, 3000
SERVE_REQUESTS, SERVE_RATE_HZ, SERVE_MAX_STEPS = 12, 20.0, 100
# Served requests live for at most a few hundred steps, so their host set-up weighs more
# than their stepping: a coarsest multigrid level of <= 256 nodes builds its dense inverse
# in milliseconds instead of about 0.1-0.2 s (17 x 65 nodes), for one more level per V-cycle.
SERVE_SOLVER = {"max_coarse": 256}


def _run_plain(sim, params, K, pushes_out=None):
    """K steps of one simulator through pb_sim_run; returns the device time (ms) and, if
    ``pushes_out`` is a list, appends the particle-pushes of those steps."""
    import ctypes as C
    from thruster_cx_code_b200 import _lib
    lib = _lib.load()
    n_p0, n_e0 = sim.num_p, sim.num_e
    it0 = sim.iteration
    plist = []
    for k in range(K):
        sim.iteration = it0 + k
        plist.append(sim.step_params(params))
    sim.iteration = it0
    P = (_lib.StepParams * K)(*plist)
    R = (_lib.StepReport * K)()
    _lib.check(lib.pb_sim_run(sim._h, P, K, R), "pb_sim_run")
    tm = (C.c_double * 9)()
    lib.pb_sim_timing(sim._h, tm)
    sim.iteration = it0 + K
    sim._invalidate()
    for r in R:
        sim._apply_report(r, params)
    if pushes_out is not None:
        pushes_out.append(pushes_of(R, n_p0, n_e0))
    return float(tm[0])


def sweep_section(device):
    """Sweep points per hour, plain (one instance at a time through pb_sim_run) against
    batched (all points together through pb_batch_run), on two identical sets of 16
    perveance-sweep points (C3 draws, 0.2M-1M macro-particles).  Rates use the device time
    of 40 steps after 2 warm-up steps, scaled to 3000 steps per point; setup is not
    included.  The same steps are also given as particle-pushes/s and as the fraction of
    HBM peak their algorithmic bytes (41 B per push) would take.  Then a served run: 12 backstreaming-limit requests arriving as a Poisson
    stream at 20 per second, admitted under a 150 GB budget, built on up to 8 setup threads
    (with a coarsest multigrid level of <= 256 nodes, SERVE_SOLVER), stepped in chunks of 10
    and retired when the saddle potential and current change less than 5% between the
    halves of a 60-step window (or at 100 steps).  Its latencies include setup."""
    from thruster_cx_code_b200 import serving as SV
    from thruster_cx_code_b200 import workloads as W
    rng = np.random.default_rng(7)
    specs = [W.sweep_point(rng, i, n_range=(2e5, 1e6)) for i in range(SWEEP_POINTS)]
    batch = SV.SweepBatch(device)
    plain = [W.make_sweep_sim(sp, device) for sp in specs]
    for s, p in plain:
        _run_plain(s, p, SWEEP_WARMUP)
    plain_pushes = []
    plain_ms = sum(_run_plain(s, p, SWEEP_STEPS, plain_pushes) for s, p in plain)
    for s, _ in plain:
        s.close()
    together = [W.make_sweep_sim(sp, device) for sp in specs]
    sims, prm = [s for s, _ in together], [p for _, p in together]
    batch.run(sims, prm, SWEEP_WARMUP)
    n0 = [(s.num_p, s.num_e) for s in sims]
    res = batch.run(sims, prm, SWEEP_STEPS)
    batched_ms = batch.last_ms
    batched_pushes = sum(SV.pushes_of([rep for _, rep in r], a, b) for r, (a, b) in zip(res, n0))
    for s in sims:
        s.close()
    per_point_plain_s = plain_ms / SWEEP_STEPS * SWEEP_REF_STEPS / 1e3 / SWEEP_POINTS
    per_point_batched_s = batched_ms / SWEEP_STEPS * SWEEP_REF_STEPS / 1e3 / SWEEP_POINTS
    out = {"points": SWEEP_POINTS, "steps_timed": SWEEP_STEPS, "steps_per_point": SWEEP_REF_STEPS,
           "grids": sorted({sp["grid"] for sp in specs}),
           "plain_points_per_hr": 3600.0 / per_point_plain_s,
           "batched_points_per_hr": 3600.0 / per_point_batched_s,
           "batched_over_plain": plain_ms / batched_ms,
           "setup": "excluded (host geometry, multigrid build and pre-load)"}
    # the same steps as particle-pushes/s, and their algorithmic bytes (41 B per push) against HBM
    peak, _ = measured_peak_gbs()
    for name, pushes, ms in (("plain", float(sum(plain_pushes)), plain_ms), ("batched", float(batched_pushes),
                                                                             batched_ms)):
        rate = pushes / (ms * 1e-3)
        out[f"{name}_pushes_per_s"] = rate
        out[f"{name}_hbm_frac"] = rate * ALG_BYTES_PER_ION / 1e9 / peak if peak else None
    # ---- served
    rs = np.random.default_rng(11)
    arrivals = []
    t = 0.0
    for i in range(SERVE_REQUESTS):
        t += rs.exponential(1.0 / SERVE_RATE_HZ)
        sp = W.sweep_point(rs, 100 + i, grids=("64x256", "128x512"), n_range=(2e5, 8e5))
        sp["params"]["grids"][1]["V"] = float(rs.uniform(-300.0, -50.0))
        sp["params"]["Te"] = 2.0
        j = rs.uniform(0.1, 1.0)  # neutralizer electron current density, A/m^2
        area = 0.5 * 0.95e-3 * 1e-3 + 0.3 * 3.75e-3 * 1e-3
        sp["params"]["neut_rate"] = max(1, int(round(j * area * sp["dt"] / (1.602e-19 * 1e3))))
        req = SV.Request(i, (lambda sp=sp: W.make_sweep_sim(sp, device, solver=SERVE_SOLVER)),
                         W.sweep_point_bytes(sp), SERVE_MAX_STEPS,
                         SV.Convergence(window=60, tol=0.05, keys=("current", "saddle")))
        arrivals.append((t, req))
    srv = SV.SweepServer(device, hbm_budget_bytes=150e9, max_active=64, chunk=10, batch=batch,
                         setup_workers=max(2, min(8, (os.cpu_count() or 2) // 2)))
    srv.serve(arrivals)
    st = srv.stats()
    st.update({"requests": SERVE_REQUESTS, "arrival_rate_hz": SERVE_RATE_HZ, "max_steps": SERVE_MAX_STEPS,
               "particle_pushes": srv.pushes, "gpu_ms": srv.gpu_ms})
    out["served"] = st
    srv.close()
    return out


# ----------------------------------------------------------------------------- CPU oracle
def _oracle_sim(name, n_ions, n_e, seed):
    from oracle.pic_oracle import OracleSimulator
    from thruster_cx_code_b200.domain import build_domain_geometry
    from thruster_cx_code_b200 import workloads as W
    o = OracleSimulator(build_domain_geometry)
    params = W.configure(o, name)
    o.build_domain(params)
    v_b, v_ti, v_te = W.thermal_speeds(o, params)
    ions, eles = W.preload(o.isBound, o.dx, o.dy, o.Lx, o.Ly, n_ions, n_e, v_b, 4 * v_ti, v_te, seed=seed,
                           x_max_ions=W.plume_boundary(o, params))
    o._add_ions(*ions, np.zeros(n_ions, bool), o.new_ion_ids(n_ions))
    o._add_electrons(*eles, o.new_e_ids(n_e))
    return o, params


def _oracle_steps(o, params, k, seed):
    from oracle.pic_oracle import PhiloxDraws
    draws = PhiloxDraws(seed)
    pushes = 0
    t0 = time.perf_counter()
    for _ in range(k):
        n_p, n_e = o.num_p, o.num_e
        o.step(params, draws)
        inj = o.injected_ions_step
        pushes += (n_p + inj) * o.n_sub_ion + (n_e + int(params.get("neut_rate", 30))) * o.n_sub_e
    return pushes, time.perf_counter() - t0


def cpu_baseline_port(name, frac=1 / 16, steps=2):
    from thruster_cx_code_b200 import workloads as W
    w = W.WORKLOADS[name]
    ni, ne = int(w["n_ions"] * frac), int(w["n_e"] * frac)
    o, params = _oracle_sim(name, ni, ne, seed=5)
    pushes, dt = _oracle_steps(o, params, steps, seed=5)
    return {"value": pushes / dt, "unit": "particle-pushes/s", "cores": 1, "kind": "port",
            "sample": f"{name} grid, {ni} ions + {ne} electrons ({frac:.4g} of the workload), {steps} steps "
                      f"(one with the 5-solve SuperLU Picard loop), NumPy/SciPy oracle of the reference step"}


def _worker(args):
    name, ni, ne, seed, warm, k, q = args
    os.environ["OMP_NUM_THREADS"] = "1"
    o, params = _oracle_sim(name, ni, ne, seed)
    if warm:
        _oracle_steps(o, params, warm, seed)
    q.put(_oracle_steps(o, params, k, seed))


def reference_arm(args):
    rank, _, world = dist_env()
    if rank != 0:
        return
    import multiprocessing as mp
    from thruster_cx_code_b200 import workloads as W
    w = W.WORKLOADS[args.workload]
    P = max(1, min(os.cpu_count() or 1, 32))
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ni, ne = w["n_ions"] // P, w["n_e"] // P
    warm = min(args.warmup, 1)
    procs = [ctx.Process(target=_worker, args=((args.workload, ni, ne, 11 + i, warm, args.steps, q),))
             for i in range(P)]
    for p in procs:
        p.start()
    res = [q.get() for _ in procs]
    for p in procs:
        p.join()
    pushes = sum(r[0] for r in res)
    wall = max(r[1] for r in res)
    value = pushes / wall
    line = {"impl": "reference", "metric": "particle-pushes/s", "value": value, "unit": "particle-pushes/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": wall / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 (NumPy, f64 potential)",
            "data": "synthetic (seeded pre-load)",
            "config": {"workload": args.workload, "processes": P},
            "cpu_baseline": {"value": value, "unit": "particle-pushes/s", "cores": P, "kind": "port",
                             "sample": f"{P} processes, each the {args.workload} grid with {ni} ions + {ne} electrons "
                                       f"(1/{P} of the workload), {args.steps} timed steps"},
            "e2e": {"value": value, "unit": "particle-pushes/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


if __name__ == "__main__":
    a = parse()
    if a.impl == "reference":
        reference_arm(a)
    else:
        gpu_arm(a)
