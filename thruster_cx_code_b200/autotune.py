"""Autotuner for the run-time knobs of one simulator.

The reference has no counterpart: it runs one fixed code path (NumPy + SuperLU).  Here a
few launch and solver settings change speed without changing what is computed, and their
best values depend on the grid size and the particle count:

* ``max_coarse``: the largest coarsest multigrid level (solved with a dense inverse).
  Fewer levels mean fewer grid-wide phases per PCG iteration; a larger coarsest level
  costs host set-up time and a larger dense product.
* ``tol_inner``: the FP32 reduction per refinement pass of the field solve.
* ``smoother_sweeps``: damped-Jacobi sweeps on the fine multigrid level on each side of the
  coarse correction (1 or 2): a second sweep costs two grid-wide phases per PCG iteration
  and may save iterations.
* ``sort_every``: steps between cell sorts of the particles (L1 locality of the field
  gathers against the cost of the sort).
* ``particle_blocks_per_sm``: the grid of the ion and electron step kernels.
* ``solve_blocks``: blocks of the field-solve launch ("all" SMs or "half").
* ``particles_per_block``: the tile of the ion and electron step kernels (1024 or 512
  particles staged, compacted and histogrammed per block).
* ``deposit_hist``, ``ion_tma_window``, ``electron_kernel``: the step kernels' variants
  (``PB_OPT_*`` bits): shared-memory cell histograms for the deposit and PPC counts, the
  TMA-staged E-corner window of the ion step, and the electron step fused, with two
  electrons per thread side by side, or split into a barrier-free push and a separate
  compaction.  Every combination computes the same bits.

Particle results are identical for every value of these knobs except ``sort_every``,
which changes only the array order, and the solver's ``max_coarse``, ``tol_inner`` and
``smoother_sweeps``: the field solve reaches the same FP64 tolerance whatever they are,
but its rounding follows them.  ``solve_blocks`` changes nothing but speed (the solve's
sums run over a fixed set of virtual blocks).

With ``horizon_steps`` set, the cost of a setting is its step time plus its multigrid
build time (host, measured) spread over that many steps: short-lived simulators, such as
served requests, favour a small coarsest level that builds in milliseconds.

``Autotuner.tune(sim, params)`` saves a checkpoint of ``sim``, then, by coordinate descent
(one knob at a time, the others at their best so far), restores a fresh copy from it for
every candidate, runs warm-up steps and times ``steps`` steps on the device
(``pb_sim_run``).  A candidate replaces the incumbent only if it is faster by more than
``min_gain``.  The best values are applied to ``sim`` and cached by grid shape and
particle count, so later simulators of the same kind take them without tuning
(``apply_cached``).
"""
import ctypes as C
import math
import os
import tempfile

from . import _lib

KNOBS = {
    "max_coarse": (256, 1536, 4096),
    "tol_inner": (1e-3, 1e-4),
    "sort_every": (10, 20, 40),
    "particle_blocks_per_sm": (4, 8, 16),
    "solve_blocks": ("all", "half"),
    "deposit_hist": (False, True),
    "ion_tma_window": (False, True),
    "electron_kernel": ("fused", "pairs", "split"),
    "particles_per_block": (1024, 512),
    "smoother_sweeps": (1, 2),
}


def current(sim):
    """The simulator's knob values."""
    s = sim.solver
    opts = C.c_uint32()
    _lib.check(_lib.load().pb_sim_get_kernel_options(sim._h, C.byref(opts)), "pb_sim_get_kernel_options")
    return {"max_coarse": int(s["max_coarse"]), "tol_inner": float(s["tol_inner"]), "smoother_sweeps": int(s["nu"]),
            "sort_every": int(sim.sort_every), "particle_blocks_per_sm": int(getattr(sim, "_pbps", 8)),
            "solve_blocks": getattr(sim, "_solve_blocks", "all"),
            "particles_per_block": int(getattr(sim, "_ppb", 1024)), **options_knobs(int(opts.value))}


def options_knobs(bits):
    """The kernel-variant knobs of PB_OPT_* bits."""
    ele = "split" if bits & _lib.PB_OPT_ELE_SPLIT else ("pairs" if bits & _lib.PB_OPT_ELE_PAIRS else "fused")
    return {"deposit_hist": bool(bits & _lib.PB_OPT_SMEM_HIST), "ion_tma_window": bool(bits & _lib.PB_OPT_TMA_TILE),
            "electron_kernel": ele}


def options_bits(knobs, base=0):
    """PB_OPT_* bits from the kernel-variant knobs present in ``knobs`` (others from ``base``)."""
    cur = options_knobs(base)
    cur.update({k: knobs[k] for k in cur if k in knobs})
    bits = (_lib.PB_OPT_SMEM_HIST if cur["deposit_hist"] else 0) | (_lib.PB_OPT_TMA_TILE if cur["ion_tma_window"] else 0)
    bits |= {"fused": 0, "pairs": _lib.PB_OPT_ELE_PAIRS, "split": _lib.PB_OPT_ELE_SPLIT}[cur["electron_kernel"]]
    return bits


def _num_sms(sim):
    import torch
    return torch.cuda.get_device_properties(sim.device).multi_processor_count


def apply(sim, knobs):
    """Set ``knobs`` (a subset of KNOBS' keys) on ``sim``.  A new ``max_coarse`` rebuilds
    the multigrid hierarchy."""
    lib = _lib.load()
    unknown = set(knobs) - set(KNOBS)
    if unknown:
        raise ValueError(f"unknown knobs: {sorted(unknown)}")
    s = dict(sim.solver)
    rebuild = "max_coarse" in knobs and int(knobs["max_coarse"]) != int(s["max_coarse"])
    s["max_coarse"] = int(knobs.get("max_coarse", s["max_coarse"]))
    s["tol_inner"] = float(knobs.get("tol_inner", s["tol_inner"]))
    s["nu"] = int(knobs.get("smoother_sweeps", s["nu"]))
    _lib.check(lib.pb_sim_set_solver(sim._h, s["tol"], s["tol_inner"], s["max_outer"], s["max_inner"], s["nu"],
                                     s["max_coarse"]), "pb_sim_set_solver")
    sim.solver = s
    if rebuild and sim.laplacian_lu:
        _lib.check(lib.pb_sim_rebuild_operator(sim._h), "rebuild_operator")
    if "sort_every" in knobs:
        sim.sort_every = int(knobs["sort_every"])
    if "particles_per_block" in knobs:
        _lib.check(lib.pb_sim_set_tile(sim._h, int(knobs["particles_per_block"])), "pb_sim_set_tile")
        sim._ppb = int(knobs["particles_per_block"])
    if any(k in knobs for k in ("deposit_hist", "ion_tma_window", "electron_kernel")):
        opts = C.c_uint32()
        _lib.check(lib.pb_sim_get_kernel_options(sim._h, C.byref(opts)), "pb_sim_get_kernel_options")
        _lib.check(lib.pb_sim_set_kernel_options(sim._h, options_bits(knobs, int(opts.value))),
                   "pb_sim_set_kernel_options")
    if "particle_blocks_per_sm" in knobs or "solve_blocks" in knobs:
        pbps = int(knobs.get("particle_blocks_per_sm", getattr(sim, "_pbps", 8)))
        sb = knobs.get("solve_blocks", getattr(sim, "_solve_blocks", "all"))
        n = _num_sms(sim)
        nblk = n if sb == "all" else max(1, n // 2) if sb == "half" else int(sb)
        _lib.check(lib.pb_sim_set_launch(sim._h, pbps, nblk), "pb_sim_set_launch")
        sim._pbps = pbps
        sim._solve_blocks = sb


def run_timed(sim, params, steps):
    """Device time (ms) of ``steps`` steps of ``sim`` through pb_sim_run."""
    lib = _lib.load()
    sim._flush()
    sim._upload_user_cs()
    it0 = sim.iteration
    plist = []
    for k in range(steps):
        sim.iteration = it0 + k
        plist.append(sim.step_params(params))
    sim.iteration = it0
    P = (_lib.StepParams * steps)(*plist)
    R = (_lib.StepReport * steps)()
    _lib.check(lib.pb_sim_run(sim._h, P, steps, R), "pb_sim_run")
    tm = (C.c_double * 9)()
    lib.pb_sim_timing(sim._h, tm)
    sim.iteration = it0 + steps
    sim._invalidate()
    for r in R:
        sim._apply_report(r, params)
    return float(tm[0])


def coordinate_descent(start, space, measure, passes=1, min_gain=0.01):
    """Minimise ``measure(knobs)`` over ``space`` (knob -> candidate values) one knob at a
    time from ``start``.  A candidate replaces the incumbent only when it is faster by
    more than ``min_gain`` (relative).  Each distinct setting is measured once.  Returns
    (best knobs, {setting tuple: time})."""
    keys = list(space)
    seen = {}

    def cost(k):
        t = tuple((n, k[n]) for n in keys)
        if t not in seen:
            seen[t] = float(measure(dict(k)))
        return seen[t]

    best = {n: start[n] for n in keys}
    best_t = cost(best)
    for _ in range(passes):
        changed = False
        for n in keys:
            for v in space[n]:
                if v == best[n]:
                    continue
                cand = dict(best, **{n: v})
                t = cost(cand)
                if t < best_t * (1.0 - min_gain):
                    best, best_t, changed = cand, t, True
        if not changed:
            break
    return best, seen


def workload_key(sim):
    """Cache key: grid shape and the particle count to the nearest power of two."""
    n = max(1, int(sim.num_p) + int(sim.num_e))
    return (int(sim.ny), int(sim.nx), int(round(math.log2(n))))


class Autotuner:
    def __init__(self, steps=6, warmup=2, passes=1, min_gain=0.01, space=None, device=0, horizon_steps=None):
        self.horizon = int(horizon_steps) if horizon_steps else None
        self.steps = int(steps)
        self.warmup = int(warmup)
        self.passes = int(passes)
        self.min_gain = float(min_gain)
        self.space = dict(space if space is not None else KNOBS)
        self.device = int(device)
        self.cache = {}
        self.last_table = {}

    def measure(self, ckpt, knobs, base_solver=None):
        """ms per step of a fresh copy restored from ``ckpt`` with ``knobs`` applied (the
        remaining solver settings taken from ``base_solver``), plus the multigrid build
        time spread over ``horizon_steps`` when that is set."""
        from .physics_engine import DigitalTwinSimulator
        trial, params = DigitalTwinSimulator.load_checkpoint(ckpt, device=self.device)
        try:
            if base_solver:
                s = dict(trial.solver)  # max_coarse stays the one the copy was built with
                s.update({k: base_solver[k] for k in ("tol", "max_outer", "max_inner")})
                trial.solver = s
            apply(trial, knobs)
            build_ms = 0.0
            if self.horizon:
                import time
                t0 = time.perf_counter()
                _lib.check(_lib.load().pb_sim_rebuild_operator(trial._h), "rebuild_operator")
                build_ms = (time.perf_counter() - t0) * 1e3
            if self.warmup:
                run_timed(trial, params, self.warmup)
            ms = run_timed(trial, params, self.steps) / self.steps
            return ms + (build_ms / self.horizon if self.horizon else 0.0)
        finally:
            trial.close()

    def tune(self, sim, params):
        """Tune ``sim``'s knobs on copies of its state; apply and cache the best.  Returns
        (best knobs, {setting: ms per step})."""
        fd, path = tempfile.mkstemp(suffix=".npz")
        os.close(fd)
        try:
            sim.save_checkpoint(path, params)
            start = current(sim)
            base = dict(sim.solver)
            best, table = coordinate_descent(start, self.space, lambda k: self.measure(path, k, base),
                                             passes=self.passes, min_gain=self.min_gain)
        finally:
            os.remove(path)
        apply(sim, best)
        self.cache[workload_key(sim)] = best
        self.last_table = {k: v for k, v in table.items()}
        return best, table

    def apply_cached(self, sim):
        """Apply the cached knobs of ``sim``'s workload kind, if any; returns them or None."""
        best = self.cache.get(workload_key(sim))
        if best is not None:
            apply(sim, best)
        return best
