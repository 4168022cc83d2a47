"""Batched and served execution of many aperture simulations on one GPU.

The reference runs a sweep (perveance, backstreaming limit) as one process per sweep point.
Each process builds a DigitalTwinSimulator, steps it until the beamlet divergence or the
saddle potential settles, and reports (Python/benchmarks/benchmark_perveance.py:17-67,
78-164; Python/benchmarks/benchmark_ebs.py:8-49).  Here the sweep points share one GPU:

* ``SweepBatch.run(sims, K)`` advances a set of simulators K steps together through
  ``pb_batch_run``.  Each instance's particle kernels run on its own stream, and the field
  solves due in a step run as one launch.
* ``Convergence`` is the retirement test: the relative change of the window means of the
  beamlet current, theta95 and the saddle potential, between the two halves of the last
  ``window`` steps.
* ``SweepServer`` does continuous batching.  Requests arrive over time and are admitted as
  soon as the device-memory budget and the instance cap allow.  An admitted request is built
  (geometry, multigrid, pre-load, upload) on a worker thread while the GPU keeps stepping
  the active ones.  The active instances advance together in chunks of steps, and an
  instance retires once it converges or reaches its step limit.  Its time-to-converged
  (retirement minus arrival, wall clock) is recorded.
"""
import ctypes as C
import math
import time
from concurrent.futures import ThreadPoolExecutor, wait, FIRST_COMPLETED

import numpy as np

from . import _lib


class SweepBatch:
    """Several DigitalTwinSimulator instances stepped together on one device."""

    def __init__(self, device=0, graphs=False):
        self._libh = _lib.load()
        h = C.c_void_p()
        _lib.check(self._libh.pb_batch_create(C.byref(h), int(device)), "pb_batch_create")
        self._h = h
        self.set_graphs(graphs)
        self.device = int(device)
        self.last_ms = 0.0
        self.last_launches = 0
        self.last_host_ms = 0.0

    def set_threads(self, threads):
        """Host threads enqueuing the members' kernels (0: the library's choice)."""
        _lib.check(self._libh.pb_batch_set_threads(self._h, int(threads)), "pb_batch_set_threads")

    def set_graphs(self, on):
        """Capture each batch step shape as a CUDA graph and replay it (pb_batch_set_graphs)."""
        _lib.check(self._libh.pb_batch_set_graphs(self._h, 1 if on else 0), "pb_batch_set_graphs")
        self.graphs = bool(on)

    def graph_stats(self):
        """(captures, replays, capture failed)."""
        out = (C.c_int64 * 3)()
        _lib.check(self._libh.pb_batch_graph_stats(self._h, out), "pb_batch_graph_stats")
        return int(out[0]), int(out[1]), bool(out[2])

    def close(self):
        if self._h is not None and self._h.value:
            self._libh.pb_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, sims, params_list, K):
        """Advance ``sims[i]`` by ``K`` steps with the step parameters of ``params_list[i]``
        (a config dict, as for ``step``).  Returns, per instance, the list of the K pairs
        (``step`` result ``(remeshed, min_pot, current_div, T_grids, trans_last_frame)``,
        step report)."""
        n = len(sims)
        if n == 0:
            return []
        P = (_lib.StepParams * (n * K))()
        for i, (s, prm) in enumerate(zip(sims, params_list)):
            s._flush()
            s._upload_user_cs()
            it0 = s.iteration
            for k in range(K):
                s.iteration = it0 + k
                P[i * K + k] = s.step_params(prm)
            s.iteration = it0
        R = (_lib.StepReport * (n * K))()
        arr = (C.c_void_p * n)(*[s._h.value for s in sims])
        _lib.check(self._libh.pb_batch_run(self._h, arr, n, P, int(K), R), "pb_batch_run")
        t = (C.c_double * 4)()
        self._libh.pb_batch_timing(self._h, t)
        self.last_ms, self.last_launches, self.last_host_ms = float(t[0]), int(t[1]), float(t[2])
        self.last_solve_ms = float(t[3])
        out = []
        for i, (s, prm) in enumerate(zip(sims, params_list)):
            res = []
            s._invalidate()
            for k in range(K):
                s.iteration += 1
                rep = _lib.StepReport()
                C.memmove(C.byref(rep), C.byref(R[i * K + k]), C.sizeof(rep))
                res.append((s._apply_report(rep, prm), rep))
            out.append(res)
        return out


def pushes_of(reports, n_p0, n_e0):
    """Particle pushes of consecutive steps of one instance, from its reports and the
    particle counts before the first step."""
    tot = 0
    np_prev, ne_prev = n_p0, n_e0
    for r in reports:
        tot += (np_prev + r.injected) * r.n_sub_ion + (ne_prev + r.rf_injected + r.neut_injected) * r.n_sub_e
        np_prev, ne_prev = r.num_p, r.num_e
    return tot


def beamlet_current(sim, rep):
    """Ions crossing the exit plane in one step as a current (A): crossed * q * w / dt."""
    return float(rep.crossed) * sim.q_ion * sim.macro_weight / sim.dt


class Convergence:
    """Relative change of window means between the halves of the last ``window`` steps,
    for each tracked quantity; converged when every change is below ``tol`` and at least
    ``min_steps`` steps have run.  Quantities that are NaN in a window (theta95 with five
    or fewer crossings) count as not converged.

    ``counts`` maps a key whose values are a count of macro-particles times a known factor
    (the beamlet current: crossings x q w / dt) to that factor.  Such a key also counts as
    settled when its change is within twice the Poisson noise of the difference of the two
    window means (sqrt(Na + Nb) / max(Na, Nb) for Na and Nb crossings in the halves): a
    current carried by a few macro-particles per step cannot settle below its own noise."""

    def __init__(self, window=500, tol=5e-3, min_steps=None, keys=("current", "theta95", "saddle"), counts=None):
        self.window = int(window)
        self.tol = float(tol)
        self.min_steps = int(min_steps if min_steps is not None else window)
        self.keys = tuple(keys)
        self.counts = dict(counts or {})
        self.hist = {k: [] for k in self.keys}
        self.steps = 0

    def add(self, **vals):
        for k in self.keys:
            self.hist[k].append(float(vals[k]))
        self.steps += 1

    def changes(self):
        h = self.window // 2
        out = {}
        for k in self.keys:
            v = self.hist[k]
            if len(v) < 2 * h or h == 0:
                out[k] = math.inf
                continue
            a = np.asarray(v[-2 * h:-h], np.float64)
            b = np.asarray(v[-h:], np.float64)
            if not (np.all(np.isfinite(a)) and np.all(np.isfinite(b))):
                out[k] = math.inf
                continue
            ma, mb = a.mean(), b.mean()
            scale = max(abs(ma), abs(mb))
            out[k] = abs(mb - ma) / scale if scale > 0 else 0.0
        return out

    def noise(self, key):
        """Twice the relative Poisson noise of the difference of the window-half means of a
        count key (inf without counts in the window); 0 for other keys."""
        f = self.counts.get(key)
        if not f:
            return 0.0
        h = self.window // 2
        v = self.hist[key]
        if len(v) < 2 * h or h == 0:
            return math.inf
        na = float(np.sum(v[-2 * h:-h])) / f
        nb = float(np.sum(v[-h:])) / f
        top = max(na, nb)
        return 2.0 * math.sqrt(na + nb) / top if top > 0 else math.inf

    def converged(self):
        if self.steps < self.min_steps:
            return False
        return all(c < max(self.tol, self.noise(k)) for k, c in self.changes().items())


class Request:
    """One sweep point: ``make()`` builds and returns (sim, params) on the device.
    ``finish(sim)``, if given, runs at retirement before the simulator is released; its
    return value is kept as ``result`` (e.g. the final state or diagnostics to report)."""

    def __init__(self, rid, make, est_bytes, max_steps, convergence, finish=None):
        self.rid = rid
        self.make = make
        self.est_bytes = int(est_bytes)
        self.max_steps = int(max_steps)
        self.conv = convergence
        self.finish = finish
        self.result = None
        self.sim = None
        self.params = None
        self.t_arrival = None
        self.t_admit = None
        self.t_done = None
        self.steps = 0
        self.converged = False
        self.last = {}


class SweepServer:
    """Continuous batching of sweep points on one GPU under a device-memory budget."""

    def __init__(self, device=0, hbm_budget_bytes=150e9, max_active=64, chunk=10, batch=None, setup_workers=2):
        self.batch = batch if batch is not None else SweepBatch(device)
        self.budget = float(hbm_budget_bytes)
        self.max_active = int(max_active)
        self.chunk = int(chunk)
        self.setup_workers = int(setup_workers)
        self.active = []
        self.preparing = {}  # future -> request
        self.done = []
        self.pushes = 0
        self.gpu_ms = 0.0

    def _in_use(self):
        return sum(r.mem for r in self.active) + sum(r.est_bytes for r in self.preparing.values())

    def _ready(self, fut, now):
        req = self.preparing.pop(fut)
        req.sim, req.params = fut.result()
        req.t_admit = now
        req.mem = max(int(req.sim.device_bytes()), req.est_bytes)
        self.active.append(req)

    def _retire(self, req, now):
        req.t_done = now
        if req.finish is not None:
            req.result = req.finish(req.sim)
        req.sim.close()
        req.sim = None
        self.active.remove(req)
        self.done.append(req)

    def serve(self, arrivals, clock=time.perf_counter):
        """``arrivals``: list of (arrival time in s from the start, Request), any order.
        Runs until every request has retired; returns the retired requests in order."""
        pending = sorted(arrivals, key=lambda a: a[0])
        t0 = clock()
        qi = 0
        waiting = []
        with ThreadPoolExecutor(max_workers=max(1, self.setup_workers)) as pool:
            while qi < len(pending) or waiting or self.preparing or self.active:
                now = clock() - t0
                while qi < len(pending) and pending[qi][0] <= now:
                    pending[qi][1].t_arrival = pending[qi][0]
                    waiting.append(pending[qi][1])
                    qi += 1
                # admission: first come, first served, while memory and slots allow
                while waiting and len(self.active) + len(self.preparing) < self.max_active and \
                        self._in_use() + waiting[0].est_bytes <= self.budget:
                    req = waiting.pop(0)
                    self.preparing[pool.submit(req.make)] = req
                if waiting and not self.active and not self.preparing:
                    raise RuntimeError(f"request {waiting[0].rid} needs {waiting[0].est_bytes} bytes, "
                                       f"more than the {self.budget:.0f}-byte budget")
                for fut in [f for f in self.preparing if f.done()]:
                    self._ready(fut, clock() - t0)
                if not self.active:
                    if self.preparing:
                        wait(list(self.preparing), timeout=0.05, return_when=FIRST_COMPLETED)
                    elif qi < len(pending):
                        time.sleep(max(0.0, min(pending[qi][0] - (clock() - t0), 0.05)))
                    continue
                k = max(1, min(self.chunk, min(r.max_steps - r.steps for r in self.active)))
                sims = [r.sim for r in self.active]
                n0 = [(s.num_p, s.num_e) for s in sims]
                results = self.batch.run(sims, [r.params for r in self.active], k)
                self.gpu_ms += self.batch.last_ms
                for r, res, (np0, ne0) in zip(list(self.active), results, n0):
                    s = r.sim
                    self.pushes += pushes_of([rep for _, rep in res], np0, ne0)
                    for (_, min_pot, div, _, _), rep in res:
                        r.conv.add(current=beamlet_current(s, rep), theta95=div, saddle=min_pot)
                    r.steps += k
                    (_, min_pot, div, _, _), rep = res[-1]
                    r.last = {"current": beamlet_current(s, rep), "theta95": float(div), "saddle": float(min_pot)}
                    if r.conv.converged() or r.steps >= r.max_steps:
                        r.converged = r.conv.converged()
                        self._retire(r, clock() - t0)
        return self.done

    def stats(self):
        lat = np.array([r.t_done - r.t_arrival for r in self.done], np.float64)
        if lat.size == 0:
            return {}
        span = max(r.t_done for r in self.done) - min(r.t_arrival for r in self.done)
        return {"completed": int(lat.size), "p50_s": float(np.percentile(lat, 50)),
                "p99_s": float(np.percentile(lat, 99)), "throughput_per_hr": lat.size / span * 3600.0,
                "converged": int(sum(r.converged for r in self.done))}

    def close(self):
        for r in list(self.active):
            r.sim.close()
        self.active = []
        self.batch.close()
