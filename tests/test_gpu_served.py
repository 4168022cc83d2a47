"""Continuous batching on the GPU: a request's result is the same alone and in the mix.

* Membership changes: request A joins a batch that is already stepping request B, C
  joins later, B retires before A finishes.  A's state after its steps is compared with
  A stepped alone.
* The served loop: three requests arrive at staggered times into a SweepServer and are
  admitted while the others are on the GPU; each retires at its step limit, and its final
  state (taken at retirement) is compared with the same request run alone.

A point in a mix shares the field-solve launch with the others and runs on fewer blocks,
but every reduction of its solve sums a fixed set of virtual-block partials in a fixed
order: its particles and potential are the solo run's, bit for bit.
"""
import numpy as np
import pytest

from thruster_cx_code_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def SV():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from thruster_cx_code_b200 import serving
    return serving


def _spec(grid, n, index, served=False):
    rng = np.random.default_rng(300 + index)
    if served:
        return W.served_point(rng, index, grids=(grid,), n_range=(n, n + 1))
    return W.sweep_point(rng, index, grids=(grid,), n_range=(n, n + 1))


def _snap(sim):
    n, ne = sim.num_p, sim.num_e
    ions = np.stack([np.asarray(getattr(sim, "p_" + k)[:n]) for k in ("x", "y", "vx", "vy", "vz")]).astype(np.float64)
    return {"ions": ions, "ids": np.asarray(sim.p_id[:n]).astype(np.int64), "num_p": n, "num_e": ne,
            "V": np.array(sim.V, copy=True)}


def _same_as(a, b):
    assert (a["num_p"], a["num_e"]) == (b["num_p"], b["num_e"])
    np.testing.assert_array_equal(a["V"], b["V"])
    np.testing.assert_array_equal(a["ids"], b["ids"])
    np.testing.assert_array_equal(a["ions"], b["ions"])


def test_join_and_retire_mid_run(SV):
    sa, sb, sc = _spec("64x256", 60000, 1), _spec("128x512", 120000, 2), _spec("64x256", 90000, 3)
    batch = SV.SweepBatch()
    alone, pal = W.make_sweep_sim(sa)
    batch.run([alone], [pal], 24)
    ref = _snap(alone)
    alone.close()
    (A, pA), (B, pB), (C, pC) = W.make_sweep_sim(sa), W.make_sweep_sim(sb), W.make_sweep_sim(sc)
    batch.run([B], [pB], 6)                   # B is running
    batch.run([B, A], [pB, pA], 8)            # A joins
    batch.run([B, A, C], [pB, pA, pC], 8)     # C joins
    B.close()                                 # B retires
    batch.run([A, C], [pA, pC], 8)            # A finishes its 24 steps beside C
    assert A.iteration == 24
    _same_as(_snap(A), ref)
    A.close()
    C.close()
    batch.close()


def test_served_requests_match_alone(SV):
    specs = [_spec("64x256", 80000, 10, served=True), _spec("128x512", 150000, 11, served=True),
             _spec("64x256", 50000, 12, served=True)]
    steps = [30, 20, 25]
    refs = []
    batch = SV.SweepBatch()
    for sp, k in zip(specs, steps):
        s, p = W.make_sweep_sim(sp, solver={"max_coarse": 256})
        batch.run([s], [p], k)
        refs.append(_snap(s))
        s.close()
    arrivals = []
    for i, (sp, k) in enumerate(zip(specs, steps)):
        req = SV.Request(i, (lambda sp=sp: W.make_sweep_sim(sp, solver={"max_coarse": 256})), W.sweep_point_bytes(sp),
                         k, SV.Convergence(window=500, tol=0.0), finish=_snap)
        arrivals.append((0.15 * i, req))
    srv = SV.SweepServer(hbm_budget_bytes=150e9, max_active=8, chunk=5, batch=batch, setup_workers=2)
    done = srv.serve(arrivals)
    assert sorted(r.rid for r in done) == [0, 1, 2]
    for r in done:
        assert r.steps == steps[r.rid] and not r.converged
        _same_as(r.result, refs[r.rid])
    srv.close()
