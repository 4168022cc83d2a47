"""Steps replayed from CUDA graphs give the same bits as steps enqueued one kernel at a time.

pb_sim_set_graphs(on) makes pb_sim_run and pb_sim_step capture each step shape once (odd
and even steps differ by the field solve, sort steps by the sort, and the particle buffers
alternate) and replay it, with the Philox step key read from device memory.  Two
simulators from the same state run 45 steps, one with graphs and one without: every
particle, the fields and every step report must agree bit for bit, the graphs must have
been replayed, and no capture may have failed.
"""
import ctypes as C

import numpy as np
import pytest

from thruster_cx_code_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mods():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from thruster_cx_code_b200 import _lib
    return _lib


def _spec():
    return W.sweep_point(np.random.default_rng(21), 0, grids=("64x256",), n_range=(120000, 120001))


def _state(sim):
    n, ne = sim.num_p, sim.num_e
    out = {k: np.asarray(getattr(sim, k)[:n]).copy() for k in ("p_x", "p_y", "p_vx", "p_vy", "p_vz", "p_id")}
    out.update({k: np.asarray(getattr(sim, k)[:ne]).copy() for k in ("e_x", "e_y", "e_vx", "e_vy", "e_vz", "e_id")})
    out.update({"V": sim.V.copy(), "rho": sim.rho.copy(), "Tmap": sim.Tmap.copy()})
    return out


def _run(sim, params, K):
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
    _lib.check(lib.pb_sim_run(sim._h, P, K, R), "pb_sim_run")
    sim.iteration = it0 + K
    sim._invalidate()
    for r in R:
        sim._apply_report(r, params)
    return [bytes(r) for r in R]


def test_graph_steps_bit_identical(mods):
    _lib = mods
    sp = _spec()
    a, pa = W.make_sweep_sim(sp)
    b, pb = W.make_sweep_sim(sp)
    _lib.check(b._libh.pb_sim_set_graphs(b._h, 1), "set_graphs")
    ra = _run(a, pa, 45)
    rb = _run(b, pb, 45)
    stats = (C.c_int64 * 4)()
    b._libh.pb_sim_graph_stats(b._h, stats)
    assert stats[3] == 0, b._libh.pb_last_error()
    assert stats[0] >= 2 and stats[1] >= 30, list(stats)
    assert ra == rb
    sa, sb = _state(a), _state(b)
    for k in sa:
        np.testing.assert_array_equal(sa[k], sb[k], err_msg=k)
    # the public step() in graph mode continues identically
    for _ in range(3):
        assert a.step(pa)[1] == b.step(pb)[1]
    sa, sb = _state(a), _state(b)
    for k in sa:
        np.testing.assert_array_equal(sa[k], sb[k], err_msg=k)
    a.close()
    b.close()
