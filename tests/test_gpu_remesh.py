"""Sputter breaks inside a multi-step run.

The reference rebuilds its field matrix in the step that breaks cells
(Python/physics_engine.py:1443-1449), so the next field solve already sees the freed
nodes.  DigitalTwinSimulator.step rebuilds the multigrid hierarchy on the host after every
step that broke cells.  Inside one pb_sim_run (or pb_batch_run, or a step graph) the node
classes and the fine-level smoother weights change on the device in the step that breaks,
and k_mg_rebuild forms the coarse levels, the transfer stencils and the dense coarsest
inverse again before the next field solve, in the host build's order of operations.

Breaks are planted: damage above the threshold on the upstream face of the first grid
(breaks in step 0) and, under a threshold lowered from step 2 on, on the downstream face of
the second grid (breaks in step 2); field solves run in steps 1, 3, 5 and 7.

* The device weights after a run with breaks equal the formula on the run's node classes
  and the host rebuild's weights, bit for bit.
* The device's hierarchy equals a host build from the same classes bit for bit (digest of
  every array the solve reads), so the run gives the same bits as the same steps taken one
  at a time with host rebuilds in between; so do the run with step graphs and the run as a
  batch of one.
* A break that makes the host build choose other levels is rebuilt on the device with the
  old level count and then by the host after the run.
"""
import ctypes as C

import numpy as np
import pytest

from thruster_cx_code_b200 import workloads as W

pytestmark = pytest.mark.gpu
K = 8
OMEGA = 0.8


@pytest.fixture(scope="module")
def lib():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from thruster_cx_code_b200 import _lib
    return _lib


THRESH_EARLY, THRESH_LATE = 1e9, 1e8


def _spec():
    return W.sweep_point(np.random.default_rng(7), 0, grids=("64x256",), n_range=(150000, 150001))


def _plant(sim):
    """Damage 2e9 on the bound cells with a free left neighbour before the second grid
    starts, 5e8 on those with a free right neighbour after it; returns the two masks."""
    ib = np.asarray(sim.isBound).astype(bool)
    free_left = np.zeros_like(ib)
    free_left[:, 1:] = ~ib[:, :-1]
    free_right = np.zeros_like(ib)
    free_right[:, :-1] = ~ib[:, 1:]
    col = np.arange(sim.nx)[None, :] * sim.dx
    x1 = sim.grid_x_starts[1]
    a = ib & free_left & (col < x1)
    b = ib & free_right & (col >= x1)
    dmg = np.zeros(ib.shape, np.float64)
    dmg[a] = 2e9
    dmg[b] = 5e8
    sim.damage_map = dmg
    return a, b


def _params(p, k):
    return dict(p, Thresh=THRESH_EARLY if k < 2 else THRESH_LATE)


def _field(lib, sim, fid, dtype):
    a = np.empty((sim.ny, sim.nx), dtype)
    lib.check(lib.load().pb_sim_get_field(sim._h, fid, a.ctypes.data_as(C.c_void_p), a.nbytes), "get_field")
    return a


def _weights_of(cls, periodic):
    """Fine-level smoother weights from node classes (0 free, 1 Dirichlet, 2 Neumann)."""
    neu = cls == 2
    ones = np.ones_like(neu)
    left, right = ones.copy(), ones.copy()
    left[:, 1:] = neu[:, :-1]
    right[:, :-1] = neu[:, 1:]
    if periodic:
        down, up = np.roll(neu, 1, axis=0), np.roll(neu, -1, axis=0)
    else:
        down, up = ones.copy(), ones.copy()
        down[1:] = neu[:-1]
        up[:-1] = neu[1:]
    nneu = left.astype(np.int32) + right + down + up
    free = (cls == 0) & (nneu < 4)
    w = np.zeros(cls.shape, np.float32)
    w[free] = (OMEGA / (4.0 - nneu[free])).astype(np.float32)
    return w


def _digest(lib, sim):
    d = C.c_uint64()
    lib.check(lib.load().pb_sim_operator_digest(sim._h, C.byref(d)), "pb_sim_operator_digest")
    return d.value


def _mg_stats(lib, sim):
    out = (C.c_int64 * 8)()
    lib.check(lib.load().pb_sim_mg_stats(sim._h, out), "pb_sim_mg_stats")
    return list(out)[:4]


def _run(lib, sim, p, steps=K, graphs=False):
    """The K planted steps of ``sim`` in one pb_sim_run; returns the reports."""
    h = lib.load()
    if graphs:
        lib.check(h.pb_sim_set_graphs(sim._h, 1), "pb_sim_set_graphs")
    sim._flush()
    sim._upload_user_cs()
    it0 = sim.iteration
    plist = []
    for k in range(steps):
        sim.iteration = it0 + k
        plist.append(sim.step_params(_params(p, k)))
    sim.iteration = it0
    P = (lib.StepParams * steps)(*plist)
    R = (lib.StepReport * steps)()
    lib.check(h.pb_sim_run(sim._h, P, steps, R), "pb_sim_run")  # raises on PB_ERR_NOCONV
    sim.iteration = it0 + steps
    sim._invalidate()
    for k, r in enumerate(R):
        sim._apply_report(r, _params(p, k))
    return list(R), [q.do_poisson for q in plist]


def _same_state(a, b):
    assert (a.num_p, a.num_e) == (b.num_p, b.num_e)
    np.testing.assert_array_equal(np.asarray(a.V), np.asarray(b.V))
    np.testing.assert_array_equal(np.asarray(a.isBound), np.asarray(b.isBound))
    for pre, n in (("p_", a.num_p), ("e_", a.num_e)):
        for k in ("x", "y", "vx", "vy", "vz", "id"):
            np.testing.assert_array_equal(np.asarray(getattr(a, pre + k)[:n]), np.asarray(getattr(b, pre + k)[:n]))


def test_breaks_inside_one_run(lib):
    from thruster_cx_code_b200 import serving as SV
    sp = _spec()
    a, pa = W.make_sweep_sim(sp)
    b, pb = W.make_sweep_sim(sp)
    c, pc = W.make_sweep_sim(sp)
    d, pd = W.make_sweep_sim(sp)
    h = lib.load()
    face_a, face_b = _plant(a)
    for m in (b, c, d):
        _plant(m)
    assert face_a.sum() > 0 and face_b.sum() > 0

    # a: one step at a time, hierarchy rebuilt on the host after each break
    broken_a = []
    for k in range(K):
        a.step(_params(pa, k))
        broken_a.append(a.last_report.broken)

    # b: all K steps in one pb_sim_run, the hierarchy rebuilt on the device
    R, solves = _run(lib, b, pb)
    broken = [r.broken for r in R]
    # a field solve follows a break inside the run
    assert any(broken[k] > 0 and any(solves[k + 1:]) for k in range(K - 1)), (broken, solves)
    assert broken[0] >= face_a.sum() and broken[2] >= face_b.sum(), broken
    rebuilds, deferred, host_runs, nc = _mg_stats(lib, b)
    assert rebuilds >= 2 and deferred == 0 and host_runs == 0, (rebuilds, deferred, host_runs)

    cls = _field(lib, b, 12, np.uint8)
    w_dev = _field(lib, b, 13, np.float32)
    np.testing.assert_array_equal(w_dev, _weights_of(cls, bool(b.periodic_y)))
    dig_dev = _digest(lib, b)
    lib.check(h.pb_sim_rebuild_operator(b._h), "rebuild_operator")
    np.testing.assert_array_equal(_field(lib, b, 13, np.float32), w_dev)
    assert _digest(lib, b) == dig_dev
    assert _mg_stats(lib, b)[3] == nc

    # the same bits as the step-at-a-time run with host rebuilds
    assert broken == broken_a, (broken_a, broken)
    _same_state(a, b)

    # c: the run with step graphs; d: the run as a batch of one
    _run(lib, c, pc, graphs=True)
    g = (C.c_int64 * 4)()
    lib.check(h.pb_sim_graph_stats(c._h, g), "pb_sim_graph_stats")
    assert g[0] >= 2 and g[1] >= 1 and g[3] == 0, list(g)
    _same_state(b, c)
    d._flush()
    d._upload_user_cs()
    batch = SV.SweepBatch(0)
    res = batch.run([d], [_params(pd, 0)], 2)
    batch.run([d], [_params(pd, 2)], K - 2)
    batch.close()
    assert res[0][0][1].broken == broken[0]
    _same_state(b, d)
    assert _digest(lib, d) == dig_dev
    for m in (a, b, c, d):
        m.close()


def test_rebuild_with_new_levels_left_to_host(lib):
    """A coarsest level pushed above max_coarse by the freed nodes: the host build would
    coarsen once more.  The device rebuilds with the old level count (the solves of the run
    converge), flags it, and the host rebuilds after the run."""
    sp = _spec()
    s, p = W.make_sweep_sim(sp)
    h = lib.load()
    nc0 = _mg_stats(lib, s)[3]
    sv = s.solver
    lib.check(h.pb_sim_set_solver(s._h, sv["tol"], sv["tol_inner"], sv["max_outer"], sv["max_inner"], sv["nu"],
                                  int(nc0)), "pb_sim_set_solver")
    lib.check(h.pb_sim_rebuild_operator(s._h), "rebuild_operator")
    assert _mg_stats(lib, s)[3] == nc0
    # every bound cell of the first grid breaks in step 0
    ib = np.asarray(s.isBound).astype(bool)
    col = np.arange(s.nx)[None, :] * s.dx
    first = ib & (col < s.grid_x_starts[1])
    dmg = np.zeros(ib.shape, np.float64)
    dmg[first] = 2e9
    s.damage_map = dmg
    R, solves = _run(lib, s, p, steps=4)
    assert R[0].broken == first.sum() and any(solves[1:])
    rebuilds, deferred, host_runs, nc = _mg_stats(lib, s)
    assert rebuilds >= 1 and deferred >= 1 and host_runs >= 1, (rebuilds, deferred, host_runs)
    assert nc <= nc0  # the host build coarsened once more
    dig = _digest(lib, s)
    lib.check(h.pb_sim_rebuild_operator(s._h), "rebuild_operator")
    assert _digest(lib, s) == dig
    s.close()
