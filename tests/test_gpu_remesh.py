"""Sputter breaks inside a multi-step run.

The reference rebuilds its field matrix in the step that breaks cells
(Python/physics_engine.py:1443-1449), so the next field solve already sees the freed
nodes.  DigitalTwinSimulator.step rebuilds the multigrid hierarchy on the host after every
step that broke cells.  Inside one pb_sim_run (or pb_batch_run) the node classes change on
the device, and so do the fine-level smoother weights: every free node gets
omega / (4 - Neumann neighbours), the value the host build gives it.  Without that the
preconditioner ignores a freed node and the solve cannot converge there.

Breaks are planted: damage above the threshold on the upstream face of the first grid
(breaks in step 0) and, under a threshold lowered from step 2 on, on the downstream face of
the second grid (breaks in step 2); field solves run in steps 1, 3, 5 and 7.

* The device weights after a run with breaks equal the formula on the run's node classes
  and the host rebuild's weights, bit for bit.
* The run agrees with the same steps taken one at a time, with host rebuilds in between.
  Both solve the same operator to the same tolerance with different coarse levels, so the
  bar is the one for independent field solves: phi within 1e-6 of max|phi|, counts within
  0.2%, broken cells within 2%.
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


def test_breaks_inside_one_run(lib):
    sp = _spec()
    a, pa = W.make_sweep_sim(sp)
    b, pb = W.make_sweep_sim(sp)
    h = lib.load()
    face_a, face_b = _plant(a)
    _plant(b)
    assert face_a.sum() > 0 and face_b.sum() > 0

    # a: one step at a time, hierarchy rebuilt on the host after each break
    broken_a = []
    for k in range(K):
        a.step(_params(pa, k))
        broken_a.append(a.last_report.broken)

    # b: all K steps in one pb_sim_run
    b._flush()
    b._upload_user_cs()
    it0 = b.iteration
    plist = []
    for k in range(K):
        b.iteration = it0 + k
        plist.append(b.step_params(_params(pb, k)))
    b.iteration = it0
    P = (lib.StepParams * K)(*plist)
    R = (lib.StepReport * K)()
    lib.check(h.pb_sim_run(b._h, P, K, R), "pb_sim_run")  # raises on PB_ERR_NOCONV
    broken = [r.broken for r in R]
    solves = [p.do_poisson for p in plist]
    # a field solve follows a break inside the run
    assert any(broken[k] > 0 and any(solves[k + 1:]) for k in range(K - 1)), (broken, solves)

    cls = _field(lib, b, 12, np.uint8)
    w_dev = _field(lib, b, 13, np.float32)
    np.testing.assert_array_equal(w_dev, _weights_of(cls, bool(b.periodic_y)))
    lib.check(h.pb_sim_rebuild_operator(b._h), "rebuild_operator")
    np.testing.assert_array_equal(_field(lib, b, 13, np.float32), w_dev)

    b.iteration = it0 + K
    b._invalidate()
    for k, r in enumerate(R):
        b._apply_report(r, _params(pb, k))
    assert broken[0] >= face_a.sum() and broken[2] >= face_b.sum(), broken
    assert abs(sum(broken) - sum(broken_a)) <= max(2, 0.02 * sum(broken_a)), (broken_a, broken)
    for n_a, n_b in ((a.num_p, b.num_p), (a.num_e, b.num_e)):
        assert abs(n_a - n_b) <= 0.002 * n_a + 2, (n_a, n_b)
    va, vb = np.asarray(a.V), np.asarray(b.V)
    assert np.abs(va - vb).max() <= 1e-6 * np.abs(va).max()
    a.close()
    b.close()
