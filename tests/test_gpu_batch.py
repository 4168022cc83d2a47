"""Batched stepping on the GPU (pb_batch_run through SweepBatch).

* A batch of one is the single-instance step: particles, fields and reports bit-identical
  to K calls of DigitalTwinSimulator.step.
* A sweep point stepped in a mix with two others of different grid sizes is the same point
  stepped alone, bit for bit.  The field solves of the mix share the SMs, so each instance
  runs on fewer blocks, but every reduction of the solve sums a fixed set of virtual-block
  partials in a fixed order, whatever the block count.
* The same holds for the block shares the batch picks from measured solve times.
"""
import numpy as np
import pytest

from thruster_cx_code_b200 import workloads as W

pytestmark = pytest.mark.gpu
K = 6


@pytest.fixture(scope="module")
def mods():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from thruster_cx_code_b200 import serving
    return serving


def _spec(grid, n, index):
    rng = np.random.default_rng(100 + index)
    sp = W.sweep_point(rng, index, grids=(grid,), n_range=(n, n + 1))
    return sp


def _state(sim):
    n, ne = sim.num_p, sim.num_e
    ions = np.stack([np.asarray(getattr(sim, "p_" + k)[:n]) for k in ("x", "y", "vx", "vy", "vz")]).astype(np.float32)
    eles = np.stack([np.asarray(getattr(sim, "e_" + k)[:ne]) for k in ("x", "y", "vx", "vy", "vz")]).astype(np.float32)
    return ions, np.asarray(sim.p_id[:n]).astype(np.int64), eles, np.asarray(sim.e_id[:ne]).astype(np.int64)


def _by_id(a, ids):
    o = np.argsort(ids, kind="stable")
    return a[:, o], ids[o]


def test_batch_of_one_is_step(mods):
    sp = _spec("64x256", 150000, 1)
    a, pa = W.make_sweep_sim(sp)
    b, pb = W.make_sweep_sim(sp)
    for _ in range(K):
        a.step(pa)
    batch = mods.SweepBatch()
    out = batch.run([b], [pb], K)
    batch.close()
    assert len(out) == 1 and len(out[0]) == K
    assert a.num_p == b.num_p and a.num_e == b.num_e
    sa, sb = _state(a), _state(b)
    for x, y in zip(sa, sb):
        np.testing.assert_array_equal(np.asarray(x).view(np.uint32) if x.dtype == np.float32 else x,
                                      np.asarray(y).view(np.uint32) if y.dtype == np.float32 else y)
    np.testing.assert_array_equal(a.V, b.V)
    np.testing.assert_array_equal(a.rho, b.rho)
    a.close()
    b.close()


def _same(a, b):
    assert a.num_p == b.num_p and a.num_e == b.num_e
    for x, y in zip(_state(a), _state(b)):
        np.testing.assert_array_equal(np.asarray(x).view(np.uint32) if x.dtype == np.float32 else x,
                                      np.asarray(y).view(np.uint32) if y.dtype == np.float32 else y)
    np.testing.assert_array_equal(a.V, b.V)


def test_point_in_a_mix_matches_alone(mods):
    specs = [_spec("64x256", 200000, 2), _spec("128x512", 400000, 3), _spec("256x1024", 300000, 4)]
    alone, pal = W.make_sweep_sim(specs[0])
    batch = mods.SweepBatch()
    batch.run([alone], [pal], K)
    mix = [W.make_sweep_sim(sp) for sp in specs]
    # two runs: the second takes its block shares from the first run's measured solve times
    batch.run([m[0] for m in mix], [m[1] for m in mix], K // 2)
    batch.run([m[0] for m in mix], [m[1] for m in mix], K - K // 2)
    batch.close()
    _same(mix[0][0], alone)
    for m in mix:
        m[0].close()
    alone.close()


def test_batch_graphs_bit_identical(mods):
    """pb_batch_set_graphs: every batch step shape of a three-member mix captured once and
    replayed gives the same bits as enqueueing each kernel, over 25 steps (a sort step and
    alternating field-solve steps included)."""
    specs = [_spec("64x256", 120000, 5), _spec("128x512", 200000, 6), _spec("64x256", 80000, 7)]
    plain = [W.make_sweep_sim(sp) for sp in specs]
    graph = [W.make_sweep_sim(sp) for sp in specs]
    b0, b1 = mods.SweepBatch(), mods.SweepBatch(graphs=True)
    r0 = b0.run([m[0] for m in plain], [m[1] for m in plain], 25)
    r1 = b1.run([m[0] for m in graph], [m[1] for m in graph], 25)
    captures, replays, broken = b1.graph_stats()
    assert not broken and captures >= 2 and replays >= 15, (captures, replays, broken)
    for ra, rb in zip(r0, r1):
        assert [bytes(rep) for _, rep in ra] == [bytes(rep) for _, rep in rb]
    for (a, _), (g, _) in zip(plain, graph):
        for x, y in zip(_state(a), _state(g)):
            np.testing.assert_array_equal(np.asarray(x).view(np.uint32) if x.dtype == np.float32 else x,
                                          np.asarray(y).view(np.uint32) if y.dtype == np.float32 else y)
        np.testing.assert_array_equal(a.V, g.V)
    # a second run of the same set replays the graphs it has
    b1.run([m[0] for m in graph], [m[1] for m in graph], 4)
    assert b1.graph_stats()[1] > replays
    for m in plain + graph:
        m[0].close()
    b0.close()
    b1.close()
