"""The autotuner's knobs and a small tuning run on the GPU (thruster_cx_code_b200/autotune.py).

* The particle-kernel grid (blocks per SM) does not change results: particle state after
  three steps is bit-identical per id.
* Half the SMs for the field solve does not change results either: the solve's sums run over
  fixed virtual blocks whatever the block count, so phi and the particles are the same bits.
* Out-of-range launch shapes and smoother counts other than 1 or 2 are rejected.
* A tuning run over two knobs applies and caches the best setting, and the tuned simulator
  keeps stepping.
* With a short horizon the multigrid build time counts, and a small coarsest level wins.
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
    from thruster_cx_code_b200 import _lib, autotune
    return _lib, autotune


def _spec():
    return W.sweep_point(np.random.default_rng(11), 0, grids=("64x256",), n_range=(150000, 150001))


def _ions_by_id(sim):
    n = sim.num_p
    ids = np.asarray(sim.p_id[:n]).astype(np.int64)
    o = np.argsort(ids, kind="stable")
    st = np.stack([np.asarray(getattr(sim, "p_" + k)[:n]) for k in ("x", "y", "vx", "vy", "vz")])
    return ids[o], st[:, o].view(np.uint32)


def test_launch_knobs(mods):
    _lib, A = mods
    sp = _spec()
    a, pa = W.make_sweep_sim(sp)
    b, pb = W.make_sweep_sim(sp)
    c, pc = W.make_sweep_sim(sp)
    A.apply(b, {"particle_blocks_per_sm": 4})
    A.apply(c, {"solve_blocks": "half"})
    assert A.current(b)["particle_blocks_per_sm"] == 4 and A.current(c)["solve_blocks"] == "half"
    for _ in range(3):
        a.step(pa)
        b.step(pb)
        c.step(pc)
    ia, sa = _ions_by_id(a)
    ib, sb = _ions_by_id(b)
    np.testing.assert_array_equal(ia, ib)
    np.testing.assert_array_equal(sa, sb)
    np.testing.assert_array_equal(np.asarray(a.V), np.asarray(c.V))
    ic, sc = _ions_by_id(c)
    np.testing.assert_array_equal(ia, ic)
    np.testing.assert_array_equal(sa, sc)
    lib = _lib.load()
    assert lib.pb_sim_set_launch(a._h, 0, 8) != 0
    assert lib.pb_sim_set_launch(a._h, 8, 100000) != 0
    s = a.solver
    assert lib.pb_sim_set_solver(a._h, s["tol"], s["tol_inner"], s["max_outer"], s["max_inner"], 3,
                                 s["max_coarse"]) != 0
    for sim in (a, b, c):
        sim.close()


def test_kernel_variant_knobs(mods):
    """The kernel-variant knobs apply and read back, and a tuning run over them picks a
    setting; particle state does not depend on them."""
    _lib, A = mods
    sp = _spec()
    a, pa = W.make_sweep_sim(sp)
    b, pb = W.make_sweep_sim(sp)
    A.apply(a, {"deposit_hist": False, "ion_tma_window": False, "electron_kernel": "fused"})
    c, pc = W.make_sweep_sim(sp)
    A.apply(b, {"deposit_hist": True, "ion_tma_window": True, "electron_kernel": "split",
                "particles_per_block": 512})
    A.apply(c, {"smoother_sweeps": 2})
    cb = A.current(b)
    assert cb["deposit_hist"] and cb["ion_tma_window"] and cb["electron_kernel"] == "split"
    assert cb["particles_per_block"] == 512 and A.current(c)["smoother_sweeps"] == 2
    for _ in range(3):
        a.step(pa)
        b.step(pb)
        c.step(pc)
    ia, sa = _ions_by_id(a)
    ib, sb = _ions_by_id(b)
    np.testing.assert_array_equal(ia, ib)
    np.testing.assert_array_equal(sa, sb)
    # the second smoother sweep changes only the rounding of the field solve
    np.testing.assert_array_equal(np.asarray(a.V), np.asarray(c.V))
    ic, sc = _ions_by_id(c)
    np.testing.assert_array_equal(ia, ic)
    np.testing.assert_array_equal(sa, sc)
    c.close()
    tuner = A.Autotuner(steps=2, warmup=1, space={"electron_kernel": ("fused", "pairs", "split"),
                                                  "deposit_hist": (False, True)})
    best, table = tuner.tune(a, pa)
    assert best["electron_kernel"] in ("fused", "pairs", "split") and 3 <= len(table) <= 4
    a.close()
    b.close()


def test_tune_two_knobs(mods):
    _lib, A = mods
    sp = _spec()
    sim, params = W.make_sweep_sim(sp)
    sim.step(params)
    tuner = A.Autotuner(steps=2, warmup=1, space={"particle_blocks_per_sm": (4, 8), "max_coarse": (256, 1536)})
    best, table = tuner.tune(sim, params)
    assert set(best) == {"particle_blocks_per_sm", "max_coarse"}
    assert 3 <= len(table) <= 4 and all(t > 0 for t in table.values())
    cur = A.current(sim)
    assert cur["particle_blocks_per_sm"] == best["particle_blocks_per_sm"]
    assert cur["max_coarse"] == best["max_coarse"]
    # the tuned simulator keeps stepping (a new max_coarse rebuilt its hierarchy)
    for _ in range(2):
        sim.step(params)
    assert np.isfinite(np.asarray(sim.V)).all()
    twin, tp = W.make_sweep_sim(sp)
    twin.step(tp)
    assert tuner.apply_cached(twin) == best
    assert A.current(twin)["max_coarse"] == best["max_coarse"]
    sim.close()
    twin.close()


def test_horizon_prefers_a_quick_build(mods):
    """Over a 50-step horizon the dense inverse of a 17 x 65 coarsest level (about 0.1 s on
    the host) costs more per step than the extra V-cycle level of a <= 256-node one."""
    _lib, A = mods
    sim, params = W.make_sweep_sim(_spec())
    sim.step(params)
    tuner = A.Autotuner(steps=2, warmup=1, horizon_steps=50, space={"max_coarse": (1536, 256)})
    best, table = tuner.tune(sim, params)
    assert best["max_coarse"] == 256, table
    sim.close()
