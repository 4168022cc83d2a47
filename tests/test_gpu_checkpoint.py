"""Checkpoint and resume: a run saved after some steps and resumed in a new simulator
continues exactly as the uninterrupted run (particles, ids, potential, counters)."""
import numpy as np
import pytest

from thruster_cx_code_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from thruster_cx_code_b200 import physics_engine as PE
    return PE


def _state(sim):
    n, ne = sim.num_p, sim.num_e
    a = np.stack([np.asarray(getattr(sim, "p_" + k)[:n]) for k in ("x", "y", "vx", "vy", "vz")]).astype(np.float32)
    e = np.stack([np.asarray(getattr(sim, "e_" + k)[:ne]) for k in ("x", "y", "vx", "vy", "vz")]).astype(np.float32)
    return a, np.asarray(sim.p_id[:n]).copy(), np.asarray(sim.p_isCEX[:n]).copy(), e, np.asarray(sim.e_id[:ne]).copy()


def test_resume_continues_bit_for_bit(engine, tmp_path):
    rng = np.random.default_rng(21)
    sp = W.sweep_point(rng, 0, grids=("64x256",), n_range=(120000, 120001))
    a, params = W.make_sweep_sim(sp)
    for _ in range(5):
        a.step(params)
    path = str(tmp_path / "ckpt.npz")
    a.save_checkpoint(path, params)
    for _ in range(4):
        a.step(params)
    b, pb = engine.DigitalTwinSimulator.load_checkpoint(path)
    assert b.iteration == 5
    for _ in range(4):
        b.step(pb)
    assert (a.num_p, a.num_e, a.iteration) == (b.num_p, b.num_e, b.iteration)
    for x, y in zip(_state(a), _state(b)):
        if x.dtype == np.float32:
            np.testing.assert_array_equal(x.view(np.uint32), y.view(np.uint32))
        else:
            np.testing.assert_array_equal(x, y)
    np.testing.assert_array_equal(a.V, b.V)
    np.testing.assert_allclose(a.damage_map, b.damage_map, rtol=1e-12, atol=0)  # FP64 atomics order
    assert a.transmitted_ions == b.transmitted_ions and a.next_ion_id == b.next_ion_id
    a.close()
    b.close()
