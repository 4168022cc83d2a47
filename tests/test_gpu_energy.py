"""get_total_energy's three float32 sums on the device (pb_sim_energy_sums) against NumPy's
np.sum of the same arrays copied to the host: bit-identical for the ions, the electrons and
the field, after real steps and for particle counts at the edges of NumPy's pairwise
summation (below 8, one block of at most 128, the first splits, and large odd counts)."""
import ctypes as C

import numpy as np
import pytest

from thruster_cx_code_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from thruster_cx_code_b200 import _lib
    return _lib


def _device_sums(_lib, sim):
    out = (C.c_double * 3)()
    _lib.check(_lib.load().pb_sim_energy_sums(sim._h, out), "pb_sim_energy_sums")
    return [np.float32(v) for v in out]


def _numpy_sums(sim):
    n, m = sim.num_p, sim.num_e
    v2 = (np.asarray(sim.p_vx[:n]) ** 2 + np.asarray(sim.p_vy[:n]) ** 2 + np.asarray(sim.p_vz[:n]) ** 2)
    v2e = (np.asarray(sim.e_vx[:m]) ** 2 + np.asarray(sim.e_vy[:m]) ** 2 + np.asarray(sim.e_vz[:m]) ** 2)
    Ex, Ey = np.asarray(sim.Ex), np.asarray(sim.Ey)
    assert v2.dtype == np.float32 and Ex.dtype == np.float32
    return [np.sum(v2), np.sum(v2e), np.sum(Ex ** 2 + Ey ** 2)]


def _spec():
    return W.sweep_point(np.random.default_rng(5), 0, grids=("64x256",), n_range=(150000, 150001))


def test_sums_after_steps_equal_numpy(lib):
    sim, params = W.make_sweep_sim(_spec())
    for _ in range(3):
        sim.step(params)
    dev, ref = _device_sums(lib, sim), _numpy_sums(sim)
    for d, r in zip(dev, ref):
        assert d.tobytes() == r.tobytes(), (d, r)
    # the public diagnostic uses them with the reference's double arithmetic
    e = sim.get_total_energy()
    assert e["ke_ions_J"] == float(ref[0]) * 0.5 * sim.m_ion * sim.macro_weight
    assert e["field_J"] == float(ref[2]) * 0.5 * sim.eps0 * ((sim.dx * 1e-3) * (sim.dy * 1e-3))
    sim.close()


@pytest.mark.parametrize("n", [0, 1, 7, 8, 9, 127, 128, 129, 136, 1000, 65543, 1000003])
def test_sums_at_pairwise_edges(lib, n):
    sim, _ = W.make_sweep_sim(_spec())
    rng = np.random.default_rng(n)
    x = rng.uniform(0.5, 1.0, n).astype(np.float32)
    y = rng.uniform(0.5, 1.0, n).astype(np.float32)
    v = [(rng.standard_normal(n) * 10.0 ** rng.uniform(2, 6, n)).astype(np.float32) for _ in range(3)]
    sim.set_particles("ions", x, y, *v, sort=False)
    sim.set_particles("electrons", x[: n // 2], y[: n // 2], *[a[: n // 2] for a in v], sort=False)
    dev, ref = _device_sums(lib, sim), _numpy_sums(sim)
    for d, r in zip(dev, ref):
        assert d.tobytes() == r.tobytes(), (n, d, r)
    sim.close()


def test_energy_warning_on_a_jump(lib, capsys):
    """The reference's conservation check (physics_engine.py:1847-1856): a call whose total
    energy differs from the previous call's by more than energy_warning_threshold prints the
    warning, a smaller change does not, and every call is kept in the history."""
    sim, params = W.make_sweep_sim(_spec())
    sim.step(params)
    capsys.readouterr()
    first = sim.get_total_energy()
    again = sim.get_total_energy()  # no change
    assert again["total_J"] == first["total_J"]
    assert "[Energy Warning]" not in capsys.readouterr().out
    # the electrode field holds nearly all of the energy here: doubling it quadruples the total
    sim.Ex = np.asarray(sim.Ex) * np.float32(2.0)
    sim.Ey = np.asarray(sim.Ey) * np.float32(2.0)
    second = sim.get_total_energy()
    rel = abs(second["total_J"] - first["total_J"]) / first["total_J"]
    assert rel > sim.energy_warning_threshold, rel
    assert "[Energy Warning]" in capsys.readouterr().out
    assert len(sim.energy_history_tot) == 3
    sim.close()
