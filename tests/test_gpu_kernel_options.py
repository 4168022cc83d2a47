"""The step kernels' variants give the same bits.

PB_OPT_SMEM_HIST (deposit and PPC counts through shared-memory cell histograms per tile),
PB_OPT_TMA_TILE (the ion step stages each tile's window of the E-corner array in shared
memory with a TMA copy), PB_OPT_ELE_PAIRS (two electrons per thread pushed side by
side), PB_OPT_ELE_SPLIT (the electron step as a barrier-free push and a separate
compaction), and the tile of 512 instead of 1024 particles per block, change how the kernels move
data and schedule work, not what they compute.
Three steps of the 257 x 1025 case from the same state, with the particles re-sorted by
cell every step (so that tiles are compact and the windows and histograms are used) and
once without sorting (wide tiles take the fallback paths), must agree bit for bit in every
particle, the charge density, the PPC map and the damage map, under every
combination.  The oracle pins the default combination (tests/test_gpu_large.py)."""
import numpy as np
import pytest

from tests.helpers import CX_POWER_LAW, LARGE_CASES, M_XE, cx_store, large_case_particles

pytestmark = pytest.mark.gpu
SEED = 77


@pytest.fixture(scope="module")
def PE():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from thruster_cx_code_b200 import physics_engine
    return physics_engine


def _run(PE, flags, sort_every, steps=3, ppb=1024):
    from thruster_cx_code_b200 import _lib
    case = LARGE_CASES["large_aperture_3grid"]
    params = dict(case["params"], Thresh=1e9)
    g = PE.DigitalTwinSimulator(seed=SEED, sort_every=sort_every)
    g.dx, g.dy, g.dt = case["dx"], case["dy"], case["dt"]
    g.m_ion = M_XE
    g.m_e = M_XE / case["m_e_ratio"]
    g.user_cs = cx_store(CX_POWER_LAW)
    _lib.check(g._libh.pb_sim_set_kernel_options(g._h, flags), "set_kernel_options")
    _lib.check(g._libh.pb_sim_set_tile(g._h, ppb), "set_tile")
    g.build_domain(params)
    ions, cex, eles = large_case_particles(g.isBound, g.dx, g.dy, g.Lx, g.Ly, 60000, 20000, 5)
    g.set_particles("ions", *ions, is_cex=cex, ids=np.arange(ions.shape[1]), sort=sort_every > 0)
    g.set_particles("electrons", *eles, ids=np.arange(eles.shape[1]), sort=sort_every > 0)
    for _ in range(steps):
        g.step(params)
    n, ne = g.num_p, g.num_e
    out = {"p": np.stack([np.asarray(getattr(g, k)[:n]) for k in ("p_x", "p_y", "p_vx", "p_vy", "p_vz")]),
           "pid": np.asarray(g.p_id[:n]), "cex": np.asarray(g.p_isCEX[:n]),
           "e": np.stack([np.asarray(getattr(g, k)[:ne]) for k in ("e_x", "e_y", "e_vx", "e_vy", "e_vz")]),
           "eid": np.asarray(g.e_id[:ne]), "rho": g.rho.copy(), "ppc": g.current_ppc_map.copy(),
           "damage": g.damage_map.copy(), "V": g.V.copy()}
    g.close()
    return out


@pytest.mark.parametrize("sort_every", [1, 0])
def test_kernel_variants_bit_identical(PE, sort_every):
    from thruster_cx_code_b200 import _lib
    ref = _run(PE, 0, sort_every)
    H, T, P, S = _lib.PB_OPT_SMEM_HIST, _lib.PB_OPT_TMA_TILE, _lib.PB_OPT_ELE_PAIRS, _lib.PB_OPT_ELE_SPLIT
    cases = [(f, 1024) for f in (H, T, H | T, P, H | P, H | T | P, S, H | T | S)] + [(0, 512), (H | T | P, 512)]
    for flags, ppb in cases:
        got = _run(PE, flags, sort_every, ppb=ppb)
        for k in ("p", "e", "rho"):
            np.testing.assert_array_equal(got[k].view(np.uint32), ref[k].view(np.uint32), err_msg=f"{flags} {ppb} {k}")
        for k in ("pid", "cex", "eid", "ppc", "V"):
            np.testing.assert_array_equal(got[k], ref[k], err_msg=f"{flags} {ppb} {k}")
        # damage adds float64 atomics in whatever order the blocks reach them
        np.testing.assert_allclose(got["damage"], ref["damage"], rtol=1e-12, atol=0)


def test_unknown_option_bits_rejected(PE):
    from thruster_cx_code_b200 import _lib
    g = PE.DigitalTwinSimulator()
    assert g._libh.pb_sim_set_kernel_options(g._h, 1 << 9) == 2
    assert g._libh.pb_sim_set_tile(g._h, 768) == 2
    g.close()
