"""GPU parity on the benchmarked configurations (257 x 1025 and 513 x 2049 nodes).

* Field solve: the 30-iteration Picard potential of build_domain against the reference's
  SuperLU result (sampled rows of the fixtures that tests/golden/make_golden.py made by
  running the reference): |V - V_ref| <= 1e-7 max|V|, |E - E_ref| <= 1e-5 max|E|, and
  the electrode masks equal.
* One timestep of the 257 x 1025 case given identical fields (3 grids, the 7e-19 E^-0.1
  CX table, m_e = M_Xe / 400, dt = 2.5e-11, cells breaking under sputtering): particles
  per id bit for bit, deposit bit-exact, damage within 1e-12 (FP64 atomics order).  Again
  with the configuration's own options, the uniform neutral background and the power-law
  yield 1e-3 (E - 30)^1.2.
* Eight timesteps with each side solving its own fields: per-id state within 1e-4 of
  scale, counts within 0.2%, potential within 1e-6.
* The FP32 GPU path against the FP64 oracle on both grids: potential, particle state,
  beamlet current, theta95 and eroded mass (sum of the FP64 damage map).
"""
import json

import numpy as np
import pytest

from oracle import pic_oracle as O
from thruster_cx_code_b200.domain import build_domain_geometry
from tests.helpers import CX_POWER_LAW, LARGE_CASES, M_XE, cx_store, large_case_particles, load

pytestmark = pytest.mark.gpu
SEED = 20240611
OPTIONS = dict(neutral_profile="uniform", sputter_exponent=1.2)
MO_POWER_LAW = {'k': 138.0, 'rho': 10280.0, 'cp': 250.0, 'emissivity': 0.80, 'alpha': 4.8e-6,
                'E_mod': 329e9, 'Y_coeff': 1e-3, 'E_th': 30.0}


@pytest.fixture(scope="module")
def PE():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from thruster_cx_code_b200 import physics_engine
    return physics_engine


def _setup(s, case, cx=True, material=None):
    s.dx, s.dy, s.dt = case["dx"], case["dy"], case["dt"]
    s.m_ion = M_XE
    s.m_e = M_XE / case["m_e_ratio"]
    if material:
        s.set_material(props=dict(material))
    if cx:
        s.user_cs = cx_store(CX_POWER_LAW)


def _unpack(bits, shape):
    return np.unpackbits(bits)[: shape[0] * shape[1]].reshape(shape).astype(bool)


@pytest.mark.parametrize("name", ["large_aperture_3grid", "long_erosion_3grid"])
def test_large_potential_matches_superlu(PE, name):
    f = load(f"domain_{name}.npz")
    case = LARGE_CASES[name]
    g = PE.DigitalTwinSimulator()
    _setup(g, case, cx=False)
    g.build_domain(case["params"])
    assert (g.ny, g.nx) == (int(f["ny"]), int(f["nx"]))
    np.testing.assert_array_equal(g.isBound, _unpack(f["isBound_bits"], (g.ny, g.nx)))
    rows = f["rows"]
    V = g.V[rows]
    errV = np.abs(V - f["V_rows"]).max() / float(f["V_absmax"])
    assert errV <= 1e-7, errV
    for k in ("Ex", "Ey"):
        E = getattr(g, k)[rows].astype(np.float64)
        Eref = f[f"{k}_rows"].astype(np.float64)
        err = np.abs(E - Eref).max() / np.abs(Eref).max()
        assert err <= 1e-5, (k, err)
    assert g.poisson_stats[2] <= 1e-8
    g.close()


def _pair(PE, opts=None, thresh=None, material=None, fp=np.float32, extra_exit=0):
    case = LARGE_CASES["large_aperture_3grid"]
    params = dict(case["params"], **(opts or {}))
    if thresh is not None:
        params["Thresh"] = thresh
    g = PE.DigitalTwinSimulator(seed=SEED, sort_every=0)
    o = O.OracleSimulator(build_domain_geometry, fp=fp)
    for s in (g, o):
        _setup(s, case, material=material)
        s.build_domain(params)
    ions, cex, eles = large_case_particles(o.isBound, o.dx, o.dy, o.Lx, o.Ly, case["n_ions"], case["n_e"],
                                           case["seed"])
    if extra_exit:
        # ions just upstream of the exit plane inside the last grid's hole, moving
        # downstream, so that theta95 is defined in every step
        rs = np.random.default_rng(5)
        x_exit = float(o.grid_x_ends[-1])
        r_hole = params["grids"][-1]["r"]
        more = np.stack([rs.uniform(x_exit - 0.03, x_exit - 0.001, extra_exit),
                         rs.uniform(0.0, 0.9 * r_hole, extra_exit), rs.normal(4e4, 2e3, extra_exit),
                         rs.normal(0.0, 2e3, extra_exit), rs.normal(0.0, 1e3, extra_exit)]).astype(np.float32)
        ions = np.concatenate([ions, more], axis=1)
        cex = np.concatenate([cex, np.zeros(extra_exit, bool)])
    n, ne = ions.shape[1], eles.shape[1]
    g.set_particles("ions", *ions, is_cex=cex, ids=np.arange(n), sort=False)
    g.set_particles("electrons", *eles, ids=np.arange(ne), sort=False)
    o._add_ions(*ions.astype(fp), cex, o.new_ion_ids(n))
    o._add_electrons(*eles.astype(fp), o.new_e_ids(ne))
    return g, o, params


def _state(sim, species):
    if species == "ions":
        n = sim.num_p
        a = np.stack([np.asarray(sim.p_x[:n]), np.asarray(sim.p_y[:n]), np.asarray(sim.p_vx[:n]),
                      np.asarray(sim.p_vy[:n]), np.asarray(sim.p_vz[:n])]).astype(np.float32)
        return a, np.asarray(sim.p_id[:n]).astype(np.int64)
    n = sim.num_e
    a = np.stack([np.asarray(sim.e_x[:n]), np.asarray(sim.e_y[:n]), np.asarray(sim.e_vx[:n]),
                  np.asarray(sim.e_vy[:n]), np.asarray(sim.e_vz[:n])]).astype(np.float32)
    return a, np.asarray(sim.e_id[:n]).astype(np.int64)


@pytest.mark.parametrize("variant", ["reference_physics", "uniform_neutrals_power_law"])
def test_large_one_step_bit_exact_given_fields(PE, variant):
    opts = OPTIONS if variant != "reference_physics" else None
    mat = MO_POWER_LAW if opts else None
    g, o, params = _pair(PE, opts=opts, material=mat)
    g.V, g.Ex, g.Ey = o.V, o.Ex, o.Ey
    rg = g.step(params)
    ro = o.step(params, O.PhiloxDraws(SEED))
    assert (g.num_p, g.num_e) == (o.num_p, o.num_e)
    np.testing.assert_array_equal(g.rho, o.rho)
    for sp in ("ions", "electrons"):
        ag, ig = _state(g, sp)
        ao, io = _state(o, sp)
        np.testing.assert_array_equal(ig, io)
        np.testing.assert_array_equal(ag.view(np.uint32), ao.view(np.uint32))
    np.testing.assert_array_equal(np.asarray(g.p_isCEX[:g.num_p]).astype(bool), o.p_isCEX[:o.num_p])
    assert bool(rg[0]) == bool(ro[0]) and rg[1] == ro[1] and rg[4] == ro[4]
    np.testing.assert_allclose(g.damage_map, o.damage_map, rtol=1e-12, atol=0)
    np.testing.assert_array_equal(g.isBound, o.isBound)
    assert bool(ro[0]), "the case is set up so that cells break in the first step"
    assert g.transmitted_ions == o.transmitted_ions and g.entered_optics == o.entered_optics
    g.close()


@pytest.mark.parametrize("variant", ["reference_physics", "uniform_neutrals_power_law"])
def test_large_eight_steps_close(PE, variant):
    opts = OPTIONS if variant != "reference_physics" else None
    mat = MO_POWER_LAW if opts else None
    g, o, params = _pair(PE, opts=opts, material=mat, thresh=1e9)
    draws = O.PhiloxDraws(SEED)
    outs_g, outs_o = [], []
    for _ in range(8):
        outs_g.append(g.step(params))
        outs_o.append(o.step(params, draws))
    assert abs(g.num_p - o.num_p) <= max(2, 0.002 * o.num_p)
    assert abs(g.num_e - o.num_e) <= max(2, 0.002 * o.num_e)
    for sp in ("ions", "electrons"):
        ag, ig = _state(g, sp)
        ao, io = _state(o, sp)
        common, a_i, b_i = np.intersect1d(ig, io, return_indices=True)
        assert common.size >= 0.99 * min(ig.size, io.size)
        d = np.abs(ag[:, a_i].astype(np.float64) - ao[:, b_i].astype(np.float64))
        scale = np.abs(ao[:, b_i]).astype(np.float64).max(axis=1, keepdims=True)
        assert (d / scale).max() <= 1e-4, sp
    errV = np.abs(g.V - o.V).max() / np.abs(o.V).max()
    assert errV <= 1e-6, errV
    for a, b in zip(outs_g, outs_o):
        assert abs(a[1] - b[1]) <= 1e-6 * abs(b[1])
    g.close()


def _fp64_table(g, o, params, K, dx, dy, label, capsys):
    draws = O.PhiloxDraws(SEED)
    th_g = th_o = np.nan
    for _ in range(K):
        rg = g.step(params)
        ro = o.step(params, draws)
        if np.isfinite(rg[2]) and np.isfinite(ro[2]):
            th_g, th_o = rg[2], ro[2]
    errV = float(np.abs(g.V - o.V).max() / np.abs(o.V).max())
    ng = g.num_p
    ig = np.asarray(g.p_id[:ng]).astype(np.int64)
    io = np.asarray(o.p_id[:o.num_p]).astype(np.int64)
    common, a, b = np.intersect1d(ig, io, return_indices=True)
    share = common.size / max(ig.size, io.size)
    dxc = np.abs(np.asarray(g.p_x[:ng])[a].astype(np.float64) - o.p_x[:o.num_p][b]) / dx
    dyc = np.abs(np.asarray(g.p_y[:ng])[a].astype(np.float64) - o.p_y[:o.num_p][b]) / dy
    pos99 = float(np.percentile(np.maximum(dxc, dyc), 99))
    cur = (g.transmitted_ions, o.transmitted_ions)
    cur_err = abs(cur[0] - cur[1]) / max(cur[1], 1.0)
    dmg = (float(np.sum(g.damage_map)), float(np.sum(o.damage_map)))
    dmg_err = abs(dmg[0] - dmg[1]) / max(abs(dmg[1]), 1e-300)
    th_err = abs(th_g - th_o) / abs(th_o) if np.isfinite(th_o) else 0.0
    with capsys.disabled():
        print(f"\n[fp64 error, {label}, {K} steps] phi {errV:.2e}; ids common {share:.4f}; position p99 "
              f"{pos99:.2e} cells; crossings {cur[0]:.0f} vs {cur[1]:.0f} ({cur_err:.2e}); theta95 {th_g:.4f} vs "
              f"{th_o:.4f} ({th_err:.2e}); eroded mass (damage sum) {dmg[0]:.6e} vs {dmg[1]:.6e} ({dmg_err:.2e})")
    assert errV <= 1e-5
    assert share >= 0.995
    assert pos99 <= 1e-3
    assert cur_err <= 0.01
    assert th_err <= 0.01
    assert dmg[1] > 0.0 and dmg_err <= 0.01


def test_large_fp32_gpu_against_fp64_oracle(PE, capsys):
    """257 x 1025 with the configuration's options (uniform neutrals, power-law yield), 40
    steps, 2000 extra ions seeded at the exit plane so that theta95 is defined."""
    g, o, params = _pair(PE, opts=OPTIONS, material=MO_POWER_LAW, thresh=1e9, fp=np.float64, extra_exit=2000)
    _fp64_table(g, o, params, 40, o.dx, o.dy, "257 x 1025", capsys)
    g.close()


def test_c5_grid_fp32_gpu_against_fp64_oracle(PE, capsys):
    """513 x 2049 (the long-erosion configuration's grid and physics: uniform neutrals at
    5e18, power-law yield, heating and conduction on) with a fixture-sized particle set,
    20 steps: the eroded-mass statement on the largest grid."""
    case = dict(LARGE_CASES["long_erosion_3grid"])
    params = dict(case["params"], **OPTIONS)
    g = PE.DigitalTwinSimulator(seed=SEED, sort_every=0)
    o = O.OracleSimulator(build_domain_geometry, fp=np.float64)
    for s in (g, o):
        _setup(s, case, material=MO_POWER_LAW)
        s.build_domain(params)
    ions, cex, eles = large_case_particles(o.isBound, o.dx, o.dy, o.Lx, o.Ly, 12000, 3000, 43)
    rs = np.random.default_rng(9)
    m = 2000
    x_exit = float(o.grid_x_ends[-1])
    more = np.stack([rs.uniform(x_exit - 0.02, x_exit - 0.001, m), rs.uniform(0.0, 0.6, m),
                     rs.normal(4e4, 2e3, m), rs.normal(0.0, 2e3, m), rs.normal(0.0, 1e3, m)]).astype(np.float32)
    # and ions driven into the accel grid's upstream face, so that sputtering accumulates
    x_acc = float(o.grid_x_starts[1])
    hit = np.stack([rs.uniform(x_acc - 0.05, x_acc - 0.01, m), rs.uniform(0.55, 1.2, m),
                    rs.normal(3e4, 2e3, m), rs.normal(0.0, 2e3, m), rs.normal(0.0, 1e3, m)]).astype(np.float32)
    ions = np.concatenate([ions, more, hit], axis=1)
    cex = np.concatenate([cex, np.zeros(2 * m, bool)])
    n, ne = ions.shape[1], eles.shape[1]
    g.set_particles("ions", *ions, is_cex=cex, ids=np.arange(n), sort=False)
    g.set_particles("electrons", *eles, ids=np.arange(ne), sort=False)
    o._add_ions(*ions.astype(np.float64), cex, o.new_ion_ids(n))
    o._add_electrons(*eles.astype(np.float64), o.new_e_ids(ne))
    _fp64_table(g, o, params, 20, o.dx, o.dy, "513 x 2049", capsys)
    g.close()
