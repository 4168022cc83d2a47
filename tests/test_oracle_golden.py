"""The CPU oracle and the host domain builder against fixtures made by the reference.

Every comparison here is bit-exact: the fixtures were produced by running the
reference engine on the same inputs, and the oracle restates the same NumPy
arithmetic with the reference's random stream replayed.
"""
import json
import types

import numpy as np
import pytest

from oracle import pic_oracle as O
from thruster_cx_code_b200.domain import build_domain_geometry
from tests.helpers import load, oracle_from_run

DOMAINS = ["c1_half", "one_hole", "two_holes", "bulk"]


def _geom_sim(case):
    s = O.OracleSimulator(build_domain_geometry)
    s.dx, s.dy, s.dt = case["dx"], case["dy"], case["dt"]
    return s


@pytest.mark.parametrize("name", DOMAINS)
def test_domain_geometry_and_potential(name):
    f = load(f"domain_{name}.npz")
    case = json.loads(str(f["case"]))
    params = json.loads(str(f["params"]))
    s = _geom_sim(case)
    s.build_domain(params)
    assert (s.nx, s.ny) == (int(f["nx"]), int(f["ny"]))
    assert s.dx == float(f["dx"]) and s.dy == float(f["dy"])
    assert s.Lx == float(f["Lx"]) and s.Ly == float(f["Ly"])
    assert s.macro_weight == float(f["macro_weight"])
    np.testing.assert_array_equal(s.isBound, f["isBound"])
    np.testing.assert_array_equal(s.V_fixed, f["V_fixed"])
    np.testing.assert_array_equal(np.array(s.mask_grids), f["mask_grids"])
    np.testing.assert_array_equal(np.array(s.grid_x_starts), f["grid_x_starts"])
    np.testing.assert_array_equal(np.array(s.grid_x_ends), f["grid_x_ends"])
    assert bool(s.periodic_y) == bool(f["periodic_y"])
    # 30 Picard iterations through SuperLU on the same operator: identical bits
    np.testing.assert_array_equal(s.V, f["V"])
    np.testing.assert_array_equal(s.Ex, f["Ex"])
    np.testing.assert_array_equal(s.Ey, f["Ey"])
    # remesh with thermal bow (preserve_state)
    s.grid_deflections = [0.012 * (i + 1) for i in range(len(params["grids"]))]
    s.build_domain(params, preserve_state=True)
    np.testing.assert_array_equal(s.isBound, f["bow_isBound"])
    np.testing.assert_array_equal(s.V, f["bow_V"])


def test_domain_numerics_errors(golden_dir):
    import os
    errs = json.load(open(os.path.join(golden_dir, "domain_errors.json")))
    params = json.loads(str(load("domain_c1_half.npz")["params"]))
    for label, (dx, dt) in {"debye": (0.2, 1e-10), "cfl": (0.025, 5e-8)}.items():
        s = O.OracleSimulator(build_domain_geometry)
        s.dx = s.dy = dx
        s.dt = dt
        with pytest.raises(ValueError) as ei:
            s.build_domain(params)
        assert str(ei.value) == errs[label]


@pytest.mark.parametrize("tag", ["ion", "ele"])
@pytest.mark.parametrize("btag", ["B0", "Br"])
@pytest.mark.parametrize("nsub", [1, 3])
def test_push_matches_reference(tag, btag, nsub):
    f = load("push.npz")
    d = load("domain_c1_half.npz")
    nx, ny = int(d["nx"]), int(d["ny"])
    if btag == "B0":
        B = [np.zeros((ny, nx), np.float32)] * 3
    else:
        B = [f["Bx"], f["By"], f["Bz"]]
    a = [np.array(v, copy=True) for v in f[f"{tag}_in"]]
    dt, qm = float(f[f"{tag}_dt"]), float(f[f"{tag}_qm"])
    with np.errstate(all="ignore"):
        for _ in range(nsub):
            O.push_particles_boris(*a, d["Ex"], d["Ey"], *B, len(a[0]), float(d["dx"]), float(d["dy"]),
                                   nx, ny, dt / nsub, qm)
    np.testing.assert_array_equal(np.stack(a), f[f"{tag}_{btag}_sub{nsub}"])


def test_deposit_matches_reference():
    f = load("deposit.npz")
    d = load("domain_c1_half.npz")
    nx, ny, dx, dy = int(d["nx"]), int(d["ny"]), float(d["dx"]), float(d["dy"])
    rho = np.zeros((ny, nx), np.float32)
    cd = float(f["cd"])
    with np.errstate(all="ignore"):
        O.accumulate_rho(f["xi"], f["yi"], rho, len(f["xi"]), dx, dy, nx, ny, cd)
        np.testing.assert_array_equal(rho, f["rho_ions"])
        O.accumulate_rho(f["xe"], f["ye"], rho, len(f["xe"]), dx, dy, nx, ny, -cd)
    np.testing.assert_array_equal(rho, f["rho"])


def test_substeps_match_reference():
    f = load("substeps.npz")
    d = load("domain_c1_half.npz")
    for tag in ("ion", "ele"):
        x, y, vx, vy, vz = f[f"{tag}_in"]
        res = O.substeps(d["Ex"], d["Ey"], float(d["dx"]), float(d["dy"]), int(d["nx"]), int(d["ny"]),
                         x, y, vx, vy, vz, float(f[f"{tag}_qm"]), 1e-10)
        assert res[0] == int(f[f"{tag}_res"][0])
        assert res[1] == f[f"{tag}_res"][1]
        assert res[2] == f[f"{tag}_res"][2]


def test_segment_hits_match_reference():
    f = load("segment.npz")
    d = load("domain_c1_half.npz")
    hit, hix, hiy = O.segment_hits(d["isBound"], float(d["dx"]), float(d["dy"]), int(d["nx"]), int(d["ny"]),
                                   f["x0"], f["y0"], f["x1"], f["y1"])
    np.testing.assert_array_equal(hit, f["hit"])
    np.testing.assert_array_equal(hix, f["hix"])
    np.testing.assert_array_equal(hiy, f["hiy"])
    assert hit.sum() > 50


def test_thermal_block_matches_reference():
    f = load("thermal.npz")
    params = dict(json.loads(str(load("domain_c1_half.npz")["params"])), sim_mode="Thermal", neut_rate=0)
    s = O.OracleSimulator(build_domain_geometry)
    s.dx, s.dy, s.dt = 0.025, 0.025, 1e-10
    s.build_domain(params)
    s.Tmap[:] = f["T0"]
    s.injection_enabled = False
    res = s.step(params, O.ReplayDraws([]))
    np.testing.assert_array_equal(s.Tmap, f["T1"])
    np.testing.assert_array_equal(np.array(res[3], np.float64), f["T_grids"])
    np.testing.assert_array_equal(np.array(s.grid_deflections, np.float64), f["deflections"])
    assert bool(res[0]) == bool(f["remeshed"])


RUNS = ["c1_both", "one_hole_rf", "two_holes_thermal"]


@pytest.mark.parametrize("fp64", [False, True])
@pytest.mark.parametrize("name", RUNS)
def test_full_steps_replay_bit_exact(name, fp64):
    f = load(f"run_{name}{'_fp64' if fp64 else ''}.npz")
    sim, params, case, draws = oracle_from_run(f, fp=np.float64 if fp64 else np.float32)
    outs = f["outs"]
    for s in range(case["steps"]):
        r = sim.step(params, draws)
        got = [float(r[0]), float(r[1]), float(r[2]), float(r[4])] + [float(t) for t in r[3]]
        np.testing.assert_array_equal(np.array(got), outs[s], err_msg=f"step {s} outputs")
        n, ne = sim.num_p, sim.num_e
        p = np.stack([sim.p_x[:n], sim.p_y[:n], sim.p_vx[:n], sim.p_vy[:n], sim.p_vz[:n]])
        np.testing.assert_array_equal(p, f[f"s{s}_p"], err_msg=f"step {s} ions")
        np.testing.assert_array_equal(sim.p_isCEX[:n], f[f"s{s}_p_cex"])
        e = np.stack([sim.e_x[:ne], sim.e_y[:ne], sim.e_vx[:ne], sim.e_vy[:ne], sim.e_vz[:ne]])
        np.testing.assert_array_equal(e, f[f"s{s}_e"], err_msg=f"step {s} electrons")
        for k, attr in (("V", "V"), ("Ex", "Ex"), ("Ey", "Ey"), ("rho", "rho"), ("Tmap", "Tmap"),
                        ("damage", "damage_map"), ("isBound", "isBound")):
            np.testing.assert_array_equal(np.asarray(getattr(sim, attr), f[f"s{s}_{k}"].dtype), f[f"s{s}_{k}"],
                                          err_msg=f"step {s} {k}")
    assert draws.pos == len(draws.log)


# ---------------------------------------------------------------------------
# the benchmarked configurations (make_golden.py "large"): rows of the fixtures
# ---------------------------------------------------------------------------
def _large_oracle(name, fp=np.float32, cx=True):
    from tests.helpers import CX_POWER_LAW, LARGE_CASES, M_XE, cx_store
    case = LARGE_CASES[name]
    s = O.OracleSimulator(build_domain_geometry, fp=fp)
    s.dx, s.dy, s.dt = case["dx"], case["dy"], case["dt"]
    s.m_ion = M_XE
    s.m_e = M_XE / case["m_e_ratio"]
    if cx:
        s.user_cs = cx_store(CX_POWER_LAW)
    s.build_domain(case["params"])
    return s, case


def _unpack(bits, shape):
    return np.unpackbits(bits)[: shape[0] * shape[1]].reshape(shape).astype(bool)


@pytest.mark.parametrize("name", ["large_aperture_3grid", "long_erosion_3grid"])
def test_large_domain_and_potential(name):
    """The 257 x 1025 and 513 x 2049 domains: geometry and the 30-iteration SuperLU
    Picard potential equal the reference's bit for bit (sampled rows and sums)."""
    f = load(f"domain_{name}.npz")
    s, case = _large_oracle(name, cx=False)
    assert (s.nx, s.ny) == (int(f["nx"]), int(f["ny"]))
    assert s.dx == float(f["dx"]) and s.Lx == float(f["Lx"]) and s.Ly == float(f["Ly"])
    assert s.macro_weight == float(f["macro_weight"])
    np.testing.assert_array_equal(s.isBound, _unpack(f["isBound_bits"], (s.ny, s.nx)))
    assert float(np.sum(s.V_fixed)) == float(f["V_fixed_sum"])
    rows = f["rows"]
    np.testing.assert_array_equal(s.V[rows], f["V_rows"])
    np.testing.assert_array_equal(s.Ex[rows], f["Ex_rows"])
    np.testing.assert_array_equal(s.Ey[rows], f["Ey_rows"])
    assert float(np.sum(s.V)) == float(f["V_sum"])


@pytest.mark.parametrize("fp64", [False, True])
def test_large_aperture_steps_replay_bit_exact(fp64):
    """Two steps of the 257 x 1025 case (3 grids, the 7e-19 E^-0.1 CX table, m_e = M/400,
    dt = 2.5e-11, sputtering with cells breaking) with the reference's draws replayed."""
    from tests.helpers import large_case_particles
    from oracle.pic_oracle import ReplayDraws
    import json as _json
    name = "large_aperture_3grid"
    f = load(f"run_{name}{'_fp64' if fp64 else ''}.npz")
    fp = np.float64 if fp64 else np.float32
    s, case = _large_oracle(name, fp=fp)
    ions, cex, eles = large_case_particles(s.isBound, s.dx, s.dy, s.Lx, s.Ly, case["n_ions"], case["n_e"],
                                           case["seed"])
    s._add_ions(*ions.astype(fp), cex, s.new_ion_ids(ions.shape[1]))
    s._add_electrons(*eles.astype(fp), s.new_e_ids(eles.shape[1]))
    names = _json.loads(str(f["log_names"]))
    draws = ReplayDraws([(nm, f[f"draw_{i}"]) for i, nm in enumerate(names)])
    params = case["params"]
    rows = np.unique(np.concatenate([np.arange(0, s.ny, case["row_step"]), [s.ny - 1]]))
    for k in range(case["steps"]):
        r = s.step(params, draws)
        got = [float(r[0]), float(r[1]), float(r[2]), float(r[4])] + [float(t) for t in r[3]]
        np.testing.assert_array_equal(np.array(got), f["outs"][k], err_msg=f"step {k} outputs")
        if f"s{k}_p" not in f.files:
            continue
        n, ne = s.num_p, s.num_e
        p = np.stack([s.p_x[:n], s.p_y[:n], s.p_vx[:n], s.p_vy[:n], s.p_vz[:n]])
        np.testing.assert_array_equal(p, f[f"s{k}_p"], err_msg=f"step {k} ions")
        np.testing.assert_array_equal(s.p_isCEX[:n], f[f"s{k}_p_cex"])
        e = np.stack([s.e_x[:ne], s.e_y[:ne], s.e_vx[:ne], s.e_vy[:ne], s.e_vz[:ne]])
        np.testing.assert_array_equal(e, f[f"s{k}_e"], err_msg=f"step {k} electrons")
        for key, attr in (("V", "V"), ("rho", "rho"), ("damage", "damage_map")):
            a = np.asarray(getattr(s, attr))
            np.testing.assert_array_equal(a[rows], f[f"s{k}_{key}_rows"], err_msg=f"step {k} {key}")
            assert float(np.sum(a.astype(np.float64))) == float(f[f"s{k}_{key}_sum"]), (k, key)
        np.testing.assert_array_equal(s.isBound, _unpack(f[f"s{k}_isBound_bits"], s.isBound.shape))
    assert draws.pos == len(draws.log)
