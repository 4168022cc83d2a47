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
