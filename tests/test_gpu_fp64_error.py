"""Error of the FP32 GPU path against the FP64 oracle.

The FP64 oracle is the NumPy restatement run with float64 particles and fields.  It is
pinned bit-exact to the reference module run with _NP_FP = float64
(tests/test_oracle_golden.py).  Both sides draw from the same Philox stream and start
from the same particles (the Both-mode 2-grid case); each solves its own fields.  After
K steps the test states, and bounds:

* phi: max |V_gpu - V_fp64| / max |V_fp64|;
* particle state per id: 99th percentile of the position error in cells, and the share of
  ids present on both sides (absorption and CEX decisions can flip near thresholds);
* beamlet current: total exit-plane crossings over the K steps;
* theta95 of the last step where it is defined (2000 ions seeded just upstream of the
  exit plane make it defined);
* eroded mass: the sum of the FP64 sputter-damage map.
"""
import json

import numpy as np
import pytest

from oracle import pic_oracle as O
from thruster_cx_code_b200.domain import build_domain_geometry
from tests.helpers import cx_store, load

pytestmark = pytest.mark.gpu
SEED = 20240611
K = 60


@pytest.fixture(scope="module")
def gpu_mod():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from thruster_cx_code_b200 import physics_engine as PE
    return PE


def test_fp32_gpu_against_fp64_oracle(gpu_mod, capsys):
    f = load("run_c1_both.npz")
    case, params = json.loads(str(f["case"])), json.loads(str(f["params"]))
    g = gpu_mod.DigitalTwinSimulator(seed=SEED, sort_every=0)
    o = O.OracleSimulator(build_domain_geometry, fp=np.float64)
    for s in (g, o):
        s.dx, s.dy, s.dt = case["dx"], case["dy"], case["dt"]
        if "cx_table" in case:
            s.user_cs = cx_store(case["cx_table"])
    g.build_domain(params)
    o.build_domain(params)
    p, cex, e = f["init_p"], f["init_p_cex"], f["init_e"]
    # plus 2000 ions just upstream of the exit plane, in the last grid's hole, moving
    # downstream, so that enough cross in each step for theta95 to be defined
    rs = np.random.default_rng(5)
    m = 2000
    x_exit = float(g.grid_x_ends[-1])
    r_hole = params["grids"][-1]["r"]
    extra = np.stack([rs.uniform(x_exit - 0.03, x_exit - 0.001, m), rs.uniform(0.0, 0.9 * r_hole, m),
                      rs.normal(4e4, 2e3, m), rs.normal(0.0, 2e3, m), rs.normal(0.0, 1e3, m)]).astype(np.float32)
    p = np.concatenate([p.astype(np.float32), extra], axis=1)
    cex = np.concatenate([cex, np.zeros(m, bool)])
    n, ne = p.shape[1], e.shape[1]
    g.set_particles("ions", *p.astype(np.float32), is_cex=cex, ids=np.arange(n), sort=False)
    o._add_ions(*p.astype(np.float64), cex, o.new_ion_ids(n))
    if ne:
        g.set_particles("electrons", *e.astype(np.float32), ids=np.arange(ne), sort=False)
        o._add_electrons(*e.astype(np.float64), o.new_e_ids(ne))
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
    dxc = np.abs(np.asarray(g.p_x[:ng])[a].astype(np.float64) - o.p_x[:o.num_p][b]) / case["dx"]
    dyc = np.abs(np.asarray(g.p_y[:ng])[a].astype(np.float64) - o.p_y[:o.num_p][b]) / case["dy"]
    pos99 = float(np.percentile(np.maximum(dxc, dyc), 99))
    cur = (g.transmitted_ions, o.transmitted_ions)
    cur_err = abs(cur[0] - cur[1]) / max(cur[1], 1.0)
    dmg = (float(np.sum(g.damage_map)), float(np.sum(o.damage_map)))
    dmg_err = abs(dmg[0] - dmg[1]) / max(abs(dmg[1]), 1e-300)
    th_err = abs(th_g - th_o) / abs(th_o) if np.isfinite(th_o) else 0.0
    with capsys.disabled():
        print(f"\n[fp64 error, {K} steps] phi {errV:.2e}; ids common {share:.4f}; position p99 {pos99:.2e} cells; "
              f"crossings {cur[0]:.0f} vs {cur[1]:.0f} ({cur_err:.2e}); theta95 {th_g:.4f} vs {th_o:.4f} "
              f"({th_err:.2e}); damage sum {dmg[0]:.6e} vs {dmg[1]:.6e} ({dmg_err:.2e})")
    assert errV <= 1e-5
    assert share >= 0.995
    assert pos99 <= 1e-3
    assert cur_err <= 0.01
    assert th_err <= 0.01
    assert dmg_err <= 0.01
