"""Shared test helpers: fixture loading and oracle construction."""
import json
import os

import numpy as np

from oracle.pic_oracle import OracleSimulator, ReplayDraws
from thruster_cx_code_b200.domain import build_domain_geometry

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=False)


def cx_store(table):
    from scipy.interpolate import UnivariateSpline
    t = np.array(table, dtype=np.float64)
    e, cs = t[:, 0], t[:, 1]
    return {"CX": {"energy": e, "cs": cs, "type": "CX",
                   "spline": UnivariateSpline(np.log10(e), np.log10(cs), s=0.0, k=3)}}


def oracle_from_run(f, fp=np.float32):
    """Oracle simulator in the state a run fixture starts from, plus its params and draws."""
    case = json.loads(str(f["case"]))
    params = json.loads(str(f["params"]))
    sim = OracleSimulator(build_domain_geometry, fp=fp)
    sim.dx, sim.dy, sim.dt = case["dx"], case["dy"], case["dt"]
    if "cx_table" in case:
        sim.user_cs = cx_store(case["cx_table"])
    sim.build_domain(params)
    p = f["init_p"]
    n = p.shape[1]
    sim._add_ions(p[0], p[1], p[2], p[3], p[4], f["init_p_cex"], sim.new_ion_ids(n))
    e = f["init_e"]
    if e.shape[1]:
        sim._add_electrons(e[0], e[1], e[2], e[3], e[4], sim.new_e_ids(e.shape[1]))
    names = json.loads(str(f["log_names"]))
    log = [(nm, f[f"draw_{i}"]) for i, nm in enumerate(names)]
    return sim, params, case, ReplayDraws(log)


# ---------------------------------------------------------------------------
# the benchmarked configurations at fixture size (tests/golden/make_golden.py "large")
# ---------------------------------------------------------------------------
M_XE = 131.293 * 1.6605e-27
CX_POWER_LAW = [[float(e), float(7e-19 * e ** -0.1)] for e in np.logspace(0.0, 3.0, 16)]
LARGE_GRIDS = [dict(V=1000.0, t=0.5, gap=0.5, r=0.8, cham=0.0),
               dict(V=-250.0, t=0.5, gap=0.5, r=0.5, cham=0.0),
               dict(V=0.0, t=0.5, gap=0.5, r=0.7, cham=0.0)]
LARGE_CASES = {
    # the 257 x 1025-node 3-grid aperture at 6.25 um (the large_aperture_3grid workload's
    # physics: CX table 7e-19 E^-0.1, m_e = M_Xe / 400, dt = 2.5e-11, sputtering on) with a
    # low break threshold so that cells break within the run
    "large_aperture_3grid": dict(dx=0.00625, dy=0.00625, dt=2.5e-11, m_e_ratio=400.0, row_step=8,
                                 n_ions=16000, n_e=4000, seed=41, steps=2,
                                 params=dict(grids=LARGE_GRIDS, pitch_mm=4.0, upstream_gap_mm=0.4, Te_up=5.0,
                                             n0_plasma=1e17, Ti=0.1, Tn=300.0, n0=1e18, sim_mode="Erosion",
                                             neut_rate=30, Te=5.0, Thresh=20.0)),
    # the 513 x 2049-node stack at 3.125 um (long_erosion_3grid): domain and potential only
    "long_erosion_3grid": dict(dx=0.003125, dy=0.003125, dt=1.25e-11, m_e_ratio=400.0, row_step=16,
                               params=dict(grids=LARGE_GRIDS, pitch_mm=4.0, upstream_gap_mm=0.4, Te_up=5.0,
                                           n0_plasma=1e17, Ti=0.1, Tn=300.0, n0=5e18, sim_mode="Both",
                                           neut_rate=30, Te=5.0, Thresh=1e9)),
}


def large_case_particles(isBound, dx, dy, Lx, Ly, n_ions, n_e, seed):
    """Seeded particles of a large case (float32 SoA): ions uniform over the open cells
    upstream of x = 0.8 Lx with N(2e4, 3e3) m/s axial and N(0, 3e3) transverse
    velocities, 10% of them flagged CEX; electrons over the whole open domain at 2e6 m/s
    thermal speed.  The same bits on every machine (NumPy RandomState)."""
    rs = np.random.RandomState(seed)
    ny, nx = isBound.shape

    def pos(n, x_hi):
        xs, ys, got = [], [], 0
        while got < n:
            x = rs.uniform(1.5 * dx, x_hi, 2 * n)
            y = rs.uniform(0.0, Ly, 2 * n)
            ok = ~isBound[np.clip(np.round(y / dy).astype(np.int64), 0, ny - 1),
                          np.clip(np.round(x / dx).astype(np.int64), 0, nx - 1)]
            xs.append(x[ok]); ys.append(y[ok]); got += int(ok.sum())
        return np.concatenate(xs)[:n].astype(np.float32), np.concatenate(ys)[:n].astype(np.float32)

    xi, yi = pos(n_ions, 0.8 * Lx)
    ions = np.stack([xi, yi, (2e4 + 3e3 * rs.randn(n_ions)).astype(np.float32),
                     (3e3 * rs.randn(n_ions)).astype(np.float32), (3e3 * rs.randn(n_ions)).astype(np.float32)])
    cex = rs.rand(n_ions) < 0.1
    xe, ye = pos(n_e, Lx - dx)
    eles = np.stack([xe, ye] + [(2e6 * rs.randn(n_e)).astype(np.float32) for _ in range(3)])
    return ions, cex, eles
