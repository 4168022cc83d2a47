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
