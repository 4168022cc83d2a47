"""Named aperture workloads (params dicts in the reference's config.json vocabulary).

``single_aperture_2grid``: 2-grid screen/accel optics at 25 um spacing (65 x 284 nodes,
the geometry of the reference's own CPU-runnable case), 100k macro-particles, a uniform
neutral background of 1e18 m^-3 and a constant CEX cross-section of 5e-19 m^2 (a flat
log-log table, evaluated by the reference's own spline path).

``large_aperture_3grid``: 3-grid screen +1000 V / accel -250 V / decel 0 V, each 0.5 mm
thick, 6.25 um spacing chosen so the derived domain is exactly 257 x 1025 nodes
(256 x 1024 cells), 8M FP32 macro-particles (6M Xe+ and 2M electrons at mass ratio
1/400), CEX cross-section 7e-19 E^-0.1 m^2 as a log-log table over 1-1000 eV, sputtering
on with the Mo yield 1e-3 (E - 30)^1.2.

``long_erosion_3grid``: the same 3-grid stack at 3.125 um spacing (513 x 2049 nodes,
512 x 2048 cells), 64M FP32 macro-particles (48M Xe+ and 16M electrons), a uniform CEX
neutral density of 5e18 m^-3, sputtering with the power-law yield and grid heating with
conduction on ("Both").

Particles are pre-loaded from a seeded NumPy generator: positions uniform over the
non-electrode cells, ion velocities N(v_Bohm, v_th), electron velocities thermal.

Sweep points (batched and served runs): the 2-grid stack with screen voltage uniform in
600-1800 V, accel voltage uniform in -300..-100 V, plasma density log-uniform in
3e16-3e17 m^-3, node spacing drawn from three resolutions (about 64 x 256, 128 x 512 and
256 x 1024 cells; dt scales with the spacing) and a log-uniform macro-particle count.
"""
import numpy as np

Q = 1.602e-19
M_XE = 131.293 * 1.6605e-27


def cx_table_power_law(a=7e-19, p=-0.1, e_lo=1.0, e_hi=1000.0, n=16):
    e = np.logspace(np.log10(e_lo), np.log10(e_hi), n)
    return np.stack([e, a * e ** p], axis=1)


def cx_store(table):
    from scipy.interpolate import UnivariateSpline
    t = np.asarray(table, dtype=np.float64)
    return {"CX": {"energy": t[:, 0], "cs": t[:, 1], "type": "CX",
                   "spline": UnivariateSpline(np.log10(t[:, 0]), np.log10(t[:, 1]), s=0.0, k=3)}}


# a constant cross-section as a table for the reference's log-log cubic spline (at least
# four points for k = 3; a flat table makes the spline constant)
CX_CONSTANT_5E19 = np.array([[1.0, 5e-19], [10.0, 5e-19], [100.0, 5e-19], [1000.0, 5e-19]])
# the molybdenum preset with the yield coefficient of the power law 1e-3 (E - 30)^1.2
MO_POWER_LAW = {'k': 138.0, 'rho': 10280.0, 'cp': 250.0, 'emissivity': 0.80, 'alpha': 4.8e-6,
                'E_mod': 329e9, 'Y_coeff': 1e-3, 'E_th': 30.0}

WORKLOADS = {
    "single_aperture_2grid": dict(
        dx=0.025, dy=0.025, dt=1e-10, m_e_ratio=100.0, n_ions=80000, n_e=20000, cx=CX_CONSTANT_5E19,
        material=None,
        params=dict(grids=[dict(V=1000.0, t=0.38, gap=1.0, r=0.95, cham=0.0),
                           dict(V=-200.0, t=1.0, gap=1.0, r=0.55, cham=0.0)],
                    pitch_mm=3.75, Te_up=5.0, n0_plasma=1e17, Ti=0.1, Tn=300.0, n0=1e18,
                    neutral_profile="uniform", sim_mode="Erosion", neut_rate=30, Te=5.0, Thresh=1e9)),
    "large_aperture_3grid": dict(
        dx=0.00625, dy=0.00625, dt=2.5e-11, m_e_ratio=400.0, n_ions=6_000_000, n_e=2_000_000,
        cx=cx_table_power_law(), material=MO_POWER_LAW,
        params=dict(grids=[dict(V=1000.0, t=0.5, gap=0.5, r=0.8, cham=0.0),
                           dict(V=-250.0, t=0.5, gap=0.5, r=0.5, cham=0.0),
                           dict(V=0.0, t=0.5, gap=0.5, r=0.7, cham=0.0)],
                    pitch_mm=4.0, upstream_gap_mm=0.4, Te_up=5.0, n0_plasma=1e17, Ti=0.1, Tn=300.0,
                    n0=1e18, sim_mode="Erosion", sputter_exponent=1.2, neut_rate=30, Te=5.0, Thresh=1e9)),
    "long_erosion_3grid": dict(
        dx=0.003125, dy=0.003125, dt=1.25e-11, m_e_ratio=400.0, n_ions=48_000_000, n_e=16_000_000,
        cx=cx_table_power_law(), material=MO_POWER_LAW,
        params=dict(grids=[dict(V=1000.0, t=0.5, gap=0.5, r=0.8, cham=0.0),
                           dict(V=-250.0, t=0.5, gap=0.5, r=0.5, cham=0.0),
                           dict(V=0.0, t=0.5, gap=0.5, r=0.7, cham=0.0)],
                    pitch_mm=4.0, upstream_gap_mm=0.4, Te_up=5.0, n0_plasma=1e17, Ti=0.1, Tn=300.0,
                    n0=5e18, neutral_profile="uniform", sim_mode="Both", sputter_exponent=1.2, neut_rate=30,
                    Te=5.0, Thresh=1e9)),
}


def configure(sim, name, n_scale=1.0):
    """Apply a workload's spacing, species, material and cross-section to a simulator
    (either the GPU one or the oracle) before build_domain; returns the params dict."""
    w = WORKLOADS[name]
    sim.dx, sim.dy, sim.dt = w["dx"], w["dy"], w["dt"]
    sim.m_ion = M_XE
    sim.m_e = M_XE / w["m_e_ratio"]
    if w.get("material") is not None:
        sim.set_material(props=dict(w["material"]))
    if w["cx"] is not None:
        sim.user_cs = cx_store(w["cx"])
    return dict(w["params"])


def preload(isBound, dx, dy, Lx, Ly, n_ions, n_e, v_bohm, v_th_i, v_th_e, seed=0, x_max_ions=None):
    """Seeded initial particles over the non-electrode cells (float32 SoA).  Ions fill
    x in [1.5 dx, x_max_ions] (the plume boundary: ions beyond it leave at the first
    step), electrons the whole domain."""
    rs = np.random.RandomState(seed)
    ny, nx = isBound.shape

    def positions(n, x_hi):
        xs, ys, got = [], [], 0
        while got < n:
            m = max(2 * (n - got), 1024)
            x = rs.uniform(1.5 * dx, x_hi, m)
            y = rs.uniform(0.0, Ly, m)
            ok = ~isBound[np.clip(np.round(y / dy).astype(np.int64), 0, ny - 1),
                          np.clip(np.round(x / dx).astype(np.int64), 0, nx - 1)]
            xs.append(x[ok]); ys.append(y[ok]); got += int(ok.sum())
        return np.concatenate(xs)[:n].astype(np.float32), np.concatenate(ys)[:n].astype(np.float32)

    xi, yi = positions(n_ions, min(Lx - dx, x_max_ions) if x_max_ions else Lx - dx)
    ions = (xi, yi, (v_bohm + v_th_i * rs.randn(n_ions)).astype(np.float32),
            (v_th_i * rs.randn(n_ions)).astype(np.float32), (v_th_i * rs.randn(n_ions)).astype(np.float32))
    xe, ye = positions(n_e, Lx - dx)
    eles = (xe, ye, (v_th_e * rs.randn(n_e)).astype(np.float32), (v_th_e * rs.randn(n_e)).astype(np.float32),
            (v_th_e * rs.randn(n_e)).astype(np.float32))
    return ions, eles


def plume_boundary(sim, params):
    grids = params.get("grids", [])
    return sim.grid_x_ends[-1] + grids[-1]["gap"] if grids else None


def thermal_speeds(sim, params):
    Te = params.get("Te_up", 3.0)
    Ti = params.get("Ti", 0.1)
    v_bohm = float(np.sqrt(sim.q_ion * Te / sim.m_ion))
    v_th_i = float(np.sqrt(sim.q_ion * Ti / sim.m_ion))
    v_th_e = float(np.sqrt(sim.q * params.get("Te", 5.0) / sim.m_e))
    return v_bohm, v_th_i, v_th_e


SWEEP_SPACINGS = {"64x256": 0.025, "128x512": 0.0125, "256x1024": 0.00625}


def sweep_point(rng, index, grids=("64x256", "128x512", "256x1024"), n_range=(2e5, 4e6)):
    """One randomly drawn sweep point (a dict; ``make_sweep_sim`` builds it)."""
    grid = grids[int(rng.integers(len(grids)))]
    dx = SWEEP_SPACINGS[grid]
    lo, hi = np.log(n_range[0]), np.log(n_range[1])
    n = int(np.exp(rng.uniform(lo, hi)))
    return dict(index=int(index), grid=grid, dx=dx, dt=1e-10 * dx / 0.025, m_e_ratio=100.0,
                n_ions=int(0.75 * n), n_e=n - int(0.75 * n), seed=1000 + int(index),
                params=dict(grids=[dict(V=float(rng.uniform(600.0, 1800.0)), t=0.38, gap=1.0, r=0.95, cham=0.0),
                                   dict(V=float(rng.uniform(-300.0, -100.0)), t=1.0, gap=1.0, r=0.55, cham=0.0)],
                            pitch_mm=3.75, Te_up=5.0, n0_plasma=float(np.exp(rng.uniform(np.log(3e16), np.log(3e17)))),
                            Ti=0.1, Tn=300.0, n0=1e18, sim_mode="Erosion", neut_rate=30, Te=5.0, Thresh=1e9))


def served_point(rng, index, grids=("128x512", "256x1024"), n_range=(1e6, 6e6)):
    """One request of the served backstreaming-limit sweep: the 2-grid stack with accel
    voltage uniform in -300..-50 V, neutralizer electrons injected at 2 eV with a current
    density uniform in 0.1-1 A/m^2 (macro-electrons per step from the density, the
    neutralizer band Ly x 1 mm, dt and the macro-particle weight), a grid drawn from
    ``grids`` and a macro-particle count uniform in ``n_range``."""
    sp = sweep_point(rng, index, grids=grids, n_range=(1.0, 1.0))
    n = int(rng.uniform(n_range[0], n_range[1]))
    sp["n_ions"], sp["n_e"] = int(0.75 * n), n - int(0.75 * n)
    prm = sp["params"]
    prm["grids"][1]["V"] = float(rng.uniform(-300.0, -50.0))
    prm["Te"] = 2.0
    j = float(rng.uniform(0.1, 1.0))
    Ly_mm = 0.5 * prm["grids"][0]["r"] + 0.3 * prm["pitch_mm"]
    cell_vol = (sp["dx"] * 1e-3) ** 2 * 1e-3
    w = max(prm["n0_plasma"] * cell_vol / 80.0, 1e3)
    prm["neut_rate"] = max(1, int(round(j * (Ly_mm * 1e-3 * 1e-3) * sp["dt"] / (Q * w))))
    sp["neut_j"] = j
    return sp


def sweep_point_bytes(spec):
    """Device-memory estimate of a sweep point before it is built (for admission): two
    buffers of 25 B per ion and 24 B per electron with 25% headroom, plus about 800 B per
    grid node for fields, multigrid and sort scratch."""
    Lx_mm = 0.4 + sum(g["t"] + g["gap"] for g in spec["params"]["grids"]) + 3.0
    Ly_mm = 0.5 * spec["params"]["grids"][0]["r"] + 0.3 * spec["params"]["pitch_mm"]
    nodes = (Lx_mm / spec["dx"] + 1) * (Ly_mm / spec["dx"] + 1)
    return int(2 * 1.25 * (25 * spec["n_ions"] + 24 * spec["n_e"]) + 800 * nodes + (64 << 20))


def make_sweep_sim(spec, device=0, sort_every=20, solver=None):
    """Build a sweep point on the device: returns (simulator, params).  ``solver``: field
    solver settings other than the defaults (see DigitalTwinSimulator)."""
    from .physics_engine import DigitalTwinSimulator
    sim = DigitalTwinSimulator(device=device, seed=spec["seed"], sort_every=sort_every, solver=solver)
    sim.dx = sim.dy = spec["dx"]
    sim.dt = spec["dt"]
    sim.m_ion = M_XE
    sim.m_e = M_XE / spec["m_e_ratio"]
    params = dict(spec["params"])
    sim.build_domain(params)
    v_b, v_ti, v_te = thermal_speeds(sim, params)
    ions, eles = preload(sim.isBound, sim.dx, sim.dy, sim.Lx, sim.Ly, spec["n_ions"], spec["n_e"], v_b, 4 * v_ti,
                         v_te, seed=spec["seed"], x_max_ions=plume_boundary(sim, params))
    sim.set_particles("ions", *ions)
    sim.set_particles("electrons", *eles)
    return sim, params

