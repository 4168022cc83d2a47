"""Generate the golden fixtures by running the reference PY-BEMCS engine itself.

Run where the reference checkout is mounted, naming its root in ``PYBEMCS_REFERENCE``:

    PYBEMCS_REFERENCE=<checkout root> python tests/golden/make_golden.py

Every fixture is produced by calling the reference module (``Python/physics_engine.py``,
loaded unmodified with a taichi stand-in) on seeded synthetic inputs.  The outputs
are saved as compressed ``.npz`` files next to this script.  They pin the CPU oracle
(``oracle/pic_oracle.py``) and, through it, the GPU kernels.  The suite needs no
reference checkout at test time.

Fixture list
  domain_<case>.npz  build_domain geometry, the 30-iteration Picard potential and E field
  push.npz           push_particles_boris_cpu: one push and three sub-steps, random B
                     fields as well as the reference's zero B, edge-case particles
  deposit.npz        accumulate_rho_cpu: ions then electrons, crowded cells
  substeps.npz       compute_particle_substeps for ions and electrons
  segment.npz        _segment_hits_grid on a real electrode mask
  thermal.npz        one step with only the thermal block active (cooling + 10 sweeps)
  run_<case>.npz     short full-step runs with the reference's np.random stream recorded

With the argument ``large`` it writes the fixtures of the benchmarked configurations
instead (every 8th / 16th row of the potential, field and deposit, plus sums):
  domain_large_aperture_3grid.npz, domain_long_erosion_3grid.npz
  run_large_aperture_3grid.npz, run_large_aperture_3grid_fp64.npz
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from reference_loader import install_recorder, load_engine  # noqa: E402

# ---------------------------------------------------------------------------
# configurations (sizes small enough for the CPU suite)
# ---------------------------------------------------------------------------
C1_GRIDS = [dict(V=1000.0, t=0.38, gap=1.0, r=0.95, cham=0.0),
            dict(V=-200.0, t=1.0, gap=1.0, r=0.55, cham=0.0)]

DOMAIN_CASES = {
    # the 2-grid single-aperture configuration at 25 um, half-hole symmetry
    "c1_half": dict(dx=0.025, dy=0.025, dt=1e-10,
                    params=dict(grids=C1_GRIDS, pitch_mm=3.75, Te_up=5.0, n0_plasma=1e17, Ti=0.1)),
    # one full aperture, periodic in y, chamfered screen grid
    "one_hole": dict(dx=0.04, dy=0.04, dt=1e-10,
                     params=dict(grids=[dict(V=1200.0, t=0.5, gap=0.8, r=0.9, cham=20.0),
                                        dict(V=-250.0, t=0.6, gap=0.7, r=0.6, cham=0.0),
                                        dict(V=0.0, t=0.5, gap=1.0, r=0.8, cham=0.0)],
                                 geometry="one_hole", Te_up=5.0, n0_plasma=1e17, Ti=0.1)),
    # two apertures across one pitch, periodic in y
    "two_holes": dict(dx=0.05, dy=0.05, dt=1e-10,
                      params=dict(grids=[dict(V=1000.0, t=0.4, gap=1.0, r=0.8, cham=10.0),
                                         dict(V=-200.0, t=0.8, gap=1.0, r=0.5, cham=0.0)],
                                  geometry="two_holes", pitch_mm=2.5, Te_up=5.0, n0_plasma=1e17, Ti=0.1)),
    # Debye-gap mode (numpy float64 scalars enter the geometry)
    "bulk": dict(dx=0.03, dy=0.03, dt=1e-10,
                 params=dict(grids=C1_GRIDS, pitch_mm=3.75, Te_up=5.0, n0_plasma=1e17, Ti=0.1,
                             entire_bulk_plasma=True)),
}


def new_sim(pe, dx, dy, dt):
    sim = pe.DigitalTwinSimulator()
    sim.dx, sim.dy, sim.dt = dx, dy, dt
    return sim


def domain_arrays(sim):
    return dict(nx=sim.nx, ny=sim.ny, dx=sim.dx, dy=sim.dy, Lx=sim.Lx, Ly=sim.Ly,
                macro_weight=sim.macro_weight, upstream_gap_mm=sim.upstream_gap_mm,
                isBound=sim.isBound.copy(), V_fixed=sim.V_fixed.copy(),
                mask_grids=np.array(sim.mask_grids), grid_x_starts=np.array(sim.grid_x_starts),
                grid_x_ends=np.array(sim.grid_x_ends), hole_centers=np.array(sim.hole_centers),
                periodic_y=bool(sim.periodic_y), V=sim.V.copy(), Ex=sim.Ex.copy(), Ey=sim.Ey.copy(),
                dx_is_np64=isinstance(sim.dx, np.floating))


def make_domains(pe):
    for name, case in DOMAIN_CASES.items():
        sim = new_sim(pe, case["dx"], case["dy"], case["dt"])
        sim.build_domain(case["params"])
        d = domain_arrays(sim)
        # a rebuild with a thermal bow on every grid (preserve_state path)
        sim.grid_deflections = [0.012 * (i + 1) for i in range(len(case["params"]["grids"]))]
        sim.build_domain(case["params"], preserve_state=True)
        d["bow_isBound"] = sim.isBound.copy()
        d["bow_V"] = sim.V.copy()
        d["bow_deflections"] = np.array(sim.grid_deflections)
        np.savez_compressed(os.path.join(HERE, f"domain_{name}.npz"), params=json.dumps(case["params"]),
                            case=json.dumps({k: v for k, v in case.items() if k != "params"}), **d)
    # numerics-check errors (build_domain raises ValueError)
    errs = {}
    for label, (dx, dt) in {"debye": (0.2, 1e-10), "cfl": (0.025, 5e-8)}.items():
        sim = new_sim(pe, dx, dx, dt)
        try:
            sim.build_domain(DOMAIN_CASES["c1_half"]["params"])
            errs[label] = ""
        except ValueError as exc:
            errs[label] = str(exc)
    with open(os.path.join(HERE, "domain_errors.json"), "w") as f:
        json.dump(errs, f, indent=1)


def load_domain_fields():
    d = np.load(os.path.join(HERE, "domain_c1_half.npz"))
    return d


def open_region_particles(rs, d, n, v0, vth):
    """Uniform positions over non-electrode cells of the domain; Gaussian velocities."""
    nx, ny, dx, dy = int(d["nx"]), int(d["ny"]), float(d["dx"]), float(d["dy"])
    Lx, Ly = float(d["Lx"]), float(d["Ly"])
    xs, ys = [], []
    while sum(len(a) for a in xs) < n:
        x = rs.uniform(1.5 * dx, Lx - dx, 4 * n)
        y = rs.uniform(0.0, Ly, 4 * n)
        ok = ~d["isBound"][np.clip(np.round(y / dy).astype(int), 0, ny - 1),
                           np.clip(np.round(x / dx).astype(int), 0, nx - 1)]
        xs.append(x[ok]); ys.append(y[ok])
    x = np.concatenate(xs)[:n].astype(np.float32)
    y = np.concatenate(ys)[:n].astype(np.float32)
    vx = (v0 + vth * rs.randn(n)).astype(np.float32)
    vy = (vth * rs.randn(n)).astype(np.float32)
    vz = (vth * rs.randn(n)).astype(np.float32)
    return x, y, vx, vy, vz


def edge_particles(d):
    """Particles on nodes, on cell mid-points, outside the box, NaN and inf."""
    dx, dy, Lx, Ly = float(d["dx"]), float(d["dy"]), float(d["Lx"]), float(d["Ly"])
    xs = [0.0, dx, 2.5 * dx, 7.5 * dx, Lx, Lx + 0.3, -0.2, 0.5 * dx, 3.0, np.nan, 1.0, np.inf, -np.inf, 1e12]
    ys = [0.0, dy, 1.5 * dy, 0.5 * dy, Ly, 0.2, -0.1, Ly + 0.4, 0.8, 0.3, np.nan, 0.1, 0.2, 0.5]
    n = len(xs)
    v = np.linspace(-3e4, 5e4, n)
    return (np.array(xs, np.float32), np.array(ys, np.float32), v.astype(np.float32),
            (-0.5 * v).astype(np.float32), (0.1 * v).astype(np.float32))


def make_push(pe):
    d = load_domain_fields()
    rs = np.random.RandomState(11)
    nx, ny = int(d["nx"]), int(d["ny"])
    out = {}
    x, y, vx, vy, vz = open_region_particles(rs, d, 6000, 3e4, 4e3)
    ex = edge_particles(d)
    x, y, vx, vy, vz = [np.concatenate([a, b]) for a, b in zip((x, y, vx, vy, vz), ex)]
    # electrons get much larger speeds
    ve = rs.randn(3, 2000).astype(np.float32) * 3e5
    xe, ye, _, _, _ = open_region_particles(rs, d, 2000, 0, 0)
    Bz0 = np.zeros((ny, nx), np.float32)
    Bxr = (rs.randn(ny, nx) * 0.02).astype(np.float32)
    Byr = (rs.randn(ny, nx) * 0.02).astype(np.float32)
    Bzr = (0.3 + rs.randn(ny, nx) * 0.05).astype(np.float32)
    q = 1.602e-19
    m_ion = 131.293 * 1.6605e-27
    cases = [("ion", x, y, vx, vy, vz, q / m_ion, 1e-10),
             ("ele", xe, ye, ve[0], ve[1], ve[2], -q / (m_ion / 100.0), 1e-10)]
    for tag, x0, y0, vx0, vy0, vz0, qm, dt in cases:
        out[f"{tag}_in"] = np.stack([x0, y0, vx0, vy0, vz0])
        out[f"{tag}_qm"] = qm
        out[f"{tag}_dt"] = dt
        for btag, B in (("B0", (Bz0, Bz0, Bz0)), ("Br", (Bxr, Byr, Bzr))):
            for nsub in (1, 3):
                a = [np.array(v, copy=True) for v in (x0, y0, vx0, vy0, vz0)]
                with np.errstate(all="ignore"):
                    for _ in range(nsub):
                        pe.push_particles_boris_cpu(*a, d["Ex"], d["Ey"], *B, len(x0), float(d["dx"]),
                                                    float(d["dy"]), nx, ny, dt / nsub, qm)
                out[f"{tag}_{btag}_sub{nsub}"] = np.stack(a)
    out["Bx"], out["By"], out["Bz"] = Bxr, Byr, Bzr
    np.savez_compressed(os.path.join(HERE, "push.npz"), **out)


def make_deposit(pe):
    d = load_domain_fields()
    rs = np.random.RandomState(5)
    nx, ny, dx, dy = int(d["nx"]), int(d["ny"]), float(d["dx"]), float(d["dy"])
    xi, yi, _, _, _ = open_region_particles(rs, d, 30000, 0, 0)
    # a crowded cell: 20000 ions on one node, 7000 electrons on another
    xi = np.concatenate([xi, np.full(20000, 40 * dx, np.float32)])
    yi = np.concatenate([yi, np.full(20000, 10 * dy, np.float32)])
    xe, ye, _, _, _ = open_region_particles(rs, d, 9000, 0, 0)
    xe = np.concatenate([xe, np.full(7000, 40 * dx, np.float32), np.full(3000, 90 * dx, np.float32)])
    ye = np.concatenate([ye, np.full(7000, 10 * dy, np.float32), np.full(3000, 30 * dy, np.float32)])
    xi = np.concatenate([xi, edge_particles(d)[0][:9]])
    yi = np.concatenate([yi, edge_particles(d)[1][:9]])
    sim = new_sim(pe, 0.025, 0.025, 1e-10)
    sim.dx, sim.dy = dx, dy
    w = 1000.0
    cell_vol = (dx * 1e-3) * (dy * 1e-3) * 1e-3
    cd = sim.q * w / cell_vol
    rho = np.zeros((ny, nx), np.float32)
    with np.errstate(all="ignore"):
        pe.accumulate_rho_cpu(xi, yi, rho, len(xi), dx, dy, nx, ny, cd)
        rho_ions = rho.copy()
        pe.accumulate_rho_cpu(xe, ye, rho, len(xe), dx, dy, nx, ny, -cd)
    np.savez_compressed(os.path.join(HERE, "deposit.npz"), xi=xi, yi=yi, xe=xe, ye=ye, cd=cd,
                        rho_ions=rho_ions, rho=rho)


def make_substeps(pe):
    d = load_domain_fields()
    rs = np.random.RandomState(7)
    sim = new_sim(pe, 0.025, 0.025, 1e-10)
    sim.build_domain(DOMAIN_CASES["c1_half"]["params"])
    out = {}
    for tag, v0, vth, qm in (("ion", 3e4, 5e3, sim.q_ion / sim.m_ion), ("ele", 0.0, 4e4, -sim.q / sim.m_e)):
        x, y, vx, vy, vz = open_region_particles(rs, d, 5000, v0, vth)
        n_sub, ds_max, ds_lim = sim.compute_particle_substeps(x, y, vx, vy, vz, qm, sim.dt)
        out[f"{tag}_in"] = np.stack([x, y, vx, vy, vz])
        out[f"{tag}_res"] = np.array([n_sub, ds_max, ds_lim])
        out[f"{tag}_qm"] = qm
    np.savez_compressed(os.path.join(HERE, "substeps.npz"), **out)


def make_segment(pe):
    d = load_domain_fields()
    rs = np.random.RandomState(9)
    sim = new_sim(pe, 0.025, 0.025, 1e-10)
    sim.build_domain(DOMAIN_CASES["c1_half"]["params"])
    x0, y0, _, _, _ = open_region_particles(rs, d, 8000, 0, 0)
    # segments of up to ~3 cells in every direction, some ending inside electrodes
    x1 = (x0 + rs.uniform(-0.08, 0.08, x0.size)).astype(np.float32)
    y1 = (y0 + rs.uniform(-0.08, 0.08, y0.size)).astype(np.float32)
    hit, hix, hiy = sim._segment_hits_grid(x0, y0, x1, y1, samples=8)
    np.savez_compressed(os.path.join(HERE, "segment.npz"), x0=x0, y0=y0, x1=x1, y1=y1,
                        hit=hit, hix=hix, hiy=hiy)


def make_thermal(pe):
    sim = new_sim(pe, 0.025, 0.025, 1e-10)
    params = dict(DOMAIN_CASES["c1_half"]["params"], sim_mode="Thermal", neut_rate=0)
    sim.build_domain(params)
    rs = np.random.RandomState(3)
    T0 = sim.Tmap.copy()
    T0[sim.isBound] = (300.0 + rs.uniform(0, 300.0, int(sim.isBound.sum()))).astype(np.float32)
    sim.Tmap[:] = T0
    sim.injection_enabled = False
    res = sim.step(params)
    np.savez_compressed(os.path.join(HERE, "thermal.npz"), T0=T0, T1=sim.Tmap.copy(),
                        T_grids=np.array(res[3], dtype=np.float64),
                        deflections=np.array(sim.grid_deflections, dtype=np.float64),
                        remeshed=bool(res[0]))


RUN_CASES = {
    # 2-grid half-hole, everything on, erosion threshold low enough to break cells
    "c1_both": dict(dx=0.05, dy=0.05, dt=1e-10, steps=8, n_ions=3000, n_e=600, seed=1,
                    params=dict(grids=C1_GRIDS, pitch_mm=3.75, Te_up=5.0, n0_plasma=1e17, Ti=0.1,
                                Tn=300.0, n0=3e21, sim_mode="Both", neut_rate=30, Thresh=2e3)),
    # one periodic aperture with RF co-extraction and a tabulated CX cross-section
    "one_hole_rf": dict(dx=0.05, dy=0.05, dt=1e-10, steps=6, n_ions=2000, n_e=400, seed=2,
                        cx_table=[[1.0, 5e-19], [10.0, 5e-19], [100.0, 5e-19], [1000.0, 5e-19]],
                        params=dict(grids=DOMAIN_CASES["one_hole"]["params"]["grids"], geometry="one_hole",
                                    Te_up=5.0, n0_plasma=1e17, Ti=0.1, Tn=300.0, n0=5e21,
                                    sim_mode="Erosion", neut_rate=20, rf_enable=True, rf_grid_idx=1,
                                    rf_amp=50.0, Thresh=1e9)),
    # two apertures, thermal only, no neutralizer
    "two_holes_thermal": dict(dx=0.05, dy=0.05, dt=1e-10, steps=5, n_ions=1500, n_e=0, seed=3,
                              params=dict(grids=DOMAIN_CASES["two_holes"]["params"]["grids"],
                                          geometry="two_holes", pitch_mm=2.5, Te_up=5.0, n0_plasma=1e17,
                                          Ti=0.1, Tn=300.0, n0=1e21, sim_mode="Thermal", neut_rate=0)),
}


def cx_spline(table):
    from scipy.interpolate import UnivariateSpline
    t = np.array(table, dtype=np.float64)
    e, cs = t[:, 0], t[:, 1]
    return {"CX": {"energy": e, "cs": cs, "type": "CX",
                   "spline": UnivariateSpline(np.log10(e), np.log10(cs), s=0.0, k=3)}}


def snapshot(sim):
    """Copies of the state after a step (np.array copies: in FP64 mode the engine's
    arrays already are float64 and a plain asarray would alias them)."""
    n, ne = sim.num_p, sim.num_e
    fp = sim.p_x.dtype
    return dict(p=np.array(np.stack([sim.p_x[:n], sim.p_y[:n], sim.p_vx[:n], sim.p_vy[:n], sim.p_vz[:n]]), dtype=fp),
                p_cex=np.array(sim.p_isCEX[:n]),
                e=np.array(np.stack([sim.e_x[:ne], sim.e_y[:ne], sim.e_vx[:ne], sim.e_vy[:ne], sim.e_vz[:ne]]), dtype=fp),
                V=np.array(sim.V, dtype=np.float64), Ex=np.array(sim.Ex, dtype=fp), Ey=np.array(sim.Ey, dtype=fp),
                rho=np.array(sim.rho, dtype=fp), Tmap=np.array(sim.Tmap, dtype=fp),
                damage=np.array(sim.damage_map, dtype=np.float64), isBound=np.array(sim.isBound))


def make_runs(pe_factory, tag_suffix=""):
    for name, case in RUN_CASES.items():
        pe = pe_factory()
        fp = pe._NP_FP
        sim = new_sim(pe, case["dx"], case["dy"], case["dt"])
        if "cx_table" in case:
            sim.user_cs = cx_spline(case["cx_table"])
        params = case["params"]
        sim.build_domain(params)
        d = domain_arrays(sim)
        rs = np.random.RandomState(100 + case["seed"])
        v_b = float(np.sqrt(sim.q_ion * params["Te_up"] / sim.m_ion))
        xi, yi, vxi, vyi, vzi = open_region_particles(rs, d, case["n_ions"], 2.0e4, 3.0e3)
        sim._add_ions(xi, yi, vxi, vyi, vzi, rs.rand(case["n_ions"]) < 0.1)
        if case["n_e"]:
            xe, ye, vxe, vye, vze = open_region_particles(rs, d, case["n_e"], 0.0, 2.0e4)
            sim._add_electrons(xe, ye, vxe, vye, vze)
        init = snapshot(sim)
        rec = install_recorder(pe, 1000 + case["seed"])
        outs, snaps = [], []
        import contextlib, io
        for _ in range(case["steps"]):
            with contextlib.redirect_stdout(io.StringIO()):
                r = sim.step(params)
            outs.append([float(r[0]), float(r[1]), float(r[2]), float(r[4])] + [float(t) for t in r[3]])
            snaps.append(snapshot(sim))
        log_names = json.dumps([m for m, _ in rec.log])
        log_vals = {f"draw_{i}": v for i, (_, v) in enumerate(rec.log)}
        flat = {}
        for k, v in init.items():
            flat[f"init_{k}"] = v
        for s, sn in enumerate(snaps):
            for k, v in sn.items():
                flat[f"s{s}_{k}"] = v
        np.savez_compressed(
            os.path.join(HERE, f"run_{name}{tag_suffix}.npz"),
            case=json.dumps({k: v for k, v in case.items() if k != "params"}), params=json.dumps(params),
            outs=np.array(outs), log_names=log_names, v_bohm=v_b, fp64=(fp is np.float64), **log_vals, **flat)


def _rows(a, step):
    """Every ``step``-th row and the last one: the fixtures of the large grids keep these
    (full potentials of 263k and 1.05M nodes would be megabytes each)."""
    idx = np.unique(np.concatenate([np.arange(0, a.shape[0], step), [a.shape[0] - 1]]))
    return idx, np.array(a[idx])


def _large_sim(pe, case):
    from tests.helpers import M_XE
    sim = new_sim(pe, case["dx"], case["dy"], case["dt"])
    sim.m_ion = M_XE
    sim.m_e = M_XE / case["m_e_ratio"]
    return sim


def make_large(pe_factory):
    """The benchmarked configurations: their domains and Picard potentials, and a short
    run of the 257 x 1025 case in FP32 (snapshots after each step) and FP64 (the last)."""
    from tests.helpers import CX_POWER_LAW, LARGE_CASES, large_case_particles
    for name, case in LARGE_CASES.items():
        pe = pe_factory(False)
        sim = _large_sim(pe, case)
        sim.build_domain(case["params"])
        rows, V = _rows(sim.V, case["row_step"])
        _, Ex = _rows(sim.Ex, case["row_step"])
        _, Ey = _rows(sim.Ey, case["row_step"])
        np.savez_compressed(
            os.path.join(HERE, f"domain_{name}.npz"), params=json.dumps(case["params"]),
            case=json.dumps({k: v for k, v in case.items() if k != "params"}), nx=sim.nx, ny=sim.ny, dx=sim.dx,
            dy=sim.dy, Lx=sim.Lx, Ly=sim.Ly, macro_weight=sim.macro_weight, isBound_bits=np.packbits(sim.isBound),
            V_fixed_sum=float(np.sum(sim.V_fixed)), rows=rows, V_rows=V, Ex_rows=Ex, Ey_rows=Ey,
            V_sum=float(np.sum(sim.V)), V_absmax=float(np.abs(sim.V).max()))
        if "steps" not in case:
            continue
        import contextlib, io
        for fp64 in (False, True):
            pe = pe_factory(fp64)
            fp = pe._NP_FP
            sim = _large_sim(pe, case)
            sim.user_cs = cx_spline(CX_POWER_LAW)
            params = case["params"]
            sim.build_domain(params)
            ions, cex, eles = large_case_particles(sim.isBound, sim.dx, sim.dy, sim.Lx, sim.Ly, case["n_ions"],
                                                   case["n_e"], case["seed"])
            sim._add_ions(*ions.astype(fp), cex)
            sim._add_electrons(*eles.astype(fp))
            rec = install_recorder(pe, 2000 + case["seed"])
            out = {}
            outs = []
            for s in range(case["steps"]):
                with contextlib.redirect_stdout(io.StringIO()):
                    r = sim.step(params)
                outs.append([float(r[0]), float(r[1]), float(r[2]), float(r[4])] + [float(t) for t in r[3]])
                if fp64 and s < case["steps"] - 1:
                    continue
                n, ne = sim.num_p, sim.num_e
                out[f"s{s}_p"] = np.array(np.stack([sim.p_x[:n], sim.p_y[:n], sim.p_vx[:n], sim.p_vy[:n],
                                                    sim.p_vz[:n]]), dtype=fp)
                out[f"s{s}_p_cex"] = np.array(sim.p_isCEX[:n])
                out[f"s{s}_e"] = np.array(np.stack([sim.e_x[:ne], sim.e_y[:ne], sim.e_vx[:ne], sim.e_vy[:ne],
                                                    sim.e_vz[:ne]]), dtype=fp)
                for k, attr in (("V", "V"), ("rho", "rho"), ("damage", "damage_map")):
                    a = np.asarray(getattr(sim, attr))
                    out[f"s{s}_{k}_rows"] = _rows(a, case["row_step"])[1]
                    out[f"s{s}_{k}_sum"] = float(np.sum(a.astype(np.float64)))
                out[f"s{s}_isBound_bits"] = np.packbits(sim.isBound)
            log_names = json.dumps([m for m, _ in rec.log])
            log_vals = {f"draw_{i}": v for i, (_, v) in enumerate(rec.log)}
            np.savez_compressed(
                os.path.join(HERE, f"run_{name}{'_fp64' if fp64 else ''}.npz"),
                case=json.dumps({k: v for k, v in case.items() if k != "params"}), params=json.dumps(params),
                outs=np.array(outs), log_names=log_names, fp64=fp64, **log_vals, **out)


def main():
    if sys.argv[1:] == ["large"]:
        make_large(lambda fp64: load_engine(fp64=fp64, name="_ref_large64" if fp64 else "_ref_large32"))
        print("large fixtures written to", HERE)
        return
    pe = load_engine()
    make_domains(pe)
    make_push(pe)
    make_deposit(pe)
    make_substeps(pe)
    make_segment(pe)
    make_thermal(pe)
    make_runs(lambda: load_engine(name="_ref_run32"))
    make_runs(lambda: load_engine(fp64=True, name="_ref_run64"), tag_suffix="_fp64")
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main()
