"""Host-side domain geometry for the PIC-MCC path (runs once per build / remesh).

Restates the geometry part of ``DigitalTwinSimulator.build_domain``
(``Python/physics_engine.py:629-847``): numerics checks, domain extent from the grid
stack, node counts, electrode masks with chamfer and thermal bow, Dirichlet values,
the plasma boundary column and the macro-particle weight.  The arithmetic follows the
reference operation by operation (Python floats, NumPy float64 meshes) so that node
counts, spacings and masks come out identical; ``tests/test_oracle_golden.py`` pins them
against the reference's own outputs.

The function mutates the simulator object it is given, exactly as the reference
method mutates ``self``; the caller then assembles the field operator and runs the
initial Picard solve.
"""
import numpy as np


def debye_length_m(eps0, q, Te_up, n0):
    """``physics_engine.py:643``: sqrt(eps0 Te / (q n0 0.61))."""
    return np.sqrt(eps0 * Te_up / (q * n0 * 0.61))


def compute_debye_upstream_gap(n0, Te_up):
    """Recommended upstream gap [mm] (``physics_engine.py:270-302``)."""
    eps0 = 8.854e-12
    q = 1.6e-19
    debye_mm = np.sqrt(eps0 * Te_up / (q * n0 * 0.61)) * 1e3
    if n0 <= 1e17:
        n_debye = 80
    elif n0 <= 4e17:
        n_debye = 40
    else:
        n_debye = 30
    return n_debye * debye_mm


def _pitch(params):
    dc = params.get("discharge_chamber")
    return params.get("pitch_mm", dc.get("pitch_mm", 0.0) if isinstance(dc, dict) else 0.0)


def build_domain_geometry(sim, params, preserve_state=False, fp=np.float32):
    """Geometry and state reset of ``build_domain`` (``physics_engine.py:629-842``).

    ``sim`` must provide ``dx, dy, dt, eps0, q, q_ion, m_ion, m_e, Lx, Ly, Tmap`` and a
    ``reset_arrays()`` method; the attributes listed in the module docstring are set.
    Raises ``ValueError`` with the reference's messages when the grid does not resolve
    the Debye length or the time step is out of range (``:672-701``).
    """
    grids = params.get("grids", [])
    total_grid_thickness = sum(g["t"] + g["gap"] for g in grids) if grids else 0.0
    pitch = _pitch(params)
    Te_up = params.get("Te_up", 3.0)
    n0_n = params.get("n0_plasma", 1e17)
    entire_bulk_plasma = params.get("entire_bulk_plasma", False)

    debye_length = debye_length_m(sim.eps0, sim.q, Te_up, n0_n)
    debye_mm = debye_length * 1e3
    if entire_bulk_plasma:
        n_debye = 80 if n0_n <= 1e17 else (40 if n0_n <= 4e17 else 30)
        sim.recommended_upstream_gap_mm = n_debye * debye_mm
    else:
        screen_r = grids[0]["r"] if grids else 0.80
        sim.recommended_upstream_gap_mm = 0.75 * screen_r

    user_gap = float(params.get("upstream_gap_mm", 0.0))
    upstream_gap = user_gap if user_gap > 0.0 else sim.recommended_upstream_gap_mm
    upstream_gap = max(upstream_gap, sim.dx * 2)
    sim.upstream_gap_mm = upstream_gap

    if grids:
        sim.Lx = upstream_gap + total_grid_thickness + 3.0
    else:
        sim.Lx = params.get("Lx", sim.Lx)

    if sim.dx * 1e-3 > debye_length or sim.dy * 1e-3 > debye_length:
        raise ValueError(
            f"Grid spacing too large for Debye resolution: "
            f"dx={sim.dx:.6f} mm, dy={sim.dy:.6f} mm, "
            f"lambda_D={debye_length*1e3:.6f} mm. "
            f"Choose dx, dy <= lambda_D."
        )
    plasma_freq = np.sqrt(n0_n * sim.q ** 2 / (sim.m_ion * sim.eps0))
    dt_min = 2 * 3.14159 / plasma_freq
    if dt_min < sim.dt:
        raise ValueError(
            f"Too low time step: "
            f"dt used ={sim.dt:.8e} s, dt minimum ={dt_min:.6e} s, "
        )
    Ti = params.get("Ti", 0.1)
    v_bohm = np.sqrt(sim.q_ion * Te_up / sim.m_ion)
    v_spread = np.sqrt(sim.q_ion * Ti / sim.m_ion)
    vmax = v_bohm + 4 * v_spread
    if sim.dx * 1e-3 / sim.dt < vmax or sim.dy * 1e-3 / sim.dt < vmax:
        raise ValueError(
            f"Grid spacing and time step too large for velocity resolution: "
            f"dx/dt={sim.dx*1e-3/sim.dt:.2e} m/s, dy/dt={sim.dy*1e-3/sim.dt:.2e} m/s, "
            f"vmax={vmax:.2e} m/s. "
            f"Choose dx, dy and dt such that dx/dt >= vmax and dy/dt >= vmax."
        )

    geometry = params.get("geometry", "half_hole")
    sim.geometry = geometry
    sim.periodic_y = geometry in ("one_hole", "two_holes")
    if grids:
        screen_r = grids[0]["r"]
        if geometry == "two_holes":
            sim.Ly = screen_r + 2.0 * screen_r + pitch
        elif geometry == "one_hole":
            sim.Ly = 3.0 * screen_r
        else:
            sim.Ly = 0.5 * screen_r + 0.30 * pitch
    else:
        sim.Ly = params.get("Ly", sim.Ly)

    sim.nx = int(sim.Lx / sim.dx) + 1
    sim.ny = int(sim.Ly / sim.dy) + 1
    sim.dx = sim.Lx / (sim.nx - 1)
    sim.dy = sim.Ly / (sim.ny - 1)
    sim.xpts = np.linspace(0, sim.Lx, sim.nx)
    sim.ypts = np.linspace(0, sim.Ly, sim.ny)
    sim.X, sim.Y = np.meshgrid(sim.xpts, sim.ypts)

    if not preserve_state:
        sim.Tmap = np.full((sim.ny, sim.nx), 300.0, dtype=fp)
        sim.T_map = sim.Tmap
        sim.T_map_new = np.full((sim.ny, sim.nx), 300.0, dtype=fp)
        sim.Tmapnew = sim.T_map_new
        sim.reset_arrays()
        sim.iteration = 0
        sim.injected_ions = 0.0
        sim.injected_ions_step = 0.0
        sim.transmitted_ions = 0.0
        sim.transmitted_ions_step = 0.0
        sim.entered_optics = 0.0
        sim.entered_optics_step = 0.0
        sim._domain_built = True

    inj_time = params.get("inj_time", 0.0)
    sim.injection_stop_time = inj_time if inj_time > 0.0 else None
    sim.injection_enabled = True

    n0 = params.get("n0_plasma", 1e17)
    target_ppc = 80.0
    cell_vol = (sim.dx * 1e-3) * (sim.dy * 1e-3) * 1e-3
    sim.macro_weight = max(n0 * cell_vol / target_ppc, 1e3)
    sim.mask_grids = []
    sim.T_grids = []
    sim.isBound = np.zeros((sim.ny, sim.nx), dtype=bool)
    sim.V_fixed = np.zeros((sim.ny, sim.nx), dtype=np.float64)

    if not hasattr(sim, "grid_deflections") or len(sim.grid_deflections) != len(grids):
        sim.grid_deflections = [0.0] * len(grids)

    current_x = sim.upstream_gap_mm
    if grids:
        screen_r = grids[0]["r"]
        if geometry == "two_holes":
            y_c1 = 1.5 * screen_r
            hole_centers = [y_c1, y_c1 + pitch]
        elif geometry == "one_hole":
            hole_centers = [1.5 * screen_r]
        else:
            hole_centers = [0.0]
    else:
        hole_centers = []
    sim.hole_centers = hole_centers

    X, Y = sim.X, sim.Y
    sim.grid_x_starts = []
    sim.grid_x_ends = []
    for i, grid in enumerate(grids):
        gstart = current_x
        gend = gstart + grid["t"]
        sim.grid_x_starts.append(gstart)
        sim.grid_x_ends.append(gend)
        delta = sim.grid_deflections[i]
        dxbow = 0.0
        if abs(delta) > 1e-6:
            if geometry == "two_holes":
                y_web = 1.5 * screen_r + 0.5 * pitch
                eta = np.clip(1.0 - np.abs(Y - y_web) / max(pitch * 0.5, 1e-6), 0.0, 1.0)
                dxbow = delta * eta ** 2
            elif geometry == "one_hole":
                y_mid = 1.5 * screen_r
                eta = np.clip(1.0 - np.abs(Y - y_mid) / max(sim.Ly * 0.5, 1e-6), 0.0, 1.0)
                dxbow = delta * eta ** 2
            else:
                Lcant = sim.Ly - grid["r"]
                if Lcant > 0:
                    eta = np.clip((sim.Ly - Y) / Lcant, 0.0, 1.0)
                    dxbow = delta * eta ** 2
        ingrid_x = (X >= gstart + dxbow) & (X <= gend + dxbow)
        mask = ingrid_x.copy()
        for yc in hole_centers:
            local_r = grid["r"] - np.maximum(0.0, X - gstart - dxbow) * np.tan(np.radians(grid["cham"]))
            local_r = np.maximum(local_r, 0.0)
            hole = ingrid_x & (np.abs(Y - yc) <= local_r)
            mask &= ~hole
        sim.isBound[mask] = True
        sim.V_fixed[mask] = grid["V"]
        sim.mask_grids.append(mask)
        sim.T_grids.append(float(np.mean(sim.Tmap[mask])) if np.any(mask) else 300.0)
        current_x = gend + grid["gap"]

    sim.Vdc = np.copy(sim.V_fixed)
    v_plasma_bound = (grids[0]["V"] + params.get("V_plasma_offset", 20.0)
                      if grids else 1000.0 + params.get("V_plasma_offset", 20.0))
    sim.V_fixed[:, 0] = v_plasma_bound
    sim.isBound[:, 0] = True
    if not preserve_state:
        sim.Tmap[sim.isBound] = 300.0


def node_classes(isBound, periodic_y):
    """Row classes of the reference's field operator (``physics_engine.py:525-552``).

    Returns ``(is_bound, is_right, is_top, is_bottom, is_interior, is_per_bot,
    is_per_top)`` as flat bool arrays over the ny*nx nodes (row-major, x fastest).
    """
    ny, nx = isBound.shape
    N = nx * ny
    idx = np.arange(N)
    y_ = idx // nx
    x_ = idx % nx
    is_bound = isBound.flatten()
    is_right = (x_ == nx - 1) & ~is_bound
    if periodic_y:
        is_top = np.zeros(N, dtype=bool)
        is_bottom = np.zeros(N, dtype=bool)
        is_per_bot = (y_ == 0) & ~is_bound & ~is_right
        is_per_top = (y_ == ny - 1) & ~is_bound & ~is_right
        is_interior = ~is_bound & ~is_right & ~is_per_bot & ~is_per_top
    else:
        is_top = (y_ == ny - 1) & ~is_bound & ~is_right
        is_bottom = (y_ == 0) & ~is_bound & ~is_right & ~is_top
        is_interior = ~is_bound & ~is_right & ~is_top & ~is_bottom
        is_per_bot = np.zeros(N, dtype=bool)
        is_per_top = np.zeros(N, dtype=bool)
    return is_bound, is_right, is_top, is_bottom, is_interior, is_per_bot, is_per_top
