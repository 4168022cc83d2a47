"""CPU oracle for the PY-BEMCS PIC-MCC timestep: a NumPy restatement of the reference.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import this module,
and only as the checker or the timed CPU baseline.  The product path
(``thruster_cx_code_b200``) never imports it and fails loudly when its CUDA library is
missing.

Each function restates the algorithm of ``Python/physics_engine.py`` at the cited lines,
with the same NumPy dtype behaviour: float32 particle/field arrays, Python-float
scalars that NumPy 2 treats as weak (so ``x / dx`` is a float32 division), the float64
promotions that arise from float32-minus-int32 (the bilinear weights and velocity
update of the push are float64), float64 potential and damage map.  The random draws
that the reference takes from the global ``np.random`` are requested from a ``draws``
object instead (see ``ReplayDraws`` and ``PhiloxDraws``); particles carry ids
(``p_id``, ``e_id``) so keyed draws can follow a particle across compactions.

Pinning: ``tests/test_oracle_golden.py`` checks every function and whole steps against
fixtures produced by running the reference module itself (``tests/golden/make_golden.py``),
bit-exact, with the reference's own MT19937 draws replayed.
"""
import numpy as np
import scipy.sparse as sp
from scipy.sparse.linalg import factorized

from . import philox as _px

# ---------------------------------------------------------------------------
# module-level kernels (reference signatures)
# ---------------------------------------------------------------------------


def accumulate_rho(x, y, rho, num_p, dx, dy, nx, ny, charge_density):
    """NGP deposit, ``physics_engine.py:178-185``: cell = clip(rint(x/dx), 1, n-2), then
    sequential ``rho[iy, ix] += charge_density`` in particle order (``np.add.at``)."""
    n = int(num_p)
    if n == 0:
        return
    ix = np.clip(np.round(x[:n] / dx).astype(np.int32), 1, nx - 2)
    iy = np.clip(np.round(y[:n] / dy).astype(np.int32), 1, ny - 2)
    np.add.at(rho, (iy, ix), charge_density)


def push_particles_boris(x, y, vx, vy, vz, Ex, Ey, Bx, By, Bz,
                         num_p, dx, dy, nx, ny, dt, q_m):
    """Bilinear gather + 2D3V Boris + drift in mm, ``physics_engine.py:188-254``.

    dtype trace (NumPy 2): ``x/dx`` float32; ``fx = idx - ix0`` float32 - int32 ->
    float64; weights, gathered fields and the whole velocity update float64; the new
    velocity is rounded to float32 on store; the drift ``x += vx*dt*1000`` is float32.
    """
    n = int(num_p)
    if n == 0:
        return
    nx_m1 = nx - 1
    ny_m1 = ny - 1
    idx_x = x[:n] / dx
    idx_y = y[:n] / dy
    ix0 = np.clip(np.floor(idx_x).astype(np.int32), 0, nx_m1 - 1)
    iy0 = np.clip(np.floor(idx_y).astype(np.int32), 0, ny_m1 - 1)
    fx = idx_x - ix0
    fy = idx_y - iy0
    ix1 = np.minimum(ix0 + 1, nx_m1)
    iy1 = np.minimum(iy0 + 1, ny_m1)
    w00 = (1.0 - fx) * (1.0 - fy)
    w10 = fx * (1.0 - fy)
    w01 = (1.0 - fx) * fy
    w11 = fx * fy

    def gather(F):
        return F[iy0, ix0] * w00 + F[iy0, ix1] * w10 + F[iy1, ix0] * w01 + F[iy1, ix1] * w11

    ex = gather(Ex)
    ey = gather(Ey)
    bx = gather(Bx)
    by = gather(By)
    bz = gather(Bz)
    h = 0.5 * q_m * dt
    vmx = vx[:n] + h * ex
    vmy = vy[:n] + h * ey
    vmz = vz[:n]
    tx = h * bx
    ty = h * by
    tz = h * bz
    t2 = tx * tx + ty * ty + tz * tz
    sx = 2.0 * tx / (1.0 + t2)
    sy = 2.0 * ty / (1.0 + t2)
    sz = 2.0 * tz / (1.0 + t2)
    vpx = vmx + (vmy * tz - vmz * ty)
    vpy = vmy + (vmz * tx - vmx * tz)
    vpz = vmz + (vmx * ty - vmy * tx)
    wx = vmx + (vpy * sz - vpz * sy)
    wy = vmy + (vpz * sx - vpx * sz)
    wz = vmz + (vpx * sy - vpy * sx)
    vx[:n] = wx + h * ex
    vy[:n] = wy + h * ey
    vz[:n] = wz
    x[:n] += vx[:n] * dt * 1000.0
    y[:n] += vy[:n] * dt * 1000.0


def thermal_sweeps(T, isBound, Fo_x, Fo_y, sweeps=10):
    """Explicit FTCS conduction of the CPU path, ``physics_engine.py:1599-1613``.

    Jacobi sweeps over interior cells (1..ny-2, 1..nx-2) that are bound; a neighbour
    that is not bound is replaced by the centre value; ``T_new = max(T + dT, 300)``.
    float32 throughout (Fo_x/Fo_y are weak Python floats).  Returns the final map.
    """
    T = T.copy()
    m = isBound[1:-1, 1:-1]
    bl = isBound[1:-1, :-2]
    br = isBound[1:-1, 2:]
    bd = isBound[:-2, 1:-1]
    bu = isBound[2:, 1:-1]
    for _ in range(sweeps):
        c = T[1:-1, 1:-1]
        Tl = np.where(bl, T[1:-1, :-2], c)
        Tr = np.where(br, T[1:-1, 2:], c)
        Td = np.where(bd, T[:-2, 1:-1], c)
        Tu = np.where(bu, T[2:, 1:-1], c)
        dT = Fo_x * (Tl - 2.0 * c + Tr) + Fo_y * (Td - 2.0 * c + Tu)
        Tn = T.copy()
        Tn[1:-1, 1:-1] = np.where(m, np.maximum(c + dT, 300.0), c)
        T = Tn
    return T


def thermal_taichi_sweep(T, mask, Fo_x, Fo_y):
    """One sweep of thermal_conduction_taichi (``physics_engine.py:147-171``): every masked
    cell (edges included), a neighbour is used when it is inside the domain and masked,
    ``T_new = max(T + dT, 300)`` in float32 (Taichi default_fp f32, Fo as f32); unmasked
    cells are copied.  Restated from the source (Taichi cannot run here)."""
    T = np.asarray(T, dtype=np.float32)
    ny, nx = T.shape
    m = np.asarray(mask).astype(bool)
    fx, fy = np.float32(Fo_x), np.float32(Fo_y)
    Tl = T.copy(); Tl[:, 1:] = np.where(m[:, :-1], T[:, :-1], T[:, 1:])
    Tr = T.copy(); Tr[:, :-1] = np.where(m[:, 1:], T[:, 1:], T[:, :-1])
    Td = T.copy(); Td[1:, :] = np.where(m[:-1, :], T[:-1, :], T[1:, :])
    Tu = T.copy(); Tu[:-1, :] = np.where(m[1:, :], T[1:, :], T[:-1, :])
    c2 = np.float32(2.0) * T
    dT = fx * ((Tl - c2) + Tr) + fy * ((Td - c2) + Tu)
    return np.where(m, np.maximum(T + dT, np.float32(300.0)), T).astype(np.float32)


def segment_hits(isBound, dx, dy, nx, ny, x0, y0, x1, y1, samples=8):
    """Path absorption test, ``physics_engine.py:1880-1901``: 8 samples along the
    straight segment, cell = clip(rint(s/d), 0, n-1); first hit cell recorded."""
    hit = np.zeros(len(x0), dtype=bool)
    hit_ix = np.clip(np.round(x1 / dx).astype(int), 0, nx - 1)
    hit_iy = np.clip(np.round(y1 / dy).astype(int), 0, ny - 1)
    for i in range(1, samples + 1):
        f = i / float(samples)
        xi = x0 + (x1 - x0) * f
        yi = y0 + (y1 - y0) * f
        c_x = np.clip(np.round(xi / dx).astype(int), 0, nx - 1)
        c_y = np.clip(np.round(yi / dy).astype(int), 0, ny - 1)
        step_hit = isBound[c_y, c_x]
        new_hits = step_hit & ~hit
        hit_ix[new_hits] = c_x[new_hits]
        hit_iy[new_hits] = c_y[new_hits]
        hit |= step_hit
    return hit, hit_ix, hit_iy


def substeps(Ex, Ey, dx, dy, nx, ny, x, y, vx, vy, vz, qm, dt, frac=0.25):
    """Adaptive sub-step count, ``physics_engine.py:928-966`` (returns n_sub, ds_max, ds_lim)."""
    if len(x) == 0:
        return 1, 0.0, frac * min(dx, dy) * 1e-3
    ix0 = np.clip(np.floor(x / dx).astype(int), 0, nx - 2)
    iy0 = np.clip(np.floor(y / dy).astype(int), 0, ny - 2)
    fx = x / dx - ix0
    fy = y / dy - iy0
    ix1 = ix0 + 1
    iy1 = iy0 + 1

    def gather(F):
        return (F[iy0, ix0] * (1 - fx) * (1 - fy) + F[iy0, ix1] * fx * (1 - fy) +
                F[iy1, ix0] * (1 - fx) * fy + F[iy1, ix1] * fx * fy)

    ex = gather(Ex)
    ey = gather(Ey)
    a_mag = np.sqrt((qm * ex) ** 2 + (qm * ey) ** 2)
    v_mag = np.sqrt(vx * vx + vy * vy + vz * vz)
    ds_pred = v_mag * dt + 0.5 * a_mag * dt ** 2
    ds_max = float(np.max(ds_pred))
    ds_lim = frac * min(dx, dy) * 1e-3
    n_sub = max(1, int(np.ceil(ds_max / max(ds_lim, 1e-30))))
    return n_sub, ds_max, ds_lim


def operator_matrix(isBound, periodic_y):
    """Field operator of ``physics_engine.py:525-607`` as a CSC matrix, plus row masks
    (bound, interior, rhs-rho).  Dirichlet rows are identity, Neumann rows copy the
    inward neighbour, interior rows are the 5-point stencil (-4, +1 x4), periodic
    rows wrap in y."""
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
    rows, cols, vals = [], [], []

    def put(r, c, v):
        rows.append(r); cols.append(c); vals.append(np.full(r.shape, v, dtype=np.float64))

    b = idx[is_bound]; put(b, b, 1.0)
    r = idx[is_right]; put(r, r, 1.0); put(r, r - 1, -1.0)
    t = idx[is_top]; put(t, t, 1.0); put(t, t - nx, -1.0)
    bo = idx[is_bottom]; put(bo, bo, 1.0); put(bo, bo + nx, -1.0)
    i = idx[is_interior]
    put(i, i, -4.0); put(i, i - 1, 1.0); put(i, i + 1, 1.0); put(i, i - nx, 1.0); put(i, i + nx, 1.0)
    pb = idx[is_per_bot]
    put(pb, pb, -4.0); put(pb, pb - 1, 1.0); put(pb, pb + 1, 1.0); put(pb, pb + nx, 1.0)
    put(pb, (ny - 1) * nx + (pb % nx), 1.0)
    pt = idx[is_per_top]
    put(pt, pt, -4.0); put(pt, pt - 1, 1.0); put(pt, pt + 1, 1.0); put(pt, pt - nx, 1.0)
    put(pt, pt % nx, 1.0)
    A = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(N, N)).tocsc()
    rhs_rho = is_interior | is_per_bot | is_per_top
    return A, is_bound, is_interior, rhs_rho


def efield(V, dx, dy, periodic_y, fp=np.float32):
    """E = -grad V, ``physics_engine.py:871-884``: ``np.gradient`` (2nd-order central
    interior, 1st-order one-sided edges) with the periodic-y edge fix; cast to fp."""
    Ey, Ex = np.gradient(-V, dy * 1e-3, dx * 1e-3)
    if periodic_y:
        ny = V.shape[0]
        two_dy_m = 2.0 * dy * 1e-3
        Ey[0, :] = (V[ny - 1, :] - V[1, :]) / two_dy_m
        Ey[ny - 1, :] = (V[ny - 2, :] - V[0, :]) / two_dy_m
    return Ex.astype(fp), Ey.astype(fp)


# ---------------------------------------------------------------------------
# random-draw sources
# ---------------------------------------------------------------------------


class ReplayDraws:
    """Replays a reference run's recorded ``np.random`` stream, call by call.

    ``log`` is a list of ``(method, values)`` in the order the reference consumed them.
    Each request checks the method name and the size so a restatement that calls the
    generator in a different order fails immediately.
    """

    def __init__(self, log):
        self.log = list(log)
        self.pos = 0

    def _take(self, name, size=None):
        m, v = self.log[self.pos]
        if m != name:
            raise AssertionError(f"draw {self.pos}: expected {name}, reference used {m}")
        if size is not None and np.size(v) != size:
            raise AssertionError(f"draw {self.pos}: size {size} vs {np.size(v)}")
        self.pos += 1
        return v

    def ion_count(self, lam, step):
        return int(self._take("poisson"))

    def ion_y_two_holes(self, n, ids, step):
        return self._take("randint", n), self._take("rand", n)

    def ion_y_uniform(self, lo, hi, n, ids, step):
        return self._take("uniform", n)

    def _normals3(self, n):
        return self._take("randn", n), self._take("randn", n), self._take("randn", n)

    def ion_v(self, n, ids, step):
        return self._normals3(n)

    def rf_count_u(self, step):
        return float(self._take("rand"))

    def rf_y(self, lo, hi, n, ids, step):
        return self._take("uniform", n)

    def rf_v(self, n, ids, step):
        return self._normals3(n)

    def neut_y(self, lo, hi, n, ids, step):
        return self._take("uniform", n)

    def neut_v(self, n, ids, step):
        return self._normals3(n)

    def see_u(self, ion_ids, step):
        return self._take("rand", len(ion_ids))

    def see_v(self, n, parent_ids, step):
        return self._normals3(n)

    def cex_u(self, ion_ids, step):
        return self._take("rand", len(ion_ids))

    def cex_fm(self, ion_ids, step):
        n = len(ion_ids)
        return [self._take("rand", n) for _ in range(9)]


class PhiloxDraws:
    """Keyed Philox4x32-10 draws (seed, site, particle id, step), as on the GPU."""

    def __init__(self, seed):
        self.seed = int(seed)

    def ion_count(self, lam, step):
        return _px.poisson_count(self.seed, _px.SITE_ION_COUNT, step, lam)

    def ion_y_two_holes(self, n, ids, step):
        u = _px.uniforms(self.seed, ids, _px.SITE_ION_HOLE, step, 2)
        which = (u[0] * 2.0).astype(np.int64)
        return which, u[1]

    def ion_y_uniform(self, lo, hi, n, ids, step):
        u = _px.uniforms(self.seed, ids, _px.SITE_ION_Y, step, 1)[0]
        return lo + (hi - lo) * u

    def ion_v(self, n, ids, step):
        g = _px.normals(self.seed, ids, _px.SITE_ION_V, step, 3)
        return g[0], g[1], g[2]

    def rf_count_u(self, step):
        return float(_px.uniforms(self.seed, np.array([0]), _px.SITE_RF_COUNT, step, 1)[0, 0])

    def rf_y(self, lo, hi, n, ids, step):
        u = _px.uniforms(self.seed, ids, _px.SITE_RF_Y, step, 1)[0]
        return lo + (hi - lo) * u

    def rf_v(self, n, ids, step):
        g = _px.normals(self.seed, ids, _px.SITE_RF_V, step, 3)
        return g[0], g[1], g[2]

    def neut_y(self, lo, hi, n, ids, step):
        u = _px.uniforms(self.seed, ids, _px.SITE_NEUT_Y, step, 1)[0]
        return lo + (hi - lo) * u

    def neut_v(self, n, ids, step):
        g = _px.normals(self.seed, ids, _px.SITE_NEUT_V, step, 3)
        return g[0], g[1], g[2]

    def see_u(self, ion_ids, step):
        return _px.uniforms(self.seed, ion_ids, _px.SITE_SEE_SPAWN, step, 1)[0]

    def see_v(self, n, parent_ids, step):
        # keyed by the parent ion, so the draw does not depend on spawn order
        g = _px.normals(self.seed, parent_ids, _px.SITE_SEE_V, step, 3)
        return g[0], g[1], g[2]

    def cex_u(self, ion_ids, step):
        return _px.uniforms(self.seed, ion_ids, _px.SITE_CEX_U, step, 1)[0]

    def cex_fm(self, ion_ids, step):
        u = _px.uniforms(self.seed, ion_ids, _px.SITE_CEX_FM, step, 9)
        return [u[k] for k in range(9)]


# ---------------------------------------------------------------------------
# simulator restatement
# ---------------------------------------------------------------------------

MATERIAL_PRESETS = {
    'Molybdenum': {'k': 138.0, 'rho': 10280.0, 'cp': 250.0, 'emissivity': 0.80, 'alpha': 4.8e-6,
                   'E_mod': 329e9, 'Y_coeff': 1.05e-4, 'E_th': 30.0},
    'Steel (SS316)': {'k': 16.3, 'rho': 8000.0, 'cp': 500.0, 'emissivity': 0.60, 'alpha': 16.0e-6,
                      'E_mod': 193e9, 'Y_coeff': 2.8e-4, 'E_th': 25.0},
    'Titanium': {'k': 21.9, 'rho': 4507.0, 'cp': 520.0, 'emissivity': 0.50, 'alpha': 8.6e-6,
                 'E_mod': 116e9, 'Y_coeff': 1.8e-4, 'E_th': 20.0},
    'Graphite': {'k': 120.0, 'rho': 2200.0, 'cp': 710.0, 'emissivity': 0.85, 'alpha': 3.0e-6,
                 'E_mod': 11e9, 'Y_coeff': 3.5e-4, 'E_th': 15.0},
}


class OracleSimulator:
    """Restatement of ``DigitalTwinSimulator`` (``physics_engine.py:309-1963``).

    ``geometry_builder(sim, params, preserve_state, fp)`` supplies the domain geometry
    (``build_domain`` lines 629-842); tests pass the host builder that is itself pinned
    against the reference.  ``fp`` selects float32 (the reference as shipped) or float64
    (the reference with ``_NP_FP = float64``, the FP64 oracle).
    """

    def __init__(self, geometry_builder, fp=np.float32):
        self.fp = fp
        self._geometry_builder = geometry_builder
        self.dt = 5e-10
        self.injection_stop_time = None
        self.injection_enabled = True
        self.q = 1.602e-19
        self.m_XE = 131.293 * 1.6605e-27
        self.m_ion = self.m_XE
        self.Z_ion = 1
        self.q_ion = self.q
        self.kB = 1.380649e-23
        self.eps0 = 8.854e-12
        self.m_e = self.m_XE / 100.0
        self.user_cs = {}
        self.set_material('Molybdenum')
        self.macro_weight = 3e5
        self.sb_sigma = 5.67e-8
        self.thermal_accel = 1e7
        self.injected_ions = 0.0
        self.transmitted_ions = 0.0
        self.entered_optics = 0.0
        self.entered_optics_step = 0.0
        self.transmitted3_step = 0.0
        self.Lx = 3
        self.Ly = 3
        self.dx = 0.02
        self.dy = 0.02
        self.nx = int(self.Lx / self.dx) + 1
        self.ny = int(self.Ly / self.dy) + 1
        self.dx = self.Lx / (self.nx - 1)
        self.dy = self.Ly / (self.ny - 1)
        self._recompute_cell_constants()
        self.T_grids = []
        self.mask_grids = []
        self.iteration = 0
        self.Tmap = np.full((self.ny, self.nx), 300.0, dtype=fp)
        self.T_map_new = np.full((self.ny, self.nx), 300.0, dtype=fp)
        self.laplacian_lu = None
        self.next_ion_id = 0
        self.next_e_id = 0
        self.reset_arrays()

    # -- state ---------------------------------------------------------------
    def reset_arrays(self):
        """``physics_engine.py:404-448`` plus particle id arrays."""
        fp = self.fp
        self.max_p = 100000
        self.max_e = 100000
        self.p_x = np.zeros(self.max_p, dtype=fp)
        self.p_y = np.zeros(self.max_p, dtype=fp)
        self.p_vx = np.zeros(self.max_p, dtype=fp)
        self.p_vy = np.zeros(self.max_p, dtype=fp)
        self.p_vz = np.zeros(self.max_p, dtype=fp)
        self.p_isCEX = np.zeros(self.max_p, dtype=bool)
        self.p_id = np.zeros(self.max_p, dtype=np.int64)
        self.num_p = 0
        self.e_x = np.zeros(self.max_e, dtype=fp)
        self.e_y = np.zeros(self.max_e, dtype=fp)
        self.e_vx = np.zeros(self.max_e, dtype=fp)
        self.e_vy = np.zeros(self.max_e, dtype=fp)
        self.e_vz = np.zeros(self.max_e, dtype=fp)
        self.e_id = np.zeros(self.max_e, dtype=np.int64)
        self.num_e = 0
        self.iteration = 0
        self.next_ion_id = 0
        self.next_e_id = 0
        self.V = np.zeros((self.ny, self.nx), dtype=np.float64)
        self.rho = np.zeros((self.ny, self.nx), dtype=fp)
        self.isBound = np.zeros((self.ny, self.nx), dtype=bool)
        self.V_fixed = np.zeros((self.ny, self.nx), dtype=np.float64)
        self.damage_map = np.zeros((self.ny, self.nx), dtype=np.float64)
        self.eroded_depth = np.zeros((self.ny, self.nx), dtype=np.float64)
        self.Ex = np.zeros((self.ny, self.nx), dtype=fp)
        self.Ey = np.zeros((self.ny, self.nx), dtype=fp)
        self.Bx = np.zeros((self.ny, self.nx), dtype=fp)
        self.By = np.zeros((self.ny, self.nx), dtype=fp)
        self.Bz = np.zeros((self.ny, self.nx), dtype=fp)
        self.accum_ppc_map = np.zeros((self.ny, self.nx), dtype=np.float64)
        self.ppc_steps_count = 0
        self.current_ppc_map = np.zeros((self.ny, self.nx), dtype=int)

    def _recompute_cell_constants(self):
        """``physics_engine.py:450-452``."""
        self.C_cell = self.mat_rho * (self.dx * 1e-3) * (self.dy * 1e-3) * 1e-3 * self.mat_cp
        self.A_cell = 2 * (self.dx * 1e-3) * 1e-3

    def set_material(self, name=None, props=None):
        """``physics_engine.py:454-473``."""
        if name and name in MATERIAL_PRESETS:
            mat = MATERIAL_PRESETS[name]
        elif props:
            mat = props
        else:
            return
        self.mat_k = mat['k']
        self.mat_rho = mat['rho']
        self.mat_cp = mat['cp']
        self.emissivity = mat['emissivity']
        self.alpha_thermal = mat['alpha']
        self.E_modulus = mat['E_mod']
        self.sputter_Y_coeff = mat['Y_coeff']
        self.sputter_E_th = mat['E_th']
        if hasattr(self, 'dx'):
            self._recompute_cell_constants()

    def lookup_user_cs(self, prefix, energy_eV):
        """``physics_engine.py:475-484``: log-log spline, clipped to the table range."""
        for label, ds in self.user_cs.items():
            if label.startswith(prefix) and ds.get('spline') is not None:
                log_e = np.log10(np.maximum(energy_eV, 1e-30))
                e_min = np.log10(max(ds['energy'][0], 1e-30))
                e_max = np.log10(ds['energy'][-1])
                log_e = np.clip(log_e, e_min, e_max)
                return 10.0 ** ds['spline'](log_e)
        return None

    def _grow(self, names, n_new, count, cap):
        new_max = max(cap * 2, count + n_new)
        for nm in names:
            setattr(self, nm, np.pad(getattr(self, nm), (0, new_max - cap)))
        return new_max

    def _add_ions(self, x, y, vx, vy, vz, is_cex, ids):
        """``physics_engine.py:486-504`` (+ ids)."""
        n_new = len(x)
        if self.num_p + n_new > self.max_p:
            self.max_p = self._grow(['p_x', 'p_y', 'p_vx', 'p_vy', 'p_vz', 'p_isCEX', 'p_id'],
                                    n_new, self.num_p, self.max_p)
        s, e = self.num_p, self.num_p + n_new
        self.p_x[s:e] = x
        self.p_y[s:e] = y
        self.p_vx[s:e] = vx
        self.p_vy[s:e] = vy
        self.p_vz[s:e] = vz
        self.p_isCEX[s:e] = is_cex
        self.p_id[s:e] = ids
        self.num_p += n_new

    def _add_electrons(self, x, y, vx, vy, vz, ids):
        """``physics_engine.py:506-522`` (+ ids)."""
        n_new = len(x)
        if self.num_e + n_new > self.max_e:
            self.max_e = self._grow(['e_x', 'e_y', 'e_vx', 'e_vy', 'e_vz', 'e_id'],
                                    n_new, self.num_e, self.max_e)
        s, e = self.num_e, self.num_e + n_new
        self.e_x[s:e] = x
        self.e_y[s:e] = y
        self.e_vx[s:e] = vx
        self.e_vy[s:e] = vy
        self.e_vz[s:e] = vz
        self.e_id[s:e] = ids
        self.num_e += n_new

    def new_ion_ids(self, n):
        ids = np.arange(self.next_ion_id, self.next_ion_id + n, dtype=np.int64)
        self.next_ion_id += n
        return ids

    def new_e_ids(self, n):
        ids = np.arange(self.next_e_id, self.next_e_id + n, dtype=np.int64)
        self.next_e_id += n
        return ids

    # -- domain / fields -----------------------------------------------------
    def build_sparse_matrix(self):
        """``physics_engine.py:525-608`` (SuperLU factorisation of the same matrix)."""
        A, is_bound, is_interior, rhs = operator_matrix(self.isBound, getattr(self, 'periodic_y', False))
        self.A = A
        self.is_bound_mask = is_bound
        self.is_interior_mask = is_interior
        self.is_rhs_rho_mask = rhs
        self.laplacian_lu = factorized(A)

    def build_domain(self, params, preserve_state=False):
        """``physics_engine.py:629-847``."""
        # C_cell / A_cell are NOT recomputed here: the reference refreshes them only in
        # __init__ and set_material (physics_engine.py:372,473), so they keep the dx, dy
        # current at that time.
        self._geometry_builder(self, params, preserve_state, self.fp)
        self.build_sparse_matrix()
        self.recalc_poisson(iterations=30 if not preserve_state else 10, params=params)

    def recalc_poisson(self, iterations=5, params=None):
        """Damped Boltzmann-electron Picard loop + E field, ``physics_engine.py:850-902``."""
        if self.laplacian_lu is None:
            return
        coeff = (self.dx * 1e-3) ** 2 / self.eps0
        params = params or {}
        grids = params.get('grids', [{'V': 1000}])
        V_plasma = grids[0]['V'] + params.get('V_plasma_offset', 20.0)
        Te_up = params.get('Te_up', 3.0)
        n0 = params.get('n0_plasma', 1e17)
        omega = 0.2
        b = np.zeros(self.nx * self.ny, dtype=np.float64)
        Vf = self.V_fixed.flatten()
        for _ in range(iterations):
            rho_e = -self.q * n0 * np.exp((np.minimum(self.V, V_plasma) - V_plasma) / Te_up)
            rho_flat = (self.rho + rho_e).flatten()
            b.fill(0.0)
            b[self.is_bound_mask] = Vf[self.is_bound_mask]
            b[self.is_rhs_rho_mask] = -coeff * rho_flat[self.is_rhs_rho_mask]
            V_new = self.laplacian_lu(b).reshape((self.ny, self.nx))
            self.V = ((1 - omega) * self.V + omega * V_new).astype(np.float64)
        self.Ex, self.Ey = efield(self.V, self.dx, self.dy, getattr(self, 'periodic_y', False), self.fp)

    def compute_particle_substeps(self, x, y, vx, vy, vz, qm, dt, frac=0.25):
        return substeps(self.Ex, self.Ey, self.dx, self.dy, self.nx, self.ny, x, y, vx, vy, vz, qm, dt, frac)

    def _segment_hits_grid(self, x0, y0, x1, y1, samples=8):
        return segment_hits(self.isBound, self.dx, self.dy, self.nx, self.ny, x0, y0, x1, y1, samples)

    # -- the timestep ----------------------------------------------------------
    def step(self, params, draws):
        """One PIC-MCC timestep, ``physics_engine.py:969-1784``; returns the 5-tuple."""
        fp = self.fp
        if self.laplacian_lu is None:
            return False, np.nan, np.nan, self.T_grids, 0.0
        sim_mode = params.get('sim_mode', 'Both')
        self.iteration += 1
        it = self.iteration
        t_current = self.iteration * self.dt
        grids = params.get('grids', [])
        self.transmitted_ions_step = 0.0
        self.transmitted3_step = 0.0
        self.entered_optics_step = 0.0
        self.injected_ions_step = 0.0
        self.lost_to_grid_step = 0.0

        # RF co-extraction (:984-991)
        if params.get('rf_enable') and grids:
            rf_idx = params.get('rf_grid_idx', 0)
            if rf_idx < len(grids):
                f_hz = params.get('rf_freq', 13.56) * 1e6
                v_rf = params.get('rf_amp', 100.0) * np.sin(2.0 * np.pi * f_hz * t_current)
                m = self.mask_grids[rf_idx]
                self.V_fixed[m] = self.Vdc[m] + v_rf
                self.recalc_poisson(iterations=2, params=params)

        # A. injection (:996-1083)
        if self.injection_enabled and (self.injection_stop_time is None or t_current <= self.injection_stop_time):
            n0 = params.get('n0_plasma', 1e17)
            Te_up = params.get('Te_up', 3.0)
            Ti = params.get('Ti', 0.1)
            v_bohm = np.sqrt(self.q_ion * Te_up / self.m_ion)
            injection_area = self.Ly * 1e-3 * 0.005
            bohm_factor = 1.0 if params.get('entire_bulk_plasma', False) else 0.61
            I_ion = self.q_ion * bohm_factor * n0 * v_bohm * injection_area
            charge_per_macro = self.q_ion * self.macro_weight
            num_inject_float = (I_ion * self.dt) / charge_per_macro
            num_inject = draws.ion_count(num_inject_float, it)
            if num_inject > 0:
                ids = self.new_ion_ids(num_inject)
                geometry = getattr(self, 'geometry', 'half_hole')
                if grids:
                    screen_r = grids[0]['r']
                    pitch_inj = params.get('pitch_mm', 0.0)
                    if geometry == 'two_holes':
                        span = np.array([
                            [max(self.dy, 0.5 * screen_r), min(2.5 * screen_r, self.Ly - self.dy)],
                            [max(self.dy, 0.5 * screen_r + pitch_inj), min(2.5 * screen_r + pitch_inj, self.Ly - self.dy)],
                        ], dtype=fp)
                        which, u = draws.ion_y_two_holes(num_inject, ids, it)
                        y_lo = span[which, 0]
                        y_hi = span[which, 1]
                        new_y = (y_lo + (y_hi - y_lo) * u).astype(fp)
                    elif geometry == 'one_hole':
                        new_y = draws.ion_y_uniform(max(self.dy, 0.5 * screen_r), min(2.5 * screen_r, self.Ly - self.dy),
                                                    num_inject, ids, it).astype(fp)
                    else:
                        new_y = draws.ion_y_uniform(0.0, min(screen_r, self.Ly - self.dy), num_inject, ids, it).astype(fp)
                else:
                    new_y = draws.ion_y_uniform(self.dy, self.Ly - self.dy, num_inject, ids, it).astype(fp)
                new_x = np.full(num_inject, self.dx * 1.5, dtype=fp)
                v_spread = np.sqrt(self.q_ion * Ti / self.m_ion)
                gx, gy, gz = draws.ion_v(num_inject, ids, it)
                new_vx = np.full(num_inject, v_bohm, dtype=np.float64) + np.asarray(gx, dtype=np.float64) * v_spread
                new_vy = (gy * v_spread).astype(fp)
                new_vz = (gz * v_spread).astype(fp)
                self._add_ions(new_x, new_y, new_vx, new_vy, new_vz, np.zeros(num_inject, dtype=bool), ids)
                self.injected_ions_step += float(num_inject)
                self.injected_ions += float(num_inject)

            if params.get('rf_enable'):
                v_e_th_source = np.sqrt(2.0 * self.q * Te_up / self.m_e)
                I_e = self.q * 0.25 * n0 * v_e_th_source * injection_area
                num_e_float = (I_e * self.dt) / charge_per_macro
                num_inj_e = int(num_e_float)
                if draws.rf_count_u(it) < (num_e_float - num_inj_e):
                    num_inj_e += 1
                if num_inj_e > 0:
                    eids = self.new_e_ids(num_inj_e)
                    y_margin = max(self.dy, 1e-9)
                    y_low = y_margin
                    y_high = max(y_low, self.Ly - y_margin)
                    new_ex = np.full(num_inj_e, 0.1, dtype=fp)
                    new_ey = draws.rf_y(y_low, y_high, num_inj_e, eids, it).astype(fp)
                    gx, gy, gz = draws.rf_v(num_inj_e, eids, it)
                    new_evx = (np.abs(gx) * v_e_th_source + v_bohm).astype(fp)
                    new_evy = (gy * v_e_th_source).astype(fp)
                    new_evz = (gz * v_e_th_source).astype(fp)
                    self._add_electrons(new_ex, new_ey, new_evx, new_evy, new_evz, eids)

        # neutralizer (:1086-1099)
        num_e_neut = int(params.get('neut_rate', 30))
        Te_eV = params.get('Te', 5.0)
        neut_x = float(np.clip(params.get('neut_x', self.Lx - 0.5), self.dx, self.Lx - self.dx))
        neut_r = float(np.clip(params.get('neut_r', self.Ly), self.dy, self.Ly))
        if num_e_neut > 0:
            eids = self.new_e_ids(num_e_neut)
            new_ey = draws.neut_y(0.0, neut_r, num_e_neut, eids, it).astype(fp)
            new_ex = np.full(num_e_neut, neut_x, dtype=fp)
            v_e_th = np.sqrt(2.0 * self.q * Te_eV / self.m_e)
            gx, gy, gz = draws.neut_v(num_e_neut, eids, it)
            self._add_electrons(new_ex, new_ey, (gx * v_e_th).astype(fp), (gy * v_e_th).astype(fp),
                                (gz * v_e_th).astype(fp), eids)

        # B. deposit + Poisson (:1104-1161)
        self.rho.fill(0.0)
        cell_vol = (self.dx * 1e-3) * (self.dy * 1e-3) * 1e-3
        cpp = self.q * self.macro_weight
        if self.num_p > 0:
            accumulate_rho(self.p_x[:self.num_p], self.p_y[:self.num_p], self.rho, self.num_p,
                           self.dx, self.dy, self.nx, self.ny, cpp / cell_vol)
        if self.num_e > 0:
            accumulate_rho(self.e_x[:self.num_e], self.e_y[:self.num_e], self.rho, self.num_e,
                           self.dx, self.dy, self.nx, self.ny, -cpp / cell_vol)
        if self.iteration % 2 == 0:
            self.recalc_poisson(iterations=5, params=params)

        # C. push (:1166-1283)
        num_p_step = int(self.num_p)
        p_x_old = self.p_x[:num_p_step].copy()
        p_y_old = self.p_y[:num_p_step].copy()
        if num_p_step > 0:
            n_sub_ion, ds_ion, lim_ion = self.compute_particle_substeps(
                self.p_x[:num_p_step], self.p_y[:num_p_step], self.p_vx[:num_p_step],
                self.p_vy[:num_p_step], self.p_vz[:num_p_step], self.q_ion / self.m_ion, self.dt)
        else:
            n_sub_ion = 1
        num_e_step = int(self.num_e)
        if num_e_step > 0:
            n_sub_e, ds_e, lim_e = self.compute_particle_substeps(
                self.e_x[:num_e_step], self.e_y[:num_e_step], self.e_vx[:num_e_step],
                self.e_vy[:num_e_step], self.e_vz[:num_e_step], -self.q / self.m_e, self.dt)
        else:
            n_sub_e = 1
        self.n_sub_ion, self.n_sub_e = n_sub_ion, n_sub_e
        if num_p_step > 0:
            for _ in range(n_sub_ion):
                push_particles_boris(self.p_x[:num_p_step], self.p_y[:num_p_step], self.p_vx[:num_p_step],
                                     self.p_vy[:num_p_step], self.p_vz[:num_p_step],
                                     self.Ex, self.Ey, self.Bx, self.By, self.Bz,
                                     num_p_step, self.dx, self.dy, self.nx, self.ny,
                                     self.dt / n_sub_ion, self.q_ion / self.m_ion)
        if num_e_step > 0:
            for _ in range(n_sub_e):
                push_particles_boris(self.e_x[:num_e_step], self.e_y[:num_e_step], self.e_vx[:num_e_step],
                                     self.e_vy[:num_e_step], self.e_vz[:num_e_step],
                                     self.Ex, self.Ey, self.Bx, self.By, self.Bz,
                                     num_e_step, self.dx, self.dy, self.nx, self.ny,
                                     self.dt / n_sub_e, -self.q / self.m_e)

        # periodic wrap (:1289-1293)
        if getattr(self, 'periodic_y', False):
            if num_p_step > 0:
                self.p_y[:num_p_step] = np.mod(self.p_y[:num_p_step], self.Ly)
            if self.num_e > 0:
                self.e_y[:self.num_e] = np.mod(self.e_y[:self.num_e], self.Ly)

        p_x = self.p_x[:num_p_step].copy()
        p_y = self.p_y[:num_p_step].copy()
        p_vx = self.p_vx[:num_p_step].copy()
        p_vy = self.p_vy[:num_p_step].copy()
        p_vz = self.p_vz[:num_p_step].copy()
        p_cex = self.p_isCEX[:num_p_step].copy()
        p_ids = self.p_id[:num_p_step].copy()

        if grids and hasattr(self, "grid_x_starts") and len(self.grid_x_starts) == len(grids):
            x_entry_first_grid = self.grid_x_starts[0]
            x_exit_last = self.grid_x_ends[-1]
            x_plume_boundary = self.grid_x_ends[-1] + grids[-1]["gap"]
        else:
            x_entry_first_grid = 0.5
            x_exit_last = 3.0
            x_plume_boundary = 3.0

        # D. hits (:1316-1336)
        entered = (p_x_old < x_entry_first_grid) & (p_x >= x_entry_first_grid) & (p_vx > 0.0)
        n_entered = int(np.count_nonzero(entered))
        self.entered_optics_step = float(n_entered)
        self.entered_optics += float(n_entered)
        self.prev_entered = self.entered_optics_step
        ix = np.clip(np.round(p_x / self.dx).astype(int), 0, self.nx - 1)
        iy = np.clip(np.round(p_y / self.dy).astype(int), 0, self.ny - 1)
        hit_final = self.isBound[iy, ix]
        hit_path, path_ix, path_iy = self._segment_hits_grid(p_x_old, p_y_old, p_x, p_y, samples=8)
        hit_grid = hit_final | hit_path
        impact_ix = np.where(hit_path, path_ix, ix)
        impact_iy = np.where(hit_path, path_iy, iy)
        self.last_hit_grid = hit_grid.copy()
        self.last_impact = (impact_iy.copy(), impact_ix.copy())

        # out of bounds (:1341-1355)
        if getattr(self, 'periodic_y', False):
            oob = (p_x < 0.0) | (p_x > x_plume_boundary) | np.isnan(p_x)
        else:
            oob = (p_x < 0.0) | (p_x > x_plume_boundary) | (p_y < 0.0) | (p_y > self.Ly) | np.isnan(p_x)
        remeshed = False

        # impact heating (:1359-1388)
        hot = hit_grid & (p_x > 0.25)
        if sim_mode in ("Thermal", "Both") and np.any(hot):
            v2 = p_vx[hot] ** 2 + p_vy[hot] ** 2 + p_vz[hot] ** 2
            E_j = 0.5 * self.m_ion * v2 * self.macro_weight
            dT_heat = (E_j / self.C_cell) * self.thermal_accel
            np.add.at(self.Tmap, (impact_iy[hot], impact_ix[hot]), dT_heat)

        # SEE (:1390-1417)
        if np.any(hot):
            v2 = p_vx[hot] ** 2 + p_vy[hot] ** 2 + p_vz[hot] ** 2
            E_eV = (0.5 * self.m_ion * v2) / self.q
            see_user = self.lookup_user_cs('SEE', E_eV)
            gamma = np.clip(see_user if see_user is not None else 0.05 + 1e-4 * E_eV, 0.0, 1.0)
            spawn = draws.see_u(p_ids[hot], it) < gamma
            if np.any(spawn):
                num_see = int(np.sum(spawn))
                sx = (p_x[hot][spawn] - p_vx[hot][spawn] * self.dt * 1000.0 / 1.5).astype(fp)
                sy = (p_y[hot][spawn] - p_vy[hot][spawn] * self.dt * 1000.0 / 1.5).astype(fp)
                v_see_th = np.sqrt(2.0 * self.q * 2.0 / self.m_e)
                eids = self.new_e_ids(num_see)
                gx, gy, gz = draws.see_v(num_see, p_ids[hot][spawn], it)
                self._add_electrons(sx, sy, (gx * v_see_th).astype(fp), (gy * v_see_th).astype(fp),
                                    (gz * v_see_th).astype(fp), eids)

        # erosion (:1419-1449)
        if sim_mode in ("Erosion", "Both") and np.any(hot):
            E_eV = (0.5 * self.m_ion * (p_vx[hot] ** 2 + p_vy[hot] ** 2 + p_vz[hot] ** 2)) / self.q
            ok = E_eV > self.sputter_E_th
            if np.any(ok):
                p_exp = float(params.get('sputter_exponent', 1.0))
                if p_exp == 1.0:
                    dmg = (self.sputter_Y_coeff * (E_eV[ok] - self.sputter_E_th)) * self.macro_weight
                else:
                    # option without a reference counterpart: Y = Y_coeff (E - E_th)^p,
                    # evaluated in float64 from the float32 excess energy
                    excess = (E_eV[ok] - self.sputter_E_th).astype(np.float64)
                    dmg = (self.sputter_Y_coeff * excess ** p_exp) * self.macro_weight
                np.add.at(self.damage_map, (impact_iy[hot][ok], impact_ix[hot][ok]), dmg)
            broken = (self.damage_map > params.get('Thresh', 1e5)) & self.isBound
            if np.any(broken):
                self.eroded_depth[broken] += self.dy
                self.isBound[broken] = False
                self.damage_map[broken] = 0.0
                self.build_sparse_matrix()
                remeshed = True

        # exit diagnostics (:1451-1494)
        exited = (p_x > x_exit_last) & (p_vx > 0.0)
        crossed = (p_x_old <= x_exit_last) & (p_x > x_exit_last) & (p_vx > 0.0)
        n_cross = int(np.count_nonzero(crossed))
        if n_cross > 0:
            vxe, vye, vze = p_vx[crossed], p_vy[crossed], p_vz[crossed]
            ve = np.sqrt(vxe ** 2 + vye ** 2 + vze ** 2)
            self.exit_vx_mean = float(np.mean(vxe))
            self.exit_v_mean = float(np.mean(ve))
            self.exit_energy_mean_eV = float(np.mean(0.5 * self.m_ion * ve ** 2 / self.q))
            self.exit_count_step = n_cross
        else:
            self.exit_vx_mean = np.nan
            self.exit_v_mean = np.nan
            self.exit_energy_mean_eV = np.nan
            self.exit_count_step = 0
        self.crossed_angles = np.abs(np.arctan2(p_vy[crossed], p_vx[crossed])) * 180.0 / np.pi
        current_div = np.percentile(self.crossed_angles, 95) if n_cross > 5 else np.nan
        if np.any(exited):
            self.transmitted_ions_step = float(n_cross)
            self.transmitted_ions += float(n_cross)
            self.transmitted3_step = float(n_cross)
        self.lost_to_grid_step = float(np.count_nonzero(hit_grid & ~oob))

        # compaction (:1499-1529) — both stable masks applied in sequence
        alive = ~(hit_grid | oob)
        keep = alive.copy()
        keep[alive] = (p_x[alive] <= x_plume_boundary) | (p_vx[alive] < 0.0)
        n_keep = int(np.count_nonzero(keep))
        self.p_x[:n_keep] = p_x[keep]
        self.p_y[:n_keep] = p_y[keep]
        self.p_vx[:n_keep] = p_vx[keep]
        self.p_vy[:n_keep] = p_vy[keep]
        self.p_vz[:n_keep] = p_vz[keep]
        self.p_isCEX[:n_keep] = p_cex[keep]
        self.p_id[:n_keep] = p_ids[keep]
        self.num_p = n_keep

        # E. electrons (:1534-1561)
        if self.num_e > 0:
            n = self.num_e
            e_x, e_y = self.e_x[:n], self.e_y[:n]
            ixe = np.clip(np.round(e_x / self.dx).astype(int), 0, self.nx - 1)
            iye = np.clip(np.round(e_y / self.dy).astype(int), 0, self.ny - 1)
            dead_e = self.isBound[iye, ixe] | (e_x < 0.0) | (e_x > self.Lx) | (e_y < 0.0) | (e_y > self.Ly) | np.isnan(e_x)
            alive_e = ~dead_e
            n_alive_e = int(np.sum(alive_e))
            if n_alive_e < n:
                for nm in ('e_x', 'e_y', 'e_vx', 'e_vy', 'e_vz', 'e_id'):
                    arr = getattr(self, nm)
                    arr[:n_alive_e] = arr[:n][alive_e]
                self.num_e = n_alive_e

        # F. thermal (:1566-1647)
        if sim_mode in ('Thermal', 'Both'):
            self.Tmap = self.Tmap.copy()
            T_bound = self.Tmap[self.isBound]
            cooling_factor = (self.emissivity * self.sb_sigma * self.A_cell * self.dt * self.thermal_accel) / self.C_cell
            self.Tmap[self.isBound] -= cooling_factor * (T_bound ** 4 - 300.0 ** 4)
            self.Tmap = self.Tmap.astype(fp)
            alpha_diff = self.mat_k / (self.mat_rho * self.mat_cp)
            dt_th = self.dt * self.thermal_accel
            Fo_x = alpha_diff * dt_th / (self.dx * 1e-3) ** 2
            Fo_y = alpha_diff * dt_th / (self.dy * 1e-3) ** 2
            if Fo_x > 0.2 or Fo_y > 0.2:
                scale = 0.2 / max(Fo_x, Fo_y)
                Fo_x *= scale
                Fo_y *= scale
            self.Fo = (Fo_x, Fo_y)
            self.Tmap = thermal_sweeps(self.Tmap, self.isBound, Fo_x, Fo_y, 10)
            self.Tmap[self.isBound] = np.maximum(self.Tmap[self.isBound], 300.0)
            needs_remesh = False
            for i, mask in enumerate(self.mask_grids):
                if np.any(mask):
                    self.T_grids[i] = np.mean(self.Tmap[mask])
            geometry = getattr(self, 'geometry', 'half_hole')
            for i, grid in enumerate(grids):
                dT = self.T_grids[i] - 300.0
                if geometry == 'two_holes':
                    dc = params.get("discharge_chamber")
                    pitch_val = params.get("pitch_mm", dc.get("pitch_mm", 3.0) if isinstance(dc, dict) else 3.0)
                    L_cant_mm = max(0.2, pitch_val - 2.0 * grid['r'])
                elif geometry == 'one_hole':
                    L_cant_mm = max(0.2, 0.5 * (self.Ly - 2.0 * grid['r']))
                else:
                    L_cant_mm = max(0.2, self.Ly - grid['r'])
                L_cant_m = L_cant_mm * 1e-3
                t_m = grid['t'] * 1e-3
                new_defl = (self.alpha_thermal * dT * L_cant_m ** 2 / (2.0 * t_m)) * 1e3 if (t_m > 0 and L_cant_m > 0) else 0.0
                if abs(new_defl - self.grid_deflections[i]) > 0.005:
                    self.grid_deflections[i] = new_defl
                    needs_remesh = True
            if needs_remesh:
                self.build_domain(params, preserve_state=True)
                remeshed = True

        # G. saddle potential (:1655-1676)
        hole_centers = getattr(self, 'hole_centers', [0.0])
        if len(grids) >= 2:
            x_grid_mm = 0.5 * (self.grid_x_starts[1] + self.grid_x_ends[1])
        elif len(grids) == 1:
            x_grid_mm = 0.5 * (self.grid_x_starts[0] + self.grid_x_ends[0])
        else:
            x_grid_mm = self.Lx * 0.5
        x_idx = int(np.clip(round(x_grid_mm / self.dx), 0, self.nx - 1))
        if hole_centers:
            min_pot = min(self.V[int(np.clip(round(yc / self.dy), 0, self.ny - 1)), x_idx] for yc in hole_centers)
        else:
            min_pot = self.V[self.ny // 2, x_idx]

        # H. CEX (:1682-1739)
        self.last_collided_ids = np.zeros(0, dtype=np.int64)
        if self.num_p > 0:
            n = self.num_p
            p_x, p_y = self.p_x[:n], self.p_y[:n]
            p_vx, p_vy, p_vz = self.p_vx[:n], self.p_vy[:n], self.p_vz[:n]
            primary = (~self.p_isCEX[:n]) & (p_x >= 1.0) & (p_x <= self.Lx)
            if np.any(primary):
                px_m = p_x[primary]
                py_m = p_y[primary]
                r_T = self.Ly * 1e-3
                z_m = np.maximum((px_m - 1.0) * 1e-3, 0.0)
                r_m = py_m * 1e-3
                a_corr = 1.0 / (1.0 - 1.0 / np.sqrt(2.0))
                R_dist = np.sqrt(r_m ** 2 + (z_m + r_T) ** 2)
                theta = np.arctan2(r_m, z_m + r_T)
                if params.get('neutral_profile', 'point_source') == 'uniform':
                    # option without a reference counterpart: a uniform background n0
                    n_local = np.full(px_m.shape, float(params.get('n0', 1e20)))
                else:
                    n_local = params.get('n0', 1e20) * a_corr * (
                        1.0 - 1.0 / np.sqrt(1.0 + (r_T / np.maximum(R_dist, 1e-12)) ** 2)) * np.cos(theta)
                n_local = np.maximum(n_local, 0.0)
                v_mag = np.sqrt(p_vx[primary] ** 2 + p_vy[primary] ** 2 + p_vz[primary] ** 2)
                g = np.maximum(v_mag, 1.0)
                E_cex = (0.5 * self.m_ion * g ** 2) / self.q
                s_user = self.lookup_user_cs('CX', E_cex)
                sigma = s_user if s_user is not None else ((-0.8821 * np.log(g) + 15.1262) ** 2) * 1e-20
                prob = 1.0 - np.exp(-n_local * sigma * g * self.dt)
                prim_ids = self.p_id[:n][primary]
                u = draws.cex_u(prim_ids, it)
                collided = u < prob
                self.last_cex = (prim_ids, u, prob)
                if np.any(collided):
                    c_idx = np.where(primary)[0][collided]
                    neut_vth = np.sqrt(2.0 * self.kB * params.get('Tn', 300.0) / self.m_ion)
                    r = draws.cex_fm(self.p_id[c_idx], it)
                    fx = 2.0 * (r[0] + r[1] + r[2] - 1.5)
                    fy = 2.0 * (r[3] + r[4] + r[5] - 1.5)
                    fz = 2.0 * (r[6] + r[7] + r[8] - 1.5)
                    self.p_vx[c_idx] = (neut_vth * fx).astype(fp)
                    self.p_vy[c_idx] = (neut_vth * fy).astype(fp)
                    self.p_vz[c_idx] = (neut_vth * fz).astype(fp)
                    self.p_isCEX[c_idx] = True
                    self.last_collided_ids = self.p_id[c_idx].copy()

        trans_last_frame = self.transmitted3_step / self.entered_optics_step if self.entered_optics_step > 0.0 else 0.0

        # PPC map (:1742-1767)
        n = self.num_p
        ixp = np.clip((self.p_x[:n] / self.dx).astype(int), 0, self.nx - 1)
        iyp = np.clip((self.p_y[:n] / self.dy).astype(int), 0, self.ny - 1)
        ppc = np.bincount(iyp * self.nx + ixp, minlength=self.nx * self.ny).reshape((self.ny, self.nx))
        self.current_ppc_map = ppc
        self.accum_ppc_map += ppc
        self.ppc_steps_count += 1
        self.total_active_cells = int(np.count_nonzero(ppc > 0))
        self.low_ppc_cells = int(np.count_nonzero((ppc > 0) & (ppc < 3)))
        return remeshed, min_pot, current_div, self.T_grids, trans_last_frame

    # -- diagnostics (:1786-1878) ------------------------------------------------
    def get_total_energy_terms(self):
        """Energy sums of ``get_total_energy`` (``physics_engine.py:1800-1845``)."""
        n, ne = self.num_p, self.num_e
        ke_i = float(np.sum(self.p_vx[:n] ** 2 + self.p_vy[:n] ** 2 + self.p_vz[:n] ** 2)) * 0.5 * self.m_ion * self.macro_weight if n else 0.0
        ke_e = float(np.sum(self.e_vx[:ne] ** 2 + self.e_vy[:ne] ** 2 + self.e_vz[:ne] ** 2)) * 0.5 * self.m_e * self.macro_weight if ne else 0.0
        cell_area = (self.dx * 1e-3) * (self.dy * 1e-3)
        fe = float(np.sum(self.Ex ** 2 + self.Ey ** 2)) * 0.5 * self.eps0 * cell_area
        return ke_i, ke_e, fe

    def get_transparency(self):
        return 0.0 if self.entered_optics <= 0.0 else self.transmitted_ions / self.entered_optics
