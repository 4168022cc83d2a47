"""The skip test of the sub-step reduction (k_substep_reduce in csrc/pb_particles.cu),
restated in NumPy and checked against the displacement of compute_particle_substeps
(physics_engine.py:928-966, as the oracle computes it per particle).

A particle inside the grid, with float32 |v|^2 = v2, is passed over when
v2 < ((M (1 - 2e-4) - acc (1 + 2e-4)) / dtf)^2 (1 - 2e-4), rounded down to float32, where M
is an exact displacement already seen and acc = 0.5 |qm| Emax dt^2 with Emax the largest
float32 |Ex| + |Ey| over the nodes.  The claim is that every such particle's displacement is
below M, so the maximum is unchanged.  Here the claim is tested for many M on particle sets
where the velocity term dominates, where the acceleration term does, and in between.
"""
import numpy as np

F32 = np.float32


def _ds_each(Ex, Ey, dx, dy, nx, ny, x, y, vx, vy, vz, qm, dt):
    # the oracle's substeps(), kept per particle (same dtypes and operation order)
    ix0 = np.clip(np.floor(x / dx).astype(int), 0, nx - 2)
    iy0 = np.clip(np.floor(y / dy).astype(int), 0, ny - 2)
    fx = x / dx - ix0
    fy = y / dy - iy0

    def gather(F):
        return (F[iy0, ix0] * (1 - fx) * (1 - fy) + F[iy0, ix0 + 1] * fx * (1 - fy) +
                F[iy0 + 1, ix0] * (1 - fx) * fy + F[iy0 + 1, ix0 + 1] * fx * fy)

    a_mag = np.sqrt((qm * gather(Ex)) ** 2 + (qm * gather(Ey)) ** 2)
    v_mag = np.sqrt(vx * vx + vy * vy + vz * vz)
    return v_mag * dt + 0.5 * a_mag * dt ** 2


def _skipped(Ex, Ey, dx, dy, nx, ny, x, y, vx, vy, vz, qm, dt, M):
    emax = np.max(np.abs(Ex) + np.abs(Ey)).astype(F32)
    dtf = F32(dt)
    acc = 0.5 * abs(qm) * float(emax) * dt * dt
    R = M * (1.0 - 2e-4) - acc * (1.0 + 2e-4)
    if not R > 0.0:
        return np.zeros(x.shape, bool)
    thr = R * R / (float(dtf) * float(dtf)) * (1.0 - 2e-4)
    thr32 = F32(thr)
    if float(thr32) > thr:  # round down, as __double2float_rd
        thr32 = np.nextafter(thr32, F32(0))
    v2 = (vx * vx + vy * vy) + vz * vz  # float32, the order of the kernel
    inv_dx, inv_dy = F32(1) / F32(dx), F32(1) / F32(dy)
    inside = (x >= 0) & (y >= 0) & (x * inv_dx < F32(nx - 2)) & (y * inv_dy < F32(ny - 2))
    return (v2 < thr32) & inside


def _case(rng, scale_v, scale_e, qm, outside=False):
    nx, ny, dx, dy = 97, 41, 0.025, 0.025
    yy, xx = np.mgrid[0:ny, 0:nx]
    Ex = (scale_e * np.sin(xx / 7.0) * np.cos(yy / 5.0) + scale_e * 0.3 * rng.standard_normal((ny, nx))).astype(F32)
    Ey = (scale_e * np.cos(xx / 3.0) + scale_e * 0.3 * rng.standard_normal((ny, nx))).astype(F32)
    n = 200_000
    x = rng.uniform(0, (nx - 1) * dx, n).astype(F32)
    y = rng.uniform(0, (ny - 1) * dy, n).astype(F32)
    if outside:
        k = rng.choice(n, n // 50, replace=False)
        x[k] = rng.uniform(-(nx - 1) * dx, 2 * (nx - 1) * dx, k.size).astype(F32)
    vx, vy, vz = (rng.standard_normal((3, n)) * scale_v).astype(F32)
    return Ex, Ey, dx, dy, nx, ny, x, y, vx, vy, vz, qm, 1e-10


def test_skipped_particles_stay_below_the_running_maximum():
    rng = np.random.default_rng(3)
    qm_e = -1.602e-19 / (131.29 * 1.6605e-27 / 100)
    # (set, whether the bound is tight enough to pass over anything): where the acceleration
    # term dominates, Emax over the grid exceeds every displacement and nothing is skipped
    cases = [(_case(rng, 5e5, 1e5, qm_e), True), (_case(rng, 5e5, 1e7, qm_e), True),
             (_case(rng, 1e3, 1e8, qm_e), False), (_case(rng, 1e4, 1e6, 7.35e5), True),
             (_case(rng, 5e5, 1e6, qm_e, outside=True), True)]
    for args, expect_skips in cases:
        ds = _ds_each(*args)
        order = np.sort(ds)
        skipped_any = False
        # M taken from the exact displacements, from the median to the maximum
        for M in order[len(order) // 2::len(order) // 40]:
            sk = _skipped(*args, float(M))
            skipped_any |= bool(sk.any())
            assert not np.any(ds[sk] >= M)
        assert skipped_any == expect_skips
