"""GPU parity of the field solve and of whole timesteps.

* Field solve: the 30-iteration Picard potential of build_domain against the reference's
  SuperLU result (fixtures), |V - V_ref| <= 1e-7 max|V| and |E - E_ref| <= 1e-5 max|E|.
* One timestep given identical fields (an odd step, so no field solve inside): particles
  compared per id bit-for-bit, deposit bit-exact, counters exact, Tmap within 1e-6
  (float atomics order and the last ulp of T**4), damage within 1e-12.  Again with
  particles on and around cell boundaries and the domain edges, where the step kernels'
  exact shortcuts take their fallback branches.
* Eight timesteps with each side solving its own fields: per-id positions within 1e-4.
* The cell sort reproduces np.argsort(key, kind="stable").
"""
import json

import numpy as np
import pytest

from oracle import pic_oracle as O
from thruster_cx_code_b200.domain import build_domain_geometry
from tests.helpers import cx_store, load

pytestmark = pytest.mark.gpu

SEED = 20240611
PB_ERR_ARG = 2  # include/pbemcs.h


@pytest.fixture(scope="module")
def gpu_mod():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from thruster_cx_code_b200 import physics_engine as PE
    return PE


def _case(name):
    f = load(f"run_{name}.npz")
    return f, json.loads(str(f["case"])), json.loads(str(f["params"]))


def _pair(PE, name, sort_every=0):
    f, case, params = _case(name)
    g = PE.DigitalTwinSimulator(seed=SEED, sort_every=sort_every)
    o = O.OracleSimulator(build_domain_geometry)
    for s in (g, o):
        s.dx, s.dy, s.dt = case["dx"], case["dy"], case["dt"]
        if "cx_table" in case:
            s.user_cs = cx_store(case["cx_table"])
    g.build_domain(params)
    o.build_domain(params)
    p, cex, e = f["init_p"], f["init_p_cex"], f["init_e"]
    n, ne = p.shape[1], e.shape[1]
    g.set_particles("ions", *p.astype(np.float32), is_cex=cex, ids=np.arange(n), sort=False)
    o._add_ions(*p, cex, o.new_ion_ids(n))
    if ne:
        g.set_particles("electrons", *e.astype(np.float32), ids=np.arange(ne), sort=False)
        o._add_electrons(*e, o.new_e_ids(ne))
    return g, o, params


def _by_id(x, ids):
    order = np.argsort(ids, kind="stable")
    return x[..., order], ids[order]


def _ions(sim):
    n = sim.num_p
    a = np.stack([np.asarray(sim.p_x[:n]), np.asarray(sim.p_y[:n]), np.asarray(sim.p_vx[:n]),
                  np.asarray(sim.p_vy[:n]), np.asarray(sim.p_vz[:n])]).astype(np.float32)
    return a, np.asarray(sim.p_isCEX[:n]).astype(bool), np.asarray(sim.p_id[:n]).astype(np.int64)


def _eles(sim):
    n = sim.num_e
    a = np.stack([np.asarray(sim.e_x[:n]), np.asarray(sim.e_y[:n]), np.asarray(sim.e_vx[:n]),
                  np.asarray(sim.e_vy[:n]), np.asarray(sim.e_vz[:n])]).astype(np.float32)
    return a, np.asarray(sim.e_id[:n]).astype(np.int64)


@pytest.mark.parametrize("nu", [1, 2])
@pytest.mark.parametrize("name", ["c1_half", "one_hole", "two_holes", "bulk"])
def test_picard_potential_matches_superlu(gpu_mod, name, nu):
    """nu: damped-Jacobi sweeps on the fine level on each side of the coarse correction
    (the autotuner's smoother knob); the solve meets the same tolerance either way."""
    f = load(f"domain_{name}.npz")
    case = json.loads(str(f["case"]))
    params = json.loads(str(f["params"]))
    g = gpu_mod.DigitalTwinSimulator(solver={"nu": nu})
    g.dx, g.dy, g.dt = case["dx"], case["dy"], case["dt"]
    g.build_domain(params)
    assert (g.ny, g.nx) == f["V"].shape
    np.testing.assert_array_equal(g.isBound, f["isBound"])
    V, Vref = g.V, f["V"]
    errV = np.abs(V - Vref).max() / np.abs(Vref).max()
    assert errV <= 1e-7, errV
    for k in ("Ex", "Ey"):
        E, Eref = getattr(g, k).astype(np.float64), f[k].astype(np.float64)
        err = np.abs(E - Eref).max() / np.abs(Eref).max()
        assert err <= 1e-5, (k, err)
    assert g.poisson_stats[2] <= 1e-8  # final relative FP64 residual of the last solve (solver tol)
    # thermal-bow rebuild keeps state and re-solves
    g.grid_deflections = [0.012 * (i + 1) for i in range(len(params["grids"]))]
    g.build_domain(params, preserve_state=True)
    np.testing.assert_array_equal(g.isBound, f["bow_isBound"])
    assert np.abs(g.V - f["bow_V"]).max() / np.abs(f["bow_V"]).max() <= 1e-7


@pytest.mark.parametrize("name", ["c1_both", "two_holes_thermal"])
def test_one_step_bit_exact_given_fields(gpu_mod, name):
    g, o, params = _pair(gpu_mod, name)
    # identical fields on both sides (the step is odd: no field solve inside)
    g.V, g.Ex, g.Ey = o.V, o.Ex, o.Ey
    rg = g.step(params)
    ro = o.step(params, O.PhiloxDraws(SEED))
    assert g.num_p == o.num_p and g.num_e == o.num_e
    np.testing.assert_array_equal(g.rho, o.rho)
    ag, cg, ig = _ions(g)
    ao, co, io = _ions(o)
    # stable compaction: the survivors keep the oracle's array order (no cell sort here)
    np.testing.assert_array_equal(ig, io)
    ag, ig2 = _by_id(ag, ig)
    ao, io2 = _by_id(ao, io)
    np.testing.assert_array_equal(ig2, io2)
    np.testing.assert_array_equal(ag.view(np.uint32), ao.view(np.uint32))
    np.testing.assert_array_equal(cg[np.argsort(ig, kind="stable")], co[np.argsort(io, kind="stable")])
    eg, jg = _eles(g)
    eo, jo = _eles(o)
    np.testing.assert_array_equal(jg, jo)
    eg, jg2 = _by_id(eg, jg)
    eo, jo2 = _by_id(eo, jo)
    np.testing.assert_array_equal(jg2, jo2)
    np.testing.assert_array_equal(eg.view(np.uint32), eo.view(np.uint32))
    assert bool(rg[0]) == bool(ro[0])
    assert rg[1] == ro[1]
    if np.isnan(ro[2]):
        assert np.isnan(rg[2])
    else:
        assert abs(rg[2] - ro[2]) <= 1e-5 * abs(ro[2])
    np.testing.assert_allclose(np.array(rg[3], float), np.array(ro[3], float), rtol=1e-6)
    assert rg[4] == ro[4]
    np.testing.assert_allclose(g.Tmap, o.Tmap, rtol=1e-6)
    np.testing.assert_allclose(g.damage_map, o.damage_map, rtol=1e-12, atol=0)
    np.testing.assert_array_equal(g.isBound, o.isBound)
    assert g.transmitted_ions == o.transmitted_ions and g.entered_optics == o.entered_optics


def _edge_particles(g, n, rng):
    """Positions on exact cell boundaries k * dx (float32), one ulp either side, at zero,
    just outside the domain and on the far edges, paired over x and y; velocities small,
    zero or mixed in sign.  They reach the fallback branches of the step kernels' exact
    shortcuts (checked division, round-down floor, quotient reuse, periodic wrap)."""
    dx, dy = np.float32(g.dx), np.float32(g.dy)
    Lx, Ly = np.float32(g.Lx), np.float32(g.Ly)

    def edges(d, m, L):
        b = np.array([k * d for k in (0, 1, 2, m // 2, m - 2, m - 1)], np.float32)
        b = np.concatenate([b, np.nextafter(b, np.float32(np.inf)), np.nextafter(b, np.float32(-np.inf)),
                            np.array([-1e-6, L, np.nextafter(L, np.float32(np.inf)), L + d], np.float32)])
        return b

    xs, ys = edges(dx, g.nx, Lx), edges(dy, g.ny, Ly)
    X, Y = np.meshgrid(xs, ys, indexing="ij")
    X, Y = X.ravel(), Y.ravel()
    k = rng.choice(X.size, size=min(n, X.size), replace=False)
    X, Y = X[k], Y[k]
    v = rng.choice(np.array([0.0, 1.0, -1.0], np.float32), size=(3, X.size)).astype(np.float32)
    return X, Y, v


@pytest.mark.parametrize("name", ["c1_both", "two_holes_thermal"])
def test_one_step_bit_exact_at_cell_boundaries(gpu_mod, name):
    """One step, identical fields, with particles placed on and around cell boundaries and
    the domain edges appended to the case's own: per-id state bit-exact."""
    f, case, params = _case(name)
    PE = gpu_mod
    g = PE.DigitalTwinSimulator(seed=SEED, sort_every=0)
    o = O.OracleSimulator(build_domain_geometry)
    for s in (g, o):
        s.dx, s.dy, s.dt = case["dx"], case["dy"], case["dt"]
        if "cx_table" in case:
            s.user_cs = cx_store(case["cx_table"])
    g.build_domain(params)
    o.build_domain(params)
    rng = np.random.default_rng(3)
    p = f["init_p"].astype(np.float32)
    e = f["init_e"].astype(np.float32)
    xi, yi, vi = _edge_particles(g, 150, rng)
    xe, ye, ve = _edge_particles(g, 150, rng)
    pi = np.concatenate([p, np.stack([xi, yi, 2e3 * vi[0] + 1e3, 2e3 * vi[1], 2e3 * vi[2]]).astype(np.float32)], axis=1)
    pe = np.concatenate([e, np.stack([xe, ye, 3e5 * ve[0], 3e5 * ve[1], 3e5 * ve[2]]).astype(np.float32)], axis=1)
    cex = np.concatenate([f["init_p_cex"], np.zeros(xi.size, bool)])
    n, ne = pi.shape[1], pe.shape[1]
    g.set_particles("ions", *pi, is_cex=cex, ids=np.arange(n), sort=False)
    g.set_particles("electrons", *pe, ids=np.arange(ne), sort=False)
    o._add_ions(*pi, cex, o.new_ion_ids(n))
    o._add_electrons(*pe, o.new_e_ids(ne))
    g.V, g.Ex, g.Ey = o.V, o.Ex, o.Ey
    g.step(params)
    o.step(params, O.PhiloxDraws(SEED))
    assert g.num_p == o.num_p and g.num_e == o.num_e
    np.testing.assert_array_equal(g.rho, o.rho)
    ag, _, ig = _ions(g)
    ao, _, io = _ions(o)
    np.testing.assert_array_equal(ig, io)
    np.testing.assert_array_equal(ag.view(np.uint32), ao.view(np.uint32))
    eg, jg = _eles(g)
    eo, jo = _eles(o)
    np.testing.assert_array_equal(jg, jo)
    np.testing.assert_array_equal(eg.view(np.uint32), eo.view(np.uint32))
    np.testing.assert_array_equal(g.current_ppc_map, o.current_ppc_map)


@pytest.mark.parametrize("name", ["c1_both", "one_hole_rf", "two_holes_thermal"])
def test_eight_steps_close(gpu_mod, name):
    g, o, params = _pair(gpu_mod, name)
    draws = O.PhiloxDraws(SEED)
    outs_g, outs_o = [], []
    for _ in range(8):
        outs_g.append(g.step(params))
        outs_o.append(o.step(params, draws))
    assert abs(g.num_p - o.num_p) <= max(2, 0.002 * o.num_p)
    assert abs(g.num_e - o.num_e) <= max(2, 0.002 * o.num_e)
    ag, _, ig = _ions(g)
    ao, _, io = _ions(o)
    common, a_i, b_i = np.intersect1d(ig, io, return_indices=True)
    assert common.size >= 0.99 * min(ig.size, io.size)
    d = np.abs(ag[:, a_i].astype(np.float64) - ao[:, b_i].astype(np.float64))
    scale = np.abs(ao[:, b_i]).astype(np.float64).max(axis=1, keepdims=True)
    assert (d / scale).max() <= 1e-4
    errV = np.abs(g.V - o.V).max() / np.abs(o.V).max()
    assert errV <= 1e-6, errV
    for a, b in zip(outs_g, outs_o):
        assert abs(a[1] - b[1]) <= 1e-6 * abs(b[1])


def test_cell_sort_is_stable_argsort(gpu_mod):
    ga, _, params = _pair(gpu_mod, "c1_both", sort_every=0)
    gb, _, _ = _pair(gpu_mod, "c1_both", sort_every=1)
    for s in (ga, gb):
        s.V = ga.V
    ga.step(params)
    gb.step(params)
    a, ca, ia = _ions(ga)
    b, cb, ib = _ions(gb)
    nx, ny = ga.nx, ga.ny
    dx, dy = np.float32(ga.dx), np.float32(ga.dy)
    ix = np.clip(np.round(a[0] / dx).astype(np.int32), 1, nx - 2)
    iy = np.clip(np.round(a[1] / dy).astype(np.int32), 1, ny - 2)
    perm = np.argsort(iy.astype(np.int64) * nx + ix, kind="stable")
    np.testing.assert_array_equal(b.view(np.uint32), a[:, perm].view(np.uint32))
    np.testing.assert_array_equal(ib, ia[perm])
    np.testing.assert_array_equal(cb, ca[perm])


def test_upload_sort_is_stable_argsort(gpu_mod):
    g, _, params = _pair(gpu_mod, "c1_both")
    a, ca, ia = _ions(g)
    g.set_particles("ions", *a, is_cex=ca, ids=ia, sort=True)
    b, cb, ib = _ions(g)
    nx, ny = g.nx, g.ny
    dx, dy = np.float32(g.dx), np.float32(g.dy)
    ix = np.clip(np.round(a[0] / dx).astype(np.int32), 1, nx - 2)
    iy = np.clip(np.round(a[1] / dy).astype(np.int32), 1, ny - 2)
    perm = np.argsort(iy.astype(np.int64) * nx + ix, kind="stable")
    np.testing.assert_array_equal(b.view(np.uint32), a[:, perm].view(np.uint32))
    np.testing.assert_array_equal(ib, ia[perm])
    np.testing.assert_array_equal(cb, ca[perm])


def test_bad_step_params_rejected(gpu_mod):
    """Indices the kernels dereference are checked before anything of the step is enqueued:
    the call fails and the simulator keeps stepping."""
    import ctypes as C
    from thruster_cx_code_b200 import _lib
    g, _, params = _pair(gpu_mod, "c1_both")
    lib = _lib.load()
    n0 = g.num_p
    for field, value in (("saddle_idx", 10 ** 9), ("rf_grid", 40)):
        P = g.step_params(params)
        if field == "saddle_idx":
            P.n_saddle = 1
            P.saddle_idx[0] = value
        else:
            P.rf_grid = value
        rep = _lib.StepReport()
        assert lib.pb_sim_step(g._h, C.byref(P), C.byref(rep)) == PB_ERR_ARG
    assert g.num_p == n0
    g.step(params)
    assert g.num_p > 0
    g.close()
