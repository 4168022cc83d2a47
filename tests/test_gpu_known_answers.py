"""Known-answer tests: the reference's two test scripts, restated with assertions.

* Python/tests/particle_push_test.py:4-106: a Xe+ ion in a uniform Bz = 0.5 T with E = 0,
  v0 = 1e4 m/s, dt = 1e-9 s, 20 000 Boris pushes.  The orbit is the Larmor circle
  r = m v0 / (q B) (27.2 mm).  Asserted: final radius error below 0.1% (the Boris rotation
  preserves |v|), and speed preserved to float32 rounding.
* Python/tests/poisson_solver_test.py:6-134: the manufactured solution
  V = sin(pi x / L) sin(pi y / L), L = 20 mm, rho = 2 eps0 k^2 V (k = pi / L), on a square
  with Dirichlet edges, at dx = 0.25, 0.125, 0.1, 0.05 mm, solved to a relative residual
  of 1e-10.  Asserted: the RMS error of the linear solve falls with a fitted order of
  2 +- 0.1 (second-order five-point stencil).
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def test_larmor_circle(torch_cuda):
    torch = torch_cuda
    from thruster_cx_code_b200.physics_engine import push_particles_boris
    q, m = 1.602e-19, 131.293 * 1.6605e-27
    Bz, dt, steps, v0 = 0.5, 1e-9, 20000, 1e4
    r_mm = m * v0 / (q * Bz) * 1e3
    nx = ny = 64
    dev = torch.device("cuda")
    zeros = torch.zeros(ny, nx, dtype=torch.float32, device=dev)
    bz = torch.full((ny, nx), Bz, dtype=torch.float32, device=dev)
    x0, y0 = 32.0, 60.0  # orbit centre (32, 60 - r): the circle stays inside the 63 x 63 mm grid
    x = torch.tensor([x0], dtype=torch.float32, device=dev)
    y = torch.tensor([y0], dtype=torch.float32, device=dev)
    vx = torch.tensor([v0], dtype=torch.float32, device=dev)
    vy = torch.zeros(1, dtype=torch.float32, device=dev)
    vz = torch.zeros(1, dtype=torch.float32, device=dev)
    for _ in range(steps):
        push_particles_boris(x, y, vx, vy, vz, zeros, zeros, zeros, zeros, bz, 1, 1.0, 1.0, nx, ny, dt, q / m)
    torch.cuda.synchronize()
    xf, yf = float(x.item()), float(y.item())
    radius = np.hypot(xf - x0, yf - (y0 - r_mm))
    assert abs(radius - r_mm) / r_mm < 1e-3
    speed = np.sqrt(vx.item() ** 2 + vy.item() ** 2 + vz.item() ** 2)
    assert abs(speed - v0) / v0 < 1e-4
    # the ion turned through omega t = q B t / m rad: check the phase of the final point
    omega_t = q * Bz / m * steps * dt
    xe, ye = x0 + r_mm * np.sin(omega_t), (y0 - r_mm) + r_mm * np.cos(omega_t)
    assert np.hypot(xf - xe, yf - ye) < 1e-3 * r_mm


def _manufactured_rms(lib, _lib, dx):
    L = 20.0
    n = int(round(L / dx)) + 1
    eps0 = 8.854e-12
    k = np.pi / (L * 1e-3)
    xs = np.arange(n) * dx
    X, Y = np.meshgrid(xs, xs)
    V_exact = np.sin(np.pi * X / L) * np.sin(np.pi * Y / L)
    rho = (2.0 * eps0 * k * k * V_exact).astype(np.float32)
    isB = np.zeros((n, n), np.uint8)
    isB[0, :] = isB[-1, :] = isB[:, 0] = isB[:, -1] = 1
    Vf = np.zeros((n, n), np.float64)
    h = C.c_void_p()
    _lib.check(lib.pb_sim_create(C.byref(h), 0), "create")
    try:
        # 1e-10: below that the FP64 residual of this problem reaches its rounding floor
        # (the right-hand side scales as (k dx)^2 against O(1) operator terms)
        _lib.check(lib.pb_sim_set_solver(h, 1e-10, 1e-5, 12, 60, 1, 256), "solver")
        p = lambda a: a.ctypes.data_as(C.c_void_p)
        _lib.check(lib.pb_sim_set_domain(h, n, n, 0, p(isB), p(Vf), None, 0, None, None, None, None, 0), "domain")
        _lib.check(lib.pb_sim_set_field(h, 3, p(rho), rho.nbytes), "rho")
        P = _lib.StepParams()
        hx = dx * 1e-3
        P.coeff = hx * hx / eps0
        P.qn0_neg = 0.0  # no Boltzmann electrons: a linear problem
        P.V_plasma, P.Te_up = 0.0, 1.0
        P.omega_keep, P.omega_new = 0.8, 0.2
        P.hx, P.two_hx, P.hy, P.two_hy, P.two_hy_per = hx, 2 * hx, hx, 2 * hx, 2 * hx
        stats = (C.c_double * 4)()
        _lib.check(lib.pb_sim_poisson(h, 1, C.byref(P), stats), "poisson")
        Vn = np.empty((n, n), np.float64)
        _lib.check(lib.pb_sim_get_field(h, 11, p(Vn), Vn.nbytes), "Vnew")  # the linear solution
    finally:
        lib.pb_sim_destroy(h)
    inner = (slice(1, -1), slice(1, -1))
    return float(np.sqrt(np.mean((Vn[inner] - V_exact[inner]) ** 2))), stats[2]


def test_poisson_manufactured_second_order(torch_cuda):
    from thruster_cx_code_b200 import _lib
    lib = _lib.load()
    dxs = [0.25, 0.125, 0.1, 0.05]
    errs = []
    for dx in dxs:
        e, rel = _manufactured_rms(lib, _lib, dx)
        assert rel <= 1e-10
        errs.append(e)
    slope = np.polyfit(np.log(dxs), np.log(errs), 1)[0]
    assert 1.9 <= slope <= 2.1, (errs, slope)
