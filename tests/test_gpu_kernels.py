"""GPU parity of the kernel-level entry points against fixtures made by the reference.

Bit-exact: push (1 and 3 sub-steps, zero and random B), NGP deposit, sub-step count,
path absorption.  The inputs include particles on nodes, outside the box, NaN and inf.
"""
import json

import numpy as np
import pytest

from oracle import pic_oracle as O
from tests.helpers import load

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def same_bits(a, b):
    """Bit equality, with every NaN equal to every NaN (CUDA writes the canonical NaN,
    NumPy propagates the payload of its input)."""
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    assert a.shape == b.shape and a.dtype == b.dtype
    if a.dtype.kind != "f":
        return np.array_equal(a, b)
    na, nb = np.isnan(a), np.isnan(b)
    if not np.array_equal(na, nb):
        return False
    ib = np.uint32 if a.dtype == np.float32 else np.uint64
    return np.array_equal(a.view(ib)[~na], b.view(ib)[~nb])


@pytest.mark.parametrize("tag", ["ion", "ele"])
@pytest.mark.parametrize("btag", ["B0", "Br"])
@pytest.mark.parametrize("nsub", [1, 3])
def test_push_bit_exact(torch_cuda, tag, btag, nsub):
    torch = torch_cuda
    from thruster_cx_code_b200.physics_engine import push_particles_boris
    f = load("push.npz")
    d = load("domain_c1_half.npz")
    nx, ny, dx, dy = int(d["nx"]), int(d["ny"]), float(d["dx"]), float(d["dy"])
    dev = torch.device("cuda", 0)
    arr = [torch.tensor(np.ascontiguousarray(v), device=dev) for v in f[f"{tag}_in"]]
    Ex = torch.tensor(d["Ex"], device=dev)
    Ey = torch.tensor(d["Ey"], device=dev)
    if btag == "B0":
        B = [torch.zeros((ny, nx), dtype=torch.float32, device=dev) for _ in range(3)]
    else:
        B = [torch.tensor(f[k], device=dev) for k in ("Bx", "By", "Bz")]
    dt, qm = float(f[f"{tag}_dt"]), float(f[f"{tag}_qm"])
    n = arr[0].numel()
    for _ in range(nsub):
        push_particles_boris(*arr, Ex, Ey, *B, n, dx, dy, nx, ny, dt / nsub, qm)
    torch.cuda.synchronize()
    got = np.stack([a.cpu().numpy() for a in arr])
    assert same_bits(got, f[f"{tag}_{btag}_sub{nsub}"])


def test_deposit_bit_exact(torch_cuda):
    torch = torch_cuda
    from thruster_cx_code_b200.physics_engine import accumulate_rho
    f = load("deposit.npz")
    d = load("domain_c1_half.npz")
    nx, ny, dx, dy = int(d["nx"]), int(d["ny"]), float(d["dx"]), float(d["dy"])
    dev = torch.device("cuda", 0)
    rho = torch.zeros((ny, nx), dtype=torch.float32, device=dev)
    xi, yi = torch.tensor(f["xi"], device=dev), torch.tensor(f["yi"], device=dev)
    xe, ye = torch.tensor(f["xe"], device=dev), torch.tensor(f["ye"], device=dev)
    cd = float(f["cd"])
    accumulate_rho(xi, yi, rho, xi.numel(), dx, dy, nx, ny, cd)
    torch.cuda.synchronize()
    assert same_bits(rho.cpu().numpy(), f["rho_ions"])
    accumulate_rho(xe, ye, rho, xe.numel(), dx, dy, nx, ny, -cd)
    torch.cuda.synchronize()
    assert same_bits(rho.cpu().numpy(), f["rho"])
    # the crowded cells (20000 ions, 7000 + 3000 electrons) are the ones that exercise
    # the run-length summation; make sure they are nonzero and were compared
    assert np.count_nonzero(f["rho"]) > 1000


def test_substeps_exact(torch_cuda):
    import ctypes as C
    torch = torch_cuda
    from thruster_cx_code_b200 import _lib
    lib = _lib.load()
    f = load("substeps.npz")
    d = load("domain_c1_half.npz")
    nx, ny, dx, dy = int(d["nx"]), int(d["ny"]), float(d["dx"]), float(d["dy"])
    dev = torch.device("cuda", 0)
    Ex = torch.tensor(d["Ex"], device=dev)
    Ey = torch.tensor(d["Ey"], device=dev)
    for tag in ("ion", "ele"):
        t = [torch.tensor(np.ascontiguousarray(v), device=dev) for v in f[f"{tag}_in"]]
        out = (C.c_double * 3)()
        _lib.check(lib.pb_compute_particle_substeps(*[a.data_ptr() for a in t], t[0].numel(), Ex.data_ptr(),
                                                    Ey.data_ptr(), nx, ny, dx, dy, float(f[f"{tag}_qm"]), 1e-10,
                                                    0.25, out, None), "substeps")
        res = f[f"{tag}_res"]
        assert int(out[0]) == int(res[0])
        assert out[1] == res[1] and out[2] == res[2]
        # the same particles in arrays that start 4 bytes past a 16-byte boundary
        # (the kernel's 16-byte loads do not apply there)
        tm = [torch.zeros(a.numel() + 1, dtype=a.dtype, device=dev) for a in t]
        for a, b in zip(tm, t):
            a[1:] = b
        _lib.check(lib.pb_compute_particle_substeps(*[a[1:].data_ptr() for a in tm], t[0].numel(), Ex.data_ptr(),
                                                    Ey.data_ptr(), nx, ny, dx, dy, float(f[f"{tag}_qm"]), 1e-10,
                                                    0.25, out, None), "substeps, unaligned")
        assert int(out[0]) == int(res[0])
        assert out[1] == res[1] and out[2] == res[2]


def test_substeps_skip_equals_full(torch_cuda):
    """The reduction passes over particles whose displacement provably stays below one
    already seen (16-byte aligned arrays); the same particles 4 bytes past a 16-byte
    boundary take the full loop.  Both give the same n_sub and ds_max bits on sets built
    against the bound: a fast particle late in the array, fields large enough that the
    acceleration term dominates, positions outside the grid (clamped cells extrapolate the
    field), all velocities zero, and a NaN velocity."""
    import ctypes as C
    import struct
    torch = torch_cuda
    from thruster_cx_code_b200 import _lib
    lib = _lib.load()
    d = load("domain_c1_half.npz")
    nx, ny, dx, dy = int(d["nx"]), int(d["ny"]), float(d["dx"]), float(d["dy"])
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(21)
    n = 300_000
    Lx, Ly = (nx - 1) * dx, (ny - 1) * dy

    def run(cols, ex, ey, qm):
        Ex = torch.tensor(ex.astype(np.float32), device=dev)
        Ey = torch.tensor(ey.astype(np.float32), device=dev)
        res = []
        for off in (0, 1):
            t = [torch.zeros(n + 1, dtype=torch.float32, device=dev) for _ in cols]
            for a, c in zip(t, cols):
                a[off:off + n] = torch.tensor(c.astype(np.float32), device=dev)
            out = (C.c_double * 3)()
            _lib.check(lib.pb_compute_particle_substeps(*[a[off:].data_ptr() for a in t], n, Ex.data_ptr(),
                                                        Ey.data_ptr(), nx, ny, dx, dy, qm, 1e-10, 0.25, out, None),
                       "substeps")
            res.append((out[0], struct.pack("<d", out[1])))
        return res

    x = rng.uniform(0.0, Lx, n)
    y = rng.uniform(0.0, Ly, n)
    Ex0, Ey0 = np.asarray(d["Ex"], np.float64), np.asarray(d["Ey"], np.float64)
    qm_i, qm_e = 1.602e-19 / (131.29 * 1.6605e-27), -1.602e-19 / (131.29 * 1.6605e-27 / 100)
    cases = []
    v = rng.normal(0.0, 1e4, (3, n))
    cases.append(("ions", [x, y, *v], Ex0, Ey0, qm_i))
    ve = rng.normal(0.0, 5e5, (3, n))
    ve[:, n - 5] *= 10.0
    cases.append(("fast electron late", [x, y, *ve], Ex0, Ey0, qm_e))
    cases.append(("acceleration dominates", [x, y, *ve], Ex0 * 1e4, Ey0 * 1e4, qm_e))
    xo, yo = x.copy(), y.copy()
    k = rng.choice(n, n // 100, replace=False)
    xo[k] = rng.uniform(-Lx, 2 * Lx, k.size)
    yo[k] = rng.uniform(-Ly, 2 * Ly, k.size)
    cases.append(("outside the grid", [xo, yo, *ve], Ex0 * 1e3, Ey0 * 1e3, qm_e))
    z = np.zeros(n)
    cases.append(("no velocity", [x, y, z, z, z], Ex0, Ey0, qm_i))
    vn = ve.copy()
    vn[0, n - 1] = np.nan
    cases.append(("NaN velocity", [x, y, *vn], Ex0, Ey0, qm_e))
    for name, cols, ex, ey, qm in cases:
        skip, full = run(cols, ex, ey, qm)
        assert skip == full, name


def test_segment_hits_exact(torch_cuda):
    torch = torch_cuda
    from thruster_cx_code_b200 import _lib
    lib = _lib.load()
    f = load("segment.npz")
    d = load("domain_c1_half.npz")
    nx, ny, dx, dy = int(d["nx"]), int(d["ny"]), float(d["dx"]), float(d["dy"])
    dev = torch.device("cuda", 0)
    isb = torch.tensor(d["isBound"].astype(np.uint8), device=dev)
    t = [torch.tensor(f[k], device=dev) for k in ("x0", "y0", "x1", "y1")]
    n = t[0].numel()
    hit = torch.empty(n, dtype=torch.uint8, device=dev)
    hx = torch.empty(n, dtype=torch.int64, device=dev)
    hy = torch.empty(n, dtype=torch.int64, device=dev)
    _lib.check(lib.pb_segment_hits_grid(isb.data_ptr(), nx, ny, dx, dy, *[a.data_ptr() for a in t], n, hit.data_ptr(),
                                        hx.data_ptr(), hy.data_ptr(), None), "segment")
    torch.cuda.synchronize()
    np.testing.assert_array_equal(hit.cpu().numpy().astype(bool), f["hit"])
    np.testing.assert_array_equal(hx.cpu().numpy(), f["hix"])
    np.testing.assert_array_equal(hy.cpu().numpy(), f["hiy"])


def test_thermal_conduction_taichi_semantics(torch_cuda):
    torch = torch_cuda
    from thruster_cx_code_b200.physics_engine import thermal_conduction
    d = load("domain_c1_half.npz")
    isB = d["isBound"]
    ny, nx = isB.shape
    rs = np.random.RandomState(4)
    T = np.where(isB, 300 + rs.rand(ny, nx) * 900, 300.0).astype(np.float32)
    dev = torch.device("cuda", 0)
    Tg = torch.tensor(T, device=dev)
    Tn = torch.empty_like(Tg)
    mask = torch.tensor(isB.astype(np.int32), device=dev)
    thermal_conduction(Tg, Tn, mask, nx, ny, 0.2, 0.17)
    torch.cuda.synchronize()
    exp = O.thermal_taichi_sweep(T, isB, 0.2, 0.17)
    assert same_bits(Tn.cpu().numpy(), exp)
