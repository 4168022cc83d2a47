"""The module kernels as PyTorch operators (torch.ops.pbemcs.*) against the reference's
fixtures, bit for bit: the same deposit, push and thermal cases as tests/test_gpu_kernels.py,
called through the dispatcher instead of the Python functions."""
import numpy as np
import pytest

from oracle import pic_oracle as O
from tests.helpers import load
from tests.test_gpu_kernels import same_bits

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ops():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import thruster_cx_code_b200.torch_ops  # noqa: F401  (registers torch.ops.pbemcs)
    return torch, torch.ops.pbemcs


def test_op_deposit_bit_exact(ops):
    torch, pb = ops
    f = load("deposit.npz")
    d = load("domain_c1_half.npz")
    nx, ny, dx, dy = int(d["nx"]), int(d["ny"]), float(d["dx"]), float(d["dy"])
    dev = torch.device("cuda", 0)
    rho = torch.zeros((ny, nx), dtype=torch.float32, device=dev)
    xi, yi = torch.tensor(f["xi"], device=dev), torch.tensor(f["yi"], device=dev)
    xe, ye = torch.tensor(f["xe"], device=dev), torch.tensor(f["ye"], device=dev)
    cd = float(f["cd"])
    pb.accumulate_rho(xi, yi, rho, xi.numel(), dx, dy, nx, ny, cd)
    pb.accumulate_rho(xe, ye, rho, xe.numel(), dx, dy, nx, ny, -cd)
    torch.cuda.synchronize()
    assert same_bits(rho.cpu().numpy(), f["rho"])


@pytest.mark.parametrize("tag", ["ion", "ele"])
def test_op_push_bit_exact(ops, tag):
    torch, pb = ops
    f = load("push.npz")
    d = load("domain_c1_half.npz")
    nx, ny, dx, dy = int(d["nx"]), int(d["ny"]), float(d["dx"]), float(d["dy"])
    dev = torch.device("cuda", 0)
    arr = [torch.tensor(np.ascontiguousarray(v), device=dev) for v in f[f"{tag}_in"]]
    Ex, Ey = torch.tensor(d["Ex"], device=dev), torch.tensor(d["Ey"], device=dev)
    B = [torch.tensor(f[k], device=dev) for k in ("Bx", "By", "Bz")]
    dt, qm = float(f[f"{tag}_dt"]), float(f[f"{tag}_qm"])
    n = arr[0].numel()
    for _ in range(3):
        pb.push_particles_boris(*arr, Ex, Ey, *B, n, dx, dy, nx, ny, dt / 3, qm)
    torch.cuda.synchronize()
    assert same_bits(np.stack([a.cpu().numpy() for a in arr]), f[f"{tag}_Br_sub3"])


def test_op_thermal_bit_exact(ops):
    torch, pb = ops
    d = load("domain_c1_half.npz")
    isB = d["isBound"]
    ny, nx = isB.shape
    rs = np.random.RandomState(4)
    T = np.where(isB, 300 + rs.rand(ny, nx) * 900, 300.0).astype(np.float32)
    dev = torch.device("cuda", 0)
    Tg = torch.tensor(T, device=dev)
    Tn = torch.empty_like(Tg)
    pb.thermal_conduction(Tg, Tn, torch.tensor(isB.astype(np.int32), device=dev), nx, ny, 0.2, 0.17)
    torch.cuda.synchronize()
    assert same_bits(Tn.cpu().numpy(), O.thermal_taichi_sweep(T, isB, 0.2, 0.17))


def test_op_refuses_wrong_dtype(ops):
    torch, pb = ops
    dev = torch.device("cuda", 0)
    x = torch.zeros(4, dtype=torch.float64, device=dev)
    rho = torch.zeros((4, 4), dtype=torch.float32, device=dev)
    with pytest.raises(RuntimeError):
        pb.accumulate_rho(x, x, rho, 4, 0.1, 0.1, 4, 4, 1.0)
