"""The allocation-free deposit entry point, through the C-ABI.

pb_accumulate_rho_noalloc exists for callers that cannot allocate device memory when
they deposit charge: a host application whose device memory is already reserved by
another framework's pool, a real-time loop that has to stay off the driver's allocation
path, or a process with a device-memory budget fixed at start-up.  It keeps its count
scratch in a static device array of 2^21 cells instead of allocating.

The test compares it with the regular pb_accumulate_rho bit for bit (the tolerance all
deposit tests use) on two calls in a row on the same rho, ions then electrons, and
against the reference's deposit fixture; it also checks that a grid above the array's
size is refused before any work.  This file is collected last so that a failure here
leaves every other test already run.
"""
import numpy as np
import pytest

from tests.helpers import load

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def test_noalloc_deposit_matches_regular_entry_point(torch_cuda):
    torch = torch_cuda
    from thruster_cx_code_b200 import _lib
    lib = _lib.load()
    f = load("deposit.npz")
    d = load("domain_c1_half.npz")
    nx, ny, dx, dy = int(d["nx"]), int(d["ny"]), float(d["dx"]), float(d["dy"])
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev).cuda_stream
    cd = float(f["cd"])
    calls = [(f["xi"], f["yi"], cd), (f["xe"], f["ye"], -cd)]
    rho_a = torch.zeros((ny, nx), dtype=torch.float32, device=dev)
    rho_b = torch.zeros((ny, nx), dtype=torch.float32, device=dev)
    for x, y, c in calls:
        xt, yt = torch.tensor(x, device=dev), torch.tensor(y, device=dev)
        _lib.check(lib.pb_accumulate_rho(xt.data_ptr(), yt.data_ptr(), rho_a.data_ptr(), xt.numel(), dx, dy, nx, ny,
                                         c, stream), "accumulate_rho")
        _lib.check(lib.pb_accumulate_rho_noalloc(xt.data_ptr(), yt.data_ptr(), rho_b.data_ptr(), xt.numel(), dx, dy,
                                                 nx, ny, c, stream), "accumulate_rho_noalloc")
        torch.cuda.synchronize()
        a, b = rho_a.cpu().numpy(), rho_b.cpu().numpy()
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert np.array_equal(rho_b.cpu().numpy(), f["rho"])


def test_noalloc_rejects_grids_above_its_scratch(torch_cuda):
    torch = torch_cuda
    from thruster_cx_code_b200 import _lib
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    x = torch.zeros(4, dtype=torch.float32, device=dev)
    rho = torch.zeros(1, dtype=torch.float32, device=dev)  # never touched: the call is refused first
    rc = lib.pb_accumulate_rho_noalloc(x.data_ptr(), x.data_ptr(), rho.data_ptr(), 4, 0.01, 0.01, 2049, 1025, 1.0,
                                       None)
    assert rc == 2
    assert b"exceeds" in lib.pb_last_error()
