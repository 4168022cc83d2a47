"""The bracketed division of the step kernels against IEEE float32 division.

Every sub-step of the ion and electron pushes needs the float32 quotients x / dx and
y / dy, bit-equal to NumPy's division.  The kernels form q0 = RN(x RN(1/d)) and its FMA
residual r0, correct q0 once with each of the two floats two steps below and above RN(1/d),
and accept the quotient when both corrections round to the same float (the exact quotient
lies between them); otherwise they take the division instruction.

pb_check_division runs that test over all 2^32 float32 values of x for one spacing and
counts the accepted quotients that differ from __fdiv_rn.  There must be none, for the
benchmarked spacings, the sweep spacings and spacings chosen to be awkward (mantissas of
all ones, just above a power of two, reciprocals of exact powers of two), and nearly all
in-grid positions must be accepted.  That the kernels give the oracle's bits with it is
shown by the step parity tests (tests/test_gpu_step.py, tests/test_gpu_large.py)."""
import ctypes as C
import struct

import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from thruster_cx_code_b200 import _lib
    return _lib.load()


def _check(lib, d):
    from thruster_cx_code_b200 import _lib
    out = (C.c_int64 * 3)()
    _lib.check(lib.pb_check_division(d, out), "pb_check_division")
    return out[0], out[1], out[2]


def _f32(bits):
    return struct.unpack("<f", struct.pack("<I", bits))[0]


def _spacings():
    from thruster_cx_code_b200 import workloads
    d = {w["dx"] for w in workloads.WORKLOADS.values()} | set(workloads.SWEEP_SPACINGS.values())
    d |= {0.02, 0.01, 0.005, 0.1, 0.3, 0.7, 3.0, 0.5, 0.25}
    d |= {_f32(b) for b in (0x3FFFFFFF, 0x3F7FFFFF, 0x3FFFFFFE, 0x3FC00001, 0x3F800001, 0x3F800003,
                            0x3FAAAAAB, 0x3F555555, 0x00800000, 0x7E800000)}
    return sorted(d)


@pytest.mark.parametrize("d", _spacings())
def test_no_accepted_quotient_differs(lib, d):
    miss, rej, cand = _check(lib, d)
    assert miss == 0


@pytest.mark.parametrize("d", [0.025, 0.0125, 0.00625, 0.003125])
def test_in_grid_positions_nearly_all_accepted(lib, d):
    # every positive float from 2^-80 up to 2^22 cells (about 0.9e9 values): the bracket
    # fails only within about 2^-22 ulp of a rounding midpoint, so a few in a million at most
    miss, rej, cand = _check(lib, d)
    assert miss == 0
    assert cand > 5e8
    assert rej <= 1e-5 * cand


def test_invalid_spacings_never_accept(lib):
    for d in (0.0, -0.01, float("inf"), float("nan")):
        miss, rej, cand = _check(lib, d)
        assert miss == 0
        assert rej == cand
