"""NumPy's float32 np.sum restated as the device computes it (k_pw_leaves, k_pw_combine and
the tree of pw_build in csrc/): 0 + pw(a, n), where pw sums a block of at most 128
elements with eight running sums (a running sum from 0 below 8 elements) and otherwise
splits at n / 2 rounded down to a multiple of 8.  The restatement is checked against
np.sum itself over many sizes, 1-D and C-contiguous 2-D, so the kernels' summation order
is pinned to NumPy's."""
import numpy as np
import pytest

f32 = np.float32


def _leaf(a):
    n = len(a)
    if n < 8:
        r = f32(0.0)
        for v in a:
            r = f32(r + v)
        return r
    acc = [a[q] for q in range(8)]
    i = 8
    while i < n - (n % 8):
        for q in range(8):
            acc[q] = f32(acc[q] + a[i + q])
        i += 8
    res = f32(f32(f32(acc[0] + acc[1]) + f32(acc[2] + acc[3])) + f32(f32(acc[4] + acc[5]) + f32(acc[6] + acc[7])))
    while i < n:
        res = f32(res + a[i])
        i += 1
    return res


def _pw(a):
    n = len(a)
    if n <= 128:
        return _leaf(a)
    m = n // 2
    m -= m % 8
    return f32(_pw(a[:m]) + _pw(a[m:]))


def np_sum_restated(a):
    return f32(f32(0.0) + _pw(np.ascontiguousarray(a, dtype=f32).ravel()))


SIZES = list(range(0, 140)) + [255, 256, 257, 1000, 4097, 8191, 8192, 8193, 20011, 65543, 100003]


@pytest.mark.parametrize("scale", [1.0, 1e6])
def test_restated_pairwise_equals_numpy(scale):
    rng = np.random.default_rng(int(scale))
    for n in SIZES:
        a = (rng.standard_normal(n) * scale).astype(f32)
        v = a ** 2 + (a * f32(0.5)) ** 2
        assert np_sum_restated(v).tobytes() == np.sum(v).tobytes(), n


def test_two_dimensional_sum_is_the_flat_sum():
    rng = np.random.default_rng(3)
    for shape in [(65, 284), (99, 137), (257, 1025)]:
        Ex = rng.standard_normal(shape).astype(f32)
        Ey = rng.standard_normal(shape).astype(f32)
        e2 = Ex ** 2 + Ey ** 2
        assert np_sum_restated(e2).tobytes() == np.sum(e2).tobytes(), shape
