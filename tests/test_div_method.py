"""The electron push's division without the reciprocal instruction (div_rn_checked in
csrc/pb_particles.cu), restated in NumPy and checked against IEEE float32 division.

q = x * inv (inv = RN(1/d)), one correction q += (x - q d) inv, accepted when
|x - q d| < ulp(q) |d| / 2; anything else falls back to the division.  fmaf(a, b, c) of
float32 operands is emulated exactly in float64 here: a * b is exact in float64 and, for
q within a few ulps of x / d, so is the sum, which is then rounded once to float32.  The
full check (every float |x| < 64, ten spacings) ran on the host in C; this samples it.
"""
import numpy as np

F32 = np.float32


def _fma32(a, b, c):
    return (a.astype(np.float64) * b.astype(np.float64) + c.astype(np.float64)).astype(F32)


def div_rn_checked(x, d):
    inv = F32(1.0) / F32(d)
    q = (x * inv).astype(F32)
    q = _fma32(_fma32(-q, np.full_like(q, d), x), np.full_like(q, inv), q)
    r = _fma32(-q, np.full_like(q, d), x)
    b = q.view(np.uint32)
    e = b & np.uint32(0x7F800000)
    ok = (e > np.uint32(26 << 23)) & (e < np.uint32(0x7F800000)) & ((b & np.uint32(0x007FFFFF)) != 0)
    h = ((e - np.uint32(24 << 23)).view(F32) * np.abs(F32(d))).astype(F32)
    accept = ok & (np.abs(r) < h)
    return np.where(accept, q, (x / F32(d)).astype(F32)), accept


def test_div_rn_checked_matches_ieee():
    rng = np.random.default_rng(5)
    with np.errstate(over="ignore", invalid="ignore", under="ignore"):
        for d in (0.025, 0.0125, 0.00625, 0.05, 0.011):
            d = F32(d)
            # positions over the grid, near cell boundaries k * d, and random bit patterns below 64
            pos = rng.uniform(-1.0, 40.0, 2_000_000).astype(F32)
            k = rng.integers(-10, 6000, 500_000)
            near = (k * d).astype(F32)
            near = np.concatenate([near, np.nextafter(near, F32(np.inf)), np.nextafter(near, F32(-np.inf))])
            bits = rng.integers(0, 0x42800000, 1_000_000, dtype=np.uint32).view(F32)
            x = np.concatenate([pos, near, bits, -bits, np.array([0.0, -0.0, 1.0, 2.0, 0.5], F32)])
            got, accept = div_rn_checked(x, d)
            ref = (x / d).astype(F32)
            assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
            # nearly every position in the grid takes the fast path
            assert accept[:pos.size].mean() > 0.999
