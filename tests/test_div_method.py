"""The particle kernels' divisions without the division instruction, restated on the host and
checked against IEEE float32 division: div_rn_checked (csrc/pb_particles.cu; the ion step's
final cells and the sub-step reduction) and div_bracket (the push of both step kernels), and
the electron push's float-to-double conversion by bits (f2d_scaled).

q = x * inv (inv = RN(1/d)), one correction q += (x - q d) inv, accepted when
|x - q d| < ulp(q) |d| / 2; anything else falls back to the division.  fmaf(a, b, c) of
float32 operands is emulated exactly in float64 here: a * b is exact in float64 and, for
q within a few ulps of x / d, so is the sum, which is then rounded once to float32.  The
full check (every float |x| < 64, ten spacings) ran on the host in C; this samples it.

The other tests cover the cell-index tricks the particle kernels use beside it (floor,
fraction, rint and truncation by adding 2^23, and the one-compare range test of the floor).
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


# The integer and fraction tricks of the particle kernels (floor_frac in csrc/pb_particles.cu,
# rint_clip and trunc_clip in csrc/pb_common.cuh): for 0 <= q < 2^22 the float32 sum q + 2^23,
# rounded to nearest (rint) or down (floor), is an integer in [2^23, 2^24) whose low mantissa
# bits hold the result; q minus that integer is exact in float32.
def _sum_bits(q, down):
    if down:  # round down: the exact sum (float64) floored onto the integer grid of [2^23, 2^24)
        t = np.floor(q.astype(np.float64) + 8388608.0).astype(F32)
    else:     # float32 addition rounds to nearest, ties to even
        t = (q + F32(8388608.0)).astype(F32)
    return t, t.view(np.int32).astype(np.int64) - 0x4B000000


def _samples(rng):
    k = rng.integers(0, 4194304, 400_000).astype(F32)
    ties = (k + F32(0.5)).astype(F32)
    q = np.concatenate([rng.uniform(0.0, 4096.0, 1_000_000).astype(F32), k, ties,
                        np.nextafter(ties, F32(0)), np.nextafter(ties, F32(np.inf)),
                        rng.integers(0, 0x4A800000, 500_000, dtype=np.uint32).view(F32),
                        np.array([0.0, 0.5, 1.5, 2.5, 4194303.5, np.nextafter(F32(4194304.0), F32(0))], F32)])
    return q[(q >= 0) & (q < F32(4194304.0))]


def test_floor_frac_and_rint_by_adding_2p23():
    rng = np.random.default_rng(11)
    q = _samples(rng)
    t, fl = _sum_bits(q, down=True)
    assert np.array_equal(fl, np.floor(q).astype(np.int64))
    frac = (q - (t - F32(8388608.0)).astype(F32)).astype(F32)
    assert np.array_equal(frac.astype(np.float64), q.astype(np.float64) - np.floor(q.astype(np.float64)))
    _, rn = _sum_bits(q, down=False)
    assert np.array_equal(rn, np.rint(q).astype(np.int64))
    # trunc_clip: astype(int) of a non-negative float is its floor
    assert np.array_equal(fl, q.astype(np.int64))


def _rd_sum_bits(q):
    """float32 q + 2^23 rounded down (emulated through the float64 sum), as int32 bits."""
    with np.errstate(invalid="ignore", over="ignore"):
        s = q.astype(np.float64) + 8388608.0
        t = s.astype(F32)
    with np.errstate(invalid="ignore"):
        up = t.astype(np.float64) > s
    t = np.where(up, np.nextafter(t, F32(-np.inf)), t)
    # an exact zero sum rounds to -0 when rounding down
    t = np.where(s == 0.0, F32(-0.0), t)
    # below 2^-29 the float64 sum itself rounds; the float32 sum rounded down is then 2^23 for
    # a positive q and the float just below 2^23 for a negative one
    with np.errstate(invalid="ignore"):
        t = np.where((q < 0) & (q > -2.0 ** -29), F32(8388607.5), t)
    return t.view(np.int32).astype(np.int64)


def test_one_unsigned_compare_bounds_the_floor():
    """push_cell tests fl = bits(q + 2^23, rounded down) - 0x4B000000 with one unsigned compare,
    fl <= N (N = nx - 2 < 2^22), in place of 0 <= q < 2^22 and fl <= N: any q that passes
    (negative, huge, infinite and NaN q included) lies in [0, N + 1) and fl is its floor."""
    rng = np.random.default_rng(17)
    for N in (2, 255, 2047, 4194302):
        q = np.concatenate([
            rng.integers(0, 0xFFFFFFFF, 2_000_000, dtype=np.uint64).astype(np.uint32).view(F32),
            rng.uniform(-3.0, N + 3.0, 1_000_000).astype(F32),
            np.array([0.0, -0.0, -8388608.0, -8388607.5, 8388608.0, 4194304.0, N, N + 1, N + 0.5,
                      np.nextafter(F32(N + 1), F32(0)), np.inf, -np.inf, np.nan, -1e-45, 1e-45], F32)])
        fl = (_rd_sum_bits(q) - 0x4B000000) & 0xFFFFFFFF
        ok = fl <= N
        with np.errstate(invalid="ignore"):
            inside = (q >= 0) & (q < N + 1)
        assert np.array_equal(ok, inside)
        assert np.array_equal(fl[ok], np.floor(q[ok]).astype(np.int64))


# ---------------------------------------------------------------- bracketed division
# div_bracket (csrc/pb_particles.cu), the division of the step kernels' push: q0 = RN(x inv),
# r0 = RN(q0 d - x), qa = RN(q0 - r0 lo), qb = RN(q0 - r0 hi) with lo and hi the floats two
# steps below and above inv = RN(1/d); accepted when qa == qb and |x| >= 2^-80.  Every
# fused multiply-add is emulated exactly here (rational arithmetic, one rounding to float32,
# ties to even); pb_check_division runs the same test on the GPU over all 2^32 x.
from fractions import Fraction  # noqa: E402


def _rn32(v):
    """Fraction -> nearest float32 (ties to even), finite inputs whose result is finite."""
    if v == 0:
        return F32(0.0)
    s = -1 if v < 0 else 1
    a = abs(v)
    e = a.numerator.bit_length() - a.denominator.bit_length()
    if Fraction(2) ** e > a:
        e -= 1
    e = max(e, -126)                    # below 2^-126: subnormal spacing 2^-149
    scale = Fraction(2) ** (23 - e)     # a * scale in [2^23, 2^24) for normal results
    m = a * scale
    q, r = divmod(m.numerator, m.denominator)
    rem = Fraction(r, m.denominator)
    if rem > Fraction(1, 2) or (rem == Fraction(1, 2) and q % 2 == 1):
        q += 1
    return F32(s * float(Fraction(q) / scale))


def _fma32_exact(a, b, c):
    return _rn32(Fraction(float(a)) * Fraction(float(b)) + Fraction(float(c)))


def div_bracket(x, d):
    x, d = F32(x), F32(d)
    inv = F32(1.0) / d
    b = np.array([inv], dtype=F32).view(np.uint32)[0]
    lo = np.array([b - 2], dtype=np.uint32).view(F32)[0]
    hi = np.array([b + 2], dtype=np.uint32).view(F32)[0]
    q0 = F32(x * inv)
    r0 = _fma32_exact(q0, d, -x)
    qa = _fma32_exact(-r0, lo, q0)
    qb = _fma32_exact(-r0, hi, q0)
    return qa, bool(qa == qb and abs(float(x)) >= 2.0 ** -80)


def test_div_bracket_accepts_only_the_division():
    rng = np.random.default_rng(11)
    spacings = [F32(v) for v in (0.025, 0.00625, 0.003125, 0.011, 0.3)] + \
        [F32(v) for v in rng.uniform(1e-3, 1.0, 3)]
    n_acc = n = 0
    with np.errstate(over="ignore", invalid="ignore", under="ignore"):
        for d in spacings:
            xs = list(rng.uniform(0.0, 2048 * float(d), 400).astype(F32))                  # in the grid
            k = rng.integers(1, 2048, 300)
            xs += list((k * d).astype(F32))                                                  # cell boundaries
            xs += list(np.nextafter((k * d).astype(F32), F32(np.inf)))
            n_grid = len(xs)
            bits = rng.integers(0x0C000000, 0x4B000000, 300, dtype=np.int64).astype(np.uint32)
            xs += list(bits.view(F32))                                                       # random patterns
            for j, x in enumerate(xs):
                q, ok = div_bracket(x, d)
                if ok:
                    assert q == F32(x) / d, (float(x), float(d))
                if j < n_grid:
                    n += 1
                    n_acc += ok
    assert n_acc >= 0.999 * n  # in-grid positions: nearly all take the bracketed quotient


def test_div_bracket_zero_and_tiny_fall_back():
    for x in (0.0, -0.0, 1e-30, -1e-30):
        assert not div_bracket(x, 0.025)[1]


# ---------------------------------------------------------------- float -> double by bits
# f2d_scaled (csrc/pb_particles.cu): hi = (bits >> 3, arithmetic) & 0x8FFFFFFF, lo = bits << 29
# is the double f 2^-896 for every finite float f; the electron push multiplies it by a weight
# scaled by 2^896 (or adds it times 2^896 in an FMA), which rounds as the converted value does.
def _f2d_scaled(f):
    b = np.asarray(f, dtype=F32).view(np.int32).astype(np.int64)
    hi = ((b >> 3) & 0x8FFFFFFF) & 0xFFFFFFFF
    lo = (b << 29) & 0xFFFFFFFF
    return ((hi << 32) | lo).astype(np.uint64).view(np.float64)


def test_f2d_scaled_is_exact_for_finite_floats():
    rng = np.random.default_rng(3)
    bits = rng.integers(0, 1 << 32, 200000, dtype=np.int64).astype(np.uint32)
    bits = np.concatenate([bits, np.array([0, 0x80000000, 1, 0x80000001, 0x007FFFFF, 0x00800000, 0x7F7FFFFF,
                                           0xFF7FFFFF, 0x3F800000], dtype=np.uint32)])
    f = bits.view(F32)
    f = f[np.isfinite(f)]
    got = _f2d_scaled(f) * 2.0 ** 896
    want = f.astype(np.float64)
    assert np.array_equal(got.view(np.uint64), want.view(np.uint64))
    # the product with a scaled weight equals the product with the converted value, bit for bit
    w = rng.uniform(0.0, 1.0, f.size)
    assert np.array_equal((_f2d_scaled(f) * (w * 2.0 ** 896)).view(np.uint64), (want * w).view(np.uint64))
