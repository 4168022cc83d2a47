"""Philox4x32-10 counter-based generator and the keyed draws of the GPU path, in NumPy.

TEST INFRASTRUCTURE ONLY: this module is part of the CPU oracle.  Product code never
imports it; the GPU kernels carry their own implementation of the same arithmetic.

Generator: Philox4x32 with 10 rounds (Salmon, Moraes, Dror, Shaw, "Parallel random
numbers: as easy as 1, 2, 3", SC11).  Round function on (c0,c1,c2,c3) with key (k0,k1):
    hi0:lo0 = M0*c0, hi1:lo1 = M1*c2,
    c' = (hi1 ^ c1 ^ k0, lo1, hi0 ^ c3 ^ k1, lo0),  key += (W0, W1)
with M0=0xD2511F53, M1=0xCD9E8D57, W0=0x9E3779B9, W1=0xBB67AE85.

Keying used throughout the PIC path (``draw site``, particle id, step):
    counter = (pid & 0xffffffff, ((pid >> 32) & 0xffff) | (site << 16), step, block)
    key     = (seed & 0xffffffff, (seed >> 32) & 0xffffffff)
Each call yields four 32-bit words; a uniform double takes two of them:
    u = ((a >> 5) * 2**26 + (b >> 6)) * 2**-53          in [0, 1)
Normals use Box-Muller, N = sqrt(-2 ln(1-u1)) * cos(2 pi u2), with ln and cos written
out below as plain IEEE double series so the CPU and GPU give identical bits (the GPU
kernel evaluates the same operations in the same order with fused multiply-add off).
"""
import numpy as np

M0 = np.uint64(0xD2511F53)
M1 = np.uint64(0xCD9E8D57)
MASK32 = np.uint64(0xFFFFFFFF)

# draw sites (16-bit) — must equal the enum in the CUDA sources
SITE_ION_COUNT = 1
SITE_ION_Y = 2
SITE_ION_V = 3
SITE_RF_COUNT = 4
SITE_RF_Y = 5
SITE_RF_V = 6
SITE_NEUT_Y = 7
SITE_NEUT_V = 8
SITE_SEE_SPAWN = 9
SITE_SEE_V = 10
SITE_CEX_U = 11
SITE_CEX_FM = 12
SITE_ION_HOLE = 13
SITE_PRELOAD = 14


def philox4x32_10(c0, c1, c2, c3, k0, k1):
    """Vectorised Philox4x32-10 on uint32 arrays (broadcast); returns four uint32 arrays."""
    c0 = np.asarray(c0, dtype=np.uint32)
    c1 = np.asarray(c1, dtype=np.uint32)
    c2 = np.asarray(c2, dtype=np.uint32)
    c3 = np.asarray(c3, dtype=np.uint32)
    k0 = int(k0) & 0xFFFFFFFF
    k1 = int(k1) & 0xFFFFFFFF
    c0, c1, c2, c3 = np.broadcast_arrays(c0, c1, c2, c3)
    c0 = c0.copy(); c1 = c1.copy(); c2 = c2.copy(); c3 = c3.copy()
    for _ in range(10):
        p0 = M0 * c0.astype(np.uint64)
        p1 = M1 * c2.astype(np.uint64)
        hi0 = (p0 >> np.uint64(32)).astype(np.uint32)
        lo0 = (p0 & MASK32).astype(np.uint32)
        hi1 = (p1 >> np.uint64(32)).astype(np.uint32)
        lo1 = (p1 & MASK32).astype(np.uint32)
        c0, c1, c2, c3 = hi1 ^ c1 ^ np.uint32(k0), lo1, hi0 ^ c3 ^ np.uint32(k1), lo0
        k0 = (k0 + 0x9E3779B9) & 0xFFFFFFFF
        k1 = (k1 + 0xBB67AE85) & 0xFFFFFFFF
    return c0, c1, c2, c3


def _counter(pid, site, step, block):
    pid = np.asarray(pid, dtype=np.uint64)
    c0 = (pid & MASK32).astype(np.uint32)
    c1 = (((pid >> np.uint64(32)) & np.uint64(0xFFFF)) | np.uint64(site << 16)).astype(np.uint32)
    c2 = np.full_like(c0, np.uint32(step & 0xFFFFFFFF))
    c3 = np.full_like(c0, np.uint32(block))
    return c0, c1, c2, c3


def _u53(a, b):
    return ((a >> np.uint32(5)).astype(np.float64) * 67108864.0 +
            (b >> np.uint32(6)).astype(np.float64)) * (1.0 / 9007199254740992.0)


def uniforms(seed, pid, site, step, count):
    """``count`` uniform doubles per id: returns array of shape (count, len(pid))."""
    pid = np.atleast_1d(np.asarray(pid, dtype=np.uint64))
    k0 = np.uint32(seed & 0xFFFFFFFF)
    k1 = np.uint32((seed >> 32) & 0xFFFFFFFF)
    out = np.empty((count, pid.size), dtype=np.float64)
    nblk = (count + 1) // 2
    for blk in range(nblk):
        r0, r1, r2, r3 = philox4x32_10(*_counter(pid, site, step, blk), k0, k1)
        out[2 * blk] = _u53(r0, r1)
        if 2 * blk + 1 < count:
            out[2 * blk + 1] = _u53(r2, r3)
    return out


# ---------------------------------------------------------------------------
# Box-Muller with series ln / cos (identical operation order on the GPU)
# ---------------------------------------------------------------------------
_LN2_HI = 0.6931471805599453     # nearest double to ln 2
_SQRT_HALF = 0.7071067811865476
_PI_4 = 0.7853981633974483


def bm_log(x):
    """Natural log for x in (0, 1]: x = m 2^e with m in [sqrt(1/2), sqrt(2));
    ln m = 2 atanh(s), s = (m-1)/(m+1), atanh by its odd power series (|s| <= 0.1716,
    13 terms give < 1e-17 truncation)."""
    x = np.asarray(x, dtype=np.float64)
    m, e = np.frexp(x)                 # m in [0.5, 1)
    small = m < _SQRT_HALF
    m = np.where(small, m * 2.0, m)
    e = np.where(small, e - 1, e).astype(np.float64)
    s = (m - 1.0) / (m + 1.0)
    s2 = s * s
    acc = 1.0 / 27.0
    for k in range(25, 0, -2):
        acc = acc * s2 + 1.0 / k
    return (s * acc) * 2.0 + e * _LN2_HI


def bm_cos2pi(u):
    """cos(2 pi u) for u in [0, 1): octant reduction on 8u (exact), then the Taylor
    series of sin / cos on [0, pi/4] (11 terms each)."""
    u = np.asarray(u, dtype=np.float64)
    w = u * 8.0
    k = np.floor(w)
    f = w - k
    k = k.astype(np.int64) & 7
    # angle within the octant; odd octants measure from the far edge
    odd = (k & 1) == 1
    f = np.where(odd, 1.0 - f, f)
    r = f * _PI_4
    r2 = r * r
    c = 1.0
    s = 1.0
    for n in range(22, 0, -2):       # cos: 1 - r^2/2! + ...
        c = 1.0 - (r2 / (n * (n - 1))) * c
    for n in range(23, 1, -2):       # sin: r (1 - r^2/3! + ...)
        s = 1.0 - (r2 / (n * (n - 1))) * s
    s = r * s
    # octant map: cos(2 pi u) for octants 0..7
    use_sin = (k == 1) | (k == 2) | (k == 5) | (k == 6)
    val = np.where(use_sin, s, c)
    neg = (k == 2) | (k == 3) | (k == 4) | (k == 5)
    return np.where(neg, -val, val)


def normals(seed, pid, site, step, count):
    """``count`` standard normals per id (shape (count, n)); each takes two uniforms."""
    u = uniforms(seed, pid, site, step, 2 * count)
    out = np.empty((count, u.shape[1]), dtype=np.float64)
    for j in range(count):
        u1 = u[2 * j]
        u2 = u[2 * j + 1]
        rad = np.sqrt(-2.0 * bm_log(1.0 - u1))
        out[j] = rad * bm_cos2pi(u2)
    return out


def poisson_count(seed, site, step, lam):
    """Poisson(lam) by CDF inversion with one keyed uniform (counter pid = 0)."""
    u = float(uniforms(seed, np.array([0], dtype=np.uint64), site, step, 1)[0, 0])
    if not lam > 0.0:
        return 0
    p = float(np.exp(-lam))
    F = p
    k = 0
    kmax = int(lam + 40.0 * np.sqrt(lam) + 100.0)
    while u > F and k < kmax:
        k += 1
        p = p * lam / k
        F = F + p
    return k
