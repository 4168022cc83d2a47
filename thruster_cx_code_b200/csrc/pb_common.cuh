// Shared device helpers for the PIC-MCC kernels (sm_100a).
//
// Arithmetic here reproduces NumPy 2 semantics on x86-64 exactly where the reference
// path (Python/physics_engine.py) depends on it:
//   * float32 -> integer casts (ndarray.astype) give INT_MIN for NaN / out of range;
//   * np.round is round-half-to-even (rintf);
//   * every expression is written with explicit __f*_rn / __d*_rn intrinsics so that no
//     multiply-add is contracted (NumPy evaluates each ufunc separately);
//   * seq_add_f32() gives the exact result of n sequential float32 additions of one
//     value, which is what np.add.at produces when every particle adds the same charge.
#pragma once
#include <cstdint>
#include <climits>
#include <cstring>
#include <cuda.h>
#include <cuda_runtime.h>

#define PB_HD __host__ __device__ __forceinline__

// error flags (PB_EF_*) come from the public header
#include "pbemcs.h"

// ---------------------------------------------------------------- draw sites
// Must equal oracle/philox.py.
enum pb_site : uint32_t {
  SITE_ION_COUNT = 1, SITE_ION_Y = 2, SITE_ION_V = 3, SITE_RF_COUNT = 4, SITE_RF_Y = 5,
  SITE_RF_V = 6, SITE_NEUT_Y = 7, SITE_NEUT_V = 8, SITE_SEE_SPAWN = 9, SITE_SEE_V = 10,
  SITE_CEX_U = 11, SITE_CEX_FM = 12, SITE_ION_HOLE = 13, SITE_PRELOAD = 14,
};

// ---------------------------------------------------------------- NumPy casts
PB_HD int np_f2i32(float v) {
  return (v >= -2147483648.0f && v < 2147483648.0f) ? (int)v : INT_MIN;
}
PB_HD long long np_f2i64(float v) {
  return (v >= -9223372036854775808.0f && v < 9223372036854775808.0f) ? (long long)v : LLONG_MIN;
}
PB_HD int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
PB_HD long long clampll(long long v, long long lo, long long hi) { return v < lo ? lo : (v > hi ? hi : v); }

// Programmatic dependent launch: a kernel launched with programmatic stream serialization
// may be scheduled while the previous kernel in its stream drains.  Every kernel that such a
// launch can reach starts here.  griddepcontrol.wait returns once the previous kernel has
// completed and its memory operations are visible (at once after a plain launch), so the
// kernels' effects keep plain stream order; only the launch overlaps.  The kernel then lets
// its own successor be scheduled.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// ---------------------------------------------------------------- grid barrier
// Barrier of the nblk blocks of a cooperative launch (or of one instance's contiguous range
// of blocks in a launch that serves several) on one 32-bit word: block gb == 0 adds
// 2^31 - (nblk - 1), the others add 1, so the top bit flips once every block has arrived and
// the low bits return to their start.  Arrival is a release, the poll an acquire: stores made
// by any thread of an arriving block before the barrier are visible to every thread after
// it.  The wait is bounded: on time-out PB_EF_SPIN_TIMEOUT is set in *err, and this and every
// later barrier stop waiting, so the kernel runs to completion and the host sees the flag.
constexpr long long GRID_SPIN_LIMIT = 1ll << 22;

__device__ __forceinline__ void grid_sync(unsigned int* bar, uint32_t* err, int nblk, int gb) {
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned int inc = gb == 0 ? (0x80000000u - (unsigned int)(nblk - 1)) : 1u;
    unsigned int old, cur;
    asm volatile("atom.release.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(bar), "r"(inc) : "memory");
    for (long long spin = 0;; ++spin) {
      asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(cur) : "l"(bar) : "memory");
      if ((old ^ cur) & 0x80000000u) break;
      if ((spin & 255) == 255) {
        if ((*(volatile uint32_t*)err & PB_EF_SPIN_TIMEOUT) != 0u) break;
        if (spin > GRID_SPIN_LIMIT) { atomicOr(err, PB_EF_SPIN_TIMEOUT); break; }
      }
    }
  }
  __syncthreads();
}

// ---------------------------------------------------------------- TMA tensor copies
// A tile of a tensor in global memory copied into shared memory by the TMA unit, its
// completion tracked by an mbarrier (one arrival with the byte count, then the copy's
// transaction bytes).  Every copy lands in the issuing block's own shared memory only.
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// orders this thread's earlier shared-memory accesses (and, after a barrier, the block's)
// before later writes by the async proxy (a TMA copy into the same buffer)
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}
// 3-D tiled copy of the box at coordinates (c0, c1, c2) of `map` (innermost first)
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1,
                                            int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_addr(bar))
      : "memory");
}

// np.clip(np.rint(q).astype(int), lo, hi) for 0 <= lo <= hi < 2^22.  For 0 <= q < 2^22 the
// float sum q + 2^23 is rint(q) + 2^23 (rounded to nearest, ties to even, as rintf rounds),
// an integer held in the low mantissa bits: no rounding or conversion instruction.  Other q
// (negative, large, NaN) take NumPy's cast.
__device__ __forceinline__ int rint_clip(float q, int lo, int hi) {
  if ((q >= 0.0f) & (q < 4194304.0f)) return min(max(__float_as_int(__fadd_rn(q, 8388608.0f)) - 0x4B000000, lo), hi);
  return (int)clampll(np_f2i64(rintf(q)), lo, hi);
}
// the same for np.clip(q.astype(int), lo, hi): for q >= 0 the cast truncates, i.e. floors,
// and q + 2^23 rounded down is floor(q) + 2^23
__device__ __forceinline__ int trunc_clip(float q, int lo, int hi) {
  if ((q >= 0.0f) & (q < 4194304.0f)) return min(max(__float_as_int(__fadd_rd(q, 8388608.0f)) - 0x4B000000, lo), hi);
  return (int)clampll(np_f2i64(truncf(q)), lo, hi);
}

// cell index of np.clip(np.round(s / d).astype(int), lo, hi)   (float32 division)
__device__ __forceinline__ int cell_round(float s, float d, int lo, int hi) {
  float q = __fdiv_rn(s, d);
  return (int)clampll(np_f2i64(rintf(q)), lo, hi);
}
// same with an int32 cast (accumulate_rho uses astype(np.int32))
__device__ __forceinline__ int cell_round32(float s, float d, int lo, int hi) {
  float q = __fdiv_rn(s, d);
  return clampi(np_f2i32(rintf(q)), lo, hi);
}

// The same roundings from q = s * (1/d) instead of the division: |q - fl(s/d)| stays below
// 1.8e-7 |q| (three float roundings), so when q is farther than 4.8e-7 |q| from every
// rounding boundary (half-integers for rint, integers for trunc) fl(s/d) rounds the same
// way; otherwise (and for NaN, inf or |q| >= 2^21) the exact quotient is used.
__device__ __forceinline__ float rint_div(float s, float d, float inv_d) {
  float q = __fmul_rn(s, inv_d);
  float n = rintf(q);
  if (!(fabsf(__fsub_rn(q, n)) < __fsub_rn(0.5f, __fmul_rn(4.8e-7f, fabsf(q))))) n = rintf(__fdiv_rn(s, d));
  return n;
}
__device__ __forceinline__ float trunc_div(float s, float d, float inv_d) {
  float q = __fmul_rn(s, inv_d);
  float n = rintf(q);
  if (!(fabsf(__fsub_rn(q, n)) > __fmul_rn(4.8e-7f, fabsf(q))) || !(fabsf(q) < 2097152.0f)) return truncf(__fdiv_rn(s, d));
  return truncf(q);
}
__device__ __forceinline__ int cell_round_f(float s, float d, float inv_d, int lo, int hi) {
  return (int)clampll(np_f2i64(rint_div(s, d, inv_d)), lo, hi);
}
__device__ __forceinline__ int cell_round32_f(float s, float d, float inv_d, int lo, int hi) {
  return clampi(np_f2i32(rint_div(s, d, inv_d)), lo, hi);
}

// np.maximum / np.minimum propagate NaN (fmaxf does not)
__device__ __forceinline__ float np_maxf(float a, float b) { return (a != a || b != b) ? __int_as_float(0x7fc00000) : (a >= b ? a : b); }
__device__ __forceinline__ double np_maxd(double a, double b) { return (a != a || b != b) ? __longlong_as_double(0x7ff8000000000000ll) : (a >= b ? a : b); }

// np.mod for float32 with a positive divisor: fmod, then shift into [0, b).  For
// 0 < a < b, fmod(a, b) is a itself, which skips the remainder routine for the particles
// that did not cross the periodic boundary.
__device__ __forceinline__ float np_modf_pos(float a, float b) {
  if (a > 0.0f && a < b) return a;
  float m = fmodf(a, b);
  if (m != 0.0f) {
    if ((b < 0.0f) != (m < 0.0f)) m = __fadd_rn(m, b);
  } else {
    m = copysignf(0.0f, b);
  }
  return m;
}

// ---------------------------------------------------------------- Philox4x32-10
struct u32x4 { uint32_t x, y, z, w; };

PB_HD u32x4 philox4x32_10(u32x4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c.x;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c.z;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    u32x4 n;
    n.x = hi1 ^ c.y ^ k0;
    n.y = lo1;
    n.z = hi0 ^ c.w ^ k1;
    n.w = lo0;
    c = n;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}

PB_HD double u53(uint32_t a, uint32_t b) {
  return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6)) * (1.0 / 9007199254740992.0);
}

// counter = (pid lo, pid hi16 | site << 16, step, block); key = seed
PB_HD u32x4 philox_block(uint64_t seed, uint64_t pid, uint32_t site, uint32_t step, uint32_t block) {
  u32x4 c;
  c.x = (uint32_t)pid;
  c.y = (uint32_t)((pid >> 32) & 0xFFFFu) | (site << 16);
  c.z = step;
  c.w = block;
  return philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
}

// j-th uniform double of (seed, pid, site, step)
PB_HD double philox_uniform(uint64_t seed, uint64_t pid, uint32_t site, uint32_t step, uint32_t j) {
  u32x4 r = philox_block(seed, pid, site, step, j >> 1);
  return (j & 1) ? u53(r.z, r.w) : u53(r.x, r.y);
}

// ---------------------------------------------------------------- Box-Muller
// ln and cos from series in plain IEEE double, identical operation order to the oracle
// (oracle/philox.py: bm_log, bm_cos2pi).  Fused multiply-add is never used.
#ifdef __CUDA_ARCH__
#define DMUL(a, b) __dmul_rn((a), (b))
#define DADD(a, b) __dadd_rn((a), (b))
#define DSUB(a, b) __dsub_rn((a), (b))
#define DDIV(a, b) __ddiv_rn((a), (b))
#else
#define DMUL(a, b) ((a) * (b))
#define DADD(a, b) ((a) + (b))
#define DSUB(a, b) ((a) - (b))
#define DDIV(a, b) ((a) / (b))
#endif

PB_HD double bm_log(double x) {
  int e;
  double m = frexp(x, &e);
  if (m < 0.7071067811865476) { m = DMUL(m, 2.0); e -= 1; }
  double s = DDIV(DSUB(m, 1.0), DADD(m, 1.0));
  double s2 = DMUL(s, s);
  double acc = 1.0 / 27.0;
  for (int k = 25; k >= 1; k -= 2) acc = DADD(DMUL(acc, s2), 1.0 / (double)k);
  return DADD(DMUL(DMUL(s, acc), 2.0), DMUL((double)e, 0.6931471805599453));
}

PB_HD double bm_cos2pi(double u) {
  double w = DMUL(u, 8.0);
  double kf = floor(w);
  double f = DSUB(w, kf);
  int k = ((int)kf) & 7;
  if (k & 1) f = DSUB(1.0, f);
  double r = DMUL(f, 0.7853981633974483);
  double r2 = DMUL(r, r);
  double c = 1.0, s = 1.0;
  for (int n = 22; n >= 2; n -= 2) c = DSUB(1.0, DMUL(DDIV(r2, (double)(n * (n - 1))), c));
  for (int n = 23; n >= 3; n -= 2) s = DSUB(1.0, DMUL(DDIV(r2, (double)(n * (n - 1))), s));
  s = DMUL(r, s);
  bool use_sin = (k == 1) | (k == 2) | (k == 5) | (k == 6);
  double v = use_sin ? s : c;
  bool neg = (k == 2) | (k == 3) | (k == 4) | (k == 5);
  return neg ? -v : v;
}

// j-th standard normal of (seed, pid, site, step): uniforms 2j, 2j+1
PB_HD double philox_normal(uint64_t seed, uint64_t pid, uint32_t site, uint32_t step, uint32_t j) {
  u32x4 r = philox_block(seed, pid, site, step, j);
  double u1 = u53(r.x, r.y), u2 = u53(r.z, r.w);
  double rad = sqrt(DMUL(-2.0, bm_log(DSUB(1.0, u1))));
  return DMUL(rad, bm_cos2pi(u2));
}

// ---------------------------------------------------------------- sequential float32 sums
// Exact result of:  for (i < n) s = (float)((double)s + c);
// which is what np.add.at(rho_float32, idx, python_float) does: each partial sum is formed
// in float64 with the double addend and rounded to float32.  Within one float32 binade of
// the running sum (away from zero) every addition moves s by the same number of float32
// ulps, so whole runs are applied at once.  With u the float32 ulp of s, |c|/u = q + f;
// the float64 sum rounds f onto a grid of u/2^29 (ties to even, independent of s), then
// the float32 rounding picks q or q+1 (ties to even).  Binade changes, sign changes and
// stagnation are taken one real addition at a time.
PB_HD float f32_add_d_rn(float a, double b) {
#ifdef __CUDA_ARCH__
  return __double2float_rn(__dadd_rn((double)a, b));
#else
  volatile double t = (double)a + b;
  volatile float r = (float)t;
  return r;
#endif
}

PB_HD bool f32_signbit(float v) {
#ifdef __CUDA_ARCH__
  return (__float_as_uint(v) >> 31) != 0u;
#else
  union { float f; uint32_t u; } a; a.f = v; return (a.u >> 31) != 0u;
#endif
}

PB_HD uint32_t f32_bits(float v) {
#ifdef __CUDA_ARCH__
  return __float_as_uint(v);
#else
  union { float f; uint32_t u; } a; a.f = v; return a.u;
#endif
}

PB_HD float f32_from_bits(uint32_t b) {
#ifdef __CUDA_ARCH__
  return __uint_as_float(b);
#else
  union { float f; uint32_t u; } a; a.u = b; return a.f;
#endif
}

PB_HD float seq_add_f32d(float s, double c, uint32_t n) {
  uint32_t guard = 0;
  while (n > 0) {
    float t = f32_add_d_rn(s, c);
    --n;
    if (t == s && !(t == 0.0f && f32_signbit(t) != f32_signbit(s))) return t;  // stagnation
    float prev = s;
    s = t;
    if (!(s == s) || n == 0) return s;
    if (++guard > 4096) {  // safety net: finish the remainder one addition at a time
      while (n > 0) { s = f32_add_d_rn(s, c); --n; }
      return s;
    }
    // try a jump: source and result in the same binade, same sign, normal range
    uint32_t bp = f32_bits(prev), bs = f32_bits(s);
    uint32_t ep = (bp >> 23) & 0xFF, es = (bs >> 23) & 0xFF;
    if (ep != es || (bp >> 31) != (bs >> 31) || es == 0 || es >= 254 || !(c == c)) continue;
    int32_t S = (int32_t)((bs & 0x7FFFFF) | 0x800000);  // |s| = S u, u = 2^(es-150)
    bool up = ((bs >> 31) != 0) == (c < 0.0);          // |s| grows when c has the sign of s
    double cu = ldexp(fabs(c), 150 - (int)es);          // |c| / u, exact
    if (!(cu < 1099511627776.0)) continue;              // 2^40
    double qd = floor(cu);
    double fr = cu - qd;                                 // exact
    double jf = rint(ldexp(fr, 29));                     // f on the float64 grid of the sum
    int64_t q = (int64_t)qd;
    int frac_cmp = jf < 268435456.0 ? -1 : (jf > 268435456.0 ? 1 : 0);  // vs 2^28
    int64_t D;  // steady increment in ulps (S stays even after a tie)
    if (frac_cmp < 0) D = q;
    else if (frac_cmp > 0) D = q + 1;
    else D = (q & 1) ? q + 1 : q;
    if (D == 0) continue;
    if (frac_cmp == 0 && (S & 1)) continue;  // parity not yet settled
    int64_t room;
    if (up) room = ((int64_t)0xFFFFFF - S) / D - 1;     // keep S + m D + D <= 2^24 - 1
    else room = (S - (int64_t)0x800000 - 1) / D - 1;    // keep S - m D - D >= 2^23
    if (room <= 0) continue;
    int64_t m = room < (int64_t)n ? room : (int64_t)n;
    int64_t S2 = up ? S + m * D : S - m * D;
    s = f32_from_bits((bs & 0xFF800000u) | ((uint32_t)S2 & 0x7FFFFFu));
    n -= (uint32_t)m;
  }
  return s;
}
