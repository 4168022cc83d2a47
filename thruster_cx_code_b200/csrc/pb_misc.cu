// Remaining step kernels: injection, SEE electron spawn, exit-angle percentile, sputter
// cell break, grid thermal conduction, PPC statistics, cell-key radix sort and the
// module-level thermal_conduction (Taichi semantics).
#include "pb_kernels.cuh"
#include "pb_misc.cuh"
#include "pb_poisson.cuh"

namespace pb {

// ------------------------------------------------------------------ helpers
__device__ __forceinline__ int dep_cell(float x, float y, float dxf, float dyf, int nx, int ny) {
  int ix = cell_round32(x, dxf, 1, nx - 2);
  int iy = cell_round32(y, dyf, 1, ny - 2);
  return iy * nx + ix;
}

// Poisson(lam) by CDF inversion with one keyed uniform (oracle/philox.py: poisson_count)
__device__ int poisson_inversion(double u, double lam) {
  if (!(lam > 0.0)) return 0;
  double p = exp(-lam);
  double F = p;
  int k = 0;
  int kmax = (int)(lam + 40.0 * sqrt(lam) + 100.0);
  while (u > F && k < kmax) {
    ++k;
    p = DDIV(DMUL(p, lam), (double)k);
    F = DADD(F, p);
  }
  return k;
}

// ------------------------------------------------------------------ injection
// inject step A (physics_engine.py:996-1099): counts, slots and ids for this step
__global__ void k_inject_prep(InjectArgs a) {
  pdl_enter();
  if (a.step_dev) a.step = *a.step_dev;
  int n_ion = 0, n_rf = 0;
  if (a.ion_on) n_ion = poisson_inversion(philox_uniform(a.seed, 0, SITE_ION_COUNT, a.step, 0), a.lam);
  if (a.rf_on) {
    n_rf = (int)a.rf_num_float;
    if (philox_uniform(a.seed, 0, SITE_RF_COUNT, a.step, 0) < DSUB(a.rf_num_float, (double)n_rf)) ++n_rf;
  }
  int n_neut = a.neut_n;
  int np0 = *a.num_p, ne0 = *a.num_e;
  if (np0 + n_ion > a.cap_p) { atomicOr(a.errflags, PB_EF_CAPACITY_ION); n_ion = a.cap_p - np0; if (n_ion < 0) n_ion = 0; }
  if (ne0 + n_rf + n_neut > a.cap_e) {
    atomicOr(a.errflags, PB_EF_CAPACITY_ELE);
    int room = a.cap_e - ne0; if (room < 0) room = 0;
    if (n_rf > room) n_rf = room;
    n_neut = room - n_rf < n_neut ? room - n_rf : n_neut;
  }
  uint32_t id_i = *a.next_ion_id, id_e = *a.next_e_id;
  if ((uint64_t)id_i + n_ion > 0xFFFFFFFFull || (uint64_t)id_e + n_rf + n_neut > 0xFFFFFFFFull)
    atomicOr(a.errflags, PB_EF_ID_OVERFLOW);
  a.inj[0] = n_ion; a.inj[1] = n_rf; a.inj[2] = n_neut;
  a.inj[3] = np0; a.inj[4] = ne0;
  a.inj[5] = (int)id_i; a.inj[6] = (int)id_e;
  *a.num_p = np0 + n_ion;
  *a.num_e = ne0 + n_rf + n_neut;
  *a.next_ion_id = id_i + n_ion;
  *a.next_e_id = id_e + n_rf + n_neut;
}

// inject step B: one thread per new particle; blockIdx.y selects ions / rf / neutralizer
__global__ void k_inject_gen(InjectArgs a) {
  pdl_enter();
  if (a.step_dev) a.step = *a.step_dev;
  const int seg = blockIdx.y;
  const int n = a.inj[seg];
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    if (seg == 0) {
      uint32_t id = (uint32_t)a.inj[5] + j;
      int slot = a.inj[3] + j;
      float y;
      if (a.geometry == 2) {
        double uh = philox_uniform(a.seed, id, SITE_ION_HOLE, a.step, 0);
        double u = philox_uniform(a.seed, id, SITE_ION_HOLE, a.step, 1);
        int which = (int)DMUL(uh, 2.0);
        float lo = a.span[2 * which], hi = a.span[2 * which + 1];
        y = __double2float_rn(DADD((double)lo, DMUL((double)__fsub_rn(hi, lo), u)));
      } else {
        double u = philox_uniform(a.seed, id, SITE_ION_Y, a.step, 0);
        y = __double2float_rn(DADD(a.ylo, DMUL(DSUB(a.yhi, a.ylo), u)));
      }
      double g0 = philox_normal(a.seed, id, SITE_ION_V, a.step, 0);
      double g1 = philox_normal(a.seed, id, SITE_ION_V, a.step, 1);
      double g2 = philox_normal(a.seed, id, SITE_ION_V, a.step, 2);
      float x = a.x_inj;
      a.ions.x[slot] = x;
      a.ions.y[slot] = y;
      a.ions.vx[slot] = __double2float_rn(DADD(a.v_bohm, DMUL(g0, a.v_spread)));
      a.ions.vy[slot] = __double2float_rn(DMUL(g1, a.v_spread));
      a.ions.vz[slot] = __double2float_rn(DMUL(g2, a.v_spread));
      a.ions.cex[slot] = 0;
      a.ions.id[slot] = id;
      atomicAdd(a.cnt_i + dep_cell(x, y, a.dxf, a.dyf, a.nx, a.ny), 1);
    } else {
      bool rf = seg == 1;
      int off = rf ? 0 : a.inj[1];
      uint32_t id = (uint32_t)a.inj[6] + off + j;
      int slot = a.inj[4] + off + j;
      float x, y, vx, vy, vz;
      if (rf) {
        double u = philox_uniform(a.seed, id, SITE_RF_Y, a.step, 0);
        y = __double2float_rn(DADD(a.rf_ylo, DMUL(DSUB(a.rf_yhi, a.rf_ylo), u)));
        double g0 = philox_normal(a.seed, id, SITE_RF_V, a.step, 0);
        double g1 = philox_normal(a.seed, id, SITE_RF_V, a.step, 1);
        double g2 = philox_normal(a.seed, id, SITE_RF_V, a.step, 2);
        x = 0.1f;
        vx = __double2float_rn(DADD(DMUL(fabs(g0), a.v_e_src), a.v_bohm));
        vy = __double2float_rn(DMUL(g1, a.v_e_src));
        vz = __double2float_rn(DMUL(g2, a.v_e_src));
      } else {
        double u = philox_uniform(a.seed, id, SITE_NEUT_Y, a.step, 0);
        y = __double2float_rn(DADD(0.0, DMUL(DSUB(a.neut_r, 0.0), u)));
        double g0 = philox_normal(a.seed, id, SITE_NEUT_V, a.step, 0);
        double g1 = philox_normal(a.seed, id, SITE_NEUT_V, a.step, 1);
        double g2 = philox_normal(a.seed, id, SITE_NEUT_V, a.step, 2);
        x = a.neut_x;
        vx = __double2float_rn(DMUL(g0, a.v_e_th));
        vy = __double2float_rn(DMUL(g1, a.v_e_th));
        vz = __double2float_rn(DMUL(g2, a.v_e_th));
      }
      a.eles.x[slot] = x; a.eles.y[slot] = y;
      a.eles.vx[slot] = vx; a.eles.vy[slot] = vy; a.eles.vz[slot] = vz;
      a.eles.id[slot] = id;
      atomicAdd(a.cnt_e + dep_cell(x, y, a.dxf, a.dyf, a.nx, a.ny), 1);
    }
  }
}

// ------------------------------------------------------------------ single-block bitonic sort
// Sorts keys[0..n) ascending in place (global memory; one block, any n <= cap).
__device__ void block_sort_u64(uint64_t* keys, int n) {
  int m = 1;
  while (m < n) m <<= 1;
  for (int i = n + threadIdx.x; i < m; i += blockDim.x) keys[i] = ~0ull;
  __syncthreads();
  for (int k = 2; k <= m; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < m; i += blockDim.x) {
        int l = i ^ j;
        if (l > i) {
          uint64_t a = keys[i], b = keys[l];
          bool up = (i & k) == 0;
          if ((a > b) == up) { keys[i] = b; keys[l] = a; }
        }
      }
      __syncthreads();
    }
  }
}

// ------------------------------------------------------------------ SEE electrons
// Spawned electrons in parent-id order (= the reference's array order), keyed draws by
// the parent ion, purge test against the current isBound, appended after the step's
// surviving electrons (physics_engine.py:1400-1417, 1541-1561).
__global__ void k_see_finish(SeeArgs a) {
  pdl_enter();
  if (a.step_dev) a.step = *a.step_dev;
  __shared__ int sm[32];
  __shared__ int s_base, s_total;
  int n = *a.see_count;
  if (n > a.see_cap) n = a.see_cap;
  block_sort_u64(a.see_key, n);
  const int ne0 = *a.num_e;
  const uint32_t id0 = *a.next_e_id;
  int done = 0;
  for (int c0 = 0; c0 < n; c0 += blockDim.x) {
    int r = c0 + threadIdx.x;
    bool keep = false;
    float x = 0, y = 0, vx = 0, vy = 0, vz = 0;
    uint32_t parent = 0;
    if (r < n) {
      uint64_t key = a.see_key[r];
      parent = (uint32_t)(key >> 32);
      uint32_t rec = (uint32_t)key;
      x = a.see_xy[2 * rec];
      y = a.see_xy[2 * rec + 1];
      vx = __double2float_rn(DMUL(philox_normal(a.seed, parent, SITE_SEE_V, a.step, 0), a.v_see_th));
      vy = __double2float_rn(DMUL(philox_normal(a.seed, parent, SITE_SEE_V, a.step, 1), a.v_see_th));
      vz = __double2float_rn(DMUL(philox_normal(a.seed, parent, SITE_SEE_V, a.step, 2), a.v_see_th));
      int icx = cell_round(x, a.dxf, 0, a.nx - 1), icy = cell_round(y, a.dyf, 0, a.ny - 1);
      bool dead = a.isBound[(size_t)icy * a.nx + icx] != 0;
      dead = dead || (x < 0.0f) || (x > a.Lxf) || (y < 0.0f) || (y > a.Lyf) || (x != x);
      keep = !dead;
    }
    // block scan of keep flags (chunk order = parent order)
    unsigned b = __ballot_sync(0xFFFFFFFFu, keep);
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int pre = __popc(b & ((1u << lane) - 1));
    if (lane == 0) sm[w] = __popc(b);
    __syncthreads();
    if (threadIdx.x == 0) {
      int s = 0;
      for (int q = 0; q < (int)(blockDim.x >> 5); ++q) { int t = sm[q]; sm[q] = s; s += t; }
      s_base = done;
      s_total = s;
    }
    __syncthreads();
    if (keep) {
      int slot = ne0 + s_base + sm[w] + pre;
      if (slot < a.cap_e) {
        a.eles.x[slot] = x; a.eles.y[slot] = y;
        a.eles.vx[slot] = vx; a.eles.vy[slot] = vy; a.eles.vz[slot] = vz;
        a.eles.id[slot] = id0 + r;
        atomicAdd(a.cnt_e + dep_cell(x, y, a.dxf, a.dyf, a.nx, a.ny), 1);
      } else {
        atomicOr(a.errflags, PB_EF_CAPACITY_ELE);
      }
    }
    done += s_total;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    int tot = ne0 + done;
    *a.num_e = tot < a.cap_e ? tot : a.cap_e;
    *a.next_e_id = id0 + (uint32_t)n;
    *a.see_spawned = n;
  }
}

// ------------------------------------------------------------------ exit divergence
// np.percentile(angles, 95) for float32 data: q = f32(95)/f32(100), v = f32(n-1)*q,
// linear interpolation with NumPy's two-sided lerp, all in float32.
PB_HD float percentile95_sorted(const float* s, int n) {
  float q = 95.0f / 100.0f;
  float vi = (float)(n - 1) * q;
  if (vi >= (float)(n - 1)) return s[n - 1];
  float prev = floorf(vi);
  float g = vi - prev;
  int i = (int)prev;
  float lo = s[i], hi = s[i + 1];
  float d = hi - lo;
  return g >= 0.5f ? hi - d * (1.0f - g) : lo + d * g;
}

__global__ void k_theta95(float* angles, const int* count, int cap, uint64_t* scratch, double* out) {
  pdl_enter();
  int n = *count;
  if (n > cap) n = cap;
  if (n <= 5) {
    if (threadIdx.x == 0) *out = __longlong_as_double(0x7ff8000000000000ll);
    return;
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) scratch[i] = (uint64_t)__float_as_uint(angles[i]);
  __syncthreads();
  block_sort_u64(scratch, n);
  for (int i = threadIdx.x; i < n; i += blockDim.x) angles[i] = __uint_as_float((uint32_t)scratch[i]);
  __syncthreads();
  if (threadIdx.x == 0) *out = (double)percentile95_sorted(angles, n);
}

// ------------------------------------------------------------------ sputter cell break
// broken = (damage > Thresh) & isBound -> eroded_depth += dy, isBound = 0, damage = 0,
// and the node class is recomputed so the next field solve uses the new operator
// (physics_engine.py:1443-1449, 525-552).
__global__ void k_erosion_break(double* damage, uint8_t* isBound, uint8_t* cls, double* eroded, int ny, int nx,
                                int periodic, double thresh, double dy, int* broken) {
  pdl_enter();
  int N = ny * nx;
  int cntb = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    if (isBound[i] && damage[i] > thresh) {
      eroded[i] += dy;
      isBound[i] = 0;
      damage[i] = 0.0;
      int y = i / nx, x = i - y * nx;
      uint8_t c = 0;  // NC_FREE
      if (x == nx - 1) c = 2;
      else if (!periodic && (y == 0 || y == ny - 1)) c = 2;
      cls[i] = c;
      ++cntb;
    }
  }
  if (cntb) atomicAdd(broken, cntb);
}

// After a break the fine-level smoother weights follow the new node classes, and the
// hierarchy is marked dirty: k_mg_rebuild forms the coarse levels again before the next
// field solve.  (Should it leave them to the host, the V-cycle with the old coarse levels
// stays symmetric positive definite: its smoother part is, once every free node has its
// weight, and the coarse part adds a semidefinite term.)  The weights are the host build's,
// omega / (4 - Neumann neighbours) in double rounded to float, 0 off the free nodes.
__global__ void k_refresh_dinv0(const uint8_t* cls, float* dinv, int ny, int nx, int periodic, const int* broken,
                                int* mg_dirty) {
  pdl_enter();
  if (*broken == 0) return;
  if (blockIdx.x == 0 && threadIdx.x == 0) *mg_dirty = 1;  // the coarse levels follow before the next solve
  const int N = ny * nx;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    float d = 0.0f;
    if (cls[i] == NC_FREE) {
      const int y = i / nx, x = i - y * nx;
      int nneu = 0;
      // left, right, down, up; outside the grid counts as a Neumann neighbour
      nneu += x == 0 || cls[i - 1] == NC_NEU;
      nneu += x == nx - 1 || cls[i + 1] == NC_NEU;
      int yd = y - 1, yu = y + 1;
      if (periodic) { if (yd < 0) yd += ny; if (yu >= ny) yu -= ny; }
      nneu += yd < 0 || cls[yd * nx + x] == NC_NEU;
      nneu += yu >= ny || cls[yu * nx + x] == NC_NEU;
      if (nneu < 4) d = (float)(MG_JACOBI_OMEGA / (double)(4 - nneu));
    }
    dinv[i] = d;
  }
}

// ------------------------------------------------------------------ thermal
// Radiative cooling of bound cells, 10 explicit FTCS sweeps over interior bound cells
// (non-bound neighbours replaced by the centre value, T_new = max(T + dT, 300)) and the
// final clamp, fused with temporal blocking: each block owns a TT x TT output tile and
// loads a halo of SWEEPS cells (physics_engine.py:1566-1615, CPU-loop semantics).
constexpr int TT = 32;
constexpr int HALO = 10;
constexpr int TW = TT + 2 * HALO;

__global__ void __launch_bounds__(256) k_thermal(float* T, const uint8_t* isBound, int ny, int nx, float cf,
                                                 float T4_300, float Fo_x, float Fo_y, int sweeps) {
  pdl_enter();
  __shared__ float A[TW * TW], B[TW * TW];
  __shared__ uint8_t M[TW * TW];
  __shared__ int any;
  const int gx0 = blockIdx.x * TT - HALO, gy0 = blockIdx.y * TT - HALO;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  int found = 0;
  for (int k = threadIdx.x; k < TW * TW; k += blockDim.x) {
    int ly = k / TW, lx = k - ly * TW;
    int gy = gy0 + ly, gx = gx0 + lx;
    bool in = gy >= 0 && gy < ny && gx >= 0 && gx < nx;
    float t = 0.0f;
    uint8_t m = 0;
    if (in) {
      t = T[(size_t)gy * nx + gx];
      m = isBound[(size_t)gy * nx + gx];
      if (m) {
        // T -= cf * (T**4 - 300**4)   (x^4 rounded once from double)
        double td = (double)t;
        float t4 = __double2float_rn(DMUL(DMUL(td, td), DMUL(td, td)));
        t = __fsub_rn(t, __fmul_rn(cf, __fsub_rn(t4, T4_300)));
        found = 1;
      }
    }
    A[k] = t;
    M[k] = m | (in ? 2 : 0);
  }
  if (found) any = 1;
  __syncthreads();
  if (!any) return;
  float* cur = A;
  float* nxt = B;
  for (int s = 0; s < sweeps; ++s) {
    for (int k = threadIdx.x; k < TW * TW; k += blockDim.x) {
      int ly = k / TW, lx = k - ly * TW;
      int gy = gy0 + ly, gx = gx0 + lx;
      float c = cur[k];
      float v = c;
      bool upd = (M[k] & 1) && gy >= 1 && gy <= ny - 2 && gx >= 1 && gx <= nx - 2 && ly >= 1 && ly <= TW - 2 &&
                 lx >= 1 && lx <= TW - 2;
      if (upd) {
        float tl = (M[k - 1] & 1) ? cur[k - 1] : c;
        float tr = (M[k + 1] & 1) ? cur[k + 1] : c;
        float td = (M[k - TW] & 1) ? cur[k - TW] : c;
        float tu = (M[k + TW] & 1) ? cur[k + TW] : c;
        float c2 = __fmul_rn(2.0f, c);
        float dT = __fadd_rn(__fmul_rn(Fo_x, __fadd_rn(__fsub_rn(tl, c2), tr)),
                             __fmul_rn(Fo_y, __fadd_rn(__fsub_rn(td, c2), tu)));
        float nv = __fadd_rn(c, dT);
        v = (nv != nv) ? nv : (nv > 300.0f ? nv : 300.0f);
      }
      nxt[k] = v;
    }
    __syncthreads();
    float* t = cur; cur = nxt; nxt = t;
  }
  for (int k = threadIdx.x; k < TW * TW; k += blockDim.x) {
    int ly = k / TW, lx = k - ly * TW;
    if (ly < HALO || ly >= HALO + TT || lx < HALO || lx >= HALO + TT) continue;
    int gy = gy0 + ly, gx = gx0 + lx;
    if (gy >= ny || gx >= nx) continue;
    float v = cur[k];
    if (M[k] & 1) v = (v != v) ? v : (v > 300.0f ? v : 300.0f);
    T[(size_t)gy * nx + gx] = v;
  }
}

// grid means over each electrode mask (bit g of gridmask) -> sums[2g], counts[2g+1]
// Block-wide reduction with op; the result is valid in thread 0.  Ends with a barrier, so
// it can be called again at once.  blockDim.x is a multiple of 32.
template <class T, class Op>
__device__ __forceinline__ T block_reduce(T v, Op op, T ident) {
  __shared__ T sm[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) v = op(v, __shfl_down_sync(0xFFFFFFFFu, v, o));
  if (lane == 0) sm[warp] = v;
  __syncthreads();
  if (warp == 0) {
    v = lane < (int)(blockDim.x >> 5) ? sm[lane] : ident;
    for (int o = 16; o > 0; o >>= 1) v = op(v, __shfl_down_sync(0xFFFFFFFFu, v, o));
  }
  __syncthreads();
  return v;
}

__global__ void k_grid_sums(const float* T, const uint16_t* gridmask, int N, int ngrids, double* out) {
  pdl_enter();
  double s[16];
  double c[16];
  for (int g = 0; g < ngrids; ++g) { s[g] = 0; c[g] = 0; }
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    uint16_t m = gridmask[i];
    if (!m) continue;
    double t = (double)T[i];
    for (int g = 0; g < ngrids; ++g)
      if (m & (1u << g)) { s[g] += t; c[g] += 1.0; }
  }
  // one pair of atomics per block and grid (per-warp atomics on the same 2 * ngrids
  // words serialised at L2)
  const auto add = [](double a, double b) { return a + b; };
  for (int g = 0; g < ngrids; ++g) {
    const double a = block_reduce(s[g], add, 0.0), b = block_reduce(c[g], add, 0.0);
    if (threadIdx.x == 0 && b != 0.0) { atomicAdd(out + 2 * g, a); atomicAdd(out + 2 * g + 1, b); }
  }
}

// ------------------------------------------------------------------ PPC statistics
// accum += ppc; total active cells, cells with 0 < ppc < 3, min nonzero
__global__ void k_ppc_stats(const int* ppc, double* accum, int N, unsigned long long* stats) {
  pdl_enter();
  unsigned long long act = 0, low = 0;
  int mn = 0x7fffffff;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    int v = ppc[i];
    accum[i] += (double)v;
    if (v > 0) { ++act; if (v < 3) ++low; mn = v < mn ? v : mn; }
  }
  const auto add = [](unsigned long long a, unsigned long long b) { return a + b; };
  act = block_reduce(act, add, 0ull);
  low = block_reduce(low, add, 0ull);
  mn = block_reduce(mn, [](int a, int b) { return a < b ? a : b; }, 0x7fffffff);
  if (threadIdx.x == 0) {
    if (act) atomicAdd(stats, act);
    if (low) atomicAdd(stats + 1, low);
    atomicMin(stats + 2, (unsigned long long)mn);
  }
}

// ------------------------------------------------------------------ Taichi-kernel thermal sweep
// thermal_conduction_taichi (physics_engine.py:147-171): every masked cell, neighbours
// inside the domain and masked, T_new = max(T + dT, 300); unmasked cells copied.
__global__ void k_thermal_taichi(const float* T, float* Tn, const int32_t* mask, int nx, int ny, float Fo_x,
                                 float Fo_y) {
  pdl_enter();
  int N = nx * ny;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    int iy = i / nx, ix = i - iy * nx;
    float c = T[i];
    if (mask[i] == 1) {
      float tl = (ix > 0 && mask[i - 1] == 1) ? T[i - 1] : c;
      float tr = (ix < nx - 1 && mask[i + 1] == 1) ? T[i + 1] : c;
      float tu = (iy < ny - 1 && mask[i + nx] == 1) ? T[i + nx] : c;
      float td = (iy > 0 && mask[i - nx] == 1) ? T[i - nx] : c;
      float c2 = __fmul_rn(2.0f, c);
      float dT = __fadd_rn(__fmul_rn(Fo_x, __fadd_rn(__fsub_rn(tl, c2), tr)),
                           __fmul_rn(Fo_y, __fadd_rn(__fsub_rn(td, c2), tu)));
      float nv = __fadd_rn(c, dT);
      Tn[i] = nv > 300.0f ? nv : 300.0f;
    } else {
      Tn[i] = c;
    }
  }
}

// ------------------------------------------------------------------ cell-key radix sort
// Stable LSD radix sort of (key, index) pairs, RADIX_BITS per pass; identical permutation
// to np.argsort(key, kind="stable").  Three kernels per pass: tile digit histograms,
// a digit-major exclusive scan, and a stable scatter (warp-ordered ranks).
__global__ void k_sort_keys(const float* x, const float* y, const int* n_dev, int nx, int ny, float dxf, float dyf,
                            uint32_t* key, uint32_t* val) {
  pdl_enter();
  int n = *n_dev;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    key[i] = (uint32_t)dep_cell(x[i], y[i], dxf, dyf, nx, ny);
    val[i] = (uint32_t)i;
  }
}

__global__ void __launch_bounds__(SORT_NT) k_sort_hist(const uint32_t* key, const int* n_dev, int shift,
                                                       uint32_t* hist, int ntiles) {
  pdl_enter();
  __shared__ uint32_t h[RADIX];
  int n = *n_dev;
  for (int d = threadIdx.x; d < RADIX; d += blockDim.x) h[d] = 0;
  __syncthreads();
  int tile = blockIdx.x;
  int t0 = tile * SORT_TILE;
  for (int k = threadIdx.x; k < SORT_TILE; k += blockDim.x) {
    int i = t0 + k;
    if (i < n) atomicAdd(&h[(key[i] >> shift) & (RADIX - 1)], 1u);
  }
  __syncthreads();
  for (int d = threadIdx.x; d < RADIX; d += blockDim.x) hist[(size_t)d * ntiles + tile] = h[d];
}

// exclusive scan of hist (RADIX * ntiles, digit-major) in one block
__global__ void __launch_bounds__(1024) k_sort_scan(uint32_t* hist, int total) {
  pdl_enter();
  __shared__ uint32_t carry;
  __shared__ uint32_t sm[32];
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int c0 = 0; c0 < total; c0 += blockDim.x) {
    int i = c0 + threadIdx.x;
    uint32_t v = i < total ? hist[i] : 0u;
    uint32_t inc = v;
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t t = __shfl_up_sync(0xFFFFFFFFu, inc, o);
      if (lane >= o) inc += t;
    }
    if (lane == 31) sm[w] = inc;
    __syncthreads();
    if (w == 0) {
      uint32_t s = lane < (int)(blockDim.x >> 5) ? sm[lane] : 0u;
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xFFFFFFFFu, s, o);
        if (lane >= o) s += t;
      }
      sm[lane] = s;
    }
    __syncthreads();
    uint32_t ex = carry + (w ? sm[w - 1] : 0u) + inc - v;
    if (i < total) hist[i] = ex;
    __syncthreads();
    if (threadIdx.x == 0) carry += sm[(blockDim.x >> 5) - 1];
    __syncthreads();
  }
}

// Multi-block exclusive scan of a long uint32 array: per-chunk sums, a one-block scan of
// the sums (k_sort_scan), then each chunk scanned from its base.
constexpr int SCAN_NT = 1024, SCAN_PER = 8, SCAN_CHUNK = SCAN_NT * SCAN_PER;

__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* total) {
  __shared__ uint32_t sm[SCAN_NT / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t inc = v;
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t t = __shfl_up_sync(0xFFFFFFFFu, inc, o);
    if (lane >= o) inc += t;
  }
  if (lane == 31) sm[w] = inc;
  __syncthreads();
  if (w == 0) {
    uint32_t s = lane < SCAN_NT / 32 ? sm[lane] : 0u;
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t t = __shfl_up_sync(0xFFFFFFFFu, s, o);
      if (lane >= o) s += t;
    }
    sm[lane] = s;
  }
  __syncthreads();
  const uint32_t ex = (w ? sm[w - 1] : 0u) + inc - v;
  if (total) *total = sm[SCAN_NT / 32 - 1];
  __syncthreads();
  return ex;
}

__global__ void __launch_bounds__(SCAN_NT) k_scan_partials(const uint32_t* a, int total, uint32_t* bsum) {
  pdl_enter();
  const int base = blockIdx.x * SCAN_CHUNK + threadIdx.x * SCAN_PER;
  uint32_t s = 0u;
#pragma unroll
  for (int k = 0; k < SCAN_PER; ++k)
    if (base + k < total) s += a[base + k];
  uint32_t t;
  block_excl_scan(s, &t);
  if (threadIdx.x == 0) bsum[blockIdx.x] = t;
}

__global__ void __launch_bounds__(SCAN_NT) k_scan_apply(uint32_t* a, int total, const uint32_t* bsum) {
  pdl_enter();
  const int base = blockIdx.x * SCAN_CHUNK + threadIdx.x * SCAN_PER;
  uint32_t v[SCAN_PER];
  uint32_t s = 0u;
#pragma unroll
  for (int k = 0; k < SCAN_PER; ++k) {
    v[k] = base + k < total ? a[base + k] : 0u;
    s += v[k];
  }
  uint32_t ex = block_excl_scan(s, nullptr) + bsum[blockIdx.x];
#pragma unroll
  for (int k = 0; k < SCAN_PER; ++k) {
    if (base + k < total) a[base + k] = ex;
    ex += v[k];
  }
}

// stable scatter: within a tile, elements are ranked per digit in index order
__global__ void __launch_bounds__(SORT_NT) k_sort_scatter(const uint32_t* key, const uint32_t* val, const int* n_dev,
                                                          int shift, const uint32_t* offs, int ntiles,
                                                          uint32_t* key_out, uint32_t* val_out) {
  pdl_enter();
  __shared__ uint32_t base[RADIX];
  __shared__ uint32_t wcount[SORT_NT / 32][RADIX];
  int n = *n_dev;
  int tile = blockIdx.x;
  int t0 = tile * SORT_TILE;
  for (int d = threadIdx.x; d < RADIX; d += blockDim.x) base[d] = offs[(size_t)d * ntiles + tile];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int NW = SORT_NT / 32;
  // process the tile in rounds of SORT_NT consecutive elements (index order)
  for (int r0 = 0; r0 < SORT_TILE; r0 += SORT_NT) {
    for (int d = lane; d < RADIX; d += 32) wcount[w][d] = 0;
    __syncthreads();
    int i = t0 + r0 + threadIdx.x;
    bool v = i < n;
    uint32_t k = v ? key[i] : 0u;
    uint32_t d = (k >> shift) & (RADIX - 1);
    unsigned peers = __match_any_sync(0xFFFFFFFFu, v ? d : 0xFFFFFFFFu);
    int rank_in_warp = __popc(peers & ((1u << lane) - 1));
    if (v && rank_in_warp == 0) wcount[w][d] = __popc(peers);
    __syncthreads();
    if (v) {
      uint32_t before = 0;
      for (int q = 0; q < w; ++q) before += wcount[q][d];
      uint32_t pos = base[d] + before + rank_in_warp;
      key_out[pos] = k;
      val_out[pos] = val[i];
    }
    __syncthreads();
    // advance digit bases by this round's counts
    for (int dd = threadIdx.x; dd < RADIX; dd += blockDim.x) {
      uint32_t s = 0;
      for (int q = 0; q < NW; ++q) s += wcount[q][dd];
      base[dd] += s;
    }
    __syncthreads();
  }
}

// gather one species' SoA through the permutation
__global__ void k_sort_gather(Soa src, Soa dst, const uint32_t* perm, const int* n_dev) {
  pdl_enter();
  int n = *n_dev;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint32_t j = perm[i];
    dst.x[i] = src.x[j]; dst.y[i] = src.y[j];
    dst.vx[i] = src.vx[j]; dst.vy[i] = src.vy[j]; dst.vz[i] = src.vz[j];
    dst.id[i] = src.id[j];
    if (src.cex) dst.cex[i] = src.cex[j];
  }
}

// copy the device count to another slot (num_dst of a sort = num_src)
__global__ void k_copy_int(const int* a, int* b) { pdl_enter(); *b = *a; }

// ------------------------------------------------------------------ distance to electrodes
// Chebyshev distance (in cells, capped at BDIST_CAP) from every node to the nearest bound
// node; the ion step uses it to skip path samples that cannot reach a bound cell.  Cells
// only ever leave isBound during a run (erosion), so the map stays a lower bound.
constexpr int BDIST_CAP = 15;

__global__ void k_bdist_rows(const uint8_t* __restrict__ isBound, uint8_t* hrow, int ny, int nx) {
  pdl_enter();
  const int N = ny * nx;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const int y = i / nx, x = i - y * nx;
    int best = BDIST_CAP;
    for (int d = 0; d < BDIST_CAP; ++d)
      if ((x - d >= 0 && isBound[i - d]) || (x + d < nx && isBound[i + d])) { best = d; break; }
    hrow[i] = (uint8_t)best;
  }
}

__global__ void k_bdist_cols(const uint8_t* __restrict__ hrow, uint8_t* dist, int ny, int nx) {
  pdl_enter();
  const int N = ny * nx;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const int y = i / nx, x = i - y * nx;
    int best = BDIST_CAP;
    for (int dy = -(BDIST_CAP - 1); dy <= BDIST_CAP - 1; ++dy) {
      const int yy = y + dy;
      if (yy < 0 || yy >= ny) continue;
      const int ady = dy < 0 ? -dy : dy;
      const int v = max(ady, (int)hrow[yy * nx + x]);
      best = min(best, v);
    }
    dist[i] = (uint8_t)best;
  }
}

// ------------------------------------------------------------------ NumPy float32 sums
// np.sum of a C-contiguous float32 array is 0 + pw(a, n), where pw is NumPy's pairwise
// summation: for n < 8 a running sum from 0; for 8 <= n <= 128 eight running sums over
// a[q], a[q + 8], ... (q = 0..7, started at a[q]) while a full group of eight remains,
// combined as ((r0 + r1) + (r2 + r3)) + ((r4 + r5) + (r6 + r7)), then the remaining
// elements in order; above 128, pw(a, m) + pw(a + m, n - m) with m = n / 2 rounded down to
// a multiple of 8.  All in float32.  The host lays out that tree for n (leaf ranges, and
// the internal nodes by height); k_pw_leaves sums the leaves and k_pw_combine the internal
// nodes, so the result is NumPy's, bit for bit.  Element i is a_i^2 + b_i^2 (+ c_i^2),
// rounded as NumPy evaluates a**2 + b**2 + c**2 on float32 arrays.
struct PwSrc {
  const float* a;
  const float* b;
  const float* c;  // may be null
};

__device__ __forceinline__ float pw_elem(const PwSrc& s, long long i) {
  const float a = __ldg(s.a + i), b = __ldg(s.b + i);
  float v = __fadd_rn(__fmul_rn(a, a), __fmul_rn(b, b));
  if (s.c) {
    const float c = __ldg(s.c + i);
    v = __fadd_rn(v, __fmul_rn(c, c));
  }
  return v;
}

__global__ void k_pw_leaves(PwSrc src, const long long* __restrict__ leaf_lo, int nleaves, float* vals) {
  pdl_enter();
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nleaves; k += gridDim.x * blockDim.x) {
    const long long lo = leaf_lo[k];
    const int n = (int)(leaf_lo[k + 1] - lo);
    float res;
    if (n < 8) {
      res = 0.0f;
      for (int i = 0; i < n; ++i) res = __fadd_rn(res, pw_elem(src, lo + i));
    } else {
      float r[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) r[q] = pw_elem(src, lo + q);
      int i = 8;
      for (; i < n - (n % 8); i += 8) {
#pragma unroll
        for (int q = 0; q < 8; ++q) r[q] = __fadd_rn(r[q], pw_elem(src, lo + i + q));
      }
      res = __fadd_rn(__fadd_rn(__fadd_rn(r[0], r[1]), __fadd_rn(r[2], r[3])),
                      __fadd_rn(__fadd_rn(r[4], r[5]), __fadd_rn(r[6], r[7])));
      for (; i < n; ++i) res = __fadd_rn(res, pw_elem(src, lo + i));
    }
    vals[k] = res;
  }
}

// one block: internal node j (height order) = vals[left[j]] + vals[right[j]], stored at
// vals[nleaves + j]; then *out = 0 + the root (root < 0: no elements)
__global__ void k_pw_combine(float* vals, const int* __restrict__ left, const int* __restrict__ right,
                             const int* __restrict__ height_off, int nheights, int nleaves, int root, float* out) {
  pdl_enter();
  for (int h = 0; h < nheights; ++h) {
    for (int j = height_off[h] + (int)threadIdx.x; j < height_off[h + 1]; j += blockDim.x)
      vals[nleaves + j] = __fadd_rn(vals[left[j]], vals[right[j]]);
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = __fadd_rn(0.0f, root >= 0 ? vals[root] : 0.0f);
}

}  // namespace pb
