// Damped Boltzmann-electron Picard loop with a geometric-multigrid-preconditioned CG
// linear solver, in one cooperative (persistent) kernel.
//
// Reference: DigitalTwinSimulator.recalc_poisson / _recalc_poisson_cpu
// (Python/physics_engine.py:850-902) solves, each Picard iteration,
//     A V_new = b,  b = V_fixed on Dirichlet rows, -coeff * (rho + rho_e(V)) on free rows,
// with Neumann rows copying the inward neighbour (:556-574), by SuperLU; then
//     V <- (1 - omega) V + omega V_new   (omega = 0.2)
// and finally E = -grad V with np.gradient (:871-884).
//
// Here the Dirichlet and Neumann rows are eliminated, which leaves the SPD operator
//     (4 - n_neumann_nbrs) V_i - sum_{free nbrs} V_j = coeff*rho_total_i + sum_{Dirichlet nbrs} V_fixed_j
// on the free nodes.  It is solved by FP32 MG-PCG inside an FP64 iterative-refinement
// loop (FP64 residual f - A x, FP64 dot products).  The multigrid hierarchy is
// Galerkin (coarse = P^T A P, 9-point stencils) with bilinear P, red-black Gauss-Seidel
// on the 5-point fine level, 4- or 6-colour Gauss-Seidel on coarse levels (symmetric
// ordering, so the V-cycle is an SPD preconditioner) and a dense inverse on the coarsest.
//
// Grid-wide phases are separated by a software grid barrier (cooperative launch
// guarantees co-residency).  Every wait is bounded: on time-out the kernel sets
// PB_EF_SPIN_TIMEOUT, stops waiting at later barriers and runs to completion.
// Reductions are deterministic: one partial per block, summed in block order.
// Data written by other blocks within the launch is read only after a grid barrier,
// which ends with an acquire fence in every thread.
#include "pb_common.cuh"
#include "pb_poisson.cuh"

namespace pb {

constexpr int PT = 512;  // threads per block
constexpr long long BAR_SPIN_LIMIT = 1ll << 22;

__device__ __forceinline__ void grid_barrier(unsigned int* bar, uint32_t* err) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned int* vgen = bar + 1;
    volatile uint32_t* verr = err;
    unsigned int gen = *vgen;
    __threadfence();
    unsigned int arrived = atomicAdd(bar, 1u);
    if (arrived == gridDim.x - 1) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      long long spin = 0;
      while (*vgen == gen) {
        if ((*verr & PB_EF_SPIN_TIMEOUT) != 0u) break;
        if (++spin > BAR_SPIN_LIMIT) { atomicOr(err, PB_EF_SPIN_TIMEOUT); break; }
      }
    }
    __threadfence();
  }
  __syncthreads();
  // every thread acquires at gpu scope, so its later (L1-cached) loads observe the
  // stores other blocks made before arriving
  asm volatile("fence.acq_rel.gpu;" ::: "memory");
}

// phase tracing (block 0, thread 0): time since the previous mark is added to trace[k]
__device__ __forceinline__ void tmark(const PoissonArgs& a, int k) {
  if (a.trace && blockIdx.x == 0 && threadIdx.x == 0) {
    unsigned long long now;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
    unsigned long long last = a.trace[31];
    if (last) a.trace[k] += now - last;
    a.trace[31] = now;
  }
}

// deterministic grid-wide sum; contains one barrier
__device__ double grid_sum(double v, const PoissonArgs& a, int& slot) {
  __shared__ double sm[PT / 32];
  __shared__ double bc;
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, o);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
  __syncthreads();
  double* part = a.partials + (size_t)(slot & 3) * gridDim.x;
  if (threadIdx.x < 32) {
    double s = threadIdx.x < PT / 32 ? sm[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xFFFFFFFFu, s, o);
    if (threadIdx.x == 0) __stcg(part + blockIdx.x, s);
  }
  grid_barrier(a.bar, a.errflags);
  if (threadIdx.x < 32) {
    // lanes take fixed strided subsets, then a fixed shuffle tree: same order in every block
    double s = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += 32) s += (*(part + b));
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xFFFFFFFFu, s, o);
    if (threadIdx.x == 0) bc = s;
  }
  __syncthreads();
  double r = bc;
  __syncthreads();
  ++slot;
  return r;
}

// ----------------------------------------------------------------- level-0 (5-point) helpers
struct Nb { int j; uint8_t c; };  // neighbour index and class (NC_NEU when outside)

__device__ __forceinline__ Nb nb0(const PoissonArgs& a, int y, int x, int dy, int dx) {
  Nb r;
  int yy = y + dy, xx = x + dx;
  if (a.periodic) { if (yy < 0) yy += a.ny; else if (yy >= a.ny) yy -= a.ny; }
  if (yy < 0 || yy >= a.ny || xx < 0 || xx >= a.nx) { r.j = -1; r.c = NC_NEU; return r; }
  r.j = yy * a.nx + xx;
  r.c = __ldg(a.cls + r.j);
  return r;
}

// (A v)_i and diag_i on the fine level for a free node i (float vector, read via L2)
__device__ __forceinline__ float apply0f(const PoissonArgs& a, const float* v, int i, int y, int x, float& diag) {
  const int DY[4] = {0, 0, -1, 1}, DX[4] = {-1, 1, 0, 0};
  float s = 0.0f;
  int nneu = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    Nb n = nb0(a, y, x, DY[k], DX[k]);
    if (n.c == NC_FREE) s += (*(v + n.j));
    else if (n.c == NC_NEU) ++nneu;
  }
  diag = (float)(4 - nneu);
  return diag * (*(v + i)) - s;
}

__device__ __forceinline__ double apply0d(const PoissonArgs& a, const double* v, int i, int y, int x) {
  const int DY[4] = {0, 0, -1, 1}, DX[4] = {-1, 1, 0, 0};
  double s = 0.0;
  int nneu = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    Nb n = nb0(a, y, x, DY[k], DX[k]);
    if (n.c == NC_FREE) s += (*(v + n.j));
    else if (n.c == NC_NEU) ++nneu;
  }
  return (double)(4 - nneu) * (*(v + i)) - s;
}

// ----------------------------------------------------------------- coarse (9-point) helpers
__device__ __forceinline__ int nbc(const MgLevel& L, int y, int x, int dI, int dJ) {
  int yy = y + dI, xx = x + dJ;
  if (L.per) { if (yy < 0) yy += L.ny; else if (yy >= L.ny) yy -= L.ny; }
  if (yy < 0 || yy >= L.ny || xx < 0 || xx >= L.nx) return -1;
  return yy * L.nx + xx;
}

// Loads and stores of level vectors.  PRIV: data only block 0 touches (the small
// levels).  Loads go through L1 in both cases: data written by other blocks is read only
// after a grid barrier, whose acquire fence orders the load after those stores.
template <bool PRIV> __device__ __forceinline__ float ldv(const float* p) { return *p; }
template <bool PRIV> __device__ __forceinline__ void stv(float* p, float v) { if (PRIV) *p = v; else __stcg(p, v); }

__device__ __forceinline__ bool active(const PoissonArgs& a, int level, int i) {
  return level == 0 ? (__ldg(a.cls + i) == NC_FREE) : (__ldg(a.lev[level].act + i) != 0);
}

// (A_l v)_i for an active node i, with v_j supplied by the callable vj(j) (inactive
// neighbours contribute nothing: their value is zero in every vector of the cycle)
template <class V>
__device__ __forceinline__ float apply_A(const PoissonArgs& a, int level, int i, int y, int x, V vj) {
  if (level == 0) {
    const int DY[4] = {0, 0, -1, 1}, DX[4] = {-1, 1, 0, 0};
    float s = 0.0f;
    int nneu = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      Nb n = nb0(a, y, x, DY[k], DX[k]);
      if (n.c == NC_FREE) s += vj(n.j);
      else if (n.c == NC_NEU) ++nneu;
    }
    return (float)(4 - nneu) * vj(i) - s;
  }
  const MgLevel& L = a.lev[level];
  const int N = L.ny * L.nx;
  float s = 0.0f;
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    int j = (k == 4) ? i : nbc(L, y, x, k / 3 - 1, k % 3 - 1);
    if (j >= 0) s += __ldg(L.st + (size_t)k * N + i) * vj(j);
  }
  return s;
}

// (P z_{l+1}) at fine node (y, x) of level l
template <bool PRIV>
__device__ __forceinline__ float prolong_at(const MgLevel& C, int y, int x) {
  int I0 = y >> 1, J0 = x >> 1, ai = y & 1, bj = x & 1;
  float s = 0.0f;
  for (int da = 0; da <= ai; ++da) {
    int I = I0 + da;
    if (I >= C.ny) { if (C.wrapP) I -= C.ny; else continue; }
    float wy = ai ? 0.5f : 1.0f;
    for (int db = 0; db <= bj; ++db) {
      int J = J0 + db;
      if (J >= C.nx) continue;
      float wx = bj ? 0.5f : 1.0f;
      s += wy * wx * ldv<PRIV>(C.z + I * C.nx + J);
    }
  }
  return s;
}

// Down leg of the V-cycle on level l: with the pre-smoothed z = omega D^-1 r (one damped
// Jacobi sweep from zero), r_{l+1} = P^T (r_l - A_l z), all evaluated from r_l.
template <bool PRIV>
__device__ __forceinline__ void down_leg(const PoissonArgs& a, int level, int tid, int nth) {
  const MgLevel& F = a.lev[level];
  const MgLevel& C = a.lev[level + 1];
  const int Nc = C.ny * C.nx;
  const bool wrap = C.wrapP;
  const float* r = F.r;
  const float* dinv = F.dinv;
  auto zpre = [&](int j) { return __ldg(dinv + j) * ldv<PRIV>(r + j); };
  for (int ic = tid; ic < Nc; ic += nth) {
    if (!__ldg(C.act + ic)) { stv<PRIV>(C.r + ic, 0.0f); continue; }
    int I = ic / C.nx, J = ic - I * C.nx;
    float s = 0.0f;
#pragma unroll
    for (int da = -1; da <= 1; ++da) {
      int yf = 2 * I + da;
      if (yf < 0) { if (wrap) yf += F.ny; else continue; }
      if (yf >= F.ny) continue;
      float wy = da == 0 ? 1.0f : 0.5f;
#pragma unroll
      for (int db = -1; db <= 1; ++db) {
        int xf = 2 * J + db;
        if (xf < 0 || xf >= F.nx) continue;
        int f = yf * F.nx + xf;
        if (!active(a, level, f)) continue;
        float wx = db == 0 ? 1.0f : 0.5f;
        float res = ldv<PRIV>(r + f) - apply_A(a, level, f, yf, xf, zpre);
        s += wy * wx * res;
      }
    }
    stv<PRIV>(C.r + ic, s);
  }
}

// Up leg on level l: z_mid = omega D^-1 r + P z_{l+1}; one damped Jacobi sweep,
// z = z_mid + omega D^-1 (r - A z_mid), all evaluated from r_l and z_{l+1}.
// PRIV_C: the coarse correction is private to block 0 as well.
template <bool PRIV, bool PRIV_C>
__device__ __forceinline__ void up_leg(const PoissonArgs& a, int level, int tid, int nth) {
  const MgLevel& F = a.lev[level];
  const MgLevel& C = a.lev[level + 1];
  const int N = F.ny * F.nx;
  const float* r = F.r;
  const float* dinv = F.dinv;
  auto zmid = [&](int j) {
    int yj = j / F.nx, xj = j - yj * F.nx;
    return __ldg(dinv + j) * ldv<PRIV>(r + j) + prolong_at<PRIV_C>(C, yj, xj);
  };
  for (int i = tid; i < N; i += nth) {
    if (!active(a, level, i)) { stv<PRIV>(F.z + i, 0.0f); continue; }
    int y = i / F.nx, x = i - y * F.nx;
    float zm = zmid(i);
    float az = apply_A(a, level, i, y, x, zmid);
    stv<PRIV>(F.z + i, zm + __ldg(dinv + i) * (ldv<PRIV>(r + i) - az));
  }
}

// coarsest level: z = A_c^{-1} r (dense, one block)
template <bool PRIV>
__device__ void coarse_solve(const PoissonArgs& a, int level) {
  const MgLevel& L = a.lev[level];
  const int N = L.ny * L.nx;
  __shared__ float rc[1024];
  for (int i = threadIdx.x; i < N; i += blockDim.x) stv<PRIV>(L.z + i, 0.0f);
  for (int k = threadIdx.x; k < a.nc; k += blockDim.x) rc[k] = ldv<PRIV>(L.r + a.cidx[k]);
  __syncthreads();
  for (int k = threadIdx.x; k < a.nc; k += blockDim.x) {
    float s = 0.0f;
    for (int j = 0; j < a.nc; ++j) s += __ldg(a.cinvT + (size_t)j * a.nc + k) * rc[j];
    stv<PRIV>(L.z + a.cidx[k], s);
  }
  __syncthreads();
}

// The levels from first_small down, run by block 0 with block-level syncs.
__device__ void small_vcycle(const PoissonArgs& a) {
  const int last = a.nlevels - 1;
  for (int l = a.first_small; l < last; ++l) {
    down_leg<true>(a, l, threadIdx.x, blockDim.x);
    __syncthreads();
  }
  coarse_solve<true>(a, last);
  for (int l = last - 1; l >= a.first_small; --l) {
    up_leg<true, true>(a, l, threadIdx.x, blockDim.x);
    __syncthreads();
  }
  // the first small level's correction is read by other blocks through L2
  __threadfence();
}

// z0 = M^{-1} r0 (lev[0].r = r32, lev[0].z = z32): a V(1,1) cycle with damped Jacobi
// smoothing, two grid barriers per grid-wide level
__device__ void vcycle(const PoissonArgs& a) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  if (a.nlevels == 1) {
    if (blockIdx.x == 0) coarse_solve<false>(a, 0);
    grid_barrier(a.bar, a.errflags);
    return;
  }
  for (int l = 0; l < a.first_small; ++l) {
    down_leg<false>(a, l, tid, nth);
    grid_barrier(a.bar, a.errflags);
    tmark(a, l < 7 ? l : 6);
  }
  if (a.first_small < a.nlevels - 1 || a.first_small == a.nlevels - 1) {
    if (blockIdx.x == 0) {
      if (a.first_small == a.nlevels - 1) {
        coarse_solve<true>(a, a.first_small);
        __threadfence();
      } else {
        small_vcycle(a);
      }
    }
    grid_barrier(a.bar, a.errflags);
  }
  tmark(a, 7);
  for (int l = a.first_small - 1; l >= 0; --l) {
    up_leg<false, false>(a, l, tid, nth);
    grid_barrier(a.bar, a.errflags);
    tmark(a, 8 + (l < 7 ? l : 6));
  }
}

// ----------------------------------------------------------------- the persistent kernel
__global__ void __launch_bounds__(PT) k_poisson(PoissonArgs a) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  const int N = a.ny * a.nx;
  const int DY[4] = {0, 0, -1, 1}, DX[4] = {-1, 1, 0, 0};
  int slot = 0;
  double n_outer = 0, n_inner = 0, last_rel = 0;
  tmark(a, 20);

  // Dirichlet-neighbour sums (V_fixed is constant during the launch)
  for (int i = tid; i < N; i += nth) {
    if (__ldg(a.cls + i) != NC_FREE) continue;
    int y = i / a.nx, x = i - y * a.nx;
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      Nb n = nb0(a, y, x, DY[k], DX[k]);
      if (n.c == NC_DIR) s += __ldg(a.Vfixed + n.j);
    }
    a.dirsum[i] = s;
  }

  for (int pic = 0; pic < a.iterations; ++pic) {
    // right-hand side from the Boltzmann electron density of the current V, residual
    double ff = 0.0, rr = 0.0;
    for (int i = tid; i < N; i += nth) {
      if (__ldg(a.cls + i) != NC_FREE) continue;
      double Vi = (*(a.V + i));
      double vm = Vi < a.V_plasma ? Vi : a.V_plasma;
      double rho_e = DMUL(a.qn0_neg, exp(DDIV(DSUB(vm, a.V_plasma), a.Te_up)));
      double rt = DADD((double)__ldg(a.rho + i), rho_e);
      double fi = DMUL(a.coeff, rt) + a.dirsum[i];
      __stcg(a.f + i, fi);
      ff += fi * fi;
    }
    for (int i = tid; i < N; i += nth) {
      if (__ldg(a.cls + i) != NC_FREE) { __stcg(a.r32 + i, 0.0f); continue; }
      int y = i / a.nx, x = i - y * a.nx;
      double res = (*(a.f + i)) - apply0d(a, a.x, i, y, x);
      __stcg(a.r32 + i, (float)res);
      rr += res * res;
    }
    double fnorm2 = grid_sum(ff, a, slot);
    double rnorm2 = grid_sum(rr, a, slot);
    tmark(a, 17);
    double target2 = a.tol * a.tol * fnorm2;

    for (int outer = 0; outer < a.max_outer && rnorm2 > target2 && fnorm2 > 0.0; ++outer) {
      n_outer += 1;
      // ---- FP32 MG-PCG on A e = r32
      for (int i = tid; i < N; i += nth) __stcg(a.e32 + i, 0.0f);
      double rz_old = 0.0, rr0 = rnorm2;
      for (int k = 0; k < a.max_inner; ++k) {
        n_inner += 1;
        tmark(a, 15);
        vcycle(a);  // z32 = M r32; ends with a barrier
        double rz_p = 0.0;
        for (int i = tid; i < N; i += nth) rz_p += (double)(*(a.r32 + i)) * (double)(*(a.z32 + i));
        double rz = grid_sum(rz_p, a, slot);
        double beta = k == 0 ? 0.0 : rz / rz_old;
        double pq_p = 0.0;
        for (int i = tid; i < N; i += nth) {
          if (__ldg(a.cls + i) != NC_FREE) { __stcg(a.p32 + i, 0.0f); __stcg(a.q32 + i, 0.0f); continue; }
          int y = i / a.nx, x = i - y * a.nx;
          float diag;
          float az = apply0f(a, a.z32, i, y, x, diag);
          float p = (*(a.z32 + i)) + (float)beta * (k == 0 ? 0.0f : (*(a.p32 + i)));
          float q = az + (float)beta * (k == 0 ? 0.0f : (*(a.q32 + i)));
          __stcg(a.p32 + i, p);
          __stcg(a.q32 + i, q);
          pq_p += (double)p * (double)q;
        }
        double pq = grid_sum(pq_p, a, slot);
        double alpha = pq != 0.0 ? rz / pq : 0.0;
        double rr_p = 0.0;
        for (int i = tid; i < N; i += nth) {
          if (__ldg(a.cls + i) != NC_FREE) continue;
          float e = (*(a.e32 + i)) + (float)alpha * (*(a.p32 + i));
          float r = (*(a.r32 + i)) - (float)alpha * (*(a.q32 + i));
          __stcg(a.e32 + i, e);
          __stcg(a.r32 + i, r);
          rr_p += (double)r * (double)r;
        }
        double rrk = grid_sum(rr_p, a, slot);
        tmark(a, 15);
        rz_old = rz;
        if (rrk <= a.tol_inner * a.tol_inner * rr0 || rrk <= target2 * 1e-4) break;
      }
      // ---- FP64 correction and true residual
      for (int i = tid; i < N; i += nth)
        if (__ldg(a.cls + i) == NC_FREE) __stcg(a.x + i, (*(a.x + i)) + (double)(*(a.e32 + i)));
      grid_barrier(a.bar, a.errflags);
      rr = 0.0;
      for (int i = tid; i < N; i += nth) {
        if (__ldg(a.cls + i) != NC_FREE) { __stcg(a.r32 + i, 0.0f); continue; }
        int y = i / a.nx, x = i - y * a.nx;
        double res = (*(a.f + i)) - apply0d(a, a.x, i, y, x);
        __stcg(a.r32 + i, (float)res);
        rr += res * res;
      }
      rnorm2 = grid_sum(rr, a, slot);
      tmark(a, 16);
    }
    if (!(rnorm2 <= target2) && fnorm2 > 0.0 && tid == 0) atomicOr(a.errflags, PB_EF_POISSON_NOCONV);
    last_rel = fnorm2 > 0.0 ? sqrt(rnorm2 / fnorm2) : 0.0;

    // ---- V_new on every node, then the damped Picard update
    for (int i = tid; i < N; i += nth) {
      uint8_t c = __ldg(a.cls + i);
      double vn;
      if (c == NC_FREE) vn = (*(a.x + i));
      else if (c == NC_DIR) vn = __ldg(a.Vfixed + i);
      else {
        int y = i / a.nx, x = i - y * a.nx;
        int sy = y, sx = x;
        if (x == a.nx - 1) {
          sx = x - 1;  // right: copy (y, nx-2), which may itself be a top/bottom copy
          uint8_t cs = __ldg(a.cls + sy * a.nx + sx);
          if (cs == NC_NEU && !a.periodic) sy = (sy == 0) ? 1 : (sy == a.ny - 1 ? a.ny - 2 : sy);
        } else if (y == 0) sy = 1;
        else sy = a.ny - 2;
        int j = sy * a.nx + sx;
        uint8_t cj = __ldg(a.cls + j);
        vn = (cj == NC_DIR) ? __ldg(a.Vfixed + j) : (*(a.x + j));
      }
      if (c != NC_FREE) __stcg(a.x + i, vn);
      double Vi = (*(a.V + i));
      __stcg(a.V + i, DADD(DMUL(a.omega_keep, Vi), DMUL(a.omega_new, vn)));
    }
    grid_barrier(a.bar, a.errflags);
    tmark(a, 18);
  }

  // ---- E = -grad V (np.gradient: central inside, one-sided at the edges; periodic y fix)
  if (a.compute_field) {
    for (int i = tid; i < N; i += nth) {
      int y = i / a.nx, x = i - y * a.nx;
      const double* V = a.V;
      double ex, ey;
      if (x == 0) ex = DDIV(DSUB(-(*(V + i + 1)), -(*(V + i))), a.hx);
      else if (x == a.nx - 1) ex = DDIV(DSUB(-(*(V + i)), -(*(V + i - 1))), a.hx);
      else ex = DDIV(DSUB(-(*(V + i + 1)), -(*(V + i - 1))), a.two_hx);
      if (a.periodic && y == 0) ey = DDIV(DSUB((*(V + (size_t)(a.ny - 1) * a.nx + x)), (*(V + a.nx + x))), a.two_hy_per);
      else if (a.periodic && y == a.ny - 1) ey = DDIV(DSUB((*(V + (size_t)(a.ny - 2) * a.nx + x)), (*(V + x))), a.two_hy_per);
      else if (y == 0) ey = DDIV(DSUB(-(*(V + i + a.nx)), -(*(V + i))), a.hy);
      else if (y == a.ny - 1) ey = DDIV(DSUB(-(*(V + i)), -(*(V + i - a.nx))), a.hy);
      else ey = DDIV(DSUB(-(*(V + i + a.nx)), -(*(V + i - a.nx))), a.two_hy);
      a.Ex[i] = __double2float_rn(ex);
      a.Ey[i] = __double2float_rn(ey);
    }
  }
  tmark(a, 19);
  if (tid == 0) {
    a.stats[0] += n_outer;
    a.stats[1] += n_inner;
    a.stats[2] = last_rel;
    a.stats[3] += (double)a.iterations;
  }
}

}  // namespace pb
