// The multigrid hierarchy rebuilt on the device after sputtered cells break.
//
// Reference: the step that breaks cells rebuilds the field matrix, so the next field solve
// sees the freed nodes (Python/physics_engine.py:1443-1449, build_sparse_matrix :525-608).
// The host build (pb_mg_host.hpp: Galerkin levels, smoother weights, the fused cycle's
// transfer stencils, the dense coarsest inverse) runs once per domain.  After a break the
// cell-break kernel has updated the node classes and the fine-level smoother weights and
// set *dirty; this kernel, launched before the next field solve, forms the coarse levels
// again from the new classes and writes the arrays the solve reads.  It follows the host
// build's order of operations term by term: every double product and sum is an explicitly
// rounded intrinsic, each sum takes its terms in the host's order, and the Cholesky
// factorisation and the inverse use the host's four-way partial dot products, with one
// four-lane group per dot product (lane t keeps partial sum t).  Its arrays are bit-equal to
// a host build from the same classes.
//
// The level count is the last host build's, and the coarsest level has a fixed capacity.
// When the freed nodes would make the host build choose other levels (a coarsest level it
// would coarsen once more), the kernel still rebuilds with the same levels, a valid cycle,
// and sets MG_STATUS_HOST so that the host rebuilds after the run.  When they cannot be
// represented (a coarsest level above its capacity, a coupling outside the 9-point pattern,
// a coarsest operator that is not positive definite) it leaves the hierarchy as it was and
// sets MG_STATUS_HOST.  Every grid-wide step ends at a bounded barrier (grid_sync).
#include "pb_common.cuh"
#include "pb_poisson.cuh"

namespace pb {
namespace {

__device__ __forceinline__ int mgb(const MgRebuildArgs& a) { return (int)blockIdx.x - a.blk0; }
__device__ __forceinline__ int mg_tid(const MgRebuildArgs& a) { return mgb(a) * (int)blockDim.x + (int)threadIdx.x; }
__device__ __forceinline__ int mg_nth(const MgRebuildArgs& a) { return a.nblk * (int)blockDim.x; }
__device__ __forceinline__ void mg_sync(const MgRebuildArgs& a) { grid_sync(a.bar, a.errflags, a.nblk, mgb(a)); }

__device__ __forceinline__ double dmul(double x, double y) { return __dmul_rn(x, y); }
__device__ __forceinline__ double dadd(double x, double y) { return __dadd_rn(x, y); }

// active node of level l (level 0: a free node)
__device__ __forceinline__ bool act_of(const MgRebuildArgs& a, int l, int i) {
  return l == 0 ? a.cls[i] == NC_FREE : (a.lev[l].act[i] & 2) != 0;
}

// neighbour (y + dy, x + dx) with the y wrap of a periodic level; -1 outside
__device__ __forceinline__ int mg_nb(int ny, int nx, int per, int y, int x, int dy, int dx) {
  int yy = y + dy;
  const int xx = x + dx;
  if (per) { if (yy < 0) yy += ny; else if (yy >= ny) yy -= ny; }
  if (yy < 0 || yy >= ny || xx < 0 || xx >= nx) return -1;
  return yy * nx + xx;
}

// prolongation parents of fine node (y, x) in the host's order (p_row): up to four
// (coarse index, weight)
__device__ __forceinline__ int mg_parents(int wrap, int nyc, int nxc, int y, int x, int* c, double* w) {
  const int I0 = y >> 1, ay = y & 1, J0 = x >> 1, bx = x & 1;
  int n = 0;
  for (int da = 0; da <= ay; ++da) {
    int I = I0 + da;
    if (I >= nyc) { if (wrap) I -= nyc; else continue; }
    const double wy = ay ? 0.5 : 1.0;
    for (int db = 0; db <= bx; ++db) {
      const int J = J0 + db;
      if (J >= nxc) continue;
      c[n] = I * nxc + J;
      w[n] = dmul(wy, bx ? 0.5 : 1.0);
      ++n;
    }
  }
  return n;
}

// The operator row of active node i of level l in the host's entry order (row_of):
// level 0 the 5-point row (free neighbours left, right, down, up at -1, then the diagonal
// 4 - Neumann neighbours), coarser levels the nonzero stencil entries to active nodes.
template <class Fn>
__device__ __forceinline__ void for_row(const MgRebuildArgs& a, int l, int i, Fn fn) {
  const MgBuildLevel& L = a.lev[l];
  const int y = i / L.nx, x = i - y * L.nx;
  if (l == 0) {
    const int DY[4] = {0, 0, -1, 1}, DX[4] = {-1, 1, 0, 0};
    int nneu = 0;
    for (int k = 0; k < 4; ++k) {
      const int j = mg_nb(L.ny, L.nx, L.per, y, x, DY[k], DX[k]);
      const uint8_t c = j < 0 ? (uint8_t)NC_NEU : a.cls[j];
      if (c == NC_FREE) fn(j, -1.0);
      else if (c == NC_NEU) ++nneu;
    }
    fn(i, (double)(4 - nneu));
    return;
  }
  const int N = L.ny * L.nx;
  for (int k = 0; k < 9; ++k) {
    const float v = L.st[(size_t)k * N + i];
    if (v == 0.0f) continue;
    const int j = mg_nb(L.ny, L.nx, L.per, y, x, k / 3 - 1, k % 3 - 1);
    if (j >= 0 && act_of(a, l, j)) fn(j, (double)v);
  }
}

// stencil entry k of active node f of level l >= 1 as the host keeps it: zero to an
// inactive or missing neighbour
__device__ __forceinline__ double st_eff(const MgRebuildArgs& a, int l, int f, int y, int x, int k) {
  const MgBuildLevel& L = a.lev[l];
  const int j = mg_nb(L.ny, L.nx, L.per, y, x, k / 3 - 1, k % 3 - 1);
  if (j < 0 || !act_of(a, l, j)) return 0.0;
  return (double)L.st[(size_t)k * L.ny * L.nx + f];
}

// Fine rows of coarse row I whose prolongation reaches it, ascending (a wrapped row -1
// comes last): returns the count, rows in ys[]
__device__ __forceinline__ int child_rows(int I, int nyf, int wrapC, int* ys) {
  int n = 0, wrapped = -1;
  for (int da = -1; da <= 1; ++da) {
    int y = 2 * I + da;
    if (y < 0) {
      if (!wrapC) continue;
      wrapped = y + nyf;
      continue;
    }
    if (y >= nyf) continue;
    ys[n++] = y;
  }
  if (wrapped >= 0) ys[n++] = wrapped;
  return n;
}

// Four-way partial dot product of the host (dot4): sum t over terms k = t mod 4 below the
// last multiple of four, the tail added to sum 0, then (s0 + s1) + (s2 + s3).  Lane t of a
// four-lane group keeps sum t; every lane of the group gets the result.  ga(k), gb(k) give
// the terms.  quad_dot4_from continues chains that already hold the terms below p (p a
// multiple of four, at most the last multiple of four below len; s is lane t's chain);
// chain_prefix forms those first p terms of lane t's chain.  Eight terms of a chain are
// loaded before they are added, in order, so the loads of a dot product overlap.
template <class GA, class GB>
__device__ __forceinline__ double chain_run(double s, GA ga, GB gb, int k, int end) {
  for (; k + 28 < end; k += 32) {
    double pa[8], pb[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      pa[u] = ga(k + 4 * u);
      pb[u] = gb(k + 4 * u);
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) s = dadd(s, dmul(pa[u], pb[u]));
  }
  for (; k < end; k += 4) s = dadd(s, dmul(ga(k), gb(k)));
  return s;
}

template <class GA, class GB>
__device__ __forceinline__ double chain_prefix(GA ga, GB gb, int p, int t) {
  return chain_run(0.0, ga, gb, t, p);
}

template <class GA, class GB>
__device__ __forceinline__ double quad_dot4_from(double s, GA ga, GB gb, int p, int len, int t, unsigned qmask) {
  const int m4 = len & ~3;
  s = chain_run(s, ga, gb, p + t, m4);
  if (t == 0)
    for (int k = m4; k < len; ++k) s = dadd(s, dmul(ga(k), gb(k)));
  const double nxt = __shfl_down_sync(qmask, s, 1, 4);
  const double pair = dadd(s, nxt);                     // lanes 0 and 2: s0 + s1, s2 + s3
  const double far = __shfl_down_sync(qmask, pair, 2, 4);
  const double tot = dadd(pair, far);                   // lane 0
  return __shfl_sync(qmask, tot, 0, 4);
}

template <class GA, class GB>
__device__ __forceinline__ double quad_dot4(GA ga, GB gb, int len, int t, unsigned qmask) {
  return quad_dot4_from(0.0, ga, gb, 0, len, t, qmask);
}

// ---- the level structure: act and Galerkin stencils of level l + 1 from level l
// Phase A: parents of active finer nodes (bit 0), less centres on Dirichlet nodes (level 1).
__device__ void phase_parents(const MgRebuildArgs& a, int l) {
  const MgBuildLevel& F = a.lev[l];
  const MgBuildLevel& C = a.lev[l + 1];
  const int Nc = C.ny * C.nx, tid = mg_tid(a), nth = mg_nth(a);
  for (int c = tid; c < Nc; c += nth) {
    const int I = c / C.nx, J = c - I * C.nx;
    int ys[3];
    const int nr = child_rows(I, F.ny, C.wrapP, ys);
    bool pre = false;
    for (int r = 0; r < nr && !pre; ++r)
      for (int db = -1; db <= 1 && !pre; ++db) {
        const int x = 2 * J + db;
        if (x < 0 || x >= F.nx) continue;
        pre = act_of(a, l, ys[r] * F.nx + x);
      }
    if (l == 0 && 2 * I < F.ny && 2 * J < F.nx && a.cls[(2 * I) * F.nx + 2 * J] == NC_DIR) pre = false;
    C.act[c] = pre ? 1 : 0;
  }
}

// Phase B: the Galerkin stencil of every node with bit 0, summed in the host's order (fine
// nodes ascending, their row entries in order, the entry's parents in order), then bit 1 =
// positive diagonal.  Returns this thread's count of active nodes.
__device__ int phase_galerkin(const MgRebuildArgs& a, int l) {
  const MgBuildLevel& F = a.lev[l];
  const MgBuildLevel& C = a.lev[l + 1];
  const int nyc = C.ny, nxc = C.nx, Nc = nyc * nxc, tid = mg_tid(a), nth = mg_nth(a);
  int nact = 0;
  for (int c = tid; c < Nc; c += nth) {
    double acc[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) acc[k] = 0.0;
    const uint8_t pre = C.act[c] & 1;
    if (pre) {
      const int I = c / nxc, J = c - I * nxc;
      int ys[3];
      const int nr = child_rows(I, F.ny, C.wrapP, ys);
      for (int r = 0; r < nr; ++r) {
        const int y = ys[r];
        const double wy = (y & 1) ? 0.5 : 1.0;
        for (int db = -1; db <= 1; ++db) {
          const int x = 2 * J + db;
          if (x < 0 || x >= F.nx) continue;
          const int f = y * F.nx + x;
          if (!act_of(a, l, f)) continue;
          const double pw = dmul(wy, db ? 0.5 : 1.0);
          for_row(a, l, f, [&](int j, double v) {
            int qc[4];
            double qw[4];
            const int m = mg_parents(C.wrapP, nyc, nxc, j / F.nx, j % F.nx, qc, qw);
            for (int b = 0; b < m; ++b) {
              if (!(C.act[qc[b]] & 1)) continue;
              int dI = qc[b] / nxc - I;
              const int dJ = qc[b] % nxc - J;
              if (C.per) { if (dI > nyc / 2) dI -= nyc; else if (dI < -(nyc / 2)) dI += nyc; }
              if (dI < -1 || dI > 1 || dJ < -1 || dJ > 1) {
                atomicOr(a.counts + MG_CNT_FLAGS, 1);
                continue;
              }
              const int k = (dI + 1) * 3 + (dJ + 1);
              acc[k] = dadd(acc[k], dmul(dmul(pw, v), qw[b]));
            }
          });
        }
      }
    }
    float s4 = 0.0f;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      const float v = __double2float_rn(acc[k]);
      if (k == 4) s4 = v;
      C.st[(size_t)k * Nc + c] = v;
    }
    const bool active = pre && s4 > 0.0f;
    C.act[c] = (uint8_t)(pre | (active ? 2 : 0));
    nact += active;
  }
  return nact;
}

__device__ __forceinline__ void count_add(int* dst, int v) {
  __shared__ int cnt;
  if (threadIdx.x == 0) cnt = 0;
  __syncthreads();
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, o);
  if ((threadIdx.x & 31) == 0 && v) atomicAdd(&cnt, v);
  __syncthreads();
  if (threadIdx.x == 0 && cnt) atomicAdd(dst, cnt);
}

// ---- transfer stencils of the fused cycle (transfer_ops), for the levels l >= 1 that have
// a coarser level: R of level l + 1 and U of level l
__device__ void transfer_R(const MgRebuildArgs& a, int l, int c) {
  const MgBuildLevel& F = a.lev[l];
  const MgBuildLevel& C = a.lev[l + 1];
  const int nyf = F.ny, nxf = F.nx, Nc = C.ny * C.nx;
  double acc[25];
  for (int k = 0; k < 25; ++k) acc[k] = 0.0;
  if (act_of(a, l + 1, c)) {
    const int I = c / C.nx, J = c - I * C.nx;
    for (int da = -1; da <= 1; ++da) {
      int yf = 2 * I + da;
      if (yf < 0) { if (C.wrapP) yf += nyf; else continue; }
      if (yf >= nyf) continue;
      for (int db = -1; db <= 1; ++db) {
        const int xf = 2 * J + db;
        if (xf < 0 || xf >= nxf) continue;
        const int f = yf * nxf + xf;
        if (!act_of(a, l, f)) continue;
        const double w = dmul(da ? 0.5 : 1.0, db ? 0.5 : 1.0);
        for (int dI = -1; dI <= 1; ++dI)
          for (int dJ = -1; dJ <= 1; ++dJ) {
            const int j = mg_nb(nyf, nxf, F.per, yf, xf, dI, dJ);
            if (j < 0) continue;
            const double stv = st_eff(a, l, f, yf, xf, (dI + 1) * 3 + (dJ + 1));
            const double v = __dsub_rn((dI == 0 && dJ == 0) ? 1.0 : 0.0, dmul(stv, (double)F.dinv[j]));
            const int k = (2 + da + dI) * 5 + (2 + db + dJ);
            acc[k] = dadd(acc[k], dmul(w, v));
          }
      }
    }
  }
  for (int k = 0; k < 25; ++k) C.R[(size_t)k * Nc + c] = __double2float_rn(acc[k]);
}

__device__ void transfer_U(const MgRebuildArgs& a, int l, int f) {
  const MgBuildLevel& F = a.lev[l];
  const MgBuildLevel& C = a.lev[l + 1];
  const int nyf = F.ny, nxf = F.nx, nyc = C.ny, nxc = C.nx, Nf = nyf * nxf;
  double ur[9], uz[9];
  for (int k = 0; k < 9; ++k) ur[k] = uz[k] = 0.0;
  if (act_of(a, l, f)) {
    const int y = f / nxf, x = f - y * nxf, I0 = y >> 1, J0 = x >> 1;
    const double df = (double)F.dinv[f];
    for (int dI = -1; dI <= 1; ++dI)
      for (int dJ = -1; dJ <= 1; ++dJ) {
        const int j = mg_nb(nyf, nxf, F.per, y, x, dI, dJ);
        if (j < 0 || !act_of(a, l, j)) continue;
        const double cm =
            __dsub_rn((dI == 0 && dJ == 0) ? 1.0 : 0.0, dmul(df, st_eff(a, l, f, y, x, (dI + 1) * 3 + (dJ + 1))));
        const int kr = (dI + 1) * 3 + (dJ + 1);
        ur[kr] = dadd(ur[kr], dmul(cm, (double)F.dinv[j]));
        int pc[4];
        double pw[4];
        const int n = mg_parents(C.wrapP, nyc, nxc, j / nxf, j % nxf, pc, pw);
        for (int q = 0; q < n; ++q) {
          int oI = pc[q] / nxc - I0;
          const int oJ = pc[q] % nxc - J0;
          if (C.per) { if (oI > nyc / 2) oI -= nyc; else if (oI < -(nyc / 2)) oI += nyc; }
          if (oI < -1 || oI > 1 || oJ < -1 || oJ > 1) continue;  // excluded by the host build's geometry
          const int kz = (oI + 1) * 3 + (oJ + 1);
          uz[kz] = dadd(uz[kz], dmul(cm, pw[q]));
        }
      }
    ur[4] = dadd(ur[4], df);
  }
  for (int k = 0; k < 9; ++k) {
    F.U[(size_t)k * Nf + f] = __double2float_rn(ur[k]);
    F.U[(size_t)(9 + k) * Nf + f] = __double2float_rn(uz[k]);
  }
}

// How the new active counts fit the hierarchy's level structure: 0 as the host build would
// make it; 1 a structure the host would make differently (a level that would stop the
// coarsening, or a coarsest level it would coarsen once more), which is still a valid cycle:
// rebuilt here with the same levels, and the host rebuilds after the run; 2 not buildable
// here (a coupling outside the 9-point pattern, or a coarsest level above its capacity).
// The host coarsens a level while it has more than max_coarse active nodes and is large enough.
__device__ int structure_of(const MgRebuildArgs& a) {
  const int L = a.nlevels;
  if (__ldcg(a.counts + MG_CNT_FLAGS) & 1) return 2;
  const int n = __ldcg(a.counts + L - 1);
  if (n > a.ncap) return 2;
  int kind = 0;
  for (int l = 0; l + 1 < L; ++l)
    if (__ldcg(a.counts + l) <= a.max_coarse) kind = 1;
  const MgBuildLevel& Lc = a.lev[L - 1];
  const int nyc = Lc.per ? (Lc.ny + 1) / 2 : Lc.ny / 2 + 1;
  const bool dims_stop = Lc.ny < 4 || Lc.nx < 4 || (Lc.per && nyc < 3) || L >= 15;
  if (n > a.max_coarse && !dims_stop) kind = 1;
  return kind;
}

// Block 0: coarsest active nodes in ascending order (cidx_new) and their positions (pos).
__device__ void scan_coarsest(const MgRebuildArgs& a) {
  const int Lc = a.nlevels - 1;
  const int N = a.lev[Lc].ny * a.lev[Lc].nx;
  __shared__ int wsum[32];
  __shared__ int base, total;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (threadIdx.x == 0) base = 0;
  __syncthreads();
  for (int c0 = 0; c0 < N; c0 += blockDim.x) {
    const int i = c0 + (int)threadIdx.x;
    const bool on = i < N && act_of(a, Lc, i);
    const unsigned m = __ballot_sync(0xFFFFFFFFu, on);
    if (lane == 0) wsum[w] = __popc(m);
    __syncthreads();
    if (w == 0) {
      const int v = lane < (int)(blockDim.x >> 5) ? wsum[lane] : 0;
      int inc = v;
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xFFFFFFFFu, inc, o);
        if (lane >= o) inc += t;
      }
      wsum[lane] = inc - v;
      if (lane == 31) total = inc;
    }
    __syncthreads();
    const int idx = base + wsum[w] + __popc(m & ((1u << lane) - 1u));
    if (i < N) {
      a.pos[i] = on ? idx : -1;
      if (on && idx < a.ncap) a.cidx_new[idx] = i;
    }
    __syncthreads();
    if (threadIdx.x == 0) base += total;
    __syncthreads();
  }
}

// Rows of the symmetrised coarsest operator, lower triangle, one warp per row: entry
// 0.5 (A_rc + A_cr) below the diagonal (the host's symmetrisation), A_rr on it.
__device__ void assemble_dense(const MgRebuildArgs& a, int n) {
  const int Lc = a.nlevels - 1;
  const MgBuildLevel& L = a.lev[Lc];
  const int N = L.ny * L.nx;
  const int lane = threadIdx.x & 31, warp = mg_tid(a) >> 5, nwarp = mg_nth(a) >> 5;
  for (int r = warp; r < n; r += nwarp) {
    double* row = a.dense + (size_t)r * n;
    for (int c = lane; c <= r; c += 32) row[c] = 0.0;
    __syncwarp();
    if (lane == 0) {
      const int i = a.cidx_new[r];
      const int y = i / L.nx, x = i - y * L.nx;
      if (Lc == 0) {
        for_row(a, 0, i, [&](int j, double v) {
          if (j == i) row[r] = v;
          else if (a.pos[j] < r) row[a.pos[j]] = dmul(0.5, dadd(v, v));
        });
      } else {
        row[r] = (double)L.st[(size_t)4 * N + i];
        for (int k = 0; k < 9; ++k) {
          if (k == 4) continue;
          const int j = mg_nb(L.ny, L.nx, L.per, y, x, k / 3 - 1, k % 3 - 1);
          if (j < 0 || !act_of(a, Lc, j) || a.pos[j] >= r) continue;
          const double v = (double)L.st[(size_t)k * N + i], vt = (double)L.st[(size_t)(8 - k) * N + j];
          row[a.pos[j]] = dmul(0.5, dadd(v, vt));
        }
      }
    }
    __syncwarp();
  }
}

// Cholesky factor of the dense operator in place (lower triangle), the host's column order:
// L_jj = sqrt(A_jj - L_j . L_j), L_ij = (A_ij - L_i . L_j) / L_jj, each dot product over the
// first j terms.  Columns go in panels of MG_PANEL: (1) every pair (i >= j, j in the panel)
// forms its four chains over the terms below the panel, in parallel; (2) block 0 finishes the
// panel's diagonal block column by column; (3) every row below it finishes its panel entries
// in order.  The chains continue where their prefix stopped, so each dot product adds its
// terms in the host's order.  Three grid barriers per panel.
__device__ void cholesky(const MgRebuildArgs& a, int n) {
  double* A = a.dense;
  const int t = threadIdx.x & 3;
  const unsigned qmask = 0xFu << (threadIdx.x & 28);
  const int q = mg_tid(a) >> 2, nq = mg_nth(a) >> 2;
  const int ql = (int)threadIdx.x >> 2, nql = (int)blockDim.x >> 2;
  for (int j0 = 0; j0 < n; j0 += MG_PANEL) {
    const int j1 = min(j0 + MG_PANEL, n), w = j1 - j0;
    if (j0 > 0) {
      const long long np = (long long)(n - j0) * w;
      for (long long pid = q; pid < np; pid += nq) {
        const int r = (int)(pid / w), j = j0 + (int)(pid - (long long)r * w), i = j0 + r;
        if (i < j) continue;
        const double* Li = A + (size_t)i * n;
        const double* Lj = A + (size_t)j * n;
        a.pre[pid * 4 + t] = chain_prefix([&](int k) { return Li[k]; }, [&](int k) { return Lj[k]; }, j0, t);
      }
      mg_sync(a);
    }
    auto pre_of = [&](int i, int j) { return j0 > 0 ? a.pre[((size_t)(i - j0) * w + (j - j0)) * 4 + t] : 0.0; };
    if (mgb(a) == 0) {
      for (int j = j0; j < j1; ++j) {
        double* Lj = A + (size_t)j * n;
        if (ql == 0) {
          const double dd = quad_dot4_from(pre_of(j, j), [&](int k) { return Lj[k]; }, [&](int k) { return Lj[k]; },
                                           j0, j, t, qmask);
          if (t == 0) {
            const double s = __dsub_rn(Lj[j], dd);
            if (!(s > 0.0)) atomicOr(a.counts + MG_CNT_FLAGS, 2);
            Lj[j] = __dsqrt_rn(s);
          }
        }
        __syncthreads();
        for (int i = j + 1 + ql; i < j1; i += nql) {
          double* Li = A + (size_t)i * n;
          const double dot = quad_dot4_from(pre_of(i, j), [&](int k) { return Li[k]; }, [&](int k) { return Lj[k]; },
                                            j0, j, t, qmask);
          if (t == 0) Li[j] = __ddiv_rn(__dsub_rn(Li[j], dot), Lj[j]);
        }
        __syncthreads();
      }
    }
    mg_sync(a);
    for (int i = j1 + q; i < n; i += nq) {
      double* Li = A + (size_t)i * n;
      for (int j = j0; j < j1; ++j) {
        const double* Lj = A + (size_t)j * n;
        const double dot = quad_dot4_from(pre_of(i, j), [&](int k) { return Li[k]; }, [&](int k) { return Lj[k]; },
                                          j0, j, t, qmask);
        if (t == 0) Li[j] = __ddiv_rn(__dsub_rn(Li[j], dot), Lj[j]);
        __syncwarp(qmask);
      }
    }
    mg_sync(a);
  }
}

// Columns of M = L^-1 (the host's forward substitution): m_c = 1 / L_cc, then
// m_i = -(L_i[c..i) . m[c..i)) / L_ii.  Column c is stored in row c of the upper triangle
// (dense[c n + i], i > c) with its diagonal in mdiag[c].  Rows go in panels of MG_PANEL:
// (1) every pair (row i of the panel, column c) forms its chains over the column's entries
// below the panel, cut at a multiple of four, in parallel; (2) one group per column finishes
// the panel's rows in order.  Two grid barriers per panel.
__device__ void inverse_factor(const MgRebuildArgs& a, int n) {
  double* A = a.dense;
  const int t = threadIdx.x & 3;
  const unsigned qmask = 0xFu << (threadIdx.x & 28);
  const int q = mg_tid(a) >> 2, nq = mg_nth(a) >> 2;
  for (int i0 = 0; i0 < n; i0 += MG_PANEL) {
    const int i1 = min(i0 + MG_PANEL, n), w = i1 - i0;
    if (i0 > 0) {
      const long long np = (long long)w * i0;
      for (long long pid = q; pid < np; pid += nq) {
        const int r = (int)(pid / i0), c = (int)(pid - (long long)r * i0);
        const int p = ((i0 - c) >> 2) << 2;
        if (p == 0) continue;
        const double* Li = A + (size_t)(i0 + r) * n + c;
        const double* Mc = A + (size_t)c * n + c;
        const double mcd = a.mdiag[c];
        a.pre[pid * 4 + t] =
            chain_prefix([&](int k) { return Li[k]; }, [&](int k) { return k == 0 ? mcd : Mc[k]; }, p, t);
      }
      mg_sync(a);
    }
    for (int c = q; c < i1; c += nq) {
      double* Mc = A + (size_t)c * n + c;  // Mc[k] = m_c[c + k], k >= 1
      double mcd;
      if (c >= i0) {
        mcd = __ddiv_rn(1.0, A[(size_t)c * n + c]);
        if (t == 0) a.mdiag[c] = mcd;
      } else {
        mcd = a.mdiag[c];
      }
      const int p = c < i0 ? ((i0 - c) >> 2) << 2 : 0;
      for (int i = max(i0, c + 1); i < i1; ++i) {
        const double* Li = A + (size_t)i * n + c;
        const double s0 = p > 0 ? a.pre[((size_t)(i - i0) * i0 + c) * 4 + t] : 0.0;
        const double dot =
            quad_dot4_from(s0, [&](int k) { return Li[k]; }, [&](int k) { return k == 0 ? mcd : Mc[k]; }, p, i - c,
                           t, qmask);
        if (t == 0) Mc[i - c] = __ddiv_rn(-dot, A[(size_t)i * n + i]);
        __syncwarp(qmask);
      }
    }
    mg_sync(a);
  }
}

// A^-1 = M^T M as float, exactly symmetric: inv_rc = inv_cr = M[r][c..n) . M[c][c..n) for c >= r.
__device__ void inverse_product(const MgRebuildArgs& a, int n) {
  const double* A = a.dense;
  const int t = threadIdx.x & 3;
  const unsigned qmask = 0xFu << (threadIdx.x & 28);
  const int q = mg_tid(a) >> 2, nq = mg_nth(a) >> 2;
  const long long np = (long long)n * n;
  for (long long p = q; p < np; p += nq) {
    const int r = (int)(p / n), c = (int)(p - (long long)r * n);
    if (c < r) continue;
    const double* Mr = A + (size_t)r * n;
    const double* Mc = A + (size_t)c * n;
    const double mrd = a.mdiag[r], mcd = a.mdiag[c];
    const double dot = quad_dot4([&](int k) { return (c + k == r) ? mrd : Mr[c + k]; },
                                 [&](int k) { return k == 0 ? mcd : Mc[c + k]; }, n - c, t, qmask);
    if (t == 0) {
      const float v = __double2float_rn(dot);
      a.cinv[(size_t)r * n + c] = v;
      a.cinv[(size_t)c * n + r] = v;
    }
  }
}

// block 0's clock: microseconds since *t0 are added to counts[slot] and *t0 moves on
__device__ __forceinline__ void mg_clock(const MgRebuildArgs& a, unsigned long long* t0, int slot) {
  if (mgb(a) != 0 || threadIdx.x != 0) return;
  unsigned long long now;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
  if (slot >= 0) atomicAdd(a.counts + slot, (int)((now - *t0) / 1000ull));
  *t0 = now;
}

__device__ void mg_rebuild_body(const MgRebuildArgs& a) {
  if (*(volatile int*)a.dirty == 0) return;  // every block reads it before any barrier
  const int L = a.nlevels, tid = mg_tid(a), nth = mg_nth(a);
  unsigned long long t0 = 0;
  mg_clock(a, &t0, -1);
  if (mgb(a) == 0 && threadIdx.x < MG_CNT_REBUILDS) a.counts[threadIdx.x] = 0;
  mg_sync(a);
  {
    // level-0 active count
    const int N0 = a.lev[0].ny * a.lev[0].nx;
    int n0 = 0;
    for (int i = tid; i < N0; i += nth) n0 += a.cls[i] == NC_FREE;
    count_add(a.counts + 0, n0);
  }
  for (int l = 0; l + 1 < L; ++l) {
    phase_parents(a, l);
    mg_sync(a);
    count_add(a.counts + l + 1, phase_galerkin(a, l));
    mg_sync(a);
  }
  mg_clock(a, &t0, MG_CNT_US_LEVELS);
  const int kind = structure_of(a);
  const int n = __ldcg(a.counts + L - 1);
  if (kind == 2) {
    if (mgb(a) == 0 && threadIdx.x == 0) {
      atomicOr(a.status, MG_STATUS_HOST);
      atomicAdd(a.counts + MG_CNT_DEFERRED, 1);
    }
    mg_sync(a);
    if (mgb(a) == 0 && threadIdx.x == 0) *a.dirty = 0;
    return;
  }
  if (mgb(a) == 0) scan_coarsest(a);
  mg_sync(a);
  assemble_dense(a, n);
  mg_sync(a);
  cholesky(a, n);
  mg_clock(a, &t0, MG_CNT_US_CHOLESKY);
  if (__ldcg(a.counts + MG_CNT_FLAGS) & 2) {
    // not positive definite: the host build reports it
    if (mgb(a) == 0 && threadIdx.x == 0) {
      atomicOr(a.status, MG_STATUS_HOST);
      atomicAdd(a.counts + MG_CNT_DEFERRED, 1);
    }
    mg_sync(a);
    if (mgb(a) == 0 && threadIdx.x == 0) *a.dirty = 0;
    return;
  }
  // commit: smoother weights of the coarse levels, the coarsest index set, the inverse factor
  for (int l = 1; l < L; ++l) {
    const MgBuildLevel& C = a.lev[l];
    const int Nc = C.ny * C.nx;
    for (int i = tid; i < Nc; i += nth)
      C.dinv[i] = act_of(a, l, i) ? __double2float_rn(__ddiv_rn(MG_JACOBI_OMEGA, (double)C.st[(size_t)4 * Nc + i]))
                                  : 0.0f;
  }
  {
    const MgBuildLevel& Lc = a.lev[L - 1];
    const int Nl = Lc.ny * Lc.nx;
    if (L > 1)
      for (int i = tid; i < Nl; i += nth) Lc.z[i] = 0.0f;
    for (int r = tid; r < n; r += nth) a.cidx[r] = a.cidx_new[r];
    if (tid == 0) *a.nc_dev = n;
  }
  inverse_factor(a, n);
  mg_sync(a);
  mg_clock(a, &t0, MG_CNT_US_INVERSE);
  for (int l = 1; l + 1 < L; ++l) {
    const int Nc = a.lev[l + 1].ny * a.lev[l + 1].nx, Nf = a.lev[l].ny * a.lev[l].nx;
    for (int c = tid; c < Nc; c += nth) transfer_R(a, l, c);
    for (int f = tid; f < Nf; f += nth) transfer_U(a, l, f);
  }
  inverse_product(a, n);
  mg_sync(a);
  mg_clock(a, &t0, MG_CNT_US_TRANSFER);
  if (mgb(a) == 0 && threadIdx.x == 0) {
    *a.dirty = 0;
    atomicAdd(a.counts + MG_CNT_REBUILDS, 1);
    if (kind == 1) {
      atomicOr(a.status, MG_STATUS_HOST);
      atomicAdd(a.counts + MG_CNT_DEFERRED, 1);
    }
  }
}

}  // namespace

__global__ void __launch_bounds__(PT, 1) k_mg_rebuild(const __grid_constant__ MgRebuildArgs a) { mg_rebuild_body(a); }

__global__ void __launch_bounds__(PT, 1) k_mg_rebuild_batch(const MgRebuildArgs* __restrict__ args,
                                                            const int* __restrict__ blk_map) {
  __shared__ MgRebuildArgs sa;
  const int* lst = blk_map + blk_map[blockIdx.x];
  const int cnt = lst[0];
  for (int q = 0; q < cnt; ++q) {
    const int* src = reinterpret_cast<const int*>(args + lst[1 + q]);
    int* dst = reinterpret_cast<int*>(&sa);
    for (int k = threadIdx.x; k < (int)(sizeof(MgRebuildArgs) / sizeof(int)); k += blockDim.x) dst[k] = src[k];
    __syncthreads();
    mg_rebuild_body(sa);
    __syncthreads();
  }
}

}  // namespace pb
