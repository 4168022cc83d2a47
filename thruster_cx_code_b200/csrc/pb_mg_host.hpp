// Host-side construction of the multigrid hierarchy for the field solver.
//
// Level 0 is the fine grid with the node classes of build_sparse_matrix
// (Python/physics_engine.py:525-552): Dirichlet (bound), Neumann copy rows (right
// column, and top/bottom rows when y is not periodic), free otherwise.  Coarse levels
// use bilinear prolongation P (coarse node (I,J) <-> fine (2I,2J); y wraps when the
// fine level is periodic with even size) and Galerkin operators A_c = P^T A P stored
// as 9-point stencils (y periodic on every level when the domain is).  Coarse nodes
// centred on Dirichlet fine nodes, and coarse nodes no active fine node interpolates
// from, are inactive.  Coarsening stops at <= max_coarse active nodes; that level is
// solved with a dense inverse computed here from a Cholesky factorisation.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <thread>
#include <vector>

#include "pb_poisson.cuh"

namespace pb {
namespace mghost {

struct Level {
  int ny = 0, nx = 0, per = 0, wrapP = 0;
  std::vector<uint8_t> act;   // active nodes (level 0: free nodes)
  std::vector<float> st;      // 9 * N stencil (coarse levels)
  std::vector<float> dinv;    // omega / diagonal on active nodes (damped Jacobi smoother)
  std::vector<float> R;       // (coarse levels >= 2) restriction of the fused cycle, 25 planes
  std::vector<float> U;       // (levels >= 1 with a coarser level) prolongation + smoothing, 18 planes
};

constexpr double JACOBI_OMEGA = MG_JACOBI_OMEGA;

struct Hierarchy {
  std::vector<Level> lev;
  std::vector<int> cidx;      // coarsest active nodes
  std::vector<float> cinv;    // coarsest inverse (exactly symmetric)
};

inline std::vector<uint8_t> node_classes(int ny, int nx, int periodic, const uint8_t* isBound) {
  // 0 free, 1 Dirichlet, 2 Neumann
  std::vector<uint8_t> c((size_t)ny * nx, 0);
  for (int y = 0; y < ny; ++y)
    for (int x = 0; x < nx; ++x) {
      size_t i = (size_t)y * nx + x;
      if (isBound[i]) { c[i] = 1; continue; }
      if (x == nx - 1) { c[i] = 2; continue; }
      if (!periodic && (y == 0 || y == ny - 1)) c[i] = 2;
    }
  return c;
}

// neighbour of (y, x) by (dy, dx) with optional y wrap; -1 outside
inline long nb(int ny, int nx, int per, int y, int x, int dy, int dx) {
  int yy = y + dy, xx = x + dx;
  if (per) { if (yy < 0) yy += ny; else if (yy >= ny) yy -= ny; }
  if (yy < 0 || yy >= ny || xx < 0 || xx >= nx) return -1;
  return (long)yy * nx + xx;
}

struct Entry { long j; double v; };

// row of the operator of level l (only active columns)
inline void row_of(const Level& L, int level, const std::vector<uint8_t>& cls0, long i, std::vector<Entry>& out) {
  out.clear();
  int y = (int)(i / L.nx), x = (int)(i % L.nx);
  if (level == 0) {
    static const int DY[4] = {0, 0, -1, 1}, DX[4] = {-1, 1, 0, 0};
    int nneu = 0;
    for (int k = 0; k < 4; ++k) {
      long j = nb(L.ny, L.nx, L.per, y, x, DY[k], DX[k]);
      uint8_t c = j < 0 ? 2 : cls0[j];
      if (c == 0) out.push_back({j, -1.0});
      else if (c == 2) ++nneu;
    }
    out.push_back({i, (double)(4 - nneu)});
    return;
  }
  size_t N = (size_t)L.ny * L.nx;
  for (int k = 0; k < 9; ++k) {
    float v = L.st[k * N + i];
    if (v == 0.0f) continue;
    long j = nb(L.ny, L.nx, L.per, y, x, k / 3 - 1, k % 3 - 1);
    if (j >= 0 && L.act[j]) out.push_back({j, (double)v});
  }
}

// prolongation weights of fine node (y, x) from the coarse level: up to 4 (c, w)
inline int p_row(int nyf, int nxf, int wrap, int nyc, int nxc, int y, int x, long* c, double* w) {
  int I0 = y >> 1, a = y & 1, J0 = x >> 1, b = x & 1;
  int n = 0;
  for (int da = 0; da <= a; ++da) {
    int I = I0 + da;
    if (I >= nyc) { if (wrap) I -= nyc; else continue; }
    double wy = a ? 0.5 : 1.0;
    for (int db = 0; db <= b; ++db) {
      int J = J0 + db;
      if (J >= nxc) continue;
      double wx = b ? 0.5 : 1.0;
      c[n] = (long)I * nxc + J;
      w[n] = wy * wx;
      ++n;
    }
  }
  (void)nyf; (void)nxf;
  return n;
}

// The transfers of the fused V-cycle as explicit stencils, for fine levels l >= 1 (where
// the operator is a 9-point stencil):
//   r_{l+1}(c) = [c active] sum_f w_cf [f active] (r_f - sum_j A_fj d_j r_j)
//              = sum over the 5 x 5 fine patch centred on (2I, 2J) of R_k r_j,
//   z_f = [f active] (m_f + d_f r_f - d_f sum_j A_fj m_j),  m_j = [j active] (d_j r_j + (P z)_j)
//       = sum over the 3 x 3 fine patch of U_k r_j + sum over the 3 x 3 coarse patch centred
//         on (y >> 1, x >> 1) of U_{9+k} z_c.
// Coefficients are accumulated per patch offset (rows wrap as the device indexes them),
// so periodic levels with few rows still match the device sums term by term.
inline void transfer_ops(Hierarchy& H) {
  for (size_t l = 1; l + 1 < H.lev.size(); ++l) {
    Level& F = H.lev[l];
    Level& C = H.lev[l + 1];
    const int nyf = F.ny, nxf = F.nx, nyc = C.ny, nxc = C.nx;
    const size_t Nf = (size_t)nyf * nxf, Nc = (size_t)nyc * nxc;
    auto stF = [&](size_t f, int dI, int dJ) { return (double)F.st[(size_t)((dI + 1) * 3 + (dJ + 1)) * Nf + f]; };
    C.R.assign(25 * Nc, 0.0f);
    for (size_t c = 0; c < Nc; ++c) {
      if (!C.act[c]) continue;
      const int I = (int)(c / nxc), J = (int)(c % nxc);
      double acc[25] = {0};
      for (int da = -1; da <= 1; ++da) {
        int yf = 2 * I + da;
        if (yf < 0) { if (C.wrapP) yf += nyf; else continue; }
        if (yf >= nyf) continue;
        for (int db = -1; db <= 1; ++db) {
          const int xf = 2 * J + db;
          if (xf < 0 || xf >= nxf) continue;
          const size_t f = (size_t)yf * nxf + xf;
          if (!F.act[f]) continue;
          const double w = (da ? 0.5 : 1.0) * (db ? 0.5 : 1.0);
          for (int dI = -1; dI <= 1; ++dI)
            for (int dJ = -1; dJ <= 1; ++dJ) {
              const long j = nb(nyf, nxf, F.per, yf, xf, dI, dJ);
              if (j < 0) continue;
              const double v = ((dI == 0 && dJ == 0) ? 1.0 : 0.0) - stF(f, dI, dJ) * (double)F.dinv[j];
              acc[(2 + da + dI) * 5 + (2 + db + dJ)] += w * v;
            }
        }
      }
      for (int k = 0; k < 25; ++k) C.R[(size_t)k * Nc + c] = (float)acc[k];
    }
    F.U.assign(18 * Nf, 0.0f);
    long pc[4];
    double pw[4];
    for (size_t f = 0; f < Nf; ++f) {
      if (!F.act[f]) continue;
      const int y = (int)(f / nxf), x = (int)(f % nxf), I0 = y >> 1, J0 = x >> 1;
      const double df = F.dinv[f];
      double ur[9] = {0}, uz[9] = {0};
      for (int dI = -1; dI <= 1; ++dI)
        for (int dJ = -1; dJ <= 1; ++dJ) {
          const long j = nb(nyf, nxf, F.per, y, x, dI, dJ);
          if (j < 0 || !F.act[j]) continue;
          const double cm = ((dI == 0 && dJ == 0) ? 1.0 : 0.0) - df * stF(f, dI, dJ);  // weight of m_j
          ur[(dI + 1) * 3 + (dJ + 1)] += cm * (double)F.dinv[j];
          const int n = p_row(nyf, nxf, C.wrapP, nyc, nxc, (int)(j / nxf), (int)(j % nxf), pc, pw);
          for (int q = 0; q < n; ++q) {
            int oI = (int)(pc[q] / nxc) - I0, oJ = (int)(pc[q] % nxc) - J0;
            if (C.per) { if (oI > nyc / 2) oI -= nyc; else if (oI < -(nyc / 2)) oI += nyc; }
            if (oI < -1 || oI > 1 || oJ < -1 || oJ > 1) throw std::runtime_error("prolongation outside the 3 x 3 patch");
            uz[(oI + 1) * 3 + (oJ + 1)] += cm * pw[q];
          }
        }
      ur[4] += df;
      for (int k = 0; k < 9; ++k) {
        F.U[(size_t)k * Nf + f] = (float)ur[k];
        F.U[(size_t)(9 + k) * Nf + f] = (float)uz[k];
      }
    }
  }
}

// a . b over n terms, four partial sums (a fixed order)
inline double dot4(const double* a, const double* b, int n) {
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
  int k = 0;
  for (; k + 4 <= n; k += 4) {
    s0 += a[k] * b[k];
    s1 += a[k + 1] * b[k + 1];
    s2 += a[k + 2] * b[k + 2];
    s3 += a[k + 3] * b[k + 3];
  }
  for (; k < n; ++k) s0 += a[k] * b[k];
  return (s0 + s1) + (s2 + s3);
}

// fn(i) for i in [0, n), split over up to 8 host threads in interleaved order
template <class Fn>
inline void parallel_for(int n, Fn fn) {
  const int nt = std::max(1, std::min({8, (int)std::thread::hardware_concurrency(), n / 64}));
  if (nt == 1) {
    for (int i = 0; i < n; ++i) fn(i);
    return;
  }
  std::vector<std::thread> th;
  for (int t = 0; t < nt; ++t)
    th.emplace_back([&, t] {
      for (int i = t; i < n; i += nt) fn(i);
    });
  for (auto& x : th) x.join();
}

// Inverse of an SPD matrix (row-major n x n) as float, exactly symmetric: Cholesky
// A = L L^T, the columns of M = L^-1 by forward substitution, then A^-1 = M^T M.  Every
// inner loop is a contiguous dot product; the column stages run on host threads.
inline std::vector<float> spd_inverse(const std::vector<double>& A, int n) {
  std::vector<double> L((size_t)n * n, 0.0);  // row-major, lower
  for (int j = 0; j < n; ++j) {
    const double* Lj = &L[(size_t)j * n];
    const double s = A[(size_t)j * n + j] - dot4(Lj, Lj, j);
    if (!(s > 0.0)) throw std::runtime_error("coarsest operator is not positive definite");
    const double d = std::sqrt(s);
    L[(size_t)j * n + j] = d;
    for (int i = j + 1; i < n; ++i) L[(size_t)i * n + j] = (A[(size_t)i * n + j] - dot4(&L[(size_t)i * n], Lj, j)) / d;
  }
  std::vector<double> M((size_t)n * n, 0.0);  // column c of L^-1 in M[c * n + i], i >= c
  parallel_for(n, [&](int c) {
    double* m = &M[(size_t)c * n];
    m[c] = 1.0 / L[(size_t)c * n + c];
    for (int i = c + 1; i < n; ++i) m[i] = -dot4(&L[(size_t)i * n + c], m + c, i - c) / L[(size_t)i * n + i];
  });
  std::vector<float> inv((size_t)n * n);
  parallel_for(n, [&](int r) {
    const double* mr = &M[(size_t)r * n];
    for (int c = r; c < n; ++c) {
      const float v = (float)dot4(mr + c, &M[(size_t)c * n + c], n - c);
      inv[(size_t)r * n + c] = v;
      inv[(size_t)c * n + r] = v;
    }
  });
  return inv;
}

inline Hierarchy build(int ny, int nx, int periodic, const std::vector<uint8_t>& cls0, int max_coarse) {
  Hierarchy H;
  Level L0;
  L0.ny = ny; L0.nx = nx; L0.per = periodic; L0.wrapP = 0;
  L0.act.resize((size_t)ny * nx);
  for (size_t i = 0; i < L0.act.size(); ++i) L0.act[i] = cls0[i] == 0;
  H.lev.push_back(L0);
  std::vector<Entry> row;
  while (true) {
    Level& F = H.lev.back();
    int level = (int)H.lev.size() - 1;
    size_t nact = 0;
    for (uint8_t a : F.act) nact += a;
    int nyc = F.per ? (F.ny + 1) / 2 : F.ny / 2 + 1;
    int nxc = F.nx / 2 + 1;
    if ((long)nact <= max_coarse || F.ny < 4 || F.nx < 4 || (F.per && nyc < 3) || H.lev.size() >= 15) break;
    int wrap = F.per && (F.ny % 2 == 0);
    Level C;
    C.ny = nyc; C.nx = nxc; C.per = F.per; C.wrapP = wrap;
    size_t Nc = (size_t)nyc * nxc, Nf = (size_t)F.ny * F.nx;
    C.act.assign(Nc, 0);
    long pc[4]; double pw[4];
    for (size_t f = 0; f < Nf; ++f) {
      if (!F.act[f]) continue;
      int n = p_row(F.ny, F.nx, wrap, nyc, nxc, (int)(f / F.nx), (int)(f % F.nx), pc, pw);
      for (int k = 0; k < n; ++k) C.act[pc[k]] = 1;
    }
    if (level == 0)
      for (size_t c = 0; c < Nc; ++c) {
        int I = (int)(c / nxc), J = (int)(c % nxc);
        int yf = 2 * I, xf = 2 * J;
        if (yf < F.ny && xf < F.nx && cls0[(size_t)yf * F.nx + xf] == 1) C.act[c] = 0;
      }
    // Galerkin product, accumulated in double then stored as float stencils
    std::vector<double> st(9 * Nc, 0.0);
    long qc[4]; double qw[4];
    bool ok = true;
    for (size_t f = 0; f < Nf && ok; ++f) {
      if (!F.act[f]) continue;
      int n = p_row(F.ny, F.nx, wrap, nyc, nxc, (int)(f / F.nx), (int)(f % F.nx), pc, pw);
      row_of(F, level, cls0, (long)f, row);
      for (const Entry& e : row) {
        int m = p_row(F.ny, F.nx, wrap, nyc, nxc, (int)(e.j / F.nx), (int)(e.j % F.nx), qc, qw);
        for (int a = 0; a < n; ++a) {
          if (!C.act[pc[a]]) continue;
          int I = (int)(pc[a] / nxc), J = (int)(pc[a] % nxc);
          for (int b = 0; b < m; ++b) {
            if (!C.act[qc[b]]) continue;
            int I2 = (int)(qc[b] / nxc), J2 = (int)(qc[b] % nxc);
            int dI = I2 - I, dJ = J2 - J;
            if (C.per) { if (dI > nyc / 2) dI -= nyc; else if (dI < -(nyc / 2)) dI += nyc; }
            if (dI < -1 || dI > 1 || dJ < -1 || dJ > 1) { ok = false; break; }
            st[(size_t)((dI + 1) * 3 + (dJ + 1)) * Nc + pc[a]] += pw[a] * e.v * qw[b];
          }
          if (!ok) break;
        }
        if (!ok) break;
      }
    }
    if (!ok) break;  // coupling outside the 9-point pattern: keep the current level as coarsest
    C.st.resize(9 * Nc);
    for (size_t k = 0; k < 9 * Nc; ++k) C.st[k] = (float)st[k];
    for (size_t c = 0; c < Nc; ++c)
      if (C.act[c] && !(C.st[4 * Nc + c] > 0.0f)) C.act[c] = 0;
    // no coupling to or from inactive nodes (the device cycle reads every stencil entry)
    for (size_t c = 0; c < Nc; ++c) {
      int I = (int)(c / nxc), J = (int)(c % nxc);
      for (int k = 0; k < 9; ++k) {
        long j = nb(nyc, nxc, C.per, I, J, k / 3 - 1, k % 3 - 1);
        if (!C.act[c] || j < 0 || !C.act[j]) C.st[k * Nc + c] = 0.0f;
      }
    }
    H.lev.push_back(std::move(C));
  }
  // smoother weights omega / A_ii on every level
  for (size_t l = 0; l < H.lev.size(); ++l) {
    Level& L = H.lev[l];
    size_t N = (size_t)L.ny * L.nx;
    L.dinv.assign(N, 0.0f);
    for (size_t i = 0; i < N; ++i) {
      if (!L.act[i]) continue;
      double d;
      if (l == 0) {
        row_of(L, 0, cls0, (long)i, row);
        d = row.back().v;  // the diagonal entry is pushed last on level 0
      } else {
        d = L.st[4 * N + i];
      }
      L.dinv[i] = d > 0.0 ? (float)(JACOBI_OMEGA / d) : 0.0f;
    }
  }
  transfer_ops(H);
  // dense inverse of the coarsest operator (Cholesky, then L^-T L^-1)
  Level& Lc = H.lev.back();
  int level = (int)H.lev.size() - 1;
  size_t N = (size_t)Lc.ny * Lc.nx;
  std::vector<long> pos(N, -1);
  for (size_t i = 0; i < N; ++i)
    if (Lc.act[i]) { pos[i] = (long)H.cidx.size(); H.cidx.push_back((int)i); }
  int n = (int)H.cidx.size();
  if (n > MG_MAX_COARSE) throw std::runtime_error("coarsest level too large for the dense solve");
  std::vector<double> A((size_t)n * n, 0.0);
  for (int r = 0; r < n; ++r) {
    row_of(Lc, level, cls0, H.cidx[r], row);
    for (const Entry& e : row)
      if (pos[e.j] >= 0) A[(size_t)r * n + pos[e.j]] += e.v;
  }
  // symmetrise (round-off) and invert
  for (int r = 0; r < n; ++r)
    for (int c = r + 1; c < n; ++c) {
      double v = 0.5 * (A[(size_t)r * n + c] + A[(size_t)c * n + r]);
      A[(size_t)r * n + c] = A[(size_t)c * n + r] = v;
    }
  H.cinv = spd_inverse(A, n);
  return H;
}

}  // namespace mghost
}  // namespace pb
