// Poisson solver data layout (device pointers) shared by the kernel and the host builder.
#pragma once
#include <cstdint>

namespace pb {

constexpr int MG_MAX_LEVELS = 16;
constexpr double MG_JACOBI_OMEGA = 0.8;       // damped-Jacobi weight of the V-cycle smoother
constexpr int MG_MAX_COARSE = 4096;          // largest coarsest level (dense inverse, nc^2 floats)
enum NodeClass : uint8_t { NC_FREE = 0, NC_DIR = 1, NC_NEU = 2 };

struct MgLevel {
  int ny, nx;
  int per;        // y is periodic on this level's operator
  int wrapP;      // prolongation from the next coarser level wraps in y
  const float* dinv;      // omega / diagonal on active nodes, 0 elsewhere (Jacobi smoother; d > 0 marks
                          // the active nodes)
  const float* R;         // levels >= 2: restriction from the finer level, R[k * N + i], 5 x 5 patch
  const float* U;         // levels >= 1: prolongation + smoothing, U[k * N + i], 3 x 3 r then 3 x 3 z
  float *r, *z;           // right-hand side and correction on this level
};

struct PoissonArgs {
  // fine grid
  int ny, nx, periodic;
  const uint8_t* cls;     // NodeClass per node (level 0)
  const double* Vfixed;
  const float* rho;
  double* V;              // Picard state (all nodes)
  double* x;              // linear-solve solution (Vnew), warm start across solves
  double* f;              // reduced right-hand side
  double* dirsum;         // sum of Dirichlet neighbour values
  float *r32, *z32, *p32, *q32, *e32;
  float *Ex, *Ey;
  // physics scalars (host double precision, as the reference computes them)
  double coeff;           // (dx*1e-3)^2 / eps0
  double qn0_neg;         // -q * n0
  double V_plasma, Te_up;
  double omega_keep, omega_new;   // 1 - omega, omega
  // np.gradient spacings: hx = dx*1e-3, two_hx = 2.*hx, ...; two_hy_per = (2.0*dy)*1e-3
  double hx, two_hx, hy, two_hy, two_hy_per;
  int iterations;         // Picard iterations
  int compute_field;      // write Ex, Ey at the end
  // solver control
  double tol;             // relative FP64 residual target ||f - A x|| / ||f||
  double tol_inner;       // relative residual reduction of each FP32 MG-PCG solve
  int max_outer, max_inner;
  // hierarchy
  int nlevels;            // including level 0 and the coarsest
  MgLevel lev[MG_MAX_LEVELS];
  int nc;                 // coarsest active count (<= MG_MAX_COARSE)
  const int* cidx;        // coarsest active node indices
  const float* cinv;      // coarsest inverse (nc x nc, exactly symmetric)
  // this instance's blocks in the launch and its reductions and barrier
  int blk0, nblk;         // first block and number of blocks
  double* partials;       // 4 slots x 2 values x nblk doubles
  unsigned int* bar;      // barrier word, zero at launch (its low bits must start at zero)
  uint32_t* errflags;
  double* stats;          // [outer its, inner its, final rel residual, solves] accumulated
  unsigned long long* trace;  // optional: ns per phase category (block 0), [31] = last stamp
};

// dynamic shared memory of k_poisson: the coarsest right-hand side gathered by each block
inline size_t mg_coarse_smem_bytes(int nc) { return 4 * (size_t)(nc > 0 ? nc : 1); }

}  // namespace pb
