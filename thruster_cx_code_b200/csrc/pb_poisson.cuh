// Poisson solver data layout (device pointers) shared by the kernel and the host builder.
#pragma once
#include <algorithm>
#include <cstdint>

namespace pb {

constexpr int PT = 1024;  // threads per block of the field-solve kernels (one block per SM)
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
  float *s32, *m32;       // fine-level smoothing temporaries (nu0 = 2)
  int nu0;                // damped-Jacobi sweeps on the fine level on each side of the coarse correction
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
  const int* nc_dev;      // coarsest active count nc (<= MG_MAX_COARSE), in device memory: the
                          // hierarchy rebuild on the device may change it between launches
  const int* cidx;        // coarsest active node indices
  const float* cinv;      // coarsest inverse (nc x nc, exactly symmetric)
  // this instance's blocks in the launch and its reductions and barrier
  int blk0, nblk;         // first block and number of blocks
  int nvb;                // virtual blocks of the reductions (mg_virtual_blocks): the order of
                          // every sum, whatever nblk is
  int vb_off;             // float4 offset of the virtual-block sums in the dynamic shared memory
  int ut_y, ut_x;         // tiles of the fine-level up leg (fine_up_tiles for nblk blocks, or
                          // for nvb when nu0 = 1: its tiles then carry the (r, z) partials)
  double* partials;       // 4 slots x 2 values x nvb doubles
  unsigned int* bar;      // barrier word, zero at launch (its low bits must start at zero)
  uint32_t* errflags;
  double* stats;          // [outer its, inner its, final rel residual, solves] accumulated
  unsigned long long* solve_ns;  // [block-ns, launches] of this instance's solves (block 0's clock
                                 // times the instance's block count)
  unsigned long long* trace;  // optional: ns per phase category (block 0), [31] = last stamp
};

// dynamic shared memory of k_poisson: the coarsest right-hand side gathered by each block
// (sized for the capacity of the coarsest level, which a rebuild on the device may fill),
// then the warp sums of the virtual blocks the block runs
inline size_t mg_coarse_smem_bytes(int nc) { return 4 * (size_t)(nc > 0 ? nc : 1); }
inline int mg_vb_offset(int ncap) { return (int)((mg_coarse_smem_bytes(ncap) + 15) / 16); }
inline size_t mg_solve_smem_bytes(int ncap, int nvb, int nblk) {
  return 16 * (size_t)mg_vb_offset(ncap) + (size_t)((nvb + nblk - 1) / nblk) * 2 * 32 * sizeof(double);
}
// Virtual blocks of the reductions on an n-node fine level: about 2048 nodes each (two per
// thread of a 1024-thread block), at most the device's SM count.  A function of the grid
// alone, so every reduction of a solve has the same order on any number of blocks; with the
// full grid of blocks no block runs more than two nodes per thread of them.
inline int mg_virtual_blocks(long n, int num_sms) {
  const long v = (n + 2047) / 2048;
  return (int)std::max(1L, std::min<long>(v, num_sms));
}

// ---------------------------------------------------------------- rebuild on the device
// Arrays of one level for k_mg_rebuild: the hierarchy the solve reads (dinv, R, U, z) and
// the rebuild's own scratch (act, st).
struct MgBuildLevel {
  int ny, nx, per, wrapP;
  float* dinv;            // omega / diagonal on active nodes (levels >= 1 written here)
  float* R;               // levels >= 2: fused-cycle restriction, 25 planes (or null)
  float* U;               // levels >= 1 with a coarser level: prolongation + smoothing, 18 planes
  float* z;               // correction (the coarsest level's is cleared by a rebuild)
  uint8_t* act;           // levels >= 1, scratch: bit 0 = a parent of an active finer node, bit 1 = active
  float* st;              // levels >= 1, scratch: Galerkin 9-point stencil, st[k * N + i]
};

// slots of MgRebuildArgs::counts
enum : int {
  MG_CNT_FLAGS = MG_MAX_LEVELS,   // bit 0: coupling outside the 9-point pattern, bit 1: not SPD
  MG_CNT_REBUILDS,                // rebuilds completed on the device (cumulative)
  MG_CNT_DEFERRED,                // rebuilds left to the host (cumulative)
  MG_CNT_US_LEVELS,               // microseconds (cumulative, block 0's clock) in the coarse levels,
  MG_CNT_US_CHOLESKY,             //   the dense assembly and Cholesky factor,
  MG_CNT_US_INVERSE,              //   the inverse factor and smoother weights,
  MG_CNT_US_TRANSFER,             //   the transfer stencils and the dense inverse
  MG_CNT_SLOTS = 32
};
// MgRebuildArgs::status bit: the freed nodes change the level structure; the host rebuilds
constexpr uint32_t MG_STATUS_HOST = 1u;
// columns (rows) per panel of the rebuild's Cholesky factor (inverse factor); a multiple of 4
constexpr int MG_PANEL = 32;

struct MgRebuildArgs {
  int nlevels, max_coarse, ncap;  // ncap: capacity of the coarsest level (cidx, cinv, dense)
  const uint8_t* cls;             // level-0 node classes (updated by the cell break)
  MgBuildLevel lev[MG_MAX_LEVELS];
  int* cidx;                      // coarsest active node indices (ncap)
  float* cinv;                    // coarsest inverse (ncap^2 floats, row stride nc)
  int* nc_dev;                    // coarsest active count
  double* dense;                  // scratch ncap^2: the coarsest operator, its Cholesky factor
                                  // (lower triangle) and the columns of its inverse (upper)
  double* mdiag;                  // scratch ncap: diagonal of the inverse factor
  double* pre;                    // scratch ncap x MG_PANEL x 4: chain prefixes of a panel
  int* cidx_new;                  // scratch ncap
  int* pos;                       // scratch, one per node of the coarsest level
  int* counts;                    // MG_CNT_SLOTS ints: active counts per level, flags, totals
  int* dirty;                     // set when cells break; cleared by the rebuild
  uint32_t* status;               // MG_STATUS_HOST
  unsigned int* bar;              // barrier word, zero at launch
  uint32_t* errflags;
  int blk0, nblk;
};

// Tiling of the fine-level up leg: at most UP_TILE_MAX nodes per tile with its one-node halo.
constexpr int UP_TILE_MAX = 4096;

// Tile counts (ty rows x tx columns of nearly equal rectangles) for an ny x nx fine level
// solved by nblk blocks of 1024 threads: the fewest rounds of tiles per block times the
// passes a block makes over one tile (three units per pass that forms m, one per pass that
// forms z), then the fewest m a block forms (rounds x nodes of a tile with its halo), then the
// most tiles.  Tile counts up to about four rounds are searched; the smallest tiles (one row)
// always fit.
inline void fine_up_tiles(int ny, int nx, int nblk, int* ty_out, int* tx_out) {
  const long cap = 4L * nblk + 4L * ((long)ny * nx / 1024 + 1);
  long best_cost = -1, best_work = 0, best_tiles = 0;
  int bty = ny, btx = nx;
  for (int ty = 1; ty <= ny; ++ty) {
    const long h = (ny + ty - 1) / ty;
    const long wmax = UP_TILE_MAX / (h + 2) - 2;
    if (wmax < 1) continue;
    const long tx_min = (nx + wmax - 1) / wmax;
    const long tx_max = std::max(tx_min, std::min<long>(nx, cap / ty));
    for (long tx = tx_min; tx <= tx_max; ++tx) {
      const long w = (nx + tx - 1) / tx;
      const long tiles = (long)ty * tx;
      const long rounds = (tiles + nblk - 1) / nblk;
      const long cost = rounds * (3 * (((h + 2) * (w + 2) + 1023) / 1024) + (h * w + 1023) / 1024);
      const long work = rounds * (h + 2) * (w + 2);
      if (best_cost < 0 || cost < best_cost ||
          (cost == best_cost && (work < best_work || (work == best_work && tiles > best_tiles)))) {
        best_cost = cost;
        best_work = work;
        best_tiles = tiles;
        bty = ty;
        btx = (int)tx;
      }
    }
    if ((long)ty * tx_min > cap && best_cost >= 0) break;
  }
  *ty_out = bty;
  *tx_out = btx;
}

#ifdef __CUDACC__
// The field-solve kernels live in their own translation unit (pb_poisson.cu), compiled
// with fused multiply-add contraction: the FP32 MG-PCG is compared with SuperLU to a
// tolerance, not bit for bit, unlike the particle arithmetic.
// One instance on every block of the launch.
__global__ void k_poisson(const __grid_constant__ PoissonArgs a);
// Several instances in one launch: block b runs the instances listed at blk_map[blk_map[b]]
// (a count, then indices into args) one after another, each together with the other blocks of
// its contiguous range (args[i].blk0, args[i].nblk): an instance with blocks of its own, or
// several one-block instances packed into one block.
__global__ void k_poisson_batch(const PoissonArgs* __restrict__ args, const int* __restrict__ blk_map);
// The hierarchy rebuilt from the node classes after cells broke (no-op unless *dirty), on
// every block of the launch, or per instance as k_poisson_batch.
__global__ void k_mg_rebuild(const __grid_constant__ MgRebuildArgs a);
__global__ void k_mg_rebuild_batch(const MgRebuildArgs* __restrict__ args, const int* __restrict__ blk_map);
#endif

}  // namespace pb
