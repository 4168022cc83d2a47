// libpbemcs runtime: device state of one simulation instance, the timestep sequence and
// the C-ABI (include/pbemcs.h).  The particle and diagnostic kernel sources are included
// here (one translation unit, no multiply-add contraction); the field solve is compiled
// separately (pb_poisson.cu).
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <functional>
#include <utility>
#include <vector>

#include "pbemcs.h"
#include "pb_particles.cu"
#include "pb_poisson.cuh"
#include "pb_misc.cu"
#include "pb_mg_host.hpp"

namespace pb {

static thread_local std::string g_err;

static int32_t fail(int32_t code, const std::string& msg) {
  g_err = msg;
  return code;
}

#define CK(call)                                                                                  \
  do {                                                                                            \
    cudaError_t e_ = (call);                                                                      \
    if (e_ != cudaSuccess) return fail(PB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

template <typename T>
static cudaError_t dalloc(T** p, size_t n) {
  *p = nullptr;
  if (n == 0) n = 1;
  return cudaMalloc((void**)p, n * sizeof(T));
}
template <typename T>
static void dfree(T*& p) {
  if (p) cudaFree((void*)p);
  p = nullptr;
}

struct Species {
  Soa buf[2] = {};
  int cur = 0;
  int cap = 0;
  bool ion = false;
};

struct DevLevel {
  int ny = 0, nx = 0, per = 0, wrapP = 0;
  float* dinv = nullptr;
  float* R = nullptr;
  float* U = nullptr;
  float* r = nullptr;
  float* z = nullptr;
  uint8_t* act = nullptr;  // scratch of the device rebuild (levels >= 1)
  float* st = nullptr;
};

struct Sim {
  int device = 0;
  cudaStream_t stream = nullptr;
  int num_sms = 148;
  // grid
  int ny = 0, nx = 0, periodic = 0, ngrids = 0;
  double *V = nullptr, *Vnew = nullptr, *Vfixed = nullptr, *Vdc = nullptr, *damage = nullptr, *eroded = nullptr;
  double *accum_ppc = nullptr, *f = nullptr, *dirsum = nullptr;
  float *Ex = nullptr, *Ey = nullptr, *rho = nullptr, *Tmap = nullptr;
  float *r32 = nullptr, *z32 = nullptr, *p32 = nullptr, *q32 = nullptr, *e32 = nullptr;
  float *s32 = nullptr, *m32 = nullptr;  // fine-level smoothing temporaries (nu = 2)
  float4* ecorn = nullptr;  // per-cell corners of Ex and Ey, 2 x float4 per node
  CUtensorMap ec_map;       // TMA view of ecorn (PB_OPT_TMA_TILE), valid for the array and shape below
  const float4* ec_map_for = nullptr;
  int ec_map_ny = 0, ec_map_nx = 0;
  uint8_t *isBound = nullptr, *cls = nullptr;
  uint8_t *bdist = nullptr, *bdist_tmp = nullptr;  // Chebyshev distance to the nearest bound node
  uint16_t* gridmask = nullptr;
  int *ppc = nullptr, *cnt_i = nullptr, *cnt_e = nullptr;
  // multigrid
  std::vector<DevLevel> lev;
  int nc = 0;             // coarsest active count of the last host build (nc_dev holds the current one)
  int ncap = 0;           // capacity of the coarsest level (cidx, cinv and the rebuild's dense scratch)
  int* cidx = nullptr;
  float* cinv = nullptr;
  int* nc_dev = nullptr;
  // rebuild of the hierarchy on the device after cells break (k_mg_rebuild)
  double* mg_dense = nullptr;
  double* mg_mdiag = nullptr;
  double* mg_pre = nullptr;
  int *mg_cidx_new = nullptr, *mg_pos = nullptr;
  int* mg_counts = nullptr;      // MG_CNT_SLOTS (persist across host builds)
  int* mg_dirty = nullptr;
  uint32_t* mg_status = nullptr;
  bool erosion_seen = false;     // a step with sputter breaks was enqueued: field solves rebuild first
  long long mg_host_rebuilds = 0;
  double* partials = nullptr;
  unsigned int* bar = nullptr;
  double* pstats = nullptr;
  unsigned long long* solve_ns = nullptr;  // [block-ns, launches] of the field solves (k_poisson*)
  double solve_work = 0.0;    // block-ns of one field-solve launch, measured in the last batch run
  int batch_blocks = 0;       // this instance's block share in the last batch launch planned
  unsigned long long* ptrace = nullptr;  // field-solve phase trace (32 slots)
  int trace_on = 0;
  int pgrid = 0;      // blocks of the field-solve launch (<= num_sms)
  int ut_key[3] = {0, 0, 0}, ut[2] = {1, 1};  // fine up-leg tiling for (ny, nx, blocks)
  int pbps = 8;       // step-kernel blocks per SM (the grid; tiles are handed out by a counter)
  uint32_t kopts = PB_OPT_ELE_SPLIT;  // kernel variants of the step (PB_OPT_*; the fastest measured)
  int ppb = TILE;                     // particles per block (tile) of the step kernels
  size_t psmem = 0;  // dynamic shared memory of the field-solve kernel
  // particles
  Species sp[2];
  int* counts = nullptr;         // [ion buf0, ion buf1, ele buf0, ele buf1]
  uint32_t* next_ids = nullptr;  // [ion, electron]
  // per-step scratch
  unsigned long long* tile_status = nullptr;
  int* tile_counter = nullptr;   // [ion, ele]
  size_t tile_cap = 0;
  uint64_t* see_key = nullptr;
  float* see_xy = nullptr;
  int see_cap = 0;
  int* see_count = nullptr;
  float* angles = nullptr;
  uint64_t* angle_scratch = nullptr;
  int angle_cap = 0;
  int* angle_count = nullptr;
  unsigned long long* ds_bits = nullptr;  // [ion, ele, field bound (low word: float bits)]
  int* n_sub = nullptr;                    // [ion, ele]
  uint8_t* ekeep = nullptr;                // survivor flags of the split electron step
  size_t ekeep_cap = 0;
  int* inj = nullptr;                      // 7 ints
  int* see_spawned = nullptr;
  // sort
  uint32_t *skey[2] = {nullptr, nullptr}, *sval[2] = {nullptr, nullptr}, *shist = nullptr, *sblk = nullptr;
  size_t sort_cap = 0, hist_cap = 0;
  // report
  pb_step_report* rep_dev = nullptr;
  pb_step_report* rep_host = nullptr;
  pb_step_report* rep_run = nullptr;  // pinned per-step reports of pb_sim_run
  int rep_run_cap = 0;
  // settings
  double tol = 1e-8, tol_inner = 1e-3;
  int max_outer = 8, max_inner = 40, nu = 2, max_coarse = 1536;
  uint64_t seed = 0;
  bool counts_valid = false;
  bool domain_set = false;
  int host_num[2] = {0, 0};
  // NumPy float32 sums (pb_sim_energy_sums): the summation tree per source (ions,
  // electrons, field) and grow-only device copies of one tree at a time
  struct PwTree {
    long long n = -1;
    std::vector<long long> leaf_lo;  // leaf k covers [leaf_lo[k], leaf_lo[k + 1])
    std::vector<int> left, right;    // internal nodes in height order; node ids: leaves first
    std::vector<int> height_off;     // internal nodes of height h + 1: [height_off[h], height_off[h + 1])
    int root = -1;
  } pw[3];
  long long* pw_lo = nullptr;
  int *pw_left = nullptr, *pw_right = nullptr, *pw_hoff = nullptr;
  float *pw_vals = nullptr, *pw_out = nullptr;
  size_t pw_cap_leaves = 0, pw_cap_nodes = 0, pw_cap_h = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double last_ms = 0.0;
  // optional per-phase timing: events at 7 marks per step, reused across runs
  int profiling = 0;
  std::vector<cudaEvent_t> marks;
  size_t mark_used = 0;
  long long launches = 0;   // kernels enqueued by the last pb_sim_run / pb_sim_step
  double sp_dx = 1.0, sp_dy = 1.0;   // grid spacing of the last step (cell keys of the sort)
  // CUDA graphs of whole steps (pb_sim_set_graphs): a step is captured once per shape (its
  // parameters without the step number, and the simulator state its launches bake in) and
  // replayed; the step number the Philox draws are keyed by comes from step_dev
  int graphs_on = 0, graphs_broken = 0, capturing = 0;
  uint32_t* step_dev = nullptr;
  long long step_dev_val = -1;     // the value step_dev holds once the stream reaches this point
  struct StepGraph {
    uint64_t pkey = 0, skey = 0;   // parameter digest, state signature before the step
    cudaGraphExec_t exec = nullptr;
    long long launches = 0;
  };
  std::vector<StepGraph> graphs;
  long long graph_captures = 0, graph_replays = 0, graph_plain_steps = 0;
  std::string graph_error;
};

// A launch with programmatic stream serialization (the step's kernels): the kernel may be
// scheduled while its predecessor in the stream drains, and waits in pdl_enter() until that
// predecessor has completed.  A predecessor that is not a kernel (a copy, a memset, an
// event) orders it as a plain launch would.
template <typename... KArgs, typename... Args>
static cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                              Args&&... args) {
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// ------------------------------------------------------------------ helpers
// cuTensorMapEncodeTiled from the driver, looked up once through the runtime (no link
// against libcuda)
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

// The corner array as a 3-D tensor of floats [ny][nx][8] with a box of 8 x TB_W x TB_H
// (one cell's eight corner values innermost, 32 B; rows 32 nx B apart).  Boxes that reach
// past the grid read zeros, which no gather uses: the gathered cell is clamped into it.
static int32_t ensure_ec_map(struct Sim* s);

static int grid_for(const Sim* s, long n, int bs, int per_sm = 8) {
  long g = (n + bs - 1) / bs;
  long cap = (long)s->num_sms * per_sm;
  if (g > cap) g = cap;
  return (int)std::max(1L, g);
}

static int32_t ensure_ec_map(Sim* s) {
  if (s->ecorn && s->ec_map_for == s->ecorn && s->ec_map_ny == s->ny && s->ec_map_nx == s->nx) return PB_OK;
  EncodeTiledFn enc = encode_tiled();
  if (!enc) return fail(PB_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
  const cuuint64_t dims[3] = {8, (cuuint64_t)s->nx, (cuuint64_t)s->ny};
  const cuuint64_t strides[2] = {32, (cuuint64_t)s->nx * 32};
  const cuuint32_t box[3] = {8, (cuuint32_t)TB_W, (cuuint32_t)TB_H};
  const cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = enc(&s->ec_map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void*)s->ecorn, dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(PB_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  s->ec_map_for = s->ecorn;
  s->ec_map_ny = s->ny;
  s->ec_map_nx = s->nx;
  return PB_OK;
}

static int32_t alloc_species(Sim* s, int k, int cap, int keep_n) {
  Species& S = s->sp[k];
  if (cap <= S.cap) return PB_OK;
  cap = ((cap + 1023) / 1024) * 1024;
  for (int b = 0; b < 2; ++b) {
    Soa nb{};
    CK(dalloc(&nb.x, cap)); CK(dalloc(&nb.y, cap)); CK(dalloc(&nb.vx, cap));
    CK(dalloc(&nb.vy, cap)); CK(dalloc(&nb.vz, cap)); CK(dalloc(&nb.id, cap));
    if (S.ion) CK(dalloc(&nb.cex, cap));
    Soa& ob = S.buf[b];
    if (ob.x && keep_n > 0 && b == S.cur) {
      size_t n4 = (size_t)keep_n * 4;
      CK(cudaMemcpyAsync(nb.x, ob.x, n4, cudaMemcpyDeviceToDevice, s->stream));
      CK(cudaMemcpyAsync(nb.y, ob.y, n4, cudaMemcpyDeviceToDevice, s->stream));
      CK(cudaMemcpyAsync(nb.vx, ob.vx, n4, cudaMemcpyDeviceToDevice, s->stream));
      CK(cudaMemcpyAsync(nb.vy, ob.vy, n4, cudaMemcpyDeviceToDevice, s->stream));
      CK(cudaMemcpyAsync(nb.vz, ob.vz, n4, cudaMemcpyDeviceToDevice, s->stream));
      CK(cudaMemcpyAsync(nb.id, ob.id, n4, cudaMemcpyDeviceToDevice, s->stream));
      if (S.ion) CK(cudaMemcpyAsync(nb.cex, ob.cex, keep_n, cudaMemcpyDeviceToDevice, s->stream));
    }
    CK(cudaStreamSynchronize(s->stream));
    dfree(ob.x); dfree(ob.y); dfree(ob.vx); dfree(ob.vy); dfree(ob.vz); dfree(ob.id); dfree(ob.cex);
    ob = nb;
  }
  S.cap = cap;
  // per-step scratch sized by the largest species
  size_t tiles = (size_t)std::max(s->sp[0].cap, s->sp[1].cap) / TILE_MIN + 2;
  if (tiles > s->tile_cap) {
    dfree(s->tile_status);
    CK(dalloc(&s->tile_status, 2 * tiles));
    s->tile_cap = tiles;
  }
  if ((size_t)s->sp[1].cap > s->ekeep_cap) {
    dfree(s->ekeep);
    CK(dalloc(&s->ekeep, (size_t)s->sp[1].cap));
    s->ekeep_cap = (size_t)s->sp[1].cap;
  }
  size_t scap = (size_t)std::max(s->sp[0].cap, s->sp[1].cap);
  if (scap > s->sort_cap) {
    for (int b = 0; b < 2; ++b) { dfree(s->skey[b]); dfree(s->sval[b]); CK(dalloc(&s->skey[b], scap)); CK(dalloc(&s->sval[b], scap)); }
    s->sort_cap = scap;
    size_t hc = (size_t)RADIX * (scap / SORT_TILE + 1);
    dfree(s->shist);
    CK(dalloc(&s->shist, hc));
    dfree(s->sblk);
    CK(dalloc(&s->sblk, hc / SCAN_CHUNK + 1));
    s->hist_cap = hc;
  }
  return PB_OK;
}

static int32_t read_counts(Sim* s) {
  int h[4];
  CK(cudaMemcpyAsync(h, s->counts, sizeof(h), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  s->host_num[0] = h[s->sp[0].cur];
  s->host_num[1] = h[2 + s->sp[1].cur];
  return PB_OK;
}

// keep room for one more step: injections, neutralizer, SEE spawns
static int32_t ensure_room(Sim* s, const pb_step_params* p, int steps) {
  long inj_max = 0;
  if (p->inject_on) inj_max = (long)(p->lam + 40.0 * std::sqrt(std::max(p->lam, 0.0)) + 100.0);
  long e_max = (long)p->neut_n + (p->rf_on ? (long)p->rf_num_float + 1 : 0);
  long need_p = s->host_num[0] + (long)steps * inj_max;
  long need_e = s->host_num[1] + (long)steps * (e_max + std::min<long>(s->see_cap, s->host_num[0] + 1024));
  int32_t rc;
  if (need_p > s->sp[0].cap) {
    if ((rc = read_counts(s))) return rc;
    need_p = s->host_num[0] + (long)steps * inj_max;
    if (need_p > s->sp[0].cap && (rc = alloc_species(s, 0, (int)(need_p + need_p / 4 + 4096), s->host_num[0]))) return rc;
  }
  if (need_e > s->sp[1].cap) {
    if ((rc = read_counts(s))) return rc;
    need_e = s->host_num[1] + (long)steps * (e_max + std::min<long>(s->see_cap, s->host_num[0] + 1024));
    if (need_e > s->sp[1].cap && (rc = alloc_species(s, 1, (int)(need_e + need_e / 4 + 4096), s->host_num[1]))) return rc;
  }
  return PB_OK;
}

static void free_levels(Sim* s) {
  for (size_t l = 0; l < s->lev.size(); ++l) {
    dfree(s->lev[l].dinv);
    dfree(s->lev[l].R);
    dfree(s->lev[l].U);
    dfree(s->lev[l].act);
    dfree(s->lev[l].st);
    if (l > 0) { dfree(s->lev[l].r); dfree(s->lev[l].z); }
  }
  s->lev.clear();
  dfree(s->cidx);
  dfree(s->cinv);
  dfree(s->mg_dense);
  dfree(s->mg_mdiag);
  dfree(s->mg_pre);
  dfree(s->mg_cidx_new);
  dfree(s->mg_pos);
}

// node classes from isBound (host copy) and the multigrid hierarchy
static int32_t update_bound_dist(Sim* s) {
  const int N = s->ny * s->nx;
  k_bdist_rows<<<grid_for(s, N, 256), 256, 0, s->stream>>>(s->isBound, s->bdist_tmp, s->ny, s->nx);
  k_bdist_cols<<<grid_for(s, N, 256), 256, 0, s->stream>>>(s->bdist_tmp, s->bdist, s->ny, s->nx);
  CK(cudaGetLastError());
  return PB_OK;
}

static int32_t build_operator(Sim* s, const uint8_t* isBound_host) {
  std::vector<uint8_t> cls = mghost::node_classes(s->ny, s->nx, s->periodic, isBound_host);
  CK(cudaMemcpyAsync(s->cls, cls.data(), cls.size(), cudaMemcpyHostToDevice, s->stream));
  if (int32_t rc = update_bound_dist(s)) return rc;
  mghost::Hierarchy H;
  try {
    H = mghost::build(s->ny, s->nx, s->periodic, cls, s->max_coarse);
  } catch (const std::exception& e) {
    return fail(PB_ERR_ARG, std::string("multigrid build: ") + e.what());
  }
  CK(cudaStreamSynchronize(s->stream));
  free_levels(s);
  s->lev.resize(H.lev.size());
  for (size_t l = 0; l < H.lev.size(); ++l) {
    const auto& L = H.lev[l];
    DevLevel& D = s->lev[l];
    D.ny = L.ny; D.nx = L.nx; D.per = L.per; D.wrapP = L.wrapP;
    size_t N = (size_t)L.ny * L.nx;
    CK(dalloc(&D.dinv, N));
    CK(cudaMemcpy(D.dinv, L.dinv.data(), N * sizeof(float), cudaMemcpyHostToDevice));
    if (!L.R.empty()) {
      CK(dalloc(&D.R, L.R.size()));
      CK(cudaMemcpy(D.R, L.R.data(), L.R.size() * sizeof(float), cudaMemcpyHostToDevice));
    }
    if (!L.U.empty()) {
      CK(dalloc(&D.U, L.U.size()));
      CK(cudaMemcpy(D.U, L.U.data(), L.U.size() * sizeof(float), cudaMemcpyHostToDevice));
    }
    if (l == 0) {
      D.r = s->r32; D.z = s->z32;
    } else {
      CK(dalloc(&D.r, N)); CK(dalloc(&D.z, N));
      CK(cudaMemset(D.r, 0, N * sizeof(float)));
      CK(cudaMemset(D.z, 0, N * sizeof(float)));
      CK(dalloc(&D.act, N));
      CK(dalloc(&D.st, 9 * N));
    }
  }
  s->nc = (int)H.cidx.size();
  // the coarsest level grows as cells break (more free nodes): room for a quarter more than
  // max(nc, max_coarse) nodes for the device rebuild, within the dense solve's limit
  s->ncap = std::min(MG_MAX_COARSE, std::max(s->nc, s->max_coarse) * 5 / 4);
  s->psmem = mg_solve_smem_bytes(s->ncap, mg_virtual_blocks((long)s->ny * s->nx, s->num_sms), 1);
  int occ = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_poisson, PT, s->psmem));
  if (occ < 1) return fail(PB_ERR_ARG, "field solver: no resident block with " + std::to_string(s->psmem) +
                                           " bytes of shared memory");
  const size_t ncap = (size_t)s->ncap;
  CK(dalloc(&s->cidx, ncap));
  CK(dalloc(&s->cinv, ncap * ncap));
  CK(cudaMemcpy(s->cidx, H.cidx.data(), s->nc * sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(s->cinv, H.cinv.data(), (size_t)s->nc * s->nc * sizeof(float), cudaMemcpyHostToDevice));
  CK(dalloc(&s->mg_dense, ncap * ncap));
  CK(dalloc(&s->mg_mdiag, ncap));
  CK(dalloc(&s->mg_pre, ncap * MG_PANEL * 4));
  CK(dalloc(&s->mg_cidx_new, ncap));
  CK(dalloc(&s->mg_pos, (size_t)H.lev.back().ny * H.lev.back().nx));
  if (!s->nc_dev) CK(dalloc(&s->nc_dev, 1));
  if (!s->mg_counts) {
    CK(dalloc(&s->mg_counts, MG_CNT_SLOTS));
    CK(cudaMemset(s->mg_counts, 0, MG_CNT_SLOTS * sizeof(int)));
  }
  if (!s->mg_dirty) CK(dalloc(&s->mg_dirty, 1));
  if (!s->mg_status) CK(dalloc(&s->mg_status, 1));
  CK(cudaMemcpy(s->nc_dev, &s->nc, sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemset(s->mg_dirty, 0, sizeof(int)));
  CK(cudaMemset(s->mg_status, 0, sizeof(uint32_t)));
  return PB_OK;
}

// Arguments of k_mg_rebuild for this simulator's hierarchy (the field solve's blocks).
static MgRebuildArgs mg_rebuild_args(Sim* s) {
  MgRebuildArgs a{};
  a.nlevels = (int)s->lev.size();
  a.max_coarse = s->max_coarse;
  a.ncap = s->ncap;
  a.cls = s->cls;
  for (size_t l = 0; l < s->lev.size() && l < (size_t)MG_MAX_LEVELS; ++l) {
    const DevLevel& D = s->lev[l];
    MgBuildLevel& B = a.lev[l];
    B.ny = D.ny; B.nx = D.nx; B.per = D.per; B.wrapP = D.wrapP;
    B.dinv = D.dinv; B.R = D.R; B.U = D.U; B.z = D.z; B.act = D.act; B.st = D.st;
  }
  a.cidx = s->cidx; a.cinv = s->cinv; a.nc_dev = s->nc_dev;
  a.dense = s->mg_dense; a.mdiag = s->mg_mdiag; a.pre = s->mg_pre; a.cidx_new = s->mg_cidx_new; a.pos = s->mg_pos;
  a.counts = s->mg_counts; a.dirty = s->mg_dirty; a.status = s->mg_status;
  a.bar = s->bar;
  a.errflags = &s->rep_dev->errflags;
  a.blk0 = 0;
  a.nblk = s->pgrid;
  return a;
}

// the fine up-leg tiling, computed once per grid shape and block count: for the launch's
// a.nblk blocks, or for the a.nvb virtual blocks when one smoothing sweep (nu = 1) makes
// that leg carry the (r, z) partials
static void set_up_tiles(Sim* s, PoissonArgs* a) {
  const int nb = a->nu0 == 2 ? a->nblk : a->nvb;
  if (s->ut_key[0] != s->ny || s->ut_key[1] != s->nx || s->ut_key[2] != nb) {
    fine_up_tiles(s->ny, s->nx, nb, &s->ut[0], &s->ut[1]);
    s->ut_key[0] = s->ny; s->ut_key[1] = s->nx; s->ut_key[2] = nb;
  }
  a->ut_y = s->ut[0];
  a->ut_x = s->ut[1];
}

static PoissonArgs poisson_args(Sim* s, int iterations, const pb_step_params* p) {
  PoissonArgs a{};
  a.ny = s->ny; a.nx = s->nx; a.periodic = s->periodic;
  a.cls = s->cls; a.Vfixed = s->Vfixed; a.rho = s->rho; a.V = s->V; a.x = s->Vnew; a.f = s->f; a.dirsum = s->dirsum;
  a.r32 = s->r32; a.z32 = s->z32; a.p32 = s->p32; a.q32 = s->q32; a.e32 = s->e32;
  a.s32 = s->s32; a.m32 = s->m32; a.nu0 = s->nu;
  a.Ex = s->Ex; a.Ey = s->Ey;
  a.coeff = p->coeff; a.qn0_neg = p->qn0_neg; a.V_plasma = p->V_plasma; a.Te_up = p->Te_up;
  a.omega_keep = p->omega_keep; a.omega_new = p->omega_new;
  a.hx = p->hx; a.two_hx = p->two_hx; a.hy = p->hy; a.two_hy = p->two_hy; a.two_hy_per = p->two_hy_per;
  a.iterations = iterations; a.compute_field = 1;
  a.tol = s->tol; a.tol_inner = s->tol_inner; a.max_outer = s->max_outer; a.max_inner = s->max_inner;
  a.nlevels = (int)s->lev.size();
  for (size_t l = 0; l < s->lev.size() && l < (size_t)MG_MAX_LEVELS; ++l) {
    const DevLevel& D = s->lev[l];
    a.lev[l].ny = D.ny; a.lev[l].nx = D.nx; a.lev[l].per = D.per; a.lev[l].wrapP = D.wrapP;
    a.lev[l].r = D.r; a.lev[l].z = D.z;
    a.lev[l].dinv = D.dinv;
    a.lev[l].R = D.R;
    a.lev[l].U = D.U;
  }
  a.nc_dev = s->nc_dev; a.cidx = s->cidx; a.cinv = s->cinv;
  a.blk0 = 0; a.nblk = s->pgrid;
  a.nvb = mg_virtual_blocks((long)s->ny * s->nx, s->num_sms);
  a.vb_off = mg_vb_offset(s->ncap);
  set_up_tiles(s, &a);
  a.partials = s->partials; a.bar = s->bar;
  a.errflags = &s->rep_dev->errflags;
  a.stats = s->pstats;
  a.solve_ns = s->solve_ns;
  a.trace = s->trace_on ? s->ptrace : nullptr;
  return a;
}

// Cooperative launches on one device are chained in enqueue order: each waits for the
// previous one (whatever stream it was on), so two field-solve kernels, each of which
// needs all of its blocks resident at once, never compete for the SMs.
struct CoopChain {
  std::mutex mu;
  cudaEvent_t last = nullptr;
};
static CoopChain g_coop[64];

template <class Launch>
static int32_t coop_launch(int device, cudaStream_t st, Launch launch) {
  if (device < 0 || device >= 64) return fail(PB_ERR_ARG, "device ordinal out of range");
  CoopChain& c = g_coop[device];
  std::lock_guard<std::mutex> lk(c.mu);
  if (!c.last) CK(cudaEventCreateWithFlags(&c.last, cudaEventDisableTiming));
  CK(cudaStreamWaitEvent(st, c.last, 0));
  CK(launch());
  CK(cudaEventRecord(c.last, st));
  return PB_OK;
}

// A cooperative launch of the field-solve grid: inside a step graph ordered by the
// simulator's own stream (a graph runs its simulator alone, so no other cooperative launch
// is chained against it), otherwise through the device's chain.
static int32_t coop_field_launch(Sim* s, const void* kernel, void** args, size_t smem) {
  CK(cudaMemsetAsync(s->bar, 0, 2 * sizeof(unsigned int), s->stream));
  if (s->capturing) {
    CK(cudaLaunchCooperativeKernel(kernel, dim3(s->pgrid), dim3(PT), args, smem, s->stream));
  } else {
    int32_t rc = coop_launch(s->device, s->stream, [&]() {
      return cudaLaunchCooperativeKernel(kernel, dim3(s->pgrid), dim3(PT), args, smem, s->stream);
    });
    if (rc) return rc;
  }
  ++s->launches;
  return PB_OK;
}

static int32_t launch_poisson(Sim* s, int iterations, const pb_step_params* p) {
  if (iterations <= 0) return PB_OK;
  int32_t rc;
  if (s->erosion_seen) {
    // cells may have broken since the last solve: the hierarchy follows the node classes
    // first (k_mg_rebuild returns at once unless a break set mg_dirty)
    MgRebuildArgs m = mg_rebuild_args(s);
    void* margs[] = {&m};
    if ((rc = coop_field_launch(s, (const void*)k_mg_rebuild, margs, 0))) return rc;
  }
  PoissonArgs a = poisson_args(s, iterations, p);
  void* args[] = {&a};
  return coop_field_launch(s, (const void*)k_poisson, args, mg_solve_smem_bytes(s->ncap, a.nvb, a.nblk));
}

// The per-step resets in one launch instead of a dozen memsets (each of which is an
// operation of its own on the GPU timeline): the step report (zero, ppc_min all ones),
// the PPC map, both step kernels' tile descriptors and the small counters.
struct StepResetArgs {
  pb_step_report* rep;
  int* ppc;
  int N;
  unsigned long long* tile_status;
  long long ntile;
  int *angle_count, *see_count, *see_spawned, *tile_counter, *ni_dst, *ne_dst, *inj;
  unsigned long long* ds_bits;
};

__global__ void k_step_reset(StepResetArgs a) {
  pdl_enter();
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x, nth = (long long)gridDim.x * blockDim.x;
  static_assert(sizeof(pb_step_report) % 4 == 0 && offsetof(pb_step_report, ppc_min) % 4 == 0, "report words");
  constexpr long long nw = sizeof(pb_step_report) / 4, w0 = offsetof(pb_step_report, ppc_min) / 4;
  uint32_t* r = reinterpret_cast<uint32_t*>(a.rep);
  for (long long i = tid; i < nw; i += nth) r[i] = (i == w0 || i == w0 + 1) ? 0xFFFFFFFFu : 0u;
  for (long long i = tid; i < a.N; i += nth) a.ppc[i] = 0;
  for (long long i = tid; i < a.ntile; i += nth) a.tile_status[i] = 0ull;
  if (tid == 0) {
    *a.angle_count = 0; *a.see_count = 0; *a.see_spawned = 0;
    a.ds_bits[0] = 0ull; a.ds_bits[1] = 0ull; a.ds_bits[2] = 0ull;
    a.tile_counter[0] = 0; a.tile_counter[1] = 0;
    *a.ni_dst = 0; *a.ne_dst = 0;
    for (int k = 0; k < 7; ++k) a.inj[k] = 0;
  }
}

// RF: V_fixed on grid g = Vdc + v_rf
__global__ void k_rf_update(double* Vfixed, const double* Vdc, const uint16_t* gridmask, int N, int g, double v_rf) {
  pdl_enter();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
    if (gridmask[i] & (1u << g)) Vfixed[i] = Vdc[i] + v_rf;
}

struct SaddleIdx { int v[8]; };

// The step report's device-side fields, the saddle potential (the minimum of V over up to
// eight saddle nodes; 0 without any) and the solver statistics, in one thread.
__global__ void k_report(pb_step_report* r, const int* counts, int ci, int ce, const int* n_sub,
                         const unsigned long long* ds_bits, const int* inj, const int* see_spawned, const double* V,
                         int n_saddle, SaddleIdx sidx, const double* pstats) {
  pdl_enter();
  r->num_p = counts[ci];
  r->num_e = counts[2 + ce];
  r->n_sub_ion = n_sub[0];
  r->n_sub_e = n_sub[1];
  r->ds_ion = __longlong_as_double((long long)ds_bits[0]);
  r->ds_e = __longlong_as_double((long long)ds_bits[1]);
  r->injected = inj[0];
  r->rf_injected = inj[1];
  r->neut_injected = inj[2];
  r->see_spawned = *see_spawned;
  double mp = 0.0;
  for (int k = 0; k < n_saddle; ++k) {
    double v = V[sidx.v[k]];
    mp = (k == 0 || v < mp) ? v : mp;
  }
  r->min_pot = mp;
  for (int k = 0; k < 4; ++k) r->poisson_stats[k] = pstats[k];
}

// n_sub of both species from their reduced displacements, one thread
__global__ void k_substep_finish2(const double* ds_max, double ds_lim, int* n_sub_out, uint32_t* errflags) {
  pdl_enter();
  n_sub_out[0] = substep_count(ds_max[0], ds_lim, errflags);
  n_sub_out[1] = substep_count(ds_max[1], ds_lim, errflags);
}

}  // namespace pb

using namespace pb;

struct SplineStore {
  double* t = nullptr;
  double* c = nullptr;
  int nt = 0;
  double lo = 0.0, hi = 0.0;
  double cmax = 0.0;  // largest B-spline coefficient: the spline never exceeds it (convex hull)
};

struct pb_sim {
  Sim s;
  SplineStore cx, see;
};

static Spline spline_of(const SplineStore& st) {
  Spline sp{};
  sp.t = st.t; sp.c = st.c; sp.nt = st.nt; sp.lo = st.lo; sp.hi = st.hi; sp.enabled = st.nt > 0;
  return sp;
}

static int32_t sort_species(Sim* s, int k, int ncell_bits) {
  Species& S = s->sp[k];
  cudaStream_t st = s->stream;
  int* n_src = s->counts + 2 * k + S.cur;
  int* n_dst = s->counts + 2 * k + (1 - S.cur);
  int cap = S.cap;
  int ntiles = (cap + SORT_TILE - 1) / SORT_TILE;
  const Soa& src = S.buf[S.cur];
  CK(launch_pdl(k_sort_keys, grid_for(s, cap, 256), 256, 0, st, src.x, src.y, n_src, s->nx, s->ny, (float)s->sp_dx,
                                                     (float)s->sp_dy, s->skey[0], s->sval[0]));
  ++s->launches;
  int a = 0;
  for (int shift = 0; shift < ncell_bits; shift += RADIX_BITS) {
    CK(launch_pdl(k_sort_hist, ntiles, SORT_NT, 0, st, s->skey[a], n_src, shift, s->shist, ntiles));
    ++s->launches;
    {
      const int total = RADIX * ntiles, nb = (total + SCAN_CHUNK - 1) / SCAN_CHUNK;
      CK(launch_pdl(k_scan_partials, nb, SCAN_NT, 0, st, s->shist, total, s->sblk));
      CK(launch_pdl(k_sort_scan, 1, 1024, 0, st, s->sblk, nb));
      CK(launch_pdl(k_scan_apply, nb, SCAN_NT, 0, st, s->shist, total, s->sblk));
      s->launches += 3;
    }
    CK(launch_pdl(k_sort_scatter, ntiles, SORT_NT, 0, st, s->skey[a], s->sval[a], n_src, shift, s->shist, ntiles,
                                                s->skey[1 - a], s->sval[1 - a]));
    ++s->launches;
    a = 1 - a;
  }
  CK(launch_pdl(k_sort_gather, grid_for(s, cap, 256), 256, 0, st, src, S.buf[1 - S.cur], s->sval[a], n_src));
  ++s->launches;
  CK(launch_pdl(k_copy_int, 1, 1, 0, st, n_src, n_dst));
  ++s->launches;
  S.cur ^= 1;
  CK(cudaGetLastError());
  return PB_OK;
}

static int32_t check_flags(Sim* s, uint32_t f) {
  if (f & PB_EF_SPIN_TIMEOUT) return fail(PB_ERR_TIMEOUT, "a bounded device wait timed out");
  if (f & (PB_EF_CAPACITY_ION | PB_EF_CAPACITY_ELE | PB_EF_SEE_OVERFLOW | PB_EF_ANGLE_OVERFLOW | PB_EF_ID_OVERFLOW))
    return fail(PB_ERR_CAPACITY, "particle storage or a per-step list overflowed (flags " + std::to_string(f) + ")");
  if (f & (PB_EF_NAN_SUBSTEP | PB_EF_SUBSTEP_CAP)) return fail(PB_ERR_ARG, "sub-step count is NaN or above 65536");
  if (f & PB_EF_POISSON_NOCONV) return fail(PB_ERR_NOCONV, "field solve did not reach its tolerance");
  return PB_OK;
}

// one timestep, enqueued on the instance stream (physics_engine.py:969-1784)
// record a phase mark (profiling only); marks k..k+PB_MARKS-1 of one step bracket its
// PB_MARKS - 1 phases: inject + deposit, field solve, E corners + sub-step counts, ion
// step, sputter break, electron step, SEE spawn, thermal + grid sums, diagnostics + sort
constexpr int PB_MARKS = 10;
static void mark(Sim* s) {
  if (!s->profiling) return;
  if (s->mark_used >= s->marks.size()) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    s->marks.push_back(e);
  }
  cudaEventRecord(s->marks[s->mark_used++], s->stream);
}

// A step is enqueued in two halves around the field solve, so that a batch can solve the
// fields of several instances in one launch between them.
// Indices in the step parameters that kernels dereference, checked before anything of the
// step is enqueued.
static int32_t check_step_params(const Sim* s, const pb_step_params* p) {
  const long N = (long)s->ny * s->nx;
  const int ns = std::max(0, std::min(p->n_saddle, 8));
  for (int k = 0; k < ns; ++k)
    if (p->saddle_idx[k] < 0 || p->saddle_idx[k] >= N) return fail(PB_ERR_ARG, "step: saddle index outside the grid");
  if (p->rf_grid < -1 || p->rf_grid > 15) return fail(PB_ERR_ARG, "step: rf_grid must be -1 (off) or 0 to 15");
  return PB_OK;
}

// the step kernels' variant for the option bits and tile size
template <int TL>
static cudaError_t launch_ion(uint32_t kopts, dim3 g, cudaStream_t st, const IonStepArgs& a) {
  switch (kopts & (PB_OPT_SMEM_HIST | PB_OPT_TMA_TILE)) {
    case 0: return launch_pdl(k_ion_step<false, 0, TL>, g, NT, 0, st, a);
    case PB_OPT_SMEM_HIST: return launch_pdl(k_ion_step<false, PB_OPT_SMEM_HIST, TL>, g, NT, 0, st, a);
    case PB_OPT_TMA_TILE: return launch_pdl(k_ion_step<false, PB_OPT_TMA_TILE, TL>, g, NT, 0, st, a);
    default: return launch_pdl(k_ion_step<false, PB_OPT_SMEM_HIST | PB_OPT_TMA_TILE, TL>, g, NT, 0, st, a);
  }
}
template <int TL>
static cudaError_t launch_ele(uint32_t kopts, dim3 g, cudaStream_t st, const EleStepArgs& b) {
  switch (kopts & (PB_OPT_SMEM_HIST | PB_OPT_ELE_PAIRS)) {
    case 0: return launch_pdl(k_ele_step<false, 0, TL>, g, NT, 0, st, b);
    case PB_OPT_SMEM_HIST: return launch_pdl(k_ele_step<false, PB_OPT_SMEM_HIST, TL>, g, NT, 0, st, b);
    case PB_OPT_ELE_PAIRS: return launch_pdl(k_ele_step<false, PB_OPT_ELE_PAIRS, TL>, g, NT, 0, st, b);
    default: return launch_pdl(k_ele_step<false, PB_OPT_SMEM_HIST | PB_OPT_ELE_PAIRS, TL>, g, NT, 0, st, b);
  }
}

static int32_t enqueue_step_pre(pb_sim* h, const pb_step_params* p) {
  Sim* s = &h->s;
  if (int32_t rc = check_step_params(s, p)) return rc;
  mark(s);
  cudaStream_t st = s->stream;
  const int N = s->ny * s->nx;
  Species& I = s->sp[0];
  Species& E = s->sp[1];
  const float dxf = (float)p->dx, dyf = (float)p->dy;
  s->sp_dx = p->dx;
  s->sp_dy = p->dy;
  int* ni_src = s->counts + I.cur;
  int* ni_dst = s->counts + (1 - I.cur);
  int* ne_src = s->counts + 2 + E.cur;
  int* ne_dst = s->counts + 2 + (1 - E.cur);
  pb_step_report* rep = s->rep_dev;
  uint32_t* ef = &rep->errflags;

  // per-step resets, one launch
  {
    StepResetArgs r{};
    r.rep = rep; r.ppc = s->ppc; r.N = N;
    r.tile_status = s->tile_status; r.ntile = 2 * (long long)s->tile_cap;
    r.angle_count = s->angle_count; r.see_count = s->see_count; r.see_spawned = s->see_spawned;
    r.ds_bits = s->ds_bits; r.tile_counter = s->tile_counter; r.ni_dst = ni_dst; r.ne_dst = ne_dst; r.inj = s->inj;
    CK(launch_pdl(k_step_reset, grid_for(s, std::max<long>(N, 2 * (long)s->tile_cap), 256), 256, 0, st, r));
    ++s->launches;
  }

  if (!s->counts_valid) {
    CK(cudaMemsetAsync(s->cnt_i, 0, (size_t)N * sizeof(int), st));
    CK(cudaMemsetAsync(s->cnt_e, 0, (size_t)N * sizeof(int), st));
    CK(launch_pdl(k_count_cells, grid_for(s, I.cap, 256), 256, 0, st, I.buf[I.cur].x, I.buf[I.cur].y, ni_src, 0, 0,
                  s->cnt_i, s->nx, s->ny, dxf, dyf));
    ++s->launches;
    CK(launch_pdl(k_count_cells, grid_for(s, E.cap, 256), 256, 0, st, E.buf[E.cur].x, E.buf[E.cur].y, ne_src, 0, 0,
                  s->cnt_e, s->nx, s->ny, dxf, dyf));
    ++s->launches;
    s->counts_valid = true;
  }

  // RF co-extraction: V_fixed on one grid, then recalc_poisson(2) (:984-991)
  int32_t rc;
  if (p->rf_grid >= 0) {
    CK(launch_pdl(k_rf_update, grid_for(s, N, 256), 256, 0, st, s->Vfixed, s->Vdc, s->gridmask, N, p->rf_grid,
                  p->v_rf));
    ++s->launches;
    if ((rc = launch_poisson(s, 2, p))) return rc;
  }

  // A. injection (:996-1099)
  InjectArgs ia{};
  ia.ion_on = p->inject_on; ia.lam = p->lam; ia.geometry = p->geometry; ia.ylo = p->ylo; ia.yhi = p->yhi;
  for (int k = 0; k < 4; ++k) ia.span[k] = (float)p->span[k];
  ia.x_inj = (float)p->x_inj; ia.v_bohm = p->v_bohm; ia.v_spread = p->v_spread;
  ia.rf_on = p->rf_on; ia.rf_num_float = p->rf_num_float; ia.rf_ylo = p->rf_ylo; ia.rf_yhi = p->rf_yhi;
  ia.v_e_src = p->v_e_src;
  ia.neut_n = p->neut_n; ia.neut_r = p->neut_r; ia.v_e_th = p->v_e_th; ia.neut_x = (float)p->neut_x;
  ia.seed = s->seed; ia.step = (uint32_t)p->iteration; ia.step_dev = s->capturing ? s->step_dev : nullptr;
  ia.num_p = ni_src; ia.num_e = ne_src; ia.cap_p = I.cap; ia.cap_e = E.cap;
  ia.next_ion_id = s->next_ids; ia.next_e_id = s->next_ids + 1;
  ia.inj = s->inj;
  ia.ions = I.buf[I.cur]; ia.eles = E.buf[E.cur];
  ia.cnt_i = s->cnt_i; ia.cnt_e = s->cnt_e;
  ia.nx = s->nx; ia.ny = s->ny; ia.dxf = dxf; ia.dyf = dyf; ia.errflags = ef;
  CK(launch_pdl(k_inject_prep, 1, 1, 0, st, ia));
  ++s->launches;
  {
    long mx = std::max<long>({(long)(p->lam + 40.0 * std::sqrt(std::max(p->lam, 0.0)) + 100.0),
                              (long)p->neut_n, (long)p->rf_num_float + 1, 1L});
    CK(launch_pdl(k_inject_gen, dim3(grid_for(s, mx, 128, 2), 3), 128, 0, st, ia));
    ++s->launches;
  }

  // B. deposit (counts -> exact float32 sums) and the Picard field solve (:1104-1161)
  CK(launch_pdl(k_rho_finalize, grid_for(s, N, 256), 256, 0, st, s->rho, s->cnt_i, s->cnt_e, N, p->charge_density, 0));
  ++s->launches;
  mark(s);
  CK(cudaGetLastError());
  return PB_OK;
}

static int32_t enqueue_step_post(pb_sim* h, const pb_step_params* p) {
  Sim* s = &h->s;
  mark(s);
  cudaStream_t st = s->stream;
  const int N = s->ny * s->nx;
  Species& I = s->sp[0];
  Species& E = s->sp[1];
  const float dxf = (float)p->dx, dyf = (float)p->dy;
  int* ni_src = s->counts + I.cur;
  int* ni_dst = s->counts + (1 - I.cur);
  int* ne_src = s->counts + 2 + E.cur;
  int* ne_dst = s->counts + 2 + (1 - E.cur);
  pb_step_report* rep = s->rep_dev;
  uint32_t* ef = &rep->errflags;
  int32_t rc;

  // corners of Ex, Ey for the gathers below (rebuilt every step: fields change in the
  // solve, through pb_sim_set_field or through pb_sim_field_ptr)
  // the field bound that lets the sub-step reductions pass over slow particles
  unsigned* ebound = reinterpret_cast<unsigned*>(s->ds_bits + 2);
  CK(launch_pdl(k_e_corners, grid_for(s, N, 256), 256, 0, st, s->Ex, s->Ey, s->ecorn, s->ny, s->nx, ebound));
  ++s->launches;

  // C. sub-step counts (:1177-1209)
  const float dtf = (float)p->dt;
  CK(launch_pdl(k_substep_reduce, grid_for(s, I.cap / 4, 256, 4), 256, 0, st, I.buf[I.cur].x, I.buf[I.cur].y,
                I.buf[I.cur].vx, I.buf[I.cur].vy, I.buf[I.cur].vz, ni_src, 0, s->Ex, s->Ey, s->ecorn, s->nx, s->ny, dxf,
                dyf, p->qm_ion, dtf, p->dt2, s->ds_bits, ebound));
  ++s->launches;
  CK(launch_pdl(k_substep_reduce, grid_for(s, E.cap / 4, 256, 4), 256, 0, st, E.buf[E.cur].x, E.buf[E.cur].y,
                E.buf[E.cur].vx, E.buf[E.cur].vy, E.buf[E.cur].vz, ne_src, 0, s->Ex, s->Ey, s->ecorn, s->nx, s->ny, dxf,
                dyf, p->qm_e, dtf, p->dt2, s->ds_bits + 1, ebound));
  ++s->launches;
  CK(launch_pdl(k_substep_finish2, 1, 1, 0, st, (const double*)s->ds_bits, p->ds_lim, s->n_sub, ef));
  ++s->launches;
  mark(s);

  // ions: push, hits, tallies, exit diagnostics, compaction, CEX, PPC (:1211-1739)
  IonStepArgs a{};
  a.src = I.buf[I.cur]; a.dst = I.buf[1 - I.cur]; a.num_src = ni_src; a.num_dst = ni_dst;
  a.Ex = s->Ex; a.Ey = s->Ey; a.Ec = s->ecorn; a.Bx = a.By = a.Bz = nullptr; a.has_B = 0;
  a.isBound = s->isBound; a.bdist = s->bdist; a.nx = s->nx; a.ny = s->ny; a.dxf = dxf; a.dyf = dyf;
  a.inv_dx = 1.0f / dxf; a.inv_dy = 1.0f / dyf; a.rcp = make_rcp(dxf, dyf);
  a.dt = p->dt; a.qm = p->qm_ion; a.ds_lim = p->ds_lim; a.ds_max = (const double*)s->ds_bits; a.n_sub_out = s->n_sub;
  a.periodic = s->periodic; a.Lyf = (float)p->Ly; a.Lxf = (float)p->Lx;
  a.x_entry = (float)p->x_entry; a.x_exit = (float)p->x_exit; a.x_plume = (float)p->x_plume;
  a.thermal_on = p->thermal_on; a.erosion_on = p->erosion_on;
  a.Tmap = s->Tmap; a.damage = s->damage;
  a.k_half_m = (float)p->half_m_ion; a.mw_f = (float)p->macro_w; a.ccell_f = (float)p->C_cell;
  a.accel_f = (float)p->thermal_accel; a.q_f = (float)p->q; a.Y_f = (float)p->Y_coeff; a.Eth_f = (float)p->E_th;
  a.Y_d = p->Y_coeff; a.mw_d = p->macro_w; a.Y_exp = p->sputter_exp == 0.0 ? 1.0 : p->sputter_exp;
  a.dt_f = dtf;
  a.see_spline = spline_of(h->see);
  a.see_key = s->see_key; a.see_xy = s->see_xy; a.see_count = s->see_count; a.see_cap = s->see_cap;
  a.angles = s->angles; a.angle_count = s->angle_count; a.angle_cap = s->angle_cap;
  a.exit_sums = rep->exit_sums; a.counters = (unsigned long long*)&rep->entered;
  a.rT_f = (float)p->rT; a.n0a = p->n0a; a.neut_vth = p->neut_vth; a.cx_spline = spline_of(h->cx);
  a.n_uniform = p->neutral_uniform ? 1 : 0; a.n0u = p->n0_uniform;
  {
    // collision-probability bound: sigma <= 10^cmax (spline), or <= 2.2881e-18 for the
    // empirical law while 1 <= g <= 1e14 (|(-0.8821 ln g + 15.1262)| <= 15.1262); the
    // point-source density never exceeds |n0 a_corr| (its geometric factor is below 1)
    double sig_max = h->cx.nt > 0 ? std::pow(10.0, h->cx.cmax) : 2.2881e-18;
    const double n_max = a.n_uniform ? std::fabs(p->n0_uniform) : std::fabs(p->n0a);
    a.cex_bound = n_max * sig_max * p->dt * (1.0 + 1e-5);
    a.cex_g_max = h->cx.nt > 0 ? INFINITY : 1e14f;
  }
  a.seed = s->seed; a.step = (uint32_t)p->iteration; a.step_dev = s->capturing ? s->step_dev : nullptr;
  a.ppc = s->ppc; a.cnt = s->cnt_i;
  a.tile_status = s->tile_status; a.tile_counter = s->tile_counter; a.errflags = ef;
  {
    const dim3 g(grid_for(s, I.cap, s->ppb, s->pbps));
    if (s->kopts & PB_OPT_TMA_TILE) {
      if ((rc = ensure_ec_map(s))) return rc;
      a.ec_map = s->ec_map;
    }
    CK(s->ppb == TILE_MIN ? launch_ion<TILE_MIN>(s->kopts, g, st, a) : launch_ion<TILE>(s->kopts, g, st, a));
  }
  ++s->launches;
  mark(s);

  // sputter cell break (:1443-1449) before the electron purge, which sees the new mask
  if (p->erosion_on) {
    CK(launch_pdl(k_erosion_break, grid_for(s, N, 256), 256, 0, st, s->damage, s->isBound, s->cls, s->eroded, s->ny,
                  s->nx, s->periodic, p->thresh, p->dy, &rep->broken));
    CK(launch_pdl(k_refresh_dinv0, grid_for(s, N, 256), 256, 0, st, s->cls, s->lev[0].dinv, s->ny, s->nx, s->periodic,
                                                         &rep->broken, s->mg_dirty));
    s->launches += 2;
    s->erosion_seen = true;
  }
  mark(s);

  // electrons: push and purge (:1248-1293, 1534-1561)
  EleStepArgs b{};
  b.src = E.buf[E.cur]; b.dst = E.buf[1 - E.cur]; b.num_src = ne_src; b.num_dst = ne_dst;
  b.Ex = s->Ex; b.Ey = s->Ey; b.Ec = s->ecorn; b.Bx = b.By = b.Bz = nullptr; b.has_B = 0;
  b.isBound = s->isBound; b.nx = s->nx; b.ny = s->ny; b.dxf = dxf; b.dyf = dyf;
  b.inv_dx = 1.0f / dxf; b.inv_dy = 1.0f / dyf; b.rcp = make_rcp(dxf, dyf);
  b.ebound = ebound;
  b.dt = p->dt; b.qm = p->qm_e; b.ds_lim = p->ds_lim; b.ds_max = (const double*)(s->ds_bits + 1);
  b.n_sub_out = s->n_sub + 1; b.periodic = s->periodic; b.Lyf = (float)p->Ly; b.Lxf = (float)p->Lx;
  b.cnt = s->cnt_e; b.tile_status = s->tile_status + s->tile_cap; b.tile_counter = s->tile_counter + 1;
  b.errflags = ef;
  if (s->kopts & PB_OPT_ELE_SPLIT) {
    CK(launch_pdl(k_ele_push, grid_for(s, E.cap, NT, s->pbps), NT, 0, st, b, s->ekeep));
    CK(launch_pdl(k_ele_compact, grid_for(s, E.cap, TILE, s->pbps), NT, 0, st, b, (const uint8_t*)s->ekeep));
    ++s->launches;
  } else {
    const dim3 g(grid_for(s, E.cap, s->ppb, s->pbps));
    CK(s->ppb == TILE_MIN ? launch_ele<TILE_MIN>(s->kopts, g, st, b) : launch_ele<TILE>(s->kopts, g, st, b));
  }
  ++s->launches;
  mark(s);

  // SEE electrons, appended after the surviving electrons (:1390-1417)
  SeeArgs sa{};
  sa.see_key = s->see_key; sa.see_xy = s->see_xy; sa.see_count = s->see_count; sa.see_cap = s->see_cap;
  sa.see_spawned = s->see_spawned; sa.seed = s->seed; sa.step = (uint32_t)p->iteration;
  sa.step_dev = s->capturing ? s->step_dev : nullptr; sa.v_see_th = p->v_see_th;
  sa.eles = E.buf[1 - E.cur]; sa.num_e = ne_dst; sa.cap_e = E.cap; sa.next_e_id = s->next_ids + 1;
  sa.isBound = s->isBound; sa.nx = s->nx; sa.ny = s->ny; sa.dxf = dxf; sa.dyf = dyf;
  sa.Lxf = (float)p->Lx; sa.Lyf = (float)p->Ly; sa.cnt_e = s->cnt_e; sa.errflags = ef;
  CK(launch_pdl(k_see_finish, 1, 1024, 0, st, sa));
  ++s->launches;
  mark(s);
  I.cur ^= 1;
  E.cur ^= 1;

  // F. thermal (:1566-1620)
  if (p->thermal_on) {
    CK(launch_pdl(k_thermal, dim3((s->nx + TT - 1) / TT, (s->ny + TT - 1) / TT), 256, 0, st,
        s->Tmap, s->isBound, s->ny, s->nx, (float)p->cooling_factor, (float)p->T4_300, (float)p->Fo_x,
        (float)p->Fo_y, p->sweeps));
    ++s->launches;
  }
  if (s->ngrids > 0) {
    CK(launch_pdl(k_grid_sums, grid_for(s, N, 256), 256, 0, st, s->Tmap, s->gridmask, N, std::min(s->ngrids, 16),
                  rep->grid_sums));
    ++s->launches;
  }
  mark(s);

  // exit divergence, saddle potential, PPC map (:1482-1488, 1655-1676, 1741-1767)
  CK(launch_pdl(k_theta95, 1, 1024, 0, st, s->angles, s->angle_count, s->angle_cap, s->angle_scratch, &rep->theta95));
  ++s->launches;
  SaddleIdx sidx{};
  for (int k = 0; k < 8; ++k) sidx.v[k] = p->saddle_idx[k];
  CK(launch_pdl(k_report, 1, 1, 0, st, rep, s->counts, I.cur, E.cur, s->n_sub, s->ds_bits, s->inj, s->see_spawned, s->V,
                            std::max(0, std::min(p->n_saddle, 8)), sidx, s->pstats));
  ++s->launches;
  CK(launch_pdl(k_ppc_stats, grid_for(s, N, 256), 256, 0, st, s->ppc, s->accum_ppc, N,
                (unsigned long long*)&rep->ppc_active));
  ++s->launches;

  // periodic re-sort by cell key (locality of the gathers and deposits); the permutation
  // equals a stable argsort
  if (p->sort_now) {
    int bits = 1;
    while ((1L << bits) < (long)N) ++bits;
    if ((rc = sort_species(s, 0, bits))) return rc;
    if ((rc = sort_species(s, 1, bits))) return rc;
  }
  mark(s);
  CK(cudaGetLastError());
  return PB_OK;
}

static int32_t enqueue_step(pb_sim* h, const pb_step_params* p) {
  int32_t rc;
  if ((rc = enqueue_step_pre(h, p))) return rc;
  if (p->do_poisson && (rc = launch_poisson(&h->s, p->picard_iters, p))) return rc;
  return enqueue_step_post(h, p);
}

// ------------------------------------------------------------------ step graphs
__global__ void k_step_advance(uint32_t* step) { *step += 1u; }
__global__ void k_step_set(uint32_t* step, uint32_t v) { *step = v; }

static uint64_t fnv(uint64_t h, const void* data, size_t n) {
  const unsigned char* c = static_cast<const unsigned char*>(data);
  for (size_t i = 0; i < n; ++i) { h ^= c[i]; h *= 1099511628211ull; }
  return h;
}
template <class T>
static uint64_t fnv_v(uint64_t h, const T& v) { return fnv(h, &v, sizeof(T)); }

// The step's parameters without the step number (which the captured kernels read from
// step_dev).
static uint64_t params_digest(const pb_step_params* p) {
  pb_step_params q = *p;
  q.iteration = 0;
  return fnv(1469598103934665603ull, &q, sizeof(q));
}

// Everything of the simulator that a step's launches take as arguments: buffers, sizes,
// settings and the host-side state (buffer parity, counts validity).  A cached graph is
// replayed only while this is unchanged.
static uint64_t state_signature(const pb_sim* h) {
  const Sim* s = &h->s;
  uint64_t k = 1469598103934665603ull;
  for (int sp = 0; sp < 2; ++sp) {
    const Species& S = s->sp[sp];
    k = fnv_v(k, S.cur); k = fnv_v(k, S.cap);
    for (int b = 0; b < 2; ++b) k = fnv_v(k, S.buf[b]);
  }
  const void* ptrs[] = {s->V, s->Vnew, s->Vfixed, s->Vdc, s->damage, s->eroded, s->accum_ppc, s->f, s->dirsum,
                        s->Ex, s->Ey, s->rho, s->Tmap, s->r32, s->z32, s->p32, s->q32, s->e32, s->s32, s->m32,
                        s->ecorn,
                        s->isBound, s->cls, s->bdist, s->gridmask, s->ppc, s->cnt_i, s->cnt_e, s->cidx, s->cinv,
                        s->partials, s->bar, s->pstats, s->ptrace, s->counts, s->next_ids, s->tile_status,
                        s->tile_counter, s->see_key, s->see_xy, s->see_count, s->angles, s->angle_scratch,
                        s->angle_count, s->ds_bits, s->n_sub, s->inj, s->see_spawned, s->skey[0], s->skey[1],
                        s->sval[0], s->sval[1], s->shist, s->sblk, s->rep_dev, h->cx.t, h->cx.c, h->see.t,
                        h->see.c, s->step_dev, s->ekeep, s->nc_dev, s->mg_dense, s->mg_mdiag, s->mg_pre, s->mg_cidx_new,
                        s->mg_pos, s->mg_counts, s->mg_dirty, s->mg_status};
  k = fnv(k, ptrs, sizeof(ptrs));
  for (const DevLevel& L : s->lev) k = fnv_v(k, L);
  const long long vals[] = {s->ny, s->nx, s->periodic, s->ngrids, s->nc, s->trace_on, s->pgrid, s->ut[0], s->ut[1],
                            s->pbps, s->ppb, (long long)s->kopts, (long long)s->psmem, (long long)s->tile_cap, s->see_cap,
                            s->angle_cap, (long long)s->sort_cap, (long long)s->hist_cap, s->counts_valid ? 1 : 0,
                            s->max_outer, s->max_inner, s->nu, h->cx.nt, h->see.nt, s->profiling, s->ncap,
                            s->max_coarse, s->erosion_seen ? 1 : 0};
  k = fnv(k, vals, sizeof(vals));
  const double dv[] = {s->tol, s->tol_inner, h->cx.lo, h->cx.hi, h->cx.cmax, h->see.lo, h->see.hi};
  k = fnv(k, dv, sizeof(dv));
  k = fnv_v(k, s->seed);
  return k;
}

static void free_graphs(Sim* s) {
  for (auto& g : s->graphs)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  s->graphs.clear();
}

// A step that a graph can hold: no RF co-extraction (its grid voltage changes every step)
// and no phase marks.
static bool graph_eligible(const Sim* s, const pb_step_params* p) {
  return s->graphs_on && !s->graphs_broken && !s->profiling && p->rf_grid < 0;
}

// One step through a graph: replay the graph of this shape, or capture it first.  Sets
// *done = false (and leaves the host state as it was) when the step cannot be captured;
// the caller then enqueues it as usual.
static int32_t graph_step(pb_sim* h, const pb_step_params* p, bool* done) {
  Sim* s = &h->s;
  *done = false;
  const uint64_t pkey = params_digest(p), skey = state_signature(h);
  if ((long long)(uint32_t)p->iteration != s->step_dev_val) {
    k_step_set<<<1, 1, 0, s->stream>>>(s->step_dev, (uint32_t)p->iteration);
    CK(cudaGetLastError());
  }
  for (auto& g : s->graphs) {
    if (g.pkey != pkey || g.skey != skey) continue;
    CK(cudaGraphLaunch(g.exec, s->stream));
    // the host-side effects of the step: buffer parity, counts, spacing of the sort keys
    const int flips = 1 + (p->sort_now ? 1 : 0);
    for (int sp = 0; sp < 2; ++sp) s->sp[sp].cur ^= (flips & 1);
    s->counts_valid = true;
    s->sp_dx = p->dx;
    s->sp_dy = p->dy;
    if (p->erosion_on) s->erosion_seen = true;
    s->launches += g.launches;
    s->step_dev_val = (long long)(uint32_t)p->iteration + 1;
    ++s->graph_replays;
    *done = true;
    return PB_OK;
  }
  // capture: the step is enqueued into the graph, not run; the host state it advances is
  // kept only when the capture succeeds
  const int cur0 = s->sp[0].cur, cur1 = s->sp[1].cur;
  const bool cv0 = s->counts_valid;
  const double dx0 = s->sp_dx, dy0 = s->sp_dy;
  const bool es0 = s->erosion_seen;
  const long long l0 = s->launches;
  if (s->graphs.size() >= 8) free_graphs(s);
  cudaError_t ce = cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal);
  if (ce != cudaSuccess) {
    s->graphs_broken = 1;
    s->graph_error = std::string("cudaStreamBeginCapture: ") + cudaGetErrorString(ce);
    cudaGetLastError();
    return PB_OK;
  }
  s->capturing = 1;
  int32_t rc = enqueue_step(h, p);
  if (rc == PB_OK) {
    k_step_advance<<<1, 1, 0, s->stream>>>(s->step_dev);
    if (cudaGetLastError() != cudaSuccess) rc = PB_ERR_CUDA;
  }
  s->capturing = 0;
  cudaGraph_t graph = nullptr;
  ce = cudaStreamEndCapture(s->stream, &graph);
  cudaGraphExec_t exec = nullptr;
  if (rc == PB_OK && ce == cudaSuccess && graph) ce = cudaGraphInstantiate(&exec, graph, 0);
  if (graph) cudaGraphDestroy(graph);
  if (rc != PB_OK || ce != cudaSuccess || !exec) {
    // not capturable here: restore the host state and let the caller enqueue the step
    s->graphs_broken = 1;
    s->graph_error = rc != PB_OK ? g_err : std::string("step capture: ") + cudaGetErrorString(ce);
    cudaGetLastError();
    s->sp[0].cur = cur0; s->sp[1].cur = cur1;
    s->counts_valid = cv0; s->sp_dx = dx0; s->sp_dy = dy0; s->erosion_seen = es0; s->launches = l0;
    return PB_OK;
  }
  Sim::StepGraph g;
  g.pkey = pkey;
  g.skey = skey;
  g.exec = exec;
  g.launches = s->launches - l0 + 1;
  s->launches = l0 + g.launches;
  s->graphs.push_back(g);
  CK(cudaGraphLaunch(exec, s->stream));
  s->step_dev_val = (long long)(uint32_t)p->iteration + 1;
  ++s->graph_captures;
  *done = true;
  return PB_OK;
}

// one step of pb_sim_run / pb_sim_step: through a graph when enabled and possible
static int32_t run_one_step(pb_sim* h, const pb_step_params* p) {
  Sim* s = &h->s;
  if (graph_eligible(s, p)) {
    bool done = false;
    if (int32_t rc = graph_step(h, p, &done)) return rc;
    if (done) return PB_OK;
  }
  if (s->graphs_on) ++s->graph_plain_steps;
  return enqueue_step(h, p);
}

static int32_t finish_report(Sim* s, pb_step_report* out) {
  CK(cudaMemcpyAsync(s->rep_host, s->rep_dev, sizeof(pb_step_report), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  *out = *s->rep_host;
  s->host_num[0] = out->num_p;
  s->host_num[1] = out->num_e;
  return check_flags(s, out->errflags);
}

// ------------------------------------------------------------------ C-ABI
extern "C" {

int32_t pb_version(void) { return 10000; }
const char* pb_last_error(void) { return g_err.c_str(); }

int32_t pb_sim_create(pb_sim** out, int32_t device) {
  if (!out) return fail(PB_ERR_ARG, "null output");
  pb_sim* h = new pb_sim();
  Sim* s = &h->s;
  s->device = device;
  CK(cudaSetDevice(device));
  CK(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
  CK(cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, device));
  // field solve: one block of PT threads per SM (cooperative launch); the little shared
  // memory it uses leaves the rest of the SM's L1 to cache the grid
  CK(cudaFuncSetAttribute((const void*)k_poisson, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)mg_solve_smem_bytes(MG_MAX_COARSE, s->num_sms, 1)));
  CK(cudaFuncSetAttribute((const void*)k_poisson, cudaFuncAttributePreferredSharedMemoryCarveout,
                          (int)cudaSharedmemCarveoutMaxL1));
  s->pgrid = s->num_sms;
  CK(dalloc(&s->partials, 4 * 2 * (size_t)s->num_sms));
  CK(dalloc(&s->bar, 2));
  CK(dalloc(&s->pstats, 4));
  CK(dalloc(&s->solve_ns, 2));
  CK(cudaMemset(s->solve_ns, 0, 2 * sizeof(unsigned long long)));
  CK(dalloc(&s->ptrace, 32));
  CK(cudaMemset(s->ptrace, 0, 32 * sizeof(unsigned long long)));
  CK(cudaMemset(s->pstats, 0, 4 * sizeof(double)));
  CK(dalloc(&s->counts, 4));
  CK(cudaMemset(s->counts, 0, 4 * sizeof(int)));
  CK(dalloc(&s->next_ids, 2));
  CK(cudaMemset(s->next_ids, 0, 2 * sizeof(uint32_t)));
  CK(dalloc(&s->tile_counter, 2));
  CK(dalloc(&s->ds_bits, 3));
  CK(dalloc(&s->n_sub, 2));
  CK(dalloc(&s->inj, 7));
  CK(dalloc(&s->see_count, 1));
  CK(dalloc(&s->see_spawned, 1));
  CK(dalloc(&s->angle_count, 1));
  s->see_cap = 1 << 16;
  s->angle_cap = 1 << 16;
  CK(dalloc(&s->see_key, 2 * (size_t)s->see_cap));
  CK(dalloc(&s->see_xy, 2 * (size_t)s->see_cap));
  CK(dalloc(&s->angles, (size_t)s->angle_cap));
  CK(dalloc(&s->angle_scratch, 2 * (size_t)s->angle_cap));
  CK(dalloc(&s->rep_dev, 1));
  CK(cudaMemset(s->rep_dev, 0, sizeof(pb_step_report)));
  CK(dalloc(&s->step_dev, 1));
  CK(cudaMemset(s->step_dev, 0, sizeof(uint32_t)));
  CK(cudaMallocHost((void**)&s->rep_host, sizeof(pb_step_report)));
  s->sp[0].ion = true;
  s->sp[1].ion = false;
  CK(cudaEventCreate(&s->ev0));
  CK(cudaEventCreate(&s->ev1));
  int32_t rc;
  if ((rc = alloc_species(s, 0, 4096, 0)) || (rc = alloc_species(s, 1, 4096, 0))) return rc;
  *out = h;
  return PB_OK;
}

int32_t pb_sim_destroy(pb_sim* h) {
  if (!h) return PB_OK;
  Sim* s = &h->s;
  cudaSetDevice(s->device);
  cudaStreamSynchronize(s->stream);
  free_graphs(s);
  if (s->step_dev) cudaFree(s->step_dev);
  if (s->ekeep) cudaFree(s->ekeep);
  free_levels(s);
  double* d[] = {s->V, s->Vnew, s->Vfixed, s->Vdc, s->damage, s->eroded, s->accum_ppc, s->f, s->dirsum, s->partials, s->pstats};
  for (double* q : d) if (q) cudaFree(q);
  float* fl[] = {s->Ex, s->Ey, s->rho, s->Tmap, s->r32, s->z32, s->p32, s->q32, s->e32, s->s32, s->m32,
                 s->see_xy, s->angles};
  for (float* q : fl) if (q) cudaFree(q);
  if (s->ecorn) cudaFree(s->ecorn);
  void* v[] = {s->isBound, s->bdist, s->bdist_tmp, s->cls, s->gridmask, s->ppc, s->cnt_i, s->cnt_e, s->bar, s->counts, s->next_ids,
               s->tile_status, s->tile_counter, s->see_key, s->see_count, s->angle_scratch, s->angle_count,
               s->ds_bits, s->n_sub, s->inj, s->see_spawned, s->skey[0], s->skey[1], s->sval[0], s->sval[1],
               s->shist, s->sblk, s->rep_dev, h->cx.t, h->cx.c, h->see.t, h->see.c, s->solve_ns, s->nc_dev,
               s->mg_counts, s->mg_dirty, s->mg_status, s->ptrace};
  for (void* q : v) if (q) cudaFree(q);
  for (int k = 0; k < 2; ++k)
    for (int b = 0; b < 2; ++b) {
      Soa& o = s->sp[k].buf[b];
      dfree(o.x); dfree(o.y); dfree(o.vx); dfree(o.vy); dfree(o.vz); dfree(o.id); dfree(o.cex);
    }
  dfree(s->pw_lo); dfree(s->pw_left); dfree(s->pw_right); dfree(s->pw_hoff); dfree(s->pw_vals); dfree(s->pw_out);
  if (s->rep_host) cudaFreeHost(s->rep_host);
  if (s->rep_run) cudaFreeHost(s->rep_run);
  if (s->ev0) cudaEventDestroy(s->ev0);
  if (s->ev1) cudaEventDestroy(s->ev1);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete h;
  return PB_OK;
}

int32_t pb_sim_set_seed(pb_sim* h, uint64_t seed) { h->s.seed = seed; return PB_OK; }

int32_t pb_sim_set_solver(pb_sim* h, double tol, double tol_inner, int32_t max_outer, int32_t max_inner, int32_t nu,
                          int32_t max_coarse) {
  Sim* s = &h->s;
  if (!(tol > 0) || !(tol_inner > 0) || max_outer < 1 || max_inner < 1 || max_coarse < 4 || max_coarse > MG_MAX_COARSE)
    return fail(PB_ERR_ARG, "pb_sim_set_solver: invalid value");
  if (nu != 1 && nu != 2)
    return fail(PB_ERR_ARG, "pb_sim_set_solver: nu must be 1 or 2 (damped-Jacobi sweeps on the fine level on "
                            "each side of the coarse correction)");
  s->tol = tol; s->tol_inner = tol_inner; s->max_outer = max_outer; s->max_inner = max_inner; s->nu = nu;
  s->max_coarse = max_coarse;
  return PB_OK;
}

int32_t pb_sim_set_graphs(pb_sim* h, int32_t on) {
  Sim* s = &h->s;
  CK(cudaStreamSynchronize(s->stream));
  s->graphs_on = on ? 1 : 0;
  s->graphs_broken = 0;
  s->graph_error.clear();
  free_graphs(s);
  s->step_dev_val = -1;
  return PB_OK;
}

int32_t pb_sim_graph_stats(pb_sim* h, int64_t* out4) {
  const Sim* s = &h->s;
  out4[0] = s->graph_captures;
  out4[1] = s->graph_replays;
  out4[2] = s->graph_plain_steps;
  out4[3] = s->graphs_broken;
  if (s->graphs_broken) g_err = s->graph_error;
  return PB_OK;
}

int32_t pb_sim_set_tile(pb_sim* h, int32_t particles_per_block) {
  if (particles_per_block != TILE && particles_per_block != TILE_MIN)
    return fail(PB_ERR_ARG, "pb_sim_set_tile: particles per block must be " + std::to_string(TILE_MIN) + " or " +
                                std::to_string(TILE));
  h->s.ppb = particles_per_block;
  return PB_OK;
}

int32_t pb_sim_set_kernel_options(pb_sim* h, uint32_t flags) {
  if (flags & ~(uint32_t)(PB_OPT_SMEM_HIST | PB_OPT_TMA_TILE | PB_OPT_ELE_PAIRS | PB_OPT_ELE_SPLIT))
    return fail(PB_ERR_ARG, "pb_sim_set_kernel_options: unknown flag bits " + std::to_string(flags));
  h->s.kopts = flags;
  return PB_OK;
}

int32_t pb_sim_get_kernel_options(pb_sim* h, uint32_t* flags) {
  *flags = h->s.kopts;
  return PB_OK;
}

int32_t pb_sim_set_launch(pb_sim* h, int32_t particle_blocks_per_sm, int32_t solve_blocks) {
  Sim* s = &h->s;
  if (particle_blocks_per_sm < 1 || particle_blocks_per_sm > 32)
    return fail(PB_ERR_ARG, "pb_sim_set_launch: particle_blocks_per_sm must be 1 to 32");
  if (solve_blocks < 1 || solve_blocks > s->num_sms)
    return fail(PB_ERR_ARG, "pb_sim_set_launch: solve_blocks must be 1 to " + std::to_string(s->num_sms));
  s->pbps = particle_blocks_per_sm;
  s->pgrid = solve_blocks;
  return PB_OK;
}

int32_t pb_sim_set_spline(pb_sim* h, int32_t which, int32_t nt, const double* t, const double* c, double lo, double hi) {
  if (which != 0 && which != 1) return fail(PB_ERR_ARG, "spline: which must be 0 (CX) or 1 (SEE)");
  SplineStore& S = which == 0 ? h->cx : h->see;
  dfree(S.t);
  dfree(S.c);
  S.nt = 0;
  if (nt <= 0) return PB_OK;
  if (nt < 8) return fail(PB_ERR_ARG, "spline: a cubic spline needs at least 8 knots");
  CK(dalloc(&S.t, nt));
  CK(dalloc(&S.c, nt));
  CK(cudaMemcpy(S.t, t, nt * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(S.c, c, (nt - 4) * sizeof(double), cudaMemcpyHostToDevice));
  S.nt = nt; S.lo = lo; S.hi = hi;
  S.cmax = -INFINITY;
  for (int k = 0; k < nt - 4; ++k) {
    if (c[k] != c[k]) { S.cmax = NAN; break; }
    S.cmax = std::max(S.cmax, c[k]);
  }
  return PB_OK;
}

int32_t pb_sim_set_domain(pb_sim* h, int32_t ny, int32_t nx, int32_t periodic, const uint8_t* isBound,
                          const double* V_fixed, const uint16_t* gridmask, int32_t ngrids, const double* V,
                          const float* Tmap, const double* damage, const double* eroded, int32_t keep_state) {
  Sim* s = &h->s;
  if (ny < 3 || nx < 3 || !isBound || !V_fixed) return fail(PB_ERR_ARG, "pb_sim_set_domain: bad grid");
  CK(cudaSetDevice(s->device));
  CK(cudaStreamSynchronize(s->stream));
  size_t N = (size_t)ny * nx;
  bool realloc = (ny != s->ny || nx != s->nx);
  if (realloc) {
    if (keep_state && s->domain_set) return fail(PB_ERR_ARG, "pb_sim_set_domain: keep_state with a new grid size");
    double** dd[] = {&s->V, &s->Vnew, &s->Vfixed, &s->Vdc, &s->damage, &s->eroded, &s->accum_ppc, &s->f, &s->dirsum};
    for (double** q : dd) { dfree(*q); CK(dalloc(q, N)); CK(cudaMemset(*q, 0, N * sizeof(double))); }
    float** ff[] = {&s->Ex, &s->Ey, &s->rho, &s->Tmap, &s->r32, &s->z32, &s->p32, &s->q32, &s->e32, &s->s32,
                    &s->m32};
    for (float** q : ff) { dfree(*q); CK(dalloc(q, N)); CK(cudaMemset(*q, 0, N * sizeof(float))); }
    dfree(s->ecorn); CK(dalloc(&s->ecorn, 2 * N)); CK(cudaMemset(s->ecorn, 0, 2 * N * sizeof(float4)));
    dfree(s->isBound); CK(dalloc(&s->isBound, N));
    dfree(s->bdist); CK(dalloc(&s->bdist, N));
    dfree(s->bdist_tmp); CK(dalloc(&s->bdist_tmp, N));
    dfree(s->cls); CK(dalloc(&s->cls, N));
    dfree(s->gridmask); CK(dalloc(&s->gridmask, N));
    int** ii[] = {&s->ppc, &s->cnt_i, &s->cnt_e};
    for (int** q : ii) { dfree(*q); CK(dalloc(q, N)); CK(cudaMemset(*q, 0, N * sizeof(int))); }
    s->ny = ny; s->nx = nx;
  }
  s->periodic = periodic ? 1 : 0;
  s->ngrids = std::min<int>(ngrids, 16);
  CK(cudaMemcpy(s->isBound, isBound, N, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(s->Vfixed, V_fixed, N * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(s->Vdc, V_fixed, N * sizeof(double), cudaMemcpyHostToDevice));
  if (gridmask) CK(cudaMemcpy(s->gridmask, gridmask, N * sizeof(uint16_t), cudaMemcpyHostToDevice));
  else CK(cudaMemset(s->gridmask, 0, N * sizeof(uint16_t)));
  if (V) { CK(cudaMemcpy(s->V, V, N * sizeof(double), cudaMemcpyHostToDevice)); CK(cudaMemcpy(s->Vnew, V, N * sizeof(double), cudaMemcpyHostToDevice)); }
  if (Tmap) CK(cudaMemcpy(s->Tmap, Tmap, N * sizeof(float), cudaMemcpyHostToDevice));
  if (damage) CK(cudaMemcpy(s->damage, damage, N * sizeof(double), cudaMemcpyHostToDevice));
  if (eroded) CK(cudaMemcpy(s->eroded, eroded, N * sizeof(double), cudaMemcpyHostToDevice));
  if (!keep_state) {
    // reset_arrays (physics_engine.py:424-438): a fresh build starts from empty maps
    CK(cudaMemset(s->accum_ppc, 0, N * sizeof(double)));
    CK(cudaMemset(s->rho, 0, N * sizeof(float)));
    if (!damage) CK(cudaMemset(s->damage, 0, N * sizeof(double)));
    if (!eroded) CK(cudaMemset(s->eroded, 0, N * sizeof(double)));
    CK(cudaMemset(s->ppc, 0, N * sizeof(int)));
    CK(cudaMemset(s->Ex, 0, N * sizeof(float)));
    CK(cudaMemset(s->Ey, 0, N * sizeof(float)));
    if (!V) { CK(cudaMemset(s->V, 0, N * sizeof(double))); CK(cudaMemset(s->Vnew, 0, N * sizeof(double))); }
  }
  int32_t rc = build_operator(s, isBound);
  if (rc) return rc;
  CK(cudaStreamSynchronize(s->stream));
  s->domain_set = true;
  s->counts_valid = false;
  return PB_OK;
}

// After a run: a break whose freed nodes change the level structure was left to the host
// by k_mg_rebuild (MG_STATUS_HOST); rebuild the hierarchy here before the next solve.
static int32_t settle_mg(Sim* s) {
  if (!s->erosion_seen || !s->mg_status) return PB_OK;
  uint32_t st = 0;
  CK(cudaMemcpyAsync(&st, s->mg_status, sizeof(st), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  if (!(st & MG_STATUS_HOST)) return PB_OK;
  std::vector<uint8_t> ib((size_t)s->ny * s->nx);
  CK(cudaMemcpy(ib.data(), s->isBound, ib.size(), cudaMemcpyDeviceToHost));
  if (int32_t rc = build_operator(s, ib.data())) return rc;
  CK(cudaStreamSynchronize(s->stream));
  ++s->mg_host_rebuilds;
  return PB_OK;
}

int32_t pb_sim_rebuild_operator(pb_sim* h) {
  Sim* s = &h->s;
  if (!s->domain_set) return fail(PB_ERR_STATE, "pb_sim_rebuild_operator: no domain");
  std::vector<uint8_t> ib((size_t)s->ny * s->nx);
  CK(cudaStreamSynchronize(s->stream));
  CK(cudaMemcpy(ib.data(), s->isBound, ib.size(), cudaMemcpyDeviceToHost));
  int32_t rc = build_operator(s, ib.data());
  if (rc) return rc;
  CK(cudaStreamSynchronize(s->stream));
  return PB_OK;
}

int32_t pb_sim_reserve(pb_sim* h, int32_t species, int32_t capacity) {
  Sim* s = &h->s;
  if (species < 0 || species > 1 || capacity < 0) return fail(PB_ERR_ARG, "pb_sim_reserve");
  int32_t rc = read_counts(s);
  if (rc) return rc;
  return alloc_species(s, species, capacity, s->host_num[species]);
}

int32_t pb_sim_set_particles(pb_sim* h, int32_t species, int32_t n, const float* x, const float* y, const float* vx,
                             const float* vy, const float* vz, const uint8_t* cex, const uint32_t* id,
                             uint32_t next_id) {
  Sim* s = &h->s;
  if (species < 0 || species > 1 || n < 0) return fail(PB_ERR_ARG, "pb_sim_set_particles");
  int32_t rc;
  if ((rc = alloc_species(s, species, std::max(n + n / 4 + 4096, 4096), 0))) return rc;
  Species& S = s->sp[species];
  Soa& b = S.buf[S.cur];
  size_t n4 = (size_t)n * 4;
  if (n > 0) {
    CK(cudaMemcpy(b.x, x, n4, cudaMemcpyHostToDevice)); CK(cudaMemcpy(b.y, y, n4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(b.vx, vx, n4, cudaMemcpyHostToDevice)); CK(cudaMemcpy(b.vy, vy, n4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(b.vz, vz, n4, cudaMemcpyHostToDevice)); CK(cudaMemcpy(b.id, id, n4, cudaMemcpyHostToDevice));
    if (S.ion) {
      if (cex) CK(cudaMemcpy(b.cex, cex, n, cudaMemcpyHostToDevice));
      else CK(cudaMemset(b.cex, 0, n));
    }
  }
  CK(cudaMemcpy(s->counts + 2 * species + S.cur, &n, sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(s->next_ids + species, &next_id, sizeof(uint32_t), cudaMemcpyHostToDevice));
  s->host_num[species] = n;
  s->counts_valid = false;
  return PB_OK;
}

int32_t pb_sim_sort(pb_sim* h, int32_t species, double dx, double dy) {
  Sim* s = &h->s;
  if (!s->domain_set) return fail(PB_ERR_STATE, "pb_sim_sort: no domain");
  if (species < -1 || species > 1 || !(dx > 0.0) || !(dy > 0.0)) return fail(PB_ERR_ARG, "pb_sim_sort");
  s->sp_dx = dx;
  s->sp_dy = dy;
  const long N = (long)s->ny * s->nx;
  int bits = 1;
  while ((1L << bits) < N) ++bits;
  for (int k = 0; k < 2; ++k) {
    if (species >= 0 && k != species) continue;
    if (s->sp[k].cap <= 0) continue;
    int32_t rc = sort_species(s, k, bits);
    if (rc) return rc;
  }
  CK(cudaStreamSynchronize(s->stream));
  return PB_OK;
}

int32_t pb_sim_get_particles(pb_sim* h, int32_t species, int32_t n, float* x, float* y, float* vx, float* vy, float* vz,
                             uint8_t* cex, uint32_t* id) {
  Sim* s = &h->s;
  if (species < 0 || species > 1 || n < 0 || n > s->sp[species].cap) return fail(PB_ERR_ARG, "pb_sim_get_particles");
  CK(cudaStreamSynchronize(s->stream));
  Species& S = s->sp[species];
  const Soa& b = S.buf[S.cur];
  size_t n4 = (size_t)n * 4;
  if (n == 0) return PB_OK;
  if (x) CK(cudaMemcpy(x, b.x, n4, cudaMemcpyDeviceToHost));
  if (y) CK(cudaMemcpy(y, b.y, n4, cudaMemcpyDeviceToHost));
  if (vx) CK(cudaMemcpy(vx, b.vx, n4, cudaMemcpyDeviceToHost));
  if (vy) CK(cudaMemcpy(vy, b.vy, n4, cudaMemcpyDeviceToHost));
  if (vz) CK(cudaMemcpy(vz, b.vz, n4, cudaMemcpyDeviceToHost));
  if (id) CK(cudaMemcpy(id, b.id, n4, cudaMemcpyDeviceToHost));
  if (cex && S.ion) CK(cudaMemcpy(cex, b.cex, n, cudaMemcpyDeviceToHost));
  return PB_OK;
}

int32_t pb_sim_counts(pb_sim* h, int32_t* num_p, int32_t* num_e, uint32_t* next_ion_id, uint32_t* next_e_id) {
  Sim* s = &h->s;
  int32_t rc = read_counts(s);
  if (rc) return rc;
  uint32_t ids[2];
  CK(cudaMemcpy(ids, s->next_ids, sizeof(ids), cudaMemcpyDeviceToHost));
  if (num_p) *num_p = s->host_num[0];
  if (num_e) *num_e = s->host_num[1];
  if (next_ion_id) *next_ion_id = ids[0];
  if (next_e_id) *next_e_id = ids[1];
  return PB_OK;
}

static void* field_of(Sim* s, int which, size_t* esize) {
  switch (which) {
    case 0: *esize = 8; return s->V;
    case 1: *esize = 4; return s->Ex;
    case 2: *esize = 4; return s->Ey;
    case 3: *esize = 4; return s->rho;
    case 4: *esize = 4; return s->Tmap;
    case 5: *esize = 8; return s->damage;
    case 6: *esize = 1; return s->isBound;
    case 7: *esize = 8; return s->Vfixed;
    case 8: *esize = 4; return s->ppc;
    case 9: *esize = 8; return s->accum_ppc;
    case 10: *esize = 8; return s->eroded;
    case 11: *esize = 8; return s->Vnew;
    case 12: *esize = 1; return s->cls;
    case 13: *esize = 4; return s->lev.empty() ? nullptr : s->lev[0].dinv;
    default: *esize = 0; return nullptr;
  }
}

int32_t pb_sim_field_ptr(pb_sim* h, int32_t which, void** dptr) {
  size_t es;
  void* p = field_of(&h->s, which, &es);
  if (!p) return fail(PB_ERR_ARG, "pb_sim_field_ptr: unknown field");
  *dptr = p;
  return PB_OK;
}

int32_t pb_sim_get_field(pb_sim* h, int32_t which, void* host, int64_t nbytes) {
  Sim* s = &h->s;
  size_t es;
  void* p = field_of(s, which, &es);
  if (!p || (size_t)nbytes != es * (size_t)s->ny * s->nx) return fail(PB_ERR_ARG, "pb_sim_get_field: size");
  CK(cudaStreamSynchronize(s->stream));
  CK(cudaMemcpy(host, p, nbytes, cudaMemcpyDeviceToHost));
  return PB_OK;
}

int32_t pb_sim_set_field(pb_sim* h, int32_t which, const void* host, int64_t nbytes) {
  Sim* s = &h->s;
  size_t es;
  void* p = field_of(s, which, &es);
  if (!p || (size_t)nbytes != es * (size_t)s->ny * s->nx) return fail(PB_ERR_ARG, "pb_sim_set_field: size");
  if (which == 13) return fail(PB_ERR_ARG, "pb_sim_set_field: the smoother weights are read-only");
  CK(cudaStreamSynchronize(s->stream));
  CK(cudaMemcpy(p, host, nbytes, cudaMemcpyHostToDevice));
  if (which == 7) CK(cudaMemcpy(s->Vdc, host, nbytes, cudaMemcpyHostToDevice));
  if (which == 6) {
    if (int32_t rc = update_bound_dist(s)) return rc;
    CK(cudaStreamSynchronize(s->stream));
  }
  return PB_OK;
}

int32_t pb_sim_particle_ptr(pb_sim* h, int32_t species, int32_t which, void** dptr) {
  Sim* s = &h->s;
  if (species < 0 || species > 1) return fail(PB_ERR_ARG, "species");
  const Soa& b = s->sp[species].buf[s->sp[species].cur];
  void* p[] = {b.x, b.y, b.vx, b.vy, b.vz, b.cex, b.id};
  if (which < 0 || which > 6 || !p[which]) return fail(PB_ERR_ARG, "which");
  *dptr = p[which];
  return PB_OK;
}

int32_t pb_sim_poisson(pb_sim* h, int32_t iterations, const pb_step_params* p, double* stats4_host) {
  Sim* s = &h->s;
  if (!s->domain_set) return fail(PB_ERR_STATE, "pb_sim_poisson: no domain");
  CK(cudaMemsetAsync(&s->rep_dev->errflags, 0, sizeof(uint32_t), s->stream));
  int32_t rc = launch_poisson(s, iterations, p);
  if (rc) return rc;
  uint32_t f = 0;
  CK(cudaMemcpyAsync(&f, &s->rep_dev->errflags, sizeof(f), cudaMemcpyDeviceToHost, s->stream));
  if (stats4_host) CK(cudaMemcpyAsync(stats4_host, s->pstats, 4 * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return check_flags(s, f);
}

int32_t pb_sim_step(pb_sim* h, const pb_step_params* p, pb_step_report* report) {
  Sim* s = &h->s;
  if (!s->domain_set) return fail(PB_ERR_STATE, "pb_sim_step: no domain");
  int32_t rc;
  if ((rc = ensure_room(s, p, 1))) return rc;
  s->mark_used = 0;
  s->launches = 0;
  CK(cudaEventRecord(s->ev0, s->stream));
  if ((rc = run_one_step(h, p))) return rc;
  CK(cudaEventRecord(s->ev1, s->stream));
  if (report) {
    if ((rc = finish_report(s, report))) return rc;
    float ms = 0.0f;
    CK(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
    s->last_ms = ms;
    if ((rc = settle_mg(s))) return rc;
  }
  return PB_OK;
}

int32_t pb_sim_run(pb_sim* h, const pb_step_params* params, int32_t nsteps, pb_step_report* reports) {
  Sim* s = &h->s;
  if (!s->domain_set) return fail(PB_ERR_STATE, "pb_sim_run: no domain");
  int32_t rc;
  if (nsteps <= 0) return PB_OK;
  for (int k = 0; k < nsteps; ++k)
    if ((rc = check_step_params(s, &params[k]))) return rc;
  if ((rc = ensure_room(s, &params[0], nsteps))) return rc;
  // reports go to pinned memory, so the copies do not block the host between steps
  if (reports && s->rep_run_cap < nsteps) {
    if (s->rep_run) CK(cudaFreeHost(s->rep_run));
    s->rep_run = nullptr;
    s->rep_run_cap = 0;
    CK(cudaMallocHost((void**)&s->rep_run, (size_t)nsteps * sizeof(pb_step_report)));
    s->rep_run_cap = nsteps;
  }
  s->mark_used = 0;
  s->launches = 0;
  CK(cudaEventRecord(s->ev0, s->stream));
  for (int k = 0; k < nsteps; ++k) {
    if ((rc = run_one_step(h, &params[k]))) return rc;
    if (reports) {
      CK(cudaMemcpyAsync(&s->rep_run[k], s->rep_dev, sizeof(pb_step_report), cudaMemcpyDeviceToHost, s->stream));
    }
  }
  CK(cudaEventRecord(s->ev1, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  float ms = 0.0f;
  CK(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
  s->last_ms = ms;
  if ((rc = read_counts(s))) return rc;
  if ((rc = settle_mg(s))) return rc;
  if (reports) {
    std::memcpy(reports, s->rep_run, (size_t)nsteps * sizeof(pb_step_report));
    for (int k = 0; k < nsteps; ++k)
      if ((rc = check_flags(s, reports[k].errflags))) return rc;
  }
  return PB_OK;
}

int32_t pb_sim_synchronize(pb_sim* h) {
  CK(cudaStreamSynchronize(h->s.stream));
  return PB_OK;
}

void* pb_sim_stream(pb_sim* h) { return (void*)h->s.stream; }

// NumPy's pairwise summation tree for n elements (see k_pw_leaves): leaves of at most 128
// elements in array order, internal nodes numbered after the leaves by height.
static void pw_build(Sim::PwTree& t, long long n) {
  t.n = n;
  t.leaf_lo.clear();
  t.left.clear();
  t.right.clear();
  t.height_off.assign(1, 0);
  t.root = -1;
  if (n <= 0) { t.leaf_lo.push_back(0); return; }
  struct Node { int l, r, h; };  // children: >= 0 a leaf, < 0 internal node -(k + 1)
  std::vector<Node> in;
  std::function<std::pair<int, int>(long long, long long)> rec = [&](long long lo, long long len) {
    if (len <= 128) {
      t.leaf_lo.push_back(lo);
      return std::make_pair((int)t.leaf_lo.size() - 1, 0);
    }
    long long m = len / 2;
    m -= m % 8;
    const std::pair<int, int> a = rec(lo, m), b = rec(lo + m, len - m);
    const int h = std::max(a.second, b.second) + 1;
    in.push_back({a.first, b.first, h});
    return std::make_pair(-(int)in.size(), h);
  };
  const std::pair<int, int> top = rec(0, n);
  const int L = (int)t.leaf_lo.size();
  t.leaf_lo.push_back(n);
  const int H = top.second;
  t.height_off.assign(H + 1, 0);
  for (const Node& x : in) ++t.height_off[x.h];  // count per height, shifted by one
  for (int h = 1; h <= H; ++h) t.height_off[h] += t.height_off[h - 1];
  std::vector<int> pos(in.size()), fill(t.height_off.begin(), t.height_off.end() - 1);
  for (size_t k = 0; k < in.size(); ++k) pos[k] = fill[in[k].h - 1]++;
  auto id = [&](int c) { return c >= 0 ? c : L + pos[-c - 1]; };
  t.left.assign(in.size(), 0);
  t.right.assign(in.size(), 0);
  for (size_t k = 0; k < in.size(); ++k) {
    t.left[pos[k]] = id(in[k].l);
    t.right[pos[k]] = id(in[k].r);
  }
  t.root = id(top.first);
}

// np.sum of one float32 source on the device, NumPy's rounding; result in *out_dev
static int32_t pw_sum(Sim* s, int which, long long n, PwSrc src, float* out_dev) {
  Sim::PwTree& t = s->pw[which];
  if (t.n != n) pw_build(t, n);
  const size_t L = t.leaf_lo.size() - 1, I = t.left.size(), H = t.height_off.size();
  if (L + 1 > s->pw_cap_leaves) {
    dfree(s->pw_lo);
    CK(dalloc(&s->pw_lo, L + 1));
    s->pw_cap_leaves = L + 1;
  }
  if (L + I + 1 > s->pw_cap_nodes) {
    dfree(s->pw_vals); dfree(s->pw_left); dfree(s->pw_right);
    CK(dalloc(&s->pw_vals, L + I + 1)); CK(dalloc(&s->pw_left, L + I + 1)); CK(dalloc(&s->pw_right, L + I + 1));
    s->pw_cap_nodes = L + I + 1;
  }
  if (H > s->pw_cap_h) {
    dfree(s->pw_hoff);
    CK(dalloc(&s->pw_hoff, H));
    s->pw_cap_h = H;
  }
  cudaStream_t st = s->stream;
  CK(cudaMemcpyAsync(s->pw_lo, t.leaf_lo.data(), (L + 1) * sizeof(long long), cudaMemcpyHostToDevice, st));
  if (I) {
    CK(cudaMemcpyAsync(s->pw_left, t.left.data(), I * sizeof(int), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(s->pw_right, t.right.data(), I * sizeof(int), cudaMemcpyHostToDevice, st));
  }
  CK(cudaMemcpyAsync(s->pw_hoff, t.height_off.data(), H * sizeof(int), cudaMemcpyHostToDevice, st));
  if (L) k_pw_leaves<<<grid_for(s, (long)L, 128), 128, 0, st>>>(src, s->pw_lo, (int)L, s->pw_vals);
  k_pw_combine<<<1, 1024, 0, st>>>(s->pw_vals, s->pw_left, s->pw_right, s->pw_hoff, (int)H - 1, (int)L, t.root,
                                   out_dev);
  CK(cudaGetLastError());
  return PB_OK;
}

int32_t pb_sim_energy_sums(pb_sim* h, double* out3) {
  Sim* s = &h->s;
  if (!out3) return fail(PB_ERR_ARG, "pb_sim_energy_sums: null output");
  CK(cudaSetDevice(s->device));
  int32_t rc;
  if ((rc = read_counts(s))) return rc;
  if (!s->pw_out) CK(dalloc(&s->pw_out, 3));
  const Soa& I = s->sp[0].buf[s->sp[0].cur];
  const Soa& E = s->sp[1].buf[s->sp[1].cur];
  const PwSrc src[3] = {{I.vx, I.vy, I.vz}, {E.vx, E.vy, E.vz}, {s->Ex, s->Ey, nullptr}};
  const long long n[3] = {s->host_num[0], s->host_num[1], s->domain_set ? (long long)s->ny * s->nx : 0};
  for (int k = 0; k < 3; ++k)
    if ((rc = pw_sum(s, k, n[k], src[k], s->pw_out + k))) return rc;
  float f[3];
  CK(cudaMemcpyAsync(f, s->pw_out, sizeof(f), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  for (int k = 0; k < 3; ++k) out3[k] = (double)f[k];
  return PB_OK;
}

// summed fine phase times of the profiled steps (PB_MARKS - 1 of them) and the step count
static int32_t phase_sums(Sim* s, double* ph, double* steps_out) {
  for (int k = 0; k < PB_MARKS - 1; ++k) ph[k] = 0.0;
  *steps_out = 0.0;
  if (!s->profiling || s->mark_used < (size_t)PB_MARKS) return PB_OK;
  CK(cudaStreamSynchronize(s->stream));
  size_t steps = s->mark_used / PB_MARKS;
  for (size_t t = 0; t < steps; ++t)
    for (int k = 0; k < PB_MARKS - 1; ++k) {
      float ms = 0.0f;
      CK(cudaEventElapsedTime(&ms, s->marks[t * PB_MARKS + k], s->marks[t * PB_MARKS + k + 1]));
      ph[k] += ms;
    }
  *steps_out = (double)steps;
  return PB_OK;
}

int32_t pb_sim_timing(pb_sim* h, double* out) {
  Sim* s = &h->s;
  for (int k = 0; k < 9; ++k) out[k] = 0.0;
  out[0] = s->last_ms;
  out[8] = (double)s->launches;
  double ph[PB_MARKS - 1], steps = 0.0;
  if (int32_t rc = phase_sums(s, ph, &steps)) return rc;
  if (steps > 0.0) {
    out[1] = ph[0]; out[2] = ph[1]; out[3] = ph[2]; out[4] = ph[3];
    out[5] = ph[4] + ph[5] + ph[6];
    out[6] = ph[7] + ph[8];
    out[7] = steps;
  }
  return PB_OK;
}

int32_t pb_sim_phase_times(pb_sim* h, double* out10) {
  Sim* s = &h->s;
  double steps = 0.0;
  if (int32_t rc = phase_sums(s, out10, &steps)) return rc;
  out10[PB_MARKS - 1] = steps;
  return PB_OK;
}

int32_t pb_sim_batch_share(pb_sim* h, double* out2) {
  if (!out2) return fail(PB_ERR_ARG, "pb_sim_batch_share: null output");
  out2[0] = h->s.solve_work * 1e-6;
  out2[1] = h->s.batch_blocks;
  return PB_OK;
}

int32_t pb_sim_mg_stats(pb_sim* h, int64_t* out8) {
  Sim* s = &h->s;
  int64_t* out4 = out8;
  if (!out8) return fail(PB_ERR_ARG, "pb_sim_mg_stats: null output");
  if (!s->domain_set) return fail(PB_ERR_STATE, "pb_sim_mg_stats: no domain");
  int c[MG_CNT_SLOTS];
  int nc = 0;
  CK(cudaStreamSynchronize(s->stream));
  CK(cudaMemcpy(c, s->mg_counts, sizeof(c), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(&nc, s->nc_dev, sizeof(int), cudaMemcpyDeviceToHost));
  out4[0] = c[MG_CNT_REBUILDS];
  out4[1] = c[MG_CNT_DEFERRED];
  out4[2] = s->mg_host_rebuilds;
  out4[3] = nc;
  out8[4] = c[MG_CNT_US_LEVELS];
  out8[5] = c[MG_CNT_US_CHOLESKY];
  out8[6] = c[MG_CNT_US_INVERSE];
  out8[7] = c[MG_CNT_US_TRANSFER];
  return PB_OK;
}

// FNV-1a over the bytes the field solve reads of the hierarchy: per level the smoother
// weights and the transfer stencils, then the coarsest count, index set and inverse.
int32_t pb_sim_operator_digest(pb_sim* h, uint64_t* out) {
  Sim* s = &h->s;
  if (!out) return fail(PB_ERR_ARG, "pb_sim_operator_digest: null output");
  if (!s->domain_set) return fail(PB_ERR_STATE, "pb_sim_operator_digest: no domain");
  CK(cudaStreamSynchronize(s->stream));
  uint64_t k = 1469598103934665603ull;
  std::vector<float> buf;
  auto add_dev = [&](const float* p, size_t n) -> cudaError_t {
    buf.resize(n);
    cudaError_t e = cudaMemcpy(buf.data(), p, n * sizeof(float), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) k = fnv(k, buf.data(), n * sizeof(float));
    return e;
  };
  const int L = (int)s->lev.size();
  k = fnv_v(k, L);
  for (int l = 0; l < L; ++l) {
    const DevLevel& D = s->lev[l];
    const size_t N = (size_t)D.ny * D.nx;
    CK(add_dev(D.dinv, N));
    if (D.R) CK(add_dev(D.R, 25 * N));
    if (D.U) CK(add_dev(D.U, 18 * N));
  }
  int nc = 0;
  CK(cudaMemcpy(&nc, s->nc_dev, sizeof(int), cudaMemcpyDeviceToHost));
  k = fnv_v(k, nc);
  std::vector<int> ci((size_t)std::max(nc, 1));
  CK(cudaMemcpy(ci.data(), s->cidx, (size_t)nc * sizeof(int), cudaMemcpyDeviceToHost));
  k = fnv(k, ci.data(), (size_t)nc * sizeof(int));
  CK(add_dev(s->cinv, (size_t)nc * nc));
  *out = k;
  return PB_OK;
}

int32_t pb_sim_poisson_trace(pb_sim* h, int32_t on, double* out32) {
  Sim* s = &h->s;
  if (out32) {
    unsigned long long t[32];
    CK(cudaStreamSynchronize(s->stream));
    CK(cudaMemcpy(t, s->ptrace, sizeof(t), cudaMemcpyDeviceToHost));
    for (int k = 0; k < 32; ++k) out32[k] = (double)t[k];
  }
  CK(cudaMemset(s->ptrace, 0, 32 * sizeof(unsigned long long)));
  s->trace_on = on ? 1 : 0;
  return PB_OK;
}

int32_t pb_sim_set_profiling(pb_sim* h, int32_t on) {
  h->s.profiling = on ? 1 : 0;
  h->s.mark_used = 0;
  return PB_OK;
}

// ------------------------------------------------------------------ kernel-level entry points
int32_t pb_check_division(double d, int64_t* out3) {
  if (!out3) return fail(PB_ERR_ARG, "pb_check_division: null output");
  unsigned long long* dev = nullptr;
  CK(cudaMalloc((void**)&dev, 3 * sizeof(unsigned long long)));
  unsigned long long h[3] = {0, 0, 0};
  cudaError_t e = cudaMemset(dev, 0, sizeof(h));
  int sms = 148, dv = 0;
  if (e == cudaSuccess) e = cudaGetDevice(&dv);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dv);
  if (e == cudaSuccess) {
    k_div_check<<<sms * 8, 256>>>((float)d, dev);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(h, dev, sizeof(h), cudaMemcpyDeviceToHost);
  cudaFree(dev);
  CK(e);
  for (int k = 0; k < 3; ++k) out3[k] = (int64_t)h[k];
  return PB_OK;
}

int32_t pb_push_particles_boris(float* x, float* y, float* vx, float* vy, float* vz, const float* Ex, const float* Ey,
                                const float* Bx, const float* By, const float* Bz, int32_t num_p, double dx, double dy,
                                int32_t nx, int32_t ny, double dt, double q_m, void* stream) {
  if (num_p <= 0) return PB_OK;
  if (nx < 2 || ny < 2) return fail(PB_ERR_ARG, "push: grid must be at least 2 x 2");
  double h = (0.5 * q_m) * dt;
  int bs = 256;
  int g = (int)std::min<long>((num_p + bs - 1) / bs, 148L * 16);
  k_push_boris<<<g, bs, 0, (cudaStream_t)stream>>>(x, y, vx, vy, vz, Ex, Ey, Bx, By, Bz, num_p, nx, ny, (float)dx,
                                                   (float)dy, h, (float)dt);
  CK(cudaGetLastError());
  return PB_OK;
}

int32_t pb_accumulate_rho(const float* x, const float* y, float* rho, int32_t num_p, double dx, double dy, int32_t nx,
                          int32_t ny, double charge_density, void* stream) {
  if (nx < 3 || ny < 3) return fail(PB_ERR_ARG, "accumulate_rho: grid must be at least 3 x 3");
  const long long G64 = (long long)nx * ny;
  if (G64 > INT32_MAX) return fail(PB_ERR_ARG, "accumulate_rho: grid of " + std::to_string(G64) +
                                                   " cells exceeds 2^31 - 1");
  if (num_p <= 0) return PB_OK;
  cudaStream_t st = (cudaStream_t)stream;
  const int G = (int)G64;
  int* cnt = nullptr;
  CK(cudaMallocAsync((void**)&cnt, (size_t)G * sizeof(int), st));
  CK(cudaMemsetAsync(cnt, 0, (size_t)G * sizeof(int), st));
  int g = (int)std::min<long>((num_p + 255) / 256, 148L * 16);
  k_count_cells<<<g, 256, 0, st>>>(x, y, nullptr, num_p, 0, cnt, nx, ny, (float)dx, (float)dy);
  k_rho_finalize<<<(int)std::min<long>((G + 255) / 256, 148L * 16), 256, 0, st>>>(rho, cnt, nullptr, G,
                                                                                  charge_density, 1);
  CK(cudaFreeAsync(cnt, st));
  CK(cudaGetLastError());
  return PB_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ allocation-free deposit
// Some callers cannot allocate device memory at the point where they deposit charge: a
// host application whose memory is already reserved by another framework's pool, a
// real-time loop that must not take the driver's allocation path (it can block and
// synchronise), or an embedded process whose device memory budget is fixed at start-up.
// pb_accumulate_rho_noalloc serves them with its per-cell count scratch in this
// file-scope device array instead of a temporary allocation.  Every GPU that loads the
// library holds the array (PB_NOALLOC_MAX_CELLS int32 = 8 MiB) until the process exits.
#define PB_NOALLOC_MAX_CELLS (1 << 21)
static __device__ __align__(256) int g_noalloc_counts[PB_NOALLOC_MAX_CELLS];

// Device address of the scratch array in the context current on the calling thread.  In
// host code the array's name is only a host-side stand-in, so the address is looked up on
// every call: that is cheap once the module is loaded, and it stays right after
// cudaDeviceReset or under a context other than the device's primary one (a cached
// address would belong to the context it was taken in).  The first call in a context
// loads the module.
static int32_t noalloc_scratch(int** out) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_counts);
  if (e != cudaSuccess || !p)
    return fail(PB_ERR_CUDA, std::string("accumulate_rho_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
  *out = (int*)p;
  return PB_OK;
}

extern "C" {

int32_t pb_accumulate_rho_noalloc(const float* x, const float* y, float* rho, int32_t num_p, double dx, double dy,
                                  int32_t nx, int32_t ny, double charge_density, void* stream) {
  if (nx < 3 || ny < 3) return fail(PB_ERR_ARG, "accumulate_rho_noalloc: grid must be at least 3 x 3");
  long long G = (long long)nx * ny;
  if (G > PB_NOALLOC_MAX_CELLS)
    return fail(PB_ERR_ARG, "accumulate_rho_noalloc: grid of " + std::to_string(G) + " cells exceeds the " +
                                std::to_string(PB_NOALLOC_MAX_CELLS) + "-cell scratch; use pb_accumulate_rho");
  int* cnt = nullptr;
  int32_t rc = noalloc_scratch(&cnt);
  if (rc) return rc;
  if (num_p <= 0) return PB_OK;
  cudaStream_t st = (cudaStream_t)stream;
  // k_rho_finalize zeroes every count it reads, so after a call has completed the cells it
  // used are zero again.  This clear guards against a call that was cut off between its
  // two kernels (an error or a cancelled stream), which would leave counts behind.
  CK(cudaMemsetAsync(cnt, 0, (size_t)G * sizeof(int), st));
  int g = (int)std::min<long>((num_p + 255) / 256, 148L * 16);
  k_count_cells<<<g, 256, 0, st>>>(x, y, nullptr, num_p, 0, cnt, nx, ny, (float)dx, (float)dy);
  k_rho_finalize<<<(int)std::min<long>((G + 255) / 256, 148L * 16), 256, 0, st>>>(rho, cnt, nullptr, (int)G,
                                                                                  charge_density, 1);
  CK(cudaGetLastError());
  return PB_OK;
}

int32_t pb_thermal_conduction(const float* T, float* T_new, const int32_t* mask, int32_t nx, int32_t ny, double Fo_x,
                              double Fo_y, void* stream) {
  if (nx < 1 || ny < 1) return fail(PB_ERR_ARG, "thermal_conduction: empty grid");
  int G = nx * ny;
  k_thermal_taichi<<<(int)std::min<long>((G + 255) / 256, 148L * 16), 256, 0, (cudaStream_t)stream>>>(
      T, T_new, mask, nx, ny, (float)Fo_x, (float)Fo_y);
  CK(cudaGetLastError());
  return PB_OK;
}

int32_t pb_compute_particle_substeps(const float* x, const float* y, const float* vx, const float* vy, const float* vz,
                                     int32_t n, const float* Ex, const float* Ey, int32_t nx, int32_t ny, double dx,
                                     double dy, double qm, double dt, double frac, double* out_host, void* stream) {
  double ds_lim = frac * std::min(dx, dy) * 1e-3;
  if (n <= 0) { out_host[0] = 1; out_host[1] = 0.0; out_host[2] = ds_lim; return PB_OK; }
  if (nx < 2 || ny < 2) return fail(PB_ERR_ARG, "compute_particle_substeps: grid must be at least 2 x 2");
  cudaStream_t st = (cudaStream_t)stream;
  // the step's path: the corner array with the field bound, so that particles which cannot
  // raise the maximum are passed over (arrays 16-byte aligned; others take the full loop)
  const long long G = (long long)nx * ny;
  unsigned long long* bits = nullptr;
  float4* ec = nullptr;
  CK(cudaMallocAsync((void**)&bits, 2 * sizeof(unsigned long long), st));
  CK(cudaMemsetAsync(bits, 0, 2 * sizeof(unsigned long long), st));
  CK(cudaMallocAsync((void**)&ec, (size_t)G * 2 * sizeof(float4), st));
  unsigned* ebound = reinterpret_cast<unsigned*>(bits + 1);
  const int gc = (int)std::min<long long>((G + 255) / 256, 148LL * 8);
  k_e_corners<<<gc, 256, 0, st>>>(Ex, Ey, ec, ny, nx, ebound);
  int g = (int)std::min<long>((n + 255) / 256, 148L * 16);
  k_substep_reduce<<<g, 256, 0, st>>>(x, y, vx, vy, vz, nullptr, n, Ex, Ey, ec, nx, ny, (float)dx, (float)dy, qm,
                                      (float)dt, dt * dt, bits, ebound);
  unsigned long long hb = 0;
  CK(cudaMemcpyAsync(&hb, bits, sizeof(hb), cudaMemcpyDeviceToHost, st));
  CK(cudaFreeAsync(ec, st));
  CK(cudaFreeAsync(bits, st));
  CK(cudaStreamSynchronize(st));
  double ds_max;
  std::memcpy(&ds_max, &hb, sizeof(double));
  double q = std::ceil(ds_max / std::max(ds_lim, 1e-30));
  out_host[0] = std::max(1.0, q);
  out_host[1] = ds_max;
  out_host[2] = ds_lim;
  return PB_OK;
}

int32_t pb_segment_hits_grid(const uint8_t* isBound, int32_t nx, int32_t ny, double dx, double dy, const float* x0,
                             const float* y0, const float* x1, const float* y1, int32_t n, uint8_t* hit,
                             int64_t* hit_ix, int64_t* hit_iy, void* stream) {
  if (n <= 0) return PB_OK;
  int g = (int)std::min<long>((n + 255) / 256, 148L * 16);
  k_segment_hits<<<g, 256, 0, (cudaStream_t)stream>>>(isBound, nx, ny, (float)dx, (float)dy, x0, y0, x1, y1, n, hit,
                                                       hit_ix, hit_iy);
  CK(cudaGetLastError());
  return PB_OK;
}

// ------------------------------------------------------------------ host helpers
float pb_host_seq_add_f32d(float s, double c, uint32_t n) { return seq_add_f32d(s, c, n); }
double pb_host_philox_uniform(uint64_t seed, uint64_t pid, uint32_t site, uint32_t step, uint32_t j) {
  return philox_uniform(seed, pid, site, step, j);
}
double pb_host_philox_normal(uint64_t seed, uint64_t pid, uint32_t site, uint32_t step, uint32_t j) {
  return philox_normal(seed, pid, site, step, j);
}
float pb_host_percentile95(const float* sorted, int32_t n) {
  if (n <= 0) return NAN;
  return percentile95_sorted(sorted, n);
}

}  // extern "C"

#include "pb_batch.cu"
