/*
 * pbemcs.h — C-ABI of the B200 PIC-MCC step library (libpbemcs.so).
 *
 * The entry points replace the numeric kernels and the per-timestep loop of the
 * PY-BEMCS reference, Python/physics_engine.py (cited as file:line below).  A Python
 * host binds them with ctypes (thruster_cx_code_b200/_lib.py); the signatures use plain
 * pointers, sizes and scalars only.
 *
 * Conventions
 *   - Every function returns 0 (PB_OK) or a PB_ERR_* code; pb_last_error() gives text.
 *   - Array arguments of the kernel-level functions are DEVICE pointers (any CUDA
 *     allocation, e.g. a torch tensor's data_ptr()); `stream` is a cudaStream_t or NULL.
 *   - Fields are row-major (ny, nx) with x fastest, as NumPy's [iy, ix]; particles are
 *     1-D structure-of-arrays.  Positions are in mm, velocities in m/s.
 *   - Host helpers (pb_host_*) run on the CPU and need no GPU.
 */
#ifndef PBEMCS_H
#define PBEMCS_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  PB_OK = 0,
  PB_ERR_CUDA = 1,        /* a CUDA call failed (message in pb_last_error) */
  PB_ERR_ARG = 2,         /* invalid argument */
  PB_ERR_CAPACITY = 3,    /* particle storage or a per-step list would overflow */
  PB_ERR_TIMEOUT = 4,     /* a bounded device-side wait gave up */
  PB_ERR_NOCONV = 5,      /* the field solve did not reach its tolerance */
  PB_ERR_STATE = 6        /* call out of order (e.g. step before a domain is set) */
};

/* error flags reported by the device in pb_step_report.errflags */
enum {
  PB_EF_CAPACITY_ION = 1 << 0, PB_EF_CAPACITY_ELE = 1 << 1, PB_EF_SEE_OVERFLOW = 1 << 2,
  PB_EF_ANGLE_OVERFLOW = 1 << 3, PB_EF_SPIN_TIMEOUT = 1 << 4, PB_EF_NAN_SUBSTEP = 1 << 5,
  PB_EF_SUBSTEP_CAP = 1 << 6, PB_EF_POISSON_NOCONV = 1 << 7, PB_EF_ID_OVERFLOW = 1 << 8
};

int32_t pb_version(void);
const char* pb_last_error(void);

/* ---------------------------------------------------------------- kernel level */

/* NGP charge deposition: rho[iy, ix] += charge_density for every particle, with
 * ix = clip(rint(x/dx), 1, nx-2), iy likewise; bit-identical to the sequential float32
 * np.add.at of accumulate_rho_cpu (physics_engine.py:178-185; Taichi form :38-60).
 * Uses a temporary count array from the stream-ordered allocator. */
int32_t pb_accumulate_rho(const float* x, const float* y, float* rho, int32_t num_p, double dx, double dy,
                          int32_t nx, int32_t ny, double charge_density, void* stream);

/* The deposit of pb_accumulate_rho without any device allocation, for callers that
 * cannot allocate (memory already reserved by another framework's pool, real-time loops
 * that must stay off the driver's allocation path, fixed device-memory budgets).  It has
 * no counterpart in the reference.  The per-cell count scratch is a file-scope device
 * array of 2^21 int32 (8 MiB) that every GPU loading the library holds until exit;
 * grids of more than 2^21 cells are rejected with PB_ERR_ARG.  Each call looks up the
 * array's device address in the current context (cudaGetSymbolAddress); the first call in
 * a context loads the module and should come before any stream capture.  All calls share
 * the array, so calls that overlap on the GPU race.  A completed call leaves the cells it
 * used at zero (the rho pass clears every count it reads); each call still clears them
 * first, in case an earlier call was cut off between its count and rho passes. */
int32_t pb_accumulate_rho_noalloc(const float* x, const float* y, float* rho, int32_t num_p, double dx, double dy,
                                  int32_t nx, int32_t ny, double charge_density, void* stream);

/* Exhaustive check of the division the step kernels use for x / dx and y / dy (no
 * counterpart in the reference; a test of this library).  For the float32 spacing d, every
 * one of the 2^32 float32 values x is divided by bracketing (x * RN(1/d), its FMA residual
 * and two FMA corrections with the neighbours of RN(1/d); accepted when both corrections
 * round alike) and compared with the IEEE float32 division.  out3[0]: accepted quotients
 * that differ in any bit (0 expected for every d); out3[1]: rejected x among those a grid
 * can hold (x >= 2^-80 and x / d < 2^22, which then take the division instruction);
 * out3[2]: all such x.  Runs on the current device in a few milliseconds and allocates
 * 24 bytes of device memory. */
int32_t pb_check_division(double d, int64_t* out3);

/* Bilinear E/B gather + 2D3V Boris + drift (x += vx dt 1000), in place; bit-identical
 * to push_particles_boris_cpu (physics_engine.py:188-254; Taichi form :63-144). */
int32_t pb_push_particles_boris(float* x, float* y, float* vx, float* vy, float* vz, const float* Ex,
                                const float* Ey, const float* Bx, const float* By, const float* Bz,
                                int32_t num_p, double dx, double dy, int32_t nx, int32_t ny, double dt,
                                double q_m, void* stream);

/* One explicit conduction sweep with the Taichi kernel's edge handling
 * (thermal_conduction_taichi, physics_engine.py:147-171). */
int32_t pb_thermal_conduction(const float* T, float* T_new, const int32_t* mask, int32_t nx, int32_t ny,
                              double Fo_x, double Fo_y, void* stream);

/* compute_particle_substeps (physics_engine.py:928-966): out_host[0] = n_sub,
 * out_host[1] = ds_max [m], out_host[2] = ds_lim [m]; synchronises the stream.  Runs the
 * step's reduction (E from a temporary corner array; with 16-byte aligned arrays, particles
 * whose displacement provably stays below one already seen are passed over), so it also
 * checks that path: the result is the full maximum, bit for bit.  Grids below 2 x 2 are
 * refused with PB_ERR_ARG. */
int32_t pb_compute_particle_substeps(const float* x, const float* y, const float* vx, const float* vy,
                                     const float* vz, int32_t n, const float* Ex, const float* Ey, int32_t nx,
                                     int32_t ny, double dx, double dy, double qm, double dt, double frac,
                                     double* out_host, void* stream);

/* _segment_hits_grid (physics_engine.py:1880-1901) with samples = 8; hit_ix/hit_iy int64. */
int32_t pb_segment_hits_grid(const uint8_t* isBound, int32_t nx, int32_t ny, double dx, double dy,
                             const float* x0, const float* y0, const float* x1, const float* y1, int32_t n,
                             uint8_t* hit, int64_t* hit_ix, int64_t* hit_iy, void* stream);

/* ---------------------------------------------------------------- simulation instance */
typedef struct pb_sim pb_sim;

/* Scalars of one timestep, computed by the host in IEEE double exactly as the reference
 * does (physics_engine.py:969-1784); float32 thresholds are cast on the device. */
typedef struct pb_step_params {
  int32_t iteration;       /* self.iteration after the increment */
  int32_t do_poisson;      /* iteration % 2 == 0 */
  int32_t picard_iters;    /* 5 */
  int32_t thermal_on;      /* sim_mode in (Thermal, Both) */
  int32_t erosion_on;      /* sim_mode in (Erosion, Both) */
  int32_t sort_now;        /* re-sort particles by cell after this step */
  /* injection */
  int32_t inject_on;
  int32_t geometry;        /* 0 half_hole, 1 one_hole, 2 two_holes, 3 no grids */
  double lam, ylo, yhi, x_inj, v_bohm, v_spread;
  double span[4];          /* two_holes band limits (cast to float32) */
  int32_t rf_on;
  int32_t neut_n;
  double rf_num_float, rf_ylo, rf_yhi, v_e_src;
  double neut_r, neut_x, v_e_th;
  /* deposit and field solve */
  double charge_density;   /* q * macro_weight / V_cell */
  double coeff, qn0_neg, V_plasma, Te_up, omega_keep, omega_new;
  double hx, two_hx, hy, two_hy, two_hy_per;
  /* grid spacing [mm] (Python floats, cast to float32 where NumPy does) */
  double dx, dy;
  /* push */
  double dt, qm_ion, qm_e, ds_lim, dt2;
  /* geometry thresholds */
  double x_entry, x_exit, x_plume, Lx, Ly;
  /* tallies */
  double half_m_ion, macro_w, C_cell, thermal_accel, q, Y_coeff, E_th, thresh;
  /* CEX */
  double rT, n0a, neut_vth;
  /* SEE */
  double v_see_th;
  /* thermal */
  double cooling_factor, T4_300, Fo_x, Fo_y;
  int32_t sweeps;
  /* RF co-extraction (V_fixed on one grid = Vdc + v_rf before injection) */
  int32_t rf_grid;         /* -1: off */
  double v_rf;
  /* saddle sample indices (flat), -1 unused */
  int32_t n_saddle;
  int32_t saddle_idx[8];
  /* options without a reference counterpart (params 'neutral_profile', 'sputter_exponent'):
   * neutral_uniform = 1 takes the CEX neutral density as n0_uniform everywhere instead of
   * the point-source profile of physics_engine.py:1696-1706; sputter_exp other than 0 or 1
   * uses the yield Y_coeff (E - E_th)^sputter_exp in float64 instead of the linear law of
   * :1432 (a zero-filled struct keeps the reference's physics) */
  int32_t neutral_uniform;
  double n0_uniform;
  double sputter_exp;
} pb_step_params;

typedef struct pb_step_report {
  int32_t num_p, num_e;
  int32_t n_sub_ion, n_sub_e;
  double ds_ion, ds_e;
  int32_t injected, rf_injected, neut_injected, see_spawned;
  uint64_t entered, crossed, exited_any, lost_to_grid, hits, cex_collisions, cex_ties;
  double exit_sums[9];     /* sum vx, |v|, E_eV, |v| primary, n primary, |v| cex, n cex, vx^2, |v|^2 */
  double theta95;          /* NaN when 5 or fewer ions crossed */
  double min_pot;
  double grid_sums[32];    /* per grid: sum T, cell count */
  int32_t broken;          /* cells broken by sputtering this step */
  int32_t pad0;
  uint64_t ppc_active, ppc_low, ppc_min;
  double poisson_stats[4]; /* outer, inner iterations (cumulative), last relative residual, solves */
  uint32_t errflags;
  int32_t pad1;
} pb_step_report;

int32_t pb_sim_create(pb_sim** out, int32_t device);
int32_t pb_sim_destroy(pb_sim* s);
int32_t pb_sim_set_seed(pb_sim* s, uint64_t seed);

/* Field solver controls: FP64 relative residual target, FP32 reduction per refinement pass
 * (default 1e-3), loop caps, damped-Jacobi sweeps on the fine level on each side of the
 * coarse correction (nu = 1, fused into the transfers, or 2: one more grid-wide phase on each
 * side; the cycle stays symmetric; other values are rejected) and the largest coarsest-level
 * size (4 to 4096 active nodes; default 1536; that level is solved with a dense inverse).
 * A new max_coarse takes effect at the next pb_sim_set_domain / pb_sim_rebuild_operator.
 * Stands in for the reference's fixed SuperLU factorisation (physics_engine.py:603-608). */
int32_t pb_sim_set_solver(pb_sim* s, double tol, double tol_inner, int32_t max_outer, int32_t max_inner,
                          int32_t nu, int32_t max_coarse);
/* Launch shapes (the autotuner's knobs; the reference has no counterpart): blocks per SM
 * of the ion and electron step kernels (1-32, default 8; tiles are handed out by a counter,
 * so any grid covers every particle) and blocks of the field-solve launch (1 to the number
 * of SMs, default all). Results do not depend on either: the field solve sums over a fixed
 * set of virtual blocks whatever its block count. */
int32_t pb_sim_set_launch(pb_sim* s, int32_t particle_blocks_per_sm, int32_t solve_blocks);
/* Kernel variants of the step (the autotuner's knobs; no counterpart in the reference).
 * Every combination gives bit-identical results; they differ in speed only.
 *   PB_OPT_SMEM_HIST  deposit and PPC counts go through shared-memory cell histograms per
 *                     tile of cell-sorted particles, flushed to HBM once per tile
 *   PB_OPT_TMA_TILE   the ion step stages each tile's window of the E-corner array in
 *                     shared memory with a TMA tensor copy before pushing
 *   PB_OPT_ELE_PAIRS  the electron step pushes two particles per thread side by side, so
 *                     that one particle's field loads overlap the other's arithmetic
 *   PB_OPT_ELE_SPLIT  the electron step runs as a barrier-free push kernel followed by a
 *                     separate stable compaction (overrides the other electron variants) */
enum { PB_OPT_SMEM_HIST = 1 << 0, PB_OPT_TMA_TILE = 1 << 1, PB_OPT_ELE_PAIRS = 1 << 2, PB_OPT_ELE_SPLIT = 1 << 3 };
int32_t pb_sim_set_kernel_options(pb_sim* s, uint32_t flags);
/* CUDA graphs of whole steps in pb_sim_run and pb_sim_step (no counterpart in the
 * reference): with on != 0 each step shape (its parameters apart from the step number,
 * and the buffers and settings its launches take) is captured once and replayed; the step
 * number that keys the Philox draws is read from device memory.  Results are the same bits
 * as without graphs.  Steps with RF co-extraction and profiled steps are enqueued as usual,
 * and so are all steps after a capture fails (see pb_sim_graph_stats).  A simulator in
 * graph mode should not run concurrently with another simulator's cooperative field solve
 * on the same device (batches use pb_batch_run). */
int32_t pb_sim_set_graphs(pb_sim* s, int32_t on);
/* out4: captures, replays, steps enqueued without a graph while graph mode was on, and 1
 * if a capture failed (then pb_last_error() gives the reason). */
int32_t pb_sim_graph_stats(pb_sim* s, int64_t* out4);
int32_t pb_sim_get_kernel_options(pb_sim* s, uint32_t* flags);
/* Particles per block of the ion and electron step kernels (their tile of staging,
 * compaction and histograms): 1024 (default) or 512; an autotuner knob without a
 * counterpart in the reference.  Results do not depend on it. */
int32_t pb_sim_set_tile(pb_sim* s, int32_t particles_per_block);

/* Upload the domain of build_domain (physics_engine.py:629-847): node masks, Dirichlet
 * values, electrode masks (bit g of gridmask = grid g), plus the state arrays to keep.
 * Host pointers.  Builds the node classes of build_sparse_matrix (:525-552) and the
 * multigrid hierarchy.  keep_state != 0 keeps particles and damage. */
int32_t pb_sim_set_domain(pb_sim* s, int32_t ny, int32_t nx, int32_t periodic, const uint8_t* isBound,
                          const double* V_fixed, const uint16_t* gridmask, int32_t ngrids, const double* V,
                          const float* Tmap, const double* damage, const double* eroded, int32_t keep_state);

/* User cross-section (lookup_user_cs, physics_engine.py:475-484): the cubic B-spline of
 * the log-log table (SciPy UnivariateSpline knots t[nt], coefficients c[nt-4]) and the
 * clip range [lo, hi] in log10 eV; which = 0 charge exchange ('CX'), 1 secondary
 * emission ('SEE'); nt = 0 removes it. */
int32_t pb_sim_set_spline(pb_sim* s, int32_t which, int32_t nt, const double* t, const double* c, double lo,
                          double hi);

/* Rebuild node classes and the multigrid hierarchy from the device isBound (after cells
 * broke by sputtering; build_sparse_matrix, physics_engine.py:1448).  Inside pb_sim_run,
 * pb_sim_step and pb_batch_run the same rebuild runs on the device before the first field
 * solve after a break, bit-equal to this host build.  When the freed nodes would make this
 * build choose other levels, or the coarsest level outgrows 1.25 x max(its size at the last
 * host build, max_coarse), those calls run this host build before returning (the solves
 * before it use the device's rebuild with the old level count, or the old hierarchy). */
int32_t pb_sim_rebuild_operator(pb_sim* s);
/* out8: hierarchy rebuilds done on the device, rebuilds left to the host, host rebuilds
 * run after pb_sim_run / pb_sim_step / pb_batch_run for them, the current coarsest active
 * count, then the microseconds the device rebuilds spent in the coarse levels, in the dense
 * assembly and Cholesky factor, in the inverse factor and smoother weights, and in the
 * transfer stencils and dense inverse (cumulative). */
int32_t pb_sim_mg_stats(pb_sim* s, int64_t* out8);
/* FNV-1a digest of the hierarchy the field solve reads (per level the smoother weights and
 * the transfer stencils, then the coarsest index set and its dense inverse): equal digests
 * mean bit-equal operators (a diagnostic without a reference counterpart). */
int32_t pb_sim_operator_digest(pb_sim* s, uint64_t* out);

/* Replace one species' particles (species 0 ions, 1 electrons); host arrays; cex may be
 * NULL for electrons. */
int32_t pb_sim_set_particles(pb_sim* s, int32_t species, int32_t n, const float* x, const float* y,
                             const float* vx, const float* vy, const float* vz, const uint8_t* cex,
                             const uint32_t* id, uint32_t next_id);
/* Re-order the particles of one species (0 ions, 1 electrons, -1 both) by cell key
 * iy * nx + ix, ix = clip(rint(x / dx), 1, nx - 2), with the device radix sort the step
 * uses every sort interval (stable: equal keys keep their order).  Particle order is
 * not observable in the reference's results (draws are keyed by particle id), so this
 * only improves memory locality, e.g. right after an upload in arbitrary order.  No
 * counterpart in the reference. */
int32_t pb_sim_sort(pb_sim* s, int32_t species, double dx, double dy);
int32_t pb_sim_get_particles(pb_sim* s, int32_t species, int32_t n, float* x, float* y, float* vx, float* vy,
                             float* vz, uint8_t* cex, uint32_t* id);
int32_t pb_sim_counts(pb_sim* s, int32_t* num_p, int32_t* num_e, uint32_t* next_ion_id, uint32_t* next_e_id);
int32_t pb_sim_reserve(pb_sim* s, int32_t species, int32_t capacity);

/* Field arrays: 0 V (f64), 1 Ex, 2 Ey, 3 rho, 4 Tmap (f32), 5 damage (f64), 6 isBound (u8),
 * 7 V_fixed (f64), 8 ppc (i32), 9 accum_ppc (f64), 10 eroded (f64), 11 Vnew (f64),
 * 12 node class (u8), 13 fine-level smoother weights of the field solver (f32, omega / A_ii on
 * free nodes, 0 elsewhere; read-only). */
int32_t pb_sim_field_ptr(pb_sim* s, int32_t which, void** dptr);
int32_t pb_sim_get_field(pb_sim* s, int32_t which, void* host, int64_t nbytes);
int32_t pb_sim_set_field(pb_sim* s, int32_t which, const void* host, int64_t nbytes);
/* particle arrays of the current buffer: 0 x, 1 y, 2 vx, 3 vy, 4 vz, 5 cex, 6 id */
int32_t pb_sim_particle_ptr(pb_sim* s, int32_t species, int32_t which, void** dptr);

/* recalc_poisson(iterations) (physics_engine.py:850-884) on the current rho. */
int32_t pb_sim_poisson(pb_sim* s, int32_t iterations, const pb_step_params* p, double* stats4_host);

/* One timestep (physics_engine.py:969-1784); report may be NULL (no host sync). */
int32_t pb_sim_step(pb_sim* s, const pb_step_params* p, pb_step_report* report);
/* Steps without a host synchronisation; params[k] for k < nsteps; reports optional. */
int32_t pb_sim_run(pb_sim* s, const pb_step_params* params, int32_t nsteps, pb_step_report* reports);
int32_t pb_sim_synchronize(pb_sim* s);
void* pb_sim_stream(pb_sim* s);

/* Device time (ms) of the last pb_sim_run / pb_sim_step in out[0]; with profiling on,
 * out[1..6] = summed phase times (inject+deposit, field solve, sub-step reduction, ion
 * step kernel, sputter break + electron step + SEE, thermal/diagnostics/sort), out[7] =
 * steps profiled, out[8] = kernels enqueued by that call. */
int32_t pb_sim_timing(pb_sim* s, double* out_host9);
/* The same profiled steps by kernel group (summed ms): out[0] injection + deposit,
 * [1] field solve, [2] E corners + sub-step counts, [3] ion step kernel, [4] sputter
 * break, [5] electron step kernel, [6] SEE spawn, [7] thermal + grid sums,
 * [8] diagnostics + cell sort; out[9] = steps profiled.  No counterpart in the
 * reference (its runner prints wall time per iteration,
 * run_simulation_from_config.py:246-273). */
int32_t pb_sim_phase_times(pb_sim* s, double* out_host10);
int32_t pb_sim_set_profiling(pb_sim* s, int32_t on);
/* Field-solve phase trace: returns the accumulated nanoseconds per phase (out32 may be
 * NULL: [l] down leg of level l, [7] coarse part, [8+l] up leg of level l, [15] Krylov
 * updates, [16] FP64 refinement, [17] right-hand side, [18] Picard update, [19] field,
 * [20] set-up; [21+p] inner iterations and [26+p] refinement passes of Picard iteration p),
 * clears them and switches tracing on or off. */
int32_t pb_sim_poisson_trace(pb_sim* s, int32_t on, double* out32);
/* The three float32 sums of get_total_energy (physics_engine.py:1800-1866) on the device,
 * each equal bit for bit to NumPy's np.sum (pairwise summation) of the same float32 array:
 * out3[0] = sum(p_vx**2 + p_vy**2 + p_vz**2) over the ions, out3[1] the same over the
 * electrons, out3[2] = sum(Ex**2 + Ey**2) over the grid (0 before a domain is set).
 * Synchronises the simulator's stream. */
int32_t pb_sim_energy_sums(pb_sim* s, double* out3);

/* ---------------------------------------------------------------- host helpers */
/* n sequential additions s = (float)((double)s + c), as np.add.at on a float32 array */
float pb_host_seq_add_f32d(float s, double c, uint32_t n);
double pb_host_philox_uniform(uint64_t seed, uint64_t pid, uint32_t site, uint32_t step, uint32_t j);
double pb_host_philox_normal(uint64_t seed, uint64_t pid, uint32_t site, uint32_t step, uint32_t j);
float pb_host_percentile95(const float* sorted, int32_t n);
/* The block plan of one batched field-solve launch (pb_batch_run): m members of positive cost
 * (block-time of one launch) on total >= m blocks.  Per member: its first block, its block
 * count, and packed = 1 when it shares its one block with other members (run one after
 * another). */
int32_t pb_host_plan_blocks(const int64_t* work, int32_t m, int32_t total, int32_t* first, int32_t* count,
                            int32_t* packed);

/* ---------------------------------------------------------------- batched instances
 * Several simulators advanced together on one GPU: sweep points of a perveance or
 * backstreaming study (the reference runs one process per point,
 * Python/benchmarks/benchmark_perveance.py:78-164).  No single counterpart in the
 * reference; each instance's step is the same as pb_sim_step's. */
typedef struct pb_batch pb_batch;

int32_t pb_batch_create(pb_batch** out, int32_t device);
int32_t pb_batch_destroy(pb_batch* b);
/* Advance n simulators (all on the batch's device, each at most once in the list) by K
 * steps: params[i * K + k] is step k of simulator i and reports[i * K + k] (may be NULL)
 * receives its report.  Each instance's particle kernels run on its own stream; the field
 * solves due in a step run as one cooperative launch with the SMs shared out in
 * proportion to grid size.  Results per instance equal those of pb_sim_run.  Returns
 * after the last step has completed. */
int32_t pb_batch_run(pb_batch* b, pb_sim* const* sims, int32_t n, const pb_step_params* params, int32_t K,
                     pb_step_report* reports);
/* CUDA graphs of whole batch steps (no counterpart in the reference): with on != 0 each
 * step shape of the set (every member's step parameters apart from the step number, and
 * the state its launches take) is captured once, with every member's work on the graph's
 * branches and the shared field solve between them, and replayed; the host then issues one
 * launch per step instead of one per kernel and member.  Results are the same bits as
 * without graphs.  Steps that cannot be captured are enqueued as usual (and graphs stay
 * off for the batch until re-enabled; see pb_batch_graph_stats). */
int32_t pb_batch_set_graphs(pb_batch* b, int32_t on);
/* Host threads that enqueue the members' kernels in the streams form (the calling thread
 * included; member i goes to thread i mod threads): 1 (default) enqueues from the calling
 * thread alone, 0 picks min(8, half the host's hardware threads).  Results do not depend on
 * it; on a 64-member sweep eight threads took more host and device time than one. */
int32_t pb_batch_set_threads(pb_batch* b, int32_t threads);
/* out3: captures, replays, 1 if a capture failed (pb_last_error() gives the reason). */
int32_t pb_batch_graph_stats(pb_batch* b, int64_t* out3);
/* out4[0] = device time (ms) of the last pb_batch_run, out4[1] = kernel launches in it,
 * out4[2] = host time (ms) from its first enqueue to its last (when this approaches the
 * device time, the run is bound by launch overhead), out4[3] = device time of its
 * field-solve launches (without graphs; -1 with them: not timed inside a graph). */
int32_t pb_batch_timing(pb_batch* b, double* out4);
/* A member's field-solve cost as the batch measured it (out2[0]: block-milliseconds per
 * launch in its last batch run, 0 before one) and its block share in the last launch planned
 * (out2[1]); pb_batch_run shares each launch's blocks so that the largest cost per block
 * is as small as it can be (one block each, then each further block to the largest). */
int32_t pb_sim_batch_share(pb_sim* s, double* out2);
/* Device memory held by a simulator (bytes, estimated from its capacities). */
int32_t pb_sim_memory(pb_sim* s, int64_t* bytes);

#ifdef __cplusplus
}
#endif
#endif
