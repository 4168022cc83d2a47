// Device-side argument structures shared by the kernel translation units and the runtime.
#pragma once
#include "pb_common.cuh"

namespace pb {

// One species' structure-of-arrays particle store (one of two ping-pong buffers).
struct Soa {
  float *x, *y, *vx, *vy, *vz;
  uint8_t *cex;  // ions only, nullptr for electrons
  uint32_t *id;
};

// Cubic B-spline in (log10 E -> log10 value) form, the SciPy UnivariateSpline of a
// cross-section table (t: knots, c: coefficients, k = 3), clipped to [lo, hi].
struct Spline {
  const double *t, *c;
  int nt;      // number of knots
  double lo, hi;
  int enabled;
};

// Reciprocals of the grid spacings for the division of the particle kernels (div_bracket):
// inv = RN(1/d) and the floats two steps below and above it, which bracket 1/d with room
// for the residual's rounding.  NaN brackets (a spacing that is not a positive normal
// float) make every quotient take the division instruction.
struct Rcp {
  float ix, ix_lo, ix_hi, iy, iy_lo, iy_hi;
};

__host__ __device__ inline void rcp_axis(float d, float& inv, float& lo, float& hi) {
  inv = 1.0f / d;
  unsigned b;
  memcpy(&b, &inv, sizeof(b));
  const bool ok = d > 0.0f && b >= 0x01000000u && b < 0x7F000000u;  // inv and its neighbours normal
  const unsigned bl = ok ? b - 2u : 0x7FC00000u, bh = ok ? b + 2u : 0x7FC00000u;
  memcpy(&lo, &bl, sizeof(lo));
  memcpy(&hi, &bh, sizeof(hi));
}

__host__ __device__ inline Rcp make_rcp(float dxf, float dyf) {
  Rcp r;
  rcp_axis(dxf, r.ix, r.ix_lo, r.ix_hi);
  rcp_axis(dyf, r.iy, r.iy_lo, r.iy_hi);
  return r;
}

// Everything the ion step kernel reads besides the particles.
// E-corner window that the ion step stages per tile with a TMA copy (PB_OPT_TMA_TILE):
// TB_W x TB_H cells of 8 floats (8 KB)
constexpr int TB_W = 64, TB_H = 4;
constexpr unsigned TB_BYTES = TB_W * TB_H * 32u;

struct IonStepArgs {
  // tensor map of the corner array viewed as float [ny][nx][8], box 8 x TB_W x TB_H
  // (read by the TMA unit from the kernel's parameter space)
  CUtensorMap ec_map;
  Soa src, dst;
  const int *num_src;
  int *num_dst;
  // fields
  const float *Ex, *Ey, *Bx, *By, *Bz;
  const float4* Ec;       // per-cell corners of Ex, Ey (the gather when B = 0)
  int has_B;
  const uint8_t *isBound;
  const uint8_t *bdist;   // Chebyshev distance (cells) to the nearest bound node, capped
  int nx, ny;
  float dxf, dyf;
  float inv_dx, inv_dy;   // f32(1/dxf), f32(1/dyf)
  Rcp rcp;                // the same with their brackets (the push's division)
  // push
  double dt, qm, ds_lim;
  const double *ds_max;   // device: max predicted displacement (n_sub)
  int *n_sub_out;
  int periodic;
  float Lyf, Lxf;
  // thresholds (float32 casts of Python floats, as NumPy compares)
  float x_entry, x_exit, x_plume;
  // tallies
  int thermal_on, erosion_on;
  float *Tmap;
  double *damage;
  float k_half_m;   // f32(0.5*m_ion)
  float mw_f;       // f32(macro_weight)
  float ccell_f;    // f32(C_cell)
  float accel_f;    // f32(thermal_accel)
  float q_f;        // f32(q)
  float Y_f, Eth_f; // f32(Y_coeff), f32(E_th)
  double Y_d, mw_d; // Y_coeff, macro_weight (float64 power-law yield)
  double Y_exp;     // yield exponent: 1 = the reference's linear law in float32
  float dt_f;       // f32(dt) (SEE spawn offset)
  Spline see_spline;
  // SEE spawn records
  uint64_t *see_key;   // (parent id << 32) | record index
  float *see_xy;       // x, y per record
  int *see_count;
  int see_cap;
  // exit diagnostics
  float *angles;
  int *angle_count;
  int angle_cap;
  double *exit_sums;     // [sum vx, sum |v|, sum E, sum |v| prim, n prim, sum |v| cex, n cex, sum vx^2, sum |v|^2]
  unsigned long long *counters;  // [entered, crossed, exited_any, lost_to_grid, hits, cex_collisions, cex_ties]
  // CEX
  float rT_f;          // f32(Ly*1e-3)
  double n0a;          // n0 * a_corr
  int n_uniform;       // 1: uniform neutral density n0u (no point-source profile)
  double n0u;
  double neut_vth;
  Spline cx_spline;
  double cex_bound;    // |n0a| * sigma_max * dt * (1 + 1e-5): P <= cex_bound * g
  float cex_g_max;     // speeds above this bypass the bound
  uint64_t seed;
  uint32_t step;
  const uint32_t* step_dev;  // non-null in a captured step: the step key is read from here
  // counts for diagnostics / next deposit
  int *ppc;            // int32 (ny, nx) current PPC map (trunc cells)
  int *cnt;            // int32 (ny, nx) deposit counts for the next step (round cells)
  // single-pass compaction
  unsigned long long *tile_status;
  int *tile_counter;
  uint32_t *errflags;
};

struct EleStepArgs {
  Soa src, dst;
  const int *num_src;
  int *num_dst;
  const float *Ex, *Ey, *Bx, *By, *Bz;
  const float4* Ec;       // per-cell corners of Ex, Ey (the gather when B = 0)
  int has_B;
  const uint8_t *isBound;
  int nx, ny;
  float dxf, dyf;
  float inv_dx, inv_dy;
  Rcp rcp;
  const unsigned *ebound;  // float bits of max |Ex| + |Ey| over the corners (k_e_corners), or nullptr
  double dt, qm, ds_lim;
  const double *ds_max;
  int *n_sub_out;
  int periodic;
  float Lyf, Lxf;
  int *cnt;
  unsigned long long *tile_status;
  int *tile_counter;
  uint32_t *errflags;
};

}  // namespace pb
