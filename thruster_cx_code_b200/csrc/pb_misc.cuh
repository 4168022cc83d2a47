// Argument structures of the injection, SEE and sort kernels.
#pragma once
#include "pb_kernels.cuh"

namespace pb {

constexpr int RADIX_BITS = 7;
constexpr int RADIX = 1 << RADIX_BITS;
constexpr int SORT_NT = 256;
constexpr int SORT_TILE = 2048;

struct InjectArgs {
  // ions (physics_engine.py:996-1064)
  int ion_on;
  double lam;               // expected injections this step (num_inject_float)
  int geometry;             // 0 half_hole / 1 one_hole / 3 no grids: uniform band; 2 two_holes
  double ylo, yhi;          // uniform band
  float span[4];            // two_holes: float32 [lo0, hi0, lo1, hi1]
  float x_inj;              // f32(dx * 1.5)
  double v_bohm, v_spread;
  // RF source electrons (:1066-1083)
  int rf_on;
  double rf_num_float, rf_ylo, rf_yhi, v_e_src;
  // neutralizer (:1086-1099)
  int neut_n;
  double neut_r, v_e_th;
  float neut_x;
  // keys and state
  uint64_t seed;
  uint32_t step;
  const uint32_t* step_dev;  // non-null in a captured step: the step key is read from here
  int *num_p, *num_e;
  int cap_p, cap_e;
  uint32_t *next_ion_id, *next_e_id;
  int *inj;                 // [n_ion, n_rf, n_neut, slot_ion, slot_e, id_ion, id_e]
  Soa ions, eles;
  int *cnt_i, *cnt_e;
  int nx, ny;
  float dxf, dyf;
  uint32_t *errflags;
};

struct SeeArgs {
  uint64_t *see_key;
  const float *see_xy;
  const int *see_count;
  int see_cap;
  int *see_spawned;
  uint64_t seed;
  uint32_t step;
  const uint32_t* step_dev;  // non-null in a captured step: the step key is read from here
  double v_see_th;
  Soa eles;
  int *num_e;
  int cap_e;
  uint32_t *next_e_id;
  const uint8_t *isBound;
  int nx, ny;
  float dxf, dyf, Lxf, Lyf;
  int *cnt_e;
  uint32_t *errflags;
};

}  // namespace pb
