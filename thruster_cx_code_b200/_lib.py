"""ctypes binding of libpbemcs.so (include/pbemcs.h).

The library is built in-tree (``python -m thruster_cx_code_b200._build``).  Loading fails
with an ImportError-style RuntimeError when it is missing: there is no CPU fallback.
The host helpers (``pb_host_*``) and the structure layouts work without a GPU.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpbemcs.so")

i32, u32, u64, f64, f32, vp = C.c_int32, C.c_uint32, C.c_uint64, C.c_double, C.c_float, C.c_void_p
P = C.POINTER


class StepParams(C.Structure):
    """pb_step_params (field order and types as in include/pbemcs.h)."""
    _fields_ = [
        ("iteration", i32), ("do_poisson", i32), ("picard_iters", i32), ("thermal_on", i32),
        ("erosion_on", i32), ("sort_now", i32),
        ("inject_on", i32), ("geometry", i32),
        ("lam", f64), ("ylo", f64), ("yhi", f64), ("x_inj", f64), ("v_bohm", f64), ("v_spread", f64),
        ("span", f64 * 4),
        ("rf_on", i32), ("neut_n", i32),
        ("rf_num_float", f64), ("rf_ylo", f64), ("rf_yhi", f64), ("v_e_src", f64),
        ("neut_r", f64), ("neut_x", f64), ("v_e_th", f64),
        ("charge_density", f64),
        ("coeff", f64), ("qn0_neg", f64), ("V_plasma", f64), ("Te_up", f64), ("omega_keep", f64), ("omega_new", f64),
        ("hx", f64), ("two_hx", f64), ("hy", f64), ("two_hy", f64), ("two_hy_per", f64),
        ("dx", f64), ("dy", f64),
        ("dt", f64), ("qm_ion", f64), ("qm_e", f64), ("ds_lim", f64), ("dt2", f64),
        ("x_entry", f64), ("x_exit", f64), ("x_plume", f64), ("Lx", f64), ("Ly", f64),
        ("half_m_ion", f64), ("macro_w", f64), ("C_cell", f64), ("thermal_accel", f64), ("q", f64),
        ("Y_coeff", f64), ("E_th", f64), ("thresh", f64),
        ("rT", f64), ("n0a", f64), ("neut_vth", f64),
        ("v_see_th", f64),
        ("cooling_factor", f64), ("T4_300", f64), ("Fo_x", f64), ("Fo_y", f64),
        ("sweeps", i32),
        ("rf_grid", i32),
        ("v_rf", f64),
        ("n_saddle", i32),
        ("saddle_idx", i32 * 8),
        ("neutral_uniform", i32),
        ("n0_uniform", f64),
        ("sputter_exp", f64),
    ]


class StepReport(C.Structure):
    """pb_step_report."""
    _fields_ = [
        ("num_p", i32), ("num_e", i32), ("n_sub_ion", i32), ("n_sub_e", i32),
        ("ds_ion", f64), ("ds_e", f64),
        ("injected", i32), ("rf_injected", i32), ("neut_injected", i32), ("see_spawned", i32),
        ("entered", u64), ("crossed", u64), ("exited_any", u64), ("lost_to_grid", u64), ("hits", u64),
        ("cex_collisions", u64), ("cex_ties", u64),
        ("exit_sums", f64 * 9),
        ("theta95", f64), ("min_pot", f64),
        ("grid_sums", f64 * 32),
        ("broken", i32), ("pad0", i32),
        ("ppc_active", u64), ("ppc_low", u64), ("ppc_min", u64),
        ("poisson_stats", f64 * 4),
        ("errflags", u32), ("pad1", i32),
    ]


PROTOTYPES = {
    "pb_version": (i32, []),
    "pb_last_error": (C.c_char_p, []),
    "pb_accumulate_rho": (i32, [vp, vp, vp, i32, f64, f64, i32, i32, f64, vp]),
    "pb_accumulate_rho_noalloc": (i32, [vp, vp, vp, i32, f64, f64, i32, i32, f64, vp]),
    "pb_push_particles_boris": (i32, [vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, i32, f64, f64, i32, i32, f64, f64, vp]),
    "pb_thermal_conduction": (i32, [vp, vp, vp, i32, i32, f64, f64, vp]),
    "pb_compute_particle_substeps": (i32, [vp, vp, vp, vp, vp, i32, vp, vp, i32, i32, f64, f64, f64, f64, f64, P(f64), vp]),
    "pb_segment_hits_grid": (i32, [vp, i32, i32, f64, f64, vp, vp, vp, vp, i32, vp, vp, vp, vp]),
    "pb_sim_create": (i32, [P(vp), i32]),
    "pb_sim_destroy": (i32, [vp]),
    "pb_sim_set_seed": (i32, [vp, u64]),
    "pb_sim_set_solver": (i32, [vp, f64, f64, i32, i32, i32, i32]),
    "pb_sim_set_launch": (i32, [vp, i32, i32]),
    "pb_sim_set_spline": (i32, [vp, i32, i32, P(f64), P(f64), f64, f64]),
    "pb_sim_set_domain": (i32, [vp, i32, i32, i32, vp, vp, vp, i32, vp, vp, vp, vp, i32]),
    "pb_sim_set_particles": (i32, [vp, i32, i32, vp, vp, vp, vp, vp, vp, vp, u32]),
    "pb_sim_get_particles": (i32, [vp, i32, i32, vp, vp, vp, vp, vp, vp, vp]),
    "pb_sim_counts": (i32, [vp, P(i32), P(i32), P(u32), P(u32)]),
    "pb_sim_reserve": (i32, [vp, i32, i32]),
    "pb_sim_rebuild_operator": (i32, [vp]),
    "pb_sim_mg_stats": (i32, [vp, P(C.c_int64)]),
    "pb_sim_batch_share": (i32, [vp, P(f64)]),
    "pb_sim_operator_digest": (i32, [vp, P(u64)]),
    "pb_sim_field_ptr": (i32, [vp, i32, P(vp)]),
    "pb_sim_get_field": (i32, [vp, i32, vp, C.c_int64]),
    "pb_sim_set_field": (i32, [vp, i32, vp, C.c_int64]),
    "pb_sim_particle_ptr": (i32, [vp, i32, i32, P(vp)]),
    "pb_sim_poisson": (i32, [vp, i32, P(StepParams), P(f64)]),
    "pb_sim_step": (i32, [vp, P(StepParams), P(StepReport)]),
    "pb_sim_run": (i32, [vp, P(StepParams), i32, P(StepReport)]),
    "pb_sim_synchronize": (i32, [vp]),
    "pb_sim_stream": (vp, [vp]),
    "pb_sim_timing": (i32, [vp, P(f64)]),
    "pb_sim_phase_times": (i32, [vp, P(f64)]),
    "pb_sim_set_kernel_options": (i32, [vp, u32]),
    "pb_sim_get_kernel_options": (i32, [vp, P(u32)]),
    "pb_check_division": (i32, [f64, P(C.c_int64)]),
    "pb_sim_set_tile": (i32, [vp, i32]),
    "pb_sim_set_graphs": (i32, [vp, i32]),
    "pb_sim_graph_stats": (i32, [vp, P(C.c_int64)]),
    "pb_sim_set_profiling": (i32, [vp, i32]),
    "pb_sim_poisson_trace": (i32, [vp, i32, P(f64)]),
    "pb_sim_energy_sums": (i32, [vp, P(f64)]),
    "pb_sim_sort": (i32, [vp, i32, f64, f64]),
    "pb_batch_create": (i32, [P(vp), i32]),
    "pb_batch_destroy": (i32, [vp]),
    "pb_batch_run": (i32, [vp, P(vp), i32, P(StepParams), i32, P(StepReport)]),
    "pb_batch_timing": (i32, [vp, P(f64)]),
    "pb_batch_set_graphs": (i32, [vp, i32]),
    "pb_batch_set_threads": (i32, [vp, i32]),
    "pb_batch_graph_stats": (i32, [vp, P(C.c_int64)]),
    "pb_sim_memory": (i32, [vp, P(C.c_int64)]),
    "pb_host_seq_add_f32d": (f32, [f32, f64, u32]),
    "pb_host_plan_blocks": (i32, [P(C.c_int64), i32, i32, P(i32), P(i32), P(i32)]),
    "pb_host_philox_uniform": (f64, [u64, u64, u32, u32, u32]),
    "pb_host_philox_normal": (f64, [u64, u64, u32, u32, u32]),
    "pb_host_percentile95": (f32, [vp, i32]),
}

_lib = None


def load():
    """Load and return the library (cached); raises RuntimeError when it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"libpbemcs.so not found at {LIB_PATH}; build it with `python -m thruster_cx_code_b200._build` "
            "(the GPU path has no CPU fallback)")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


# kernel variants of the step (pb_sim_set_kernel_options)
PB_OPT_SMEM_HIST = 1 << 0
PB_OPT_TMA_TILE = 1 << 1
PB_OPT_ELE_PAIRS = 1 << 2
PB_OPT_ELE_SPLIT = 1 << 3

ERRORS = {1: "CUDA error", 2: "invalid argument", 3: "capacity", 4: "device wait timed out",
          5: "field solve did not converge", 6: "call out of order"}


class PbError(RuntimeError):
    def __init__(self, code, where):
        msg = load().pb_last_error().decode(errors="replace")
        super().__init__(f"{where}: {ERRORS.get(code, code)}: {msg}")
        self.code = code


def check(code, where):
    if code != 0:
        raise PbError(code, where)
