"""ctypes mirror of include/drmppi.h (the C ABI of the control step).

The structures follow the reference's configuration structs field by field
(include/environments/env_stratrace_defs.h:42-96, include/config.h:116-192, and for the
gate race include/environments/env_dronerace_defs.h:44-103), with the compile-time
sizes of the reference turned into runtime counts.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

DR_ABI_VERSION = 2
DR_DIM = 2
DR_MAX_OPP = 3
DR_MAX_AGENTS = 4
DR_MAX_THETA = 8
DR_MAX_KNOTS = 64
DR_MAX_T = 256
DR_GRAD_MAX_STEPS = 8
DR_GRAD_WEIGHTS = 6
DR_N_TRACK_SAMPLES = 512

DR_OK = 0
DR_ERR_INVALID_ARG = 1
DR_ERR_UNSUPPORTED = 2
DR_ERR_CUDA = 3
DR_ERR_OOM = 4
DR_ERR_NO_DEVICE = 5
DR_ERR_TIMEOUT = 6
DR_ERR_STATE = 7


class dr_opp_config(C.Structure):
    _fields_ = [
        ("s1", C.c_float * DR_MAX_OPP),
        ("s2", C.c_float * DR_MAX_OPP),
        ("s3", C.c_float * DR_MAX_OPP),
        ("speed_scale", C.c_float * DR_MAX_OPP),
        ("action_noise", C.c_float * DR_MAX_OPP),
    ]


class dr_env_config(C.Structure):
    _fields_ = [
        ("n_opp", C.c_int32),
        ("n_theta", C.c_int32),
        ("arena_min", C.c_float * DR_DIM),
        ("arena_max", C.c_float * DR_DIM),
        ("dt", C.c_float),
        ("send_states", C.c_int32),
        ("drone_radius", C.c_float),
        ("pos_noise_level", C.c_float),
        ("speed_noise_level", C.c_float),
        ("action_noise_level", C.c_float),
        ("max_speed", C.c_float * DR_MAX_AGENTS),
        ("max_accel", C.c_float * DR_MAX_AGENTS),
        ("track_width", C.c_float),
        ("n_win_laps", C.c_int32),
        ("init_belief", C.c_float * DR_MAX_THETA),
        ("opp_configs", dr_opp_config * DR_MAX_THETA),
        ("kP", C.c_float),
        ("kV", C.c_float),
        ("max_opp_lat_dist_fact", C.c_float),
        ("track_length", C.c_float),
        ("p_grid", C.POINTER(C.c_float)),
        ("dp_grid", C.POINTER(C.c_float)),
        ("t_grid", C.POINTER(C.c_float)),
        ("kappa_grid", C.POINTER(C.c_float)),
    ]


class dr_sim_state(C.Structure):
    _fields_ = [
        ("pos", C.c_float * (DR_MAX_AGENTS * DR_DIM)),
        ("vel", C.c_float * (DR_MAX_AGENTS * DR_DIM)),
        ("S", C.c_float * DR_MAX_AGENTS),
        ("lat_dist", C.c_float * DR_MAX_AGENTS),
        ("laps", C.c_int32 * DR_MAX_AGENTS),
    ]


class dr_mppi_config(C.Structure):
    _fields_ = [
        ("n_samples", C.c_int32),
        ("n_timesteps", C.c_int32),
        ("n_knots", C.c_int32),
        ("knots", C.c_int32 * DR_MAX_KNOTS),
        ("use_splines", C.c_int32),
        ("inv_temperature", C.c_float),
        ("sampling_noise", C.c_float),
        ("gate_traversal_margin", C.c_float),
        ("coll_dist_factor", C.c_float),
        ("boundary_cost", C.c_float),
        ("boundary_threshold_factor", C.c_float),
        ("outside_cost", C.c_float),
        ("win_cost", C.c_float),
        ("opp_win_cost", C.c_float),
        ("final_adv_weight", C.c_float),
        ("final_opp_adv_weight", C.c_float),
        ("min_confidence", C.c_float),
        ("n_verif_samples", C.c_int32),
        ("beta", C.c_float),
        ("verif_horizon", C.c_int32),
        ("max_verif_eps", C.c_float),
        ("sampling_noise_dim", C.c_float * DR_DIM),
        ("min_nu", C.c_float),
        ("max_nu", C.c_float),
        ("verify", C.c_int32),
    ]


class dr_prmppi_config(C.Structure):
    _fields_ = [
        ("n_samples", C.c_int32),
        ("n_timesteps", C.c_int32),
        ("inv_temperature", C.c_float),
        ("sampling_noise", C.c_float),
        ("gate_traversal_margin", C.c_float),
        ("coll_dist_factor", C.c_float),
        ("boundary_cost", C.c_float),
        ("boundary_threshold_factor", C.c_float),
        ("win_cost", C.c_float),
        ("opp_win_cost", C.c_float),
        ("final_adv_weight", C.c_float),
        ("final_opp_adv_weight", C.c_float),
        ("safety_weight", C.c_float),
        ("min_safe_dist", C.c_float),
        ("delta", C.c_float),
        ("P", C.c_int32),
        ("sampling_noise_dim", C.c_float * DR_DIM),
        ("min_nu", C.c_float),
        ("max_nu", C.c_float),
    ]


class dr_mppi_info(C.Structure):
    _fields_ = [
        ("fail_count_total", C.c_uint32),
        ("use_new_plan", C.c_int32),
        ("epsilon", C.c_double),
        ("epsilon_partial", C.c_double),
        ("certified_loss", C.c_double),
        ("branch_idx", C.c_int32),
        ("min_cost", C.c_float),
        ("nu", C.c_float),
        ("inv_temperature", C.c_float),
        ("nonfinite_costs", C.c_int32),
        ("verif_timeouts", C.c_int32),
        ("grad_cost_plain", C.c_float),
        ("grad_cost_refined", C.c_float),
        ("grad_best_step", C.c_int32),
    ]


class dr_prmppi_info(C.Structure):
    _fields_ = [
        ("use_nom_plan", C.c_int32),
        ("reset_nom", C.c_int32),
        ("cand_cost", C.c_float * 2),
        ("min_costs", C.c_float * 3),
        ("nu", C.c_float * 3),
        ("inv_temperature", C.c_float * 3),
        ("nonfinite_costs", C.c_int32),
    ]


# ---- gate race (reference EnvDroneRace, include/environments/env_dronerace_defs.h) ----
DR_GATE_AGENTS = 2
DR_GATE_RACELINES = 2
DR_GATE_MAX_GATES = 16
DR_GATE_MAX_OBSTACLES = 4


class dr_pid_config(C.Structure):
    _fields_ = [
        ("kp", C.c_float),
        ("kd", C.c_float),
        ("repulsion_factor", C.c_float),
        ("repulsion_power", C.c_float),
        ("repulsion_dist_fact", C.c_float),
        ("raceline_index", C.c_int32),
        ("action_noise", C.c_float),
    ]


class dr_gate_env_config(C.Structure):
    _fields_ = [
        ("n_theta", C.c_int32),
        ("arena_min", C.c_float * DR_DIM),
        ("arena_max", C.c_float * DR_DIM),
        ("dt", C.c_float),
        ("send_states", C.c_int32),
        ("drone_radius", C.c_float),
        ("pos_noise_level", C.c_float),
        ("speed_noise_level", C.c_float),
        ("action_noise_level", C.c_float),
        ("max_speed", C.c_float * DR_GATE_AGENTS),
        ("max_accel", C.c_float * DR_GATE_AGENTS),
        ("n_win_laps", C.c_int32),
        ("target_distance", C.c_float),
        ("n_gates", C.c_int32),
        ("gate_centers", C.c_float * (DR_GATE_MAX_GATES * DR_DIM)),
        ("gate_vectors", C.c_float * (DR_GATE_MAX_GATES * DR_DIM)),
        ("gate_radius", C.c_float * DR_GATE_MAX_GATES),
        ("n_obstacles", C.c_int32),
        ("obstacles", C.c_float * (DR_GATE_MAX_OBSTACLES * DR_DIM * 2)),
        ("n_round_obstacles", C.c_int32),
        ("round_obs_centers", C.c_float * (DR_GATE_MAX_OBSTACLES * DR_DIM)),
        ("round_obs_radius", C.c_float * DR_GATE_MAX_OBSTACLES),
        ("track_points", C.POINTER(C.c_float)),
        ("init_belief", C.c_float * DR_MAX_THETA),
        ("opp_pid", dr_pid_config * DR_MAX_THETA),
        ("i_mppi", C.c_int32),
    ]


class dr_gate_state(C.Structure):
    _fields_ = [
        ("pos", C.c_float * (DR_GATE_AGENTS * DR_DIM)),
        ("vel", C.c_float * (DR_GATE_AGENTS * DR_DIM)),
        ("S", C.c_float * (DR_GATE_AGENTS * DR_GATE_RACELINES)),
        ("laps", C.c_int32 * DR_GATE_AGENTS),
        ("gates", C.c_int32 * DR_GATE_AGENTS),
    ]


DR_TUNE_MAX_CANDIDATES = 12


class dr_tune_report(C.Structure):
    _fields_ = [
        ("rollout_ctas_per_sm", C.c_int),
        ("rollout_lockstep", C.c_int),
        ("verify_ctas_per_sm", C.c_int),
        ("grad_ckpt", C.c_int),
        ("n_rollout", C.c_int),
        ("n_verify", C.c_int),
        ("n_grad", C.c_int),
        ("rollout_cand", C.c_int * DR_TUNE_MAX_CANDIDATES),
        ("rollout_lock", C.c_int * DR_TUNE_MAX_CANDIDATES),
        ("rollout_ms", C.c_float * DR_TUNE_MAX_CANDIDATES),
        ("verify_cand", C.c_int * DR_TUNE_MAX_CANDIDATES),
        ("verify_ms", C.c_float * DR_TUNE_MAX_CANDIDATES),
        ("grad_cand", C.c_int * DR_TUNE_MAX_CANDIDATES),
        ("grad_ms", C.c_float * DR_TUNE_MAX_CANDIDATES),
    ]


def fptr(a: np.ndarray) -> C.POINTER(C.c_float):
    assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_float))


def dptr(a: np.ndarray) -> C.POINTER(C.c_double):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_double))


def iptr(a: np.ndarray) -> C.POINTER(C.c_int32):
    assert a.dtype == np.int32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def uptr(a: np.ndarray) -> C.POINTER(C.c_uint32):
    assert a.dtype == np.uint32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_uint32))


PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "lib" / "libdrmppi.so"
DR_PREDICT_RECORD = 5

# name -> (restype, argtypes)
_PROTOS = {
    "dr_abi_version": (C.c_int, []),
    "dr_supported": (C.c_int, [C.c_int, C.c_int]),
    "dr_last_error": (C.c_char_p, []),
    "dr_status_string": (C.c_char_p, [C.c_int]),
    "dr_mppi_create": (C.c_int, [C.POINTER(dr_env_config), C.POINTER(dr_mppi_config), C.c_uint64, C.POINTER(C.c_float), C.c_int, C.c_void_p, C.POINTER(C.c_void_p)]),
    "dr_mppi_destroy": (C.c_int, [C.c_void_p]),
    "dr_mppi_step": (C.c_int, [C.c_void_p, C.POINTER(dr_sim_state), C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(dr_mppi_info)]),
    "dr_mppi_get_nominal": (C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.c_size_t]),
    "dr_mppi_get_knots": (C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.c_size_t]),
    "dr_mppi_get_fail_counts": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.c_size_t]),
    "dr_mppi_get_temperature": (C.c_float, [C.c_void_p]),
    "dr_mppi_set_temperature": (C.c_int, [C.c_void_p, C.c_float]),
    "dr_mppi_get_step": (C.c_uint64, [C.c_void_p]),
    "dr_mppi_set_step": (C.c_int, [C.c_void_p, C.c_uint64]),
    "dr_mppi_io_bytes": (C.c_int, [C.c_void_p, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
    "dr_prmppi_io_bytes": (C.c_int, [C.c_void_p, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
    "dr_mppi_set_profiling": (C.c_int, [C.c_void_p, C.c_int]),
    "dr_mppi_get_kernel_times": (C.c_int, [C.c_void_p, C.POINTER(C.c_char_p), C.POINTER(C.c_float), C.c_int, C.POINTER(C.c_int)]),
    "dr_mppi_batch_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.c_void_p, C.POINTER(C.c_void_p)]),
    "dr_mppi_batch_destroy": (C.c_int, [C.c_void_p]),
    "dr_mppi_batch_step": (C.c_int, [C.c_void_p, C.POINTER(dr_sim_state), C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(dr_mppi_info)]),
    "dr_mppi_batch_step_dev": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "dr_mppi_batch_set_graph": (C.c_int, [C.c_void_p, C.c_int]),
    "dr_mppi_batch_set_profiling": (C.c_int, [C.c_void_p, C.c_int]),
    "dr_mppi_batch_set_overlap": (C.c_int, [C.c_void_p, C.c_int]),
    "dr_mppi_batch_set_priority": (C.c_int, [C.c_void_p, C.c_int]),
    "dr_mppi_batch_set_persistent": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int]),
    "dr_mppi_batch_autotune": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "dr_mppi_batch_set_side_verify": (C.c_int, [C.c_void_p, C.c_int]),
    "dr_mppi_batch_set_pdl": (C.c_int, [C.c_void_p, C.c_int]),
    "dr_prmppi_set_shard": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "dr_prmppi_shard_words": (C.c_int, [C.c_void_p, C.POINTER(C.c_size_t)]),
    "dr_prmppi_shard_begin": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "dr_prmppi_shard_finish": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "dr_mppi_batch_get_kernel_times": (C.c_int, [C.c_void_p, C.POINTER(C.c_char_p), C.POINTER(C.c_float), C.c_int, C.POINTER(C.c_int)]),
    "dr_mppi_batch_get_kernel_timeline": (C.c_int, [C.c_void_p, C.POINTER(C.c_char_p), C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int, C.POINTER(C.c_int)]),
    "dr_prmppi_batch_set_profiling": (C.c_int, [C.c_void_p, C.c_int]),
    "dr_prmppi_batch_get_kernel_times": (C.c_int, [C.c_void_p, C.POINTER(C.c_char_p), C.POINTER(C.c_float), C.c_int, C.POINTER(C.c_int)]),
    "dr_prmppi_batch_set_rollout_slots": (C.c_int, [C.c_void_p, C.c_int]),
    "dr_mppi_debug_noise": (C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.c_size_t]),
    "dr_mppi_debug_rollout": (C.c_int, [C.c_void_p, C.POINTER(dr_sim_state), C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_float)]),
    "dr_mppi_debug_update": (C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "dr_mppi_debug_verify": (C.c_int, [C.c_void_p, C.POINTER(dr_sim_state), C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int, C.POINTER(C.c_uint32), C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "dr_mppi_debug_stage_timeout": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "dr_mppi_set_verify_exact": (C.c_int, [C.c_void_p, C.c_int]),
    "dr_mppi_set_ego_table": (C.c_int, [C.c_void_p, C.c_int]),
    "dr_mppi_predict": (C.c_int, [C.c_void_p, C.POINTER(dr_sim_state), C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float),
                                  C.POINTER(C.c_int32), C.POINTER(C.c_float)]),
    "dr_mppi_batch_predict_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
    "dr_prmppi_predict": (C.c_int, [C.c_void_p, C.POINTER(dr_sim_state), C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_int32),
                                    C.POINTER(C.c_float)]),
    "dr_prmppi_create": (C.c_int, [C.POINTER(dr_env_config), C.POINTER(dr_prmppi_config), C.c_uint64, C.POINTER(C.c_float), C.c_int, C.c_void_p, C.POINTER(C.c_void_p)]),
    "dr_prmppi_destroy": (C.c_int, [C.c_void_p]),
    "dr_prmppi_step": (C.c_int, [C.c_void_p, C.POINTER(dr_sim_state), C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(dr_prmppi_info)]),
    "dr_gate_prmppi_create": (C.c_int, [C.POINTER(dr_gate_env_config), C.POINTER(dr_prmppi_config), C.c_uint64, C.POINTER(C.c_float), C.c_int, C.c_void_p,
                                        C.POINTER(C.c_void_p)]),
    "dr_gate_prmppi_step": (C.c_int, [C.c_void_p, C.POINTER(dr_gate_state), C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(dr_prmppi_info)]),
    "dr_gate_prmppi_debug_rollout": (C.c_int, [C.c_void_p, C.POINTER(dr_gate_state), C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "dr_prmppi_get_nominals": (C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_size_t]),
    "dr_prmppi_get_step": (C.c_uint64, [C.c_void_p]),
    "dr_prmppi_set_step": (C.c_int, [C.c_void_p, C.c_uint64]),
    "dr_prmppi_set_profiling": (C.c_int, [C.c_void_p, C.c_int]),
    "dr_prmppi_get_kernel_times": (C.c_int, [C.c_void_p, C.POINTER(C.c_char_p), C.POINTER(C.c_float), C.c_int, C.POINTER(C.c_int)]),
    "dr_prmppi_batch_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.c_void_p, C.POINTER(C.c_void_p)]),
    "dr_prmppi_batch_destroy": (C.c_int, [C.c_void_p]),
    "dr_prmppi_batch_step": (C.c_int, [C.c_void_p, C.POINTER(dr_sim_state), C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(dr_prmppi_info)]),
    "dr_prmppi_batch_step_dev": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "dr_prmppi_debug_noise": (C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_size_t, C.POINTER(C.c_int32)]),
    "dr_prmppi_debug_rollout": (C.c_int, [C.c_void_p, C.POINTER(dr_sim_state), C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "dr_mppi_rollout_costs_noalloc": (C.c_int, [C.POINTER(dr_env_config), C.POINTER(dr_mppi_config), C.c_uint64, C.c_uint64, C.POINTER(dr_sim_state),
                                                C.POINTER(C.c_float), C.c_void_p, C.c_void_p, C.c_void_p]),
    "dr_spline_matrix": (C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_int32), C.POINTER(C.c_float)]),
    "dr_mppi_nominal_grad": (C.c_int, [C.c_void_p, C.POINTER(dr_sim_state), C.POINTER(C.c_float), C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_void_p, C.c_int, C.c_void_p]),
    "dr_mppi_set_grad_refine": (C.c_int, [C.c_void_p, C.c_int, C.c_float, C.c_int]),
    "dr_mppi_set_shard": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "dr_mppi_shard_words": (C.c_int, [C.c_void_p, C.POINTER(C.c_size_t)]),
    "dr_mppi_shard_begin": (C.c_int, [C.c_void_p, C.POINTER(dr_sim_state), C.POINTER(C.c_float), C.c_void_p]),
    "dr_mppi_shard_update": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "dr_mppi_shard_finish": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(dr_mppi_info)]),
    "dr_mppi_batch_step_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "dr_mppi_batch_env_step_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_uint64, C.c_void_p]),
    "dr_track_grids": (C.c_int, [C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float),
                                 C.POINTER(C.c_float)]),
    "dr_debug_cp": (C.c_int, [C.POINTER(C.c_uint32), C.c_int, C.c_uint32, C.c_double, C.c_int, C.POINTER(C.c_double)]),
    "dr_debug_cp_host": (C.c_int, [C.POINTER(C.c_uint32), C.c_int, C.c_uint32, C.c_double, C.c_int, C.POINTER(C.c_double)]),
    "dr_env_step": (C.c_int, [C.POINTER(dr_env_config), C.c_int, C.POINTER(C.c_float), C.POINTER(dr_sim_state), C.POINTER(C.c_float), C.c_int, C.c_uint64, C.c_uint64, C.POINTER(C.c_int)]),
    "dr_projection_certificate": (C.c_int, [C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "dr_debug_project": (C.c_int, [C.POINTER(dr_env_config), C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int, C.c_int, C.POINTER(C.c_float),
                                   C.POINTER(C.c_float), C.POINTER(C.c_int32)]),
    "dr_gate_mppi_create": (C.c_int, [C.POINTER(dr_gate_env_config), C.POINTER(dr_mppi_config), C.c_uint64, C.POINTER(C.c_float), C.c_int, C.c_void_p, C.POINTER(C.c_void_p)]),
    "dr_gate_mppi_step": (C.c_int, [C.c_void_p, C.POINTER(dr_gate_state), C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(dr_mppi_info)]),
    "dr_gate_mppi_batch_step": (C.c_int, [C.c_void_p, C.POINTER(dr_gate_state), C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(dr_mppi_info)]),
    "dr_gate_mppi_debug_rollout": (C.c_int, [C.c_void_p, C.POINTER(dr_gate_state), C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_float)]),
    "dr_gate_mppi_debug_verify": (C.c_int, [C.c_void_p, C.POINTER(dr_gate_state), C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int, C.POINTER(C.c_uint32), C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "dr_gate_env_step": (C.c_int, [C.POINTER(dr_gate_env_config), C.c_int, C.POINTER(C.c_float), C.POINTER(dr_gate_state), C.POINTER(C.c_float), C.c_int, C.c_uint64, C.c_uint64, C.POINTER(C.c_int)]),
}

EXPORTED = sorted(_PROTOS)

_lib = None


class DrError(RuntimeError):
    def __init__(self, status: int, what: str):
        super().__init__(f"{what}: status {status} ({status_name(status)})")
        self.status = status


_STATUS_NAMES = {
    DR_OK: "ok",
    DR_ERR_INVALID_ARG: "invalid argument",
    DR_ERR_UNSUPPORTED: "unsupported configuration",
    DR_ERR_CUDA: "CUDA error",
    DR_ERR_OOM: "out of device memory",
    DR_ERR_NO_DEVICE: "no CUDA device",
    DR_ERR_TIMEOUT: "device wait timed out",
    DR_ERR_STATE: "invalid state",
}


def status_name(s: int) -> str:
    return _STATUS_NAMES.get(s, "unknown")


def lib(path: str | os.PathLike | None = None) -> C.CDLL:
    """Load libdrmppi.so (built by build.py). Raises if it is missing: there is no
    fallback implementation."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise FileNotFoundError(f"{p} not found: build it with __graft_entry__.build() (nvcc, sm_100a)")
    L = C.CDLL(str(p))
    for name, (res, args) in _PROTOS.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    if L.dr_abi_version() != DR_ABI_VERSION:
        raise RuntimeError(f"{p}: ABI version {L.dr_abi_version()}, these bindings expect {DR_ABI_VERSION}: rebuild it")
    if path is None:
        _lib = L
    return L


def check(status: int, what: str) -> None:
    if status != DR_OK:
        err = lib().dr_last_error()
        msg = err.decode() if err else ""
        raise DrError(status, f"{what} {msg}".strip())
