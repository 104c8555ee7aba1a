"""ctypes declarations of the C ABI in include/pct_api.h.

The engine is libpct_b200.so, built in-tree by pct_reconstruction_b200.build.  Loading fails
loudly when the library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libpct_b200.so"

# pct_status (include/pct_api.h)
PCT_OK, PCT_ERR_ARG, PCT_ERR_CUDA, PCT_ERR_OOB, PCT_ERR_TIMEOUT, PCT_ERR_STATE, PCT_ERR_NOMEM, PCT_ERR_IO = range(8)
PCT_HOST, PCT_DEVICE = 0, 1
PCT_RAM_LAK, PCT_SHEPP_LOGAN, PCT_UNFILTERED = 0, 1, 2
PCT_SC_HULL, PCT_MSC_HULL, PCT_SM_HULL, PCT_FBP_HULL = 0, 1, 2, 3
PCT_PRECISION_EXACT, PCT_PRECISION_MIXED, PCT_PRECISION_MIXED_COMPENSATED = 0, 1, 2
PCT_SCATTER_ATOMIC, PCT_SCATTER_DETERMINISTIC = 0, 1
PCT_SIGMOID, PCT_TANH, PCT_ATAN, PCT_ERF, PCT_LIN_OVER_ROOT = range(5)
PCT_MLP_PATH_CAP = 1312

_i32, _f64, _f32 = C.c_int32, C.c_double, C.c_float

CONFIG_FIELDS = [
    ("COLUMNS", _i32), ("ROWS", _i32), ("SLICES", _i32), ("NUM_VOXELS", _i32),
    ("VOXEL_WIDTH", _f64), ("VOXEL_HEIGHT", _f64), ("VOXEL_THICKNESS", _f64),
    ("RECON_CYL_RADIUS", _f64), ("RECON_CYL_HEIGHT", _f64),
    ("GANTRY_ANGLE_INTERVAL", _f64), ("SSD_T_SIZE", _f64), ("SSD_V_SIZE", _f64),
    ("T_BIN_SIZE", _f64), ("V_BIN_SIZE", _f64), ("ANGULAR_BIN_SIZE", _f64),
    ("T_BINS", _i32), ("V_BINS", _i32), ("ANGULAR_BINS", _i32), ("NUM_BINS", _i32),
    ("SIGMAS_TO_KEEP", _i32), ("SAMPLE_STD_DEV", _i32),
    ("SINOGRAM_FILTER", _i32), ("MEDIAN_FILTER_FBP", _i32),
    ("FBP_MED_FILTER_RADIUS", _i32), ("PATH_CTA_THREADS", _i32),
    ("SOURCE_RADIUS", _f64), ("FBP_THRESHOLD", _f64), ("RSP_AIR", _f64),
    ("SC_LOWER_THRESHOLD", _f64), ("SC_UPPER_THRESHOLD", _f64),
    ("MSC_LOWER_THRESHOLD", _f64), ("MSC_UPPER_THRESHOLD", _f64),
    ("SM_LOWER_THRESHOLD", _f64), ("SM_UPPER_THRESHOLD", _f64), ("SM_SCALE_THRESHOLD", _f64),
    ("MSC_DIFF_THRESH", _i32), ("ENDPOINTS_HULL", _i32),
    ("SC_ON", _i32), ("MSC_ON", _i32), ("SM_ON", _i32), ("PATH_ORDER_WINDOW", _i32),
    ("MLP_U_STEP", _f64), ("MIN_MLP_LENGTH", _i32),
    ("LAMBDA", _f32), ("DROP_BLOCK_SIZE", _i32), ("ITERATIONS", _i32),
    ("HISTORIES_PER_BLOCK", _i32),
    ("PRECISION", _i32), ("SCATTER_MODE", _i32), ("THREADS_PER_HISTORY", _i32),
    ("PATH_CHUNK_BLOCKS", _i32), ("EXACT_FAST_POINTS", _i32),
    ("DATA_IN_MM", _i32), ("USE_CONT_ANGLES", _i32),
    ("T_SHIFT", _f64), ("U_SHIFT", _f64), ("V_SHIFT", _f64),
    ("TVS_ON", _i32), ("TVS_OLD", _i32), ("TVS_FIRST", _i32), ("TVS_CONDITIONED", _i32),
    ("TVS_REPETITIONS", _i32), ("TVS_L_0", _i32),
    ("TVS_A", _f64), ("TVS_MIN_ETA", _f64), ("TV_THRESHOLD", _f64), ("TVS_SEED", C.c_int64),
    ("PROJECTION_ALGORITHM", _i32), ("PSI_SIGN", _i32), ("ETA", _f64),
    ("RECON_HISTORY_ORDERING", _i32), ("IDENTIFY_X_N_AIR", _i32), ("PRIME_OFFSET", C.c_int64),
    ("X_N_AIR_THRESHOLD", _f64),
    ("S_CURVE_ON", _i32), ("S_CURVE", _i32), ("DUAL_SIDED_S_CURVE", _i32), ("SIGMOID_MID_SHIFT", _i32),
    ("SIGMOID_STEEPNESS", _f64),
]


class pct_config(C.Structure):
    _fields_ = CONFIG_FIELDS


_P = C.c_void_p


class pct_histories(C.Structure):
    """Reconstruction histories, structure of arrays (B.h:1257-1271 order)."""
    _fields_ = [(name, _P) for name in (
        "x_entry", "y_entry", "z_entry", "x_exit", "y_exit", "z_exit",
        "xy_entry_angle", "xz_entry_angle", "xy_exit_angle", "xz_exit_angle",
        "WEPL", "first_MLP_voxel")]


HISTORY_FIELDS = [f[0] for f in pct_histories._fields_]


class pct_tracker_data(C.Structure):
    """Tracker hits (t/u/v on 4 planes), WEPL and the projection angle in degrees."""
    _fields_ = [(name, _P) for name in (
        "t_in_1", "t_in_2", "t_out_1", "t_out_2", "u_in_1", "u_in_2", "u_out_1", "u_out_2",
        "v_in_1", "v_in_2", "v_out_1", "v_out_2", "WEPL", "gantry_angle")]


TRACKER_FIELDS = [f[0] for f in pct_tracker_data._fields_]


class pct_projection_header(C.Structure):
    """Header of a projection data file (PCTD / PCTN, versions 0 and 1)."""
    _fields_ = [
        ("continuous", _i32), ("version", _i32), ("num_histories", _i32),
        ("projection_angle", _f32), ("beam_energy", _f32),
        ("generation_date", _i32), ("preprocess_date", _i32), ("has_angles", _i32),
        ("data_offset", C.c_int64),
        ("phantom_name", C.c_char * 256), ("data_source", C.c_char * 256),
        ("prepared_by", C.c_char * 256)]


class pct_projection_arrays(C.Structure):
    """One projection file's arrays in file order (t0..t3, v0..v3, u0..u3, WEPL, angles)."""
    _fields_ = [(name, _P) for name in (
        "t_in_1", "t_in_2", "t_out_1", "t_out_2", "v_in_1", "v_in_2", "v_out_1", "v_out_2",
        "u_in_1", "u_in_2", "u_out_1", "u_out_2", "WEPL", "projection_angle")]


PROJECTION_FIELDS = [f[0] for f in pct_projection_arrays._fields_]

# (name, restype, argtypes) for every symbol the header declares.
SIGNATURES = [
    ("pct_config_size", C.c_size_t, []),
    ("pct_config_default", None, [C.POINTER(pct_config)]),
    ("pct_config_set", C.c_int, [C.POINTER(pct_config), C.c_char_p, C.c_char_p]),
    ("pct_config_load", C.c_int, [C.POINTER(pct_config), C.c_char_p]),
    ("pct_config_finalize", C.c_int, [C.POINTER(pct_config)]),
    ("pct_create", C.c_int, [C.POINTER(pct_config), C.c_int, C.POINTER(_P)]),
    ("pct_destroy", None, [_P]),
    ("pct_status_string", C.c_char_p, [C.c_int]),
    ("pct_last_error", C.c_char_p, [_P]),
    ("pct_set_stream", C.c_int, [_P, _P]),
    ("pct_synchronize", C.c_int, [_P]),
    ("pct_set_reconstruction_histories", C.c_int, [_P, C.POINTER(pct_histories), C.c_int64, C.c_int]),
    ("pct_reconstruction_histories", C.c_int64, [_P]),
    ("pct_apply_history_sequence", C.c_int, [_P, C.c_int64]),
    ("pct_set_image", C.c_int, [_P, _P, C.c_int]),
    ("pct_get_image", C.c_int, [_P, _P, C.c_int]),
    ("pct_drop_full_tx_iteration", C.c_int, [_P, C.c_int]),
    ("pct_drop_gpu", C.c_int, [_P]),
    ("pct_ntvs_iteration", C.c_int, [_P, C.c_int]),
    ("pct_total_variation", C.c_int, [_P, C.POINTER(C.c_double)]),
    ("pct_tvs_L", C.c_int, [_P, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    ("pct_calculate_x_update", C.c_int, [_P, C.c_int64, C.c_int64]),
    ("pct_set_path_storage_limit", C.c_int, [_P, C.c_int64]),
    ("pct_profile_drop_iteration", C.c_int, [_P, C.POINTER(C.c_double), C.POINTER(C.c_int64)]),
    ("pct_path_storage_superblocks", C.c_int, [_P]),
    ("pct_set_path_reuse", C.c_int, [_P, C.c_int]),
    ("pct_image_update", C.c_int, [_P]),
    ("pct_mlp_paths", C.c_int, [_P, C.c_int64, C.c_int64, C.c_int32, _P, _P, _P, _P, C.c_int]),
    ("pct_drop_block_update_noalloc", C.c_int, [_P, C.POINTER(pct_histories), C.c_int64, _P]),
    ("pct_mlp_precision", C.c_int, [_P, C.c_int64, C.c_int64, _P, _P, _P, _P, C.c_int]),
    ("pct_load_tracker_data", C.c_int, [_P, C.POINTER(pct_tracker_data), C.c_int64, C.c_int, C.c_int]),
    ("pct_recon_volume_intersections", C.c_int, [_P]),
    ("pct_binning", C.c_int, [_P]),
    ("pct_hull_detection", C.c_int, [_P]),
    ("pct_calculate_means", C.c_int, [_P]),
    ("pct_sum_squared_deviations", C.c_int, [_P]),
    ("pct_calculate_standard_deviations", C.c_int, [_P]),
    ("pct_statistical_cuts", C.c_int, [_P]),
    ("pct_construct_sinogram", C.c_int, [_P]),
    ("pct_FBP", C.c_int, [_P]),
    ("pct_hull_detection_finish", C.c_int, [_P]),
    ("pct_hull_selection", C.c_int, [_P]),
    ("pct_define_initial_iterate", C.c_int, [_P]),
    ("pct_reconstruction_cuts", C.c_int, [_P]),
    ("pct_preprocessing", C.c_int, [_P, C.POINTER(pct_tracker_data), C.c_int64, C.c_int, C.c_int]),
    ("pct_set_history_vectors", C.c_int, [_P, C.POINTER(pct_histories), C.c_int64, C.c_int]),
    ("pct_array_length", C.c_int64, [_P, C.c_char_p]),
    ("pct_get_array", C.c_int, [_P, C.c_char_p, _P, C.c_int64, C.c_int]),
    ("pct_set_array", C.c_int, [_P, C.c_char_p, _P, C.c_int64, C.c_int]),
    ("pct_read_projection_header", C.c_int, [C.c_char_p, C.POINTER(pct_projection_header)]),
    ("pct_read_projection_file", C.c_int, [C.c_char_p, C.c_int64, C.POINTER(pct_projection_arrays),
                                           C.POINTER(pct_projection_header)]),
    ("pct_write_projection_file", C.c_int, [C.c_char_p, C.POINTER(pct_projection_header),
                                            C.POINTER(pct_projection_arrays), C.c_int64]),
    ("pct_load_projection_data", C.c_int, [_P, C.c_char_p, C.POINTER(C.c_int64)]),
    ("pct_preprocessing_from_files", C.c_int, [_P, C.c_char_p]),
    ("pct_batch_create", C.c_int, [C.POINTER(_P), C.c_int, C.POINTER(_P)]),
    ("pct_batch_destroy", None, [_P]),
    ("pct_batch_drop_iteration", C.c_int, [_P, C.c_int]),
    ("pct_batch_synchronize", C.c_int, [_P]),
    ("pct_batch_last_error", C.c_char_p, [_P]),
    ("pct_batch_stream", _P, [_P]),
    ("pct_export_preprocessed", C.c_int, [_P, C.c_char_p]),
    ("pct_import_preprocessed", C.c_int, [_P, C.c_char_p]),
    ("pct_get_counters", C.c_int, [_P, C.POINTER(C.c_int64)]),
    ("pct_reset_counters", C.c_int, [_P]),
    ("pct_get_s_curve", C.c_int, [_P, _P, C.c_int32]),
    ("pct_config_last_error", C.c_char_p, []),
    ("pct_kernel_launches", C.c_int64, [_P]),
    ("pct_selftest_powf_square", C.c_int, [C.c_int64, C.c_uint64, C.POINTER(C.c_int64)]),
    ("pct_selftest_powf_square_max_ulp", C.c_int, [C.POINTER(C.c_int64)]),
    ("pct_fp64_fma_rate", C.c_int, [C.c_int, C.POINTER(C.c_double)]),
    ("pct_mlp_steps", C.c_int, [_P, C.c_int64, C.c_int64, _P, C.c_int]),
    ("pct_set_l2_window", C.c_int, [_P, C.c_int]),
    ("pct_autotune", C.c_int, [_P, C.POINTER(C.c_int32)]),
    ("pct_autotune_schedule", C.c_int, [_P, C.POINTER(C.c_int32)]),
    ("pct_stage_reconstruction_histories", C.c_int, [_P, C.POINTER(pct_histories), C.c_int64, C.c_int]),
    ("pct_use_staged_histories", C.c_int, [_P]),
    ("pct_unet_create", C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int64, C.c_int, C.POINTER(_P)]),
    ("pct_unet_destroy", C.c_int, [_P]),
    ("pct_unet_last_error", C.c_char_p, [_P]),
    ("pct_unet_param_count", C.c_int, [_P, C.POINTER(C.c_int64)]),
    ("pct_unet_get_params", C.c_int, [_P, _P, C.c_int64]),
    ("pct_unet_set_params", C.c_int, [_P, _P, C.c_int64]),
    ("pct_unet_forward", C.c_int, [_P, _P, _P, _P]),
    ("pct_unet_gradients", C.c_int, [_P, _P, _P, _P, _P, C.POINTER(C.c_double)]),
    ("pct_unet_train_step", C.c_int, [_P, _P, _P, _P, C.c_float, C.POINTER(C.c_double)]),
    ("pct_learned_initial_iterate", C.c_int, [_P, _P]),
    ("pct_conv3d_bf16", C.c_int, [_P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _P, C.c_int, _P, _P, _P,
                                  C.c_int, _P, _P]),
    ("pct_conv3d_bf16_wgrad", C.c_int, [_P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _P, C.c_int, _P, _P]),
]

_lib = None


def load_library(path: Path | str | None = None) -> C.CDLL:
    """Load libpct_b200.so and declare its signatures.  Raises if it is missing."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(
            f"{p} is missing: build the CUDA engine first (python -m pct_reconstruction_b200.build). "
            "There is no CPU fallback.")
    lib = C.CDLL(str(p))
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.pct_config_size() != C.sizeof(pct_config):
        raise RuntimeError("pct_config layout mismatch between include/pct_api.h and _abi.py")
    if path is None:
        _lib = lib
    return lib
