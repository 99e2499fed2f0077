"""ctypes declarations of the C ABI in include/twisty_b200.h.

Loads the in-tree library twisty_b200/libtwisty_b200.so (built by twisty_b200.build).
Importing this module never falls back to anything: a missing library raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtwisty_b200.so")

# twisty_status
OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_INVALID_CONFIG = 2
ERR_INFEASIBLE_GEOMETRY = 3
ERR_LUT_INVALID = 4
ERR_CUDA = 5
ERR_DEVICE_TIMEOUT = 6
ERR_IO = 7
ERR_UNSUPPORTED = 8
ERR_NO_DEVICE = 9
ERR_OUT_OF_MEMORY = 10

# twisty_form / twisty_lut_mode
FORM_PLAIN_FP32 = 0
FORM_COMPENSATED = 1
FORM_FP64 = 2
LUT_FAITHFUL = 0
LUT_FP64 = 1
LUT_EXTERNAL = 2
LUT_MULTI_DS = 3
TABLE_FIXED_NARROW = 0
TABLE_FIXED_WIDE = 1
TABLE_EXACT_BLEND = 2
TABLE_NONE = 3


class Vec3(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float)]


class BC(C.Structure):
    _fields_ = [("start_pos", Vec3), ("start_dir", Vec3), ("end_pos", Vec3), ("end_dir", Vec3),
                ("arclength", C.c_float)]


class Params(C.Structure):
    _fields_ = [
        ("struct_size", C.c_uint32),
        ("paths_to_generate", C.c_uint64),
        ("paths_to_skip", C.c_uint64),
        ("num_segments", C.c_uint32),
        ("bootstrap_seed", C.c_uint32),
        ("perturb_seed", C.c_uint32),
        ("weight_function", C.c_int32),
        ("perturb_method", C.c_int32),
        ("mu", C.c_float),
        ("eps", C.c_float),
        ("scatter", C.c_float),
        ("absorption", C.c_float),
        ("num_steps_int", C.c_uint32),
        ("num_curvature_steps", C.c_uint32),
        ("min_bound", C.c_float),
        ("max_bound", C.c_float),
        ("bias", C.c_float),
        ("form", C.c_int32),
        ("lut_mode", C.c_int32),
        ("max_sub_chain", C.c_uint32),
        ("max_angle", C.c_float),
        ("num_chains", C.c_uint32),
        ("device", C.c_int32),
        ("chain_offset", C.c_uint32),
        ("experiment_id", C.c_uint32),
        ("bootstrap_kind", C.c_int32),
        ("eval_end_shift", Vec3),
        ("comp_group", C.c_uint32),
        ("comp_spl", C.c_uint32),
        ("comp_warps", C.c_uint32),
        ("incremental_resync", C.c_uint32),
        ("comp_table_memory", C.c_uint32),
        ("fp64_check_chains", C.c_uint32),
    ]


class Result(C.Structure):
    _fields_ = [
        ("log10_weight", C.c_double),
        ("log10_normalizer", C.c_double),
        ("log10_mean_weight", C.c_double),
        ("rel_std_error", C.c_double),
        ("total_paths", C.c_uint64),
        ("failed_paths", C.c_uint64),
        ("clamped_curvatures", C.c_uint64),
        ("num_chains", C.c_uint32),
        ("steps_per_chain", C.c_uint32),
        ("total_ms", C.c_double),
        ("setup_ms", C.c_double),
        ("perturb_ms", C.c_double),
        ("weighting_ms", C.c_double),
        ("table_form", C.c_uint32),
        ("steep_bins", C.c_uint32),
        ("weight_error_bound", C.c_double),
        ("fp64_rel_error", C.c_double),
        ("fp64_check_chains", C.c_uint32),
        ("kernel_shape", C.c_uint32),
    ]


class LutInfo(C.Structure):
    _fields_ = [("min_curvature", C.c_float), ("max_curvature", C.c_float), ("curvature_step", C.c_float),
                ("min_segment_weight", C.c_float), ("max_segment_weight", C.c_float), ("ds", C.c_float),
                ("bins", C.c_uint32)]


class Experiment(C.Structure):
    _fields_ = [("bc", BC), ("num_segments", C.c_uint32), ("scatter", C.c_float), ("eps", C.c_float),
                ("paths", C.c_uint64)]


class Tuning(C.Structure):
    _fields_ = [("num_segments", C.c_uint32), ("bins", C.c_uint32), ("group", C.c_uint32), ("spl", C.c_uint32),
                ("warps", C.c_uint32), ("path_segments_per_s", C.c_double)]


NOALLOC_MAX_CHAINS = 16384
NOALLOC_MAX_BINS = 1 << 24


class NoAllocArgs(C.Structure):
    """twisty_noalloc_args: every pointer is device memory owned by the caller."""
    _fields_ = [("table", C.c_void_p), ("bins", C.c_uint32), ("min_curvature", C.c_float),
                ("max_curvature", C.c_float), ("curvature_step", C.c_float), ("init_segments", C.c_void_p),
                ("num_segments", C.c_uint32), ("arclength", C.c_float), ("absorption", C.c_float),
                ("seed", C.c_uint64), ("experiment_id", C.c_uint32), ("chain_offset", C.c_uint32),
                ("num_chains", C.c_uint32), ("paths", C.c_uint64), ("burn_in", C.c_uint32),
                ("max_sub_chain", C.c_uint32), ("max_angle", C.c_float), ("result", C.c_void_p)]


class NoAllocResult(C.Structure):
    _fields_ = [("log10_weight", C.c_double), ("rel_std_error", C.c_double), ("max_chain_log10", C.c_double),
                ("valid_paths", C.c_uint64), ("failed_paths", C.c_uint64), ("clamped_curvatures", C.c_uint64)]


class Shape(C.Structure):
    """twisty_shape: a kernel shape and its table placement."""
    _fields_ = [("group", C.c_uint32), ("spl", C.c_uint32), ("warps", C.c_uint32), ("table_in_l1", C.c_uint32),
                ("smem_bytes", C.c_uint32), ("batched", C.c_uint32)]


# (name, restype, argtypes): every entry point declared in include/twisty_b200.h
_P = C.c_void_p
SIGNATURES = [
    ("twisty_abi_version", C.c_int, []),
    ("twisty_status_string", C.c_char_p, [C.c_int]),
    ("twisty_params_init", None, [C.POINTER(Params)]),
    ("twisty_params_from_config", C.c_int, [C.c_char_p, C.c_int, C.POINTER(Params), C.POINTER(BC)]),
    ("twisty_create", C.c_int, [C.POINTER(Params), C.POINTER(_P)]),
    ("twisty_destroy", None, [_P]),
    ("twisty_last_error", C.c_char_p, [_P]),
    ("twisty_update_params", C.c_int, [_P, C.POINTER(Params)]),
    ("twisty_run", C.c_int, [_P, C.POINTER(BC), C.POINTER(Result)]),
    ("twisty_prepare", C.c_int, [_P, C.POINTER(BC)]),
    ("twisty_launch", C.c_int, [_P, _P]),
    ("twisty_collect", C.c_int, [_P, C.POINTER(Result)]),
    ("twisty_launch_kernel_count", C.c_uint32, [_P]),
    ("twisty_chain_results", C.c_int, [_P, _P, _P, C.c_uint32]),
    ("twisty_weight_histogram", C.c_int, [_P, C.POINTER(BC), C.c_double, C.c_double, C.c_uint32, _P]),
    ("twisty_run_batch", C.c_int, [_P, C.POINTER(Experiment), C.c_uint32, C.c_uint32, C.POINTER(Result)]),
    ("twisty_run_msegment", C.c_int, [_P, C.POINTER(BC), C.POINTER(Result)]),
    ("twisty_weight_paths", C.c_int, [_P, C.POINTER(BC), _P, C.c_uint64, C.c_int32, _P, _P, _P]),
    ("twisty_build_lut", C.c_int, [_P, C.c_float, _P, C.POINTER(LutInfo)]),
    ("twisty_set_lut", C.c_int, [_P, _P, C.POINTER(LutInfo)]),
    ("twisty_normalizer_log10", C.c_int, [_P, C.c_uint32, C.c_float, C.POINTER(BC), C.POINTER(C.c_double)]),
    ("twisty_bootstrap_curve", C.c_int, [C.POINTER(Params), C.POINTER(BC), _P]),
    ("twisty_min_arclength", C.c_float, [C.POINTER(BC), C.c_uint32]),
    ("twisty_set_initial_curve", C.c_int, [_P, _P, C.c_uint32]),
    ("twisty_export_paths", C.c_int, [_P, C.POINTER(BC), C.c_char_p, C.c_uint64, _P, _P, C.POINTER(C.c_uint64),
                                      C.POINTER(Result)]),
    ("twisty_adjoint", C.c_int, [_P, C.POINTER(BC), C.POINTER(Result), C.POINTER(C.c_double)]),
    ("twisty_adjoint_batch", C.c_int, [_P, C.POINTER(Experiment), C.c_uint32, C.POINTER(Result),
                                       C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    ("twisty_run_noalloc", C.c_int, [C.POINTER(NoAllocArgs), _P]),
    ("twisty_autotune", C.c_int, [_P, C.POINTER(BC), C.c_uint64, C.POINTER(Tuning)]),
    ("twisty_multi_ds_tables", C.c_int, [_P, C.c_float, C.c_float, C.c_uint32, C.c_char_p]),
    ("twisty_tuning_cache_save", C.c_int, [C.c_char_p]),
    ("twisty_tuning_cache_load", C.c_int, [C.c_char_p]),
    ("twisty_default_shape", C.c_int, [C.c_uint32, C.c_uint32, C.POINTER(Shape)]),
    ("twisty_measure_fp32_peak", C.c_int, [C.c_int, C.POINTER(C.c_double)]),
]

_lib = None


def load(path: str = LIB_PATH) -> C.CDLL:
    """Load the CUDA library; raises OSError when it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise OSError(f"{path} not found: build it with `python -m twisty_b200.build`")
        L = C.CDLL(path)
        for name, res, args in SIGNATURES:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib
