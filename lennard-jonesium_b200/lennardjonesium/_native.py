"""ctypes binding of the engine's C ABI (include/lj_gpu.h).

The library is lib/liblj_gpu.so beside this package, built by
lennard-jonesium_b200/build.py.  There is no fallback: if the library is
missing or a GPU call fails, the call raises.
"""

import ctypes
import pathlib

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE.parent / "lib" / "liblj_gpu.so"

LJ_OK, LJ_ERR_ARG, LJ_ERR_CUDA, LJ_ERR_NONFINITE, LJ_ERR_TIMEOUT, LJ_ERR_CAPACITY = range(6)
LJ_PRECISION_FP64, LJ_PRECISION_MIXED = 0, 1
LJ_FORCE_NONE, LJ_FORCE_LJ, LJ_FORCE_CONSTANT = 0, 1, 2


class Params(ctypes.Structure):
    _fields_ = [
        ("particle_count", ctypes.c_int),
        ("box", ctypes.c_double * 3),
        ("cutoff_distance", ctypes.c_double),
        ("time_delta", ctypes.c_double),
        ("precision", ctypes.c_int),
        ("force_kind", ctypes.c_int),
        ("force_strength", ctypes.c_double),
        ("periodic", ctypes.c_int),
        ("device", ctypes.c_int),
        ("skin", ctypes.c_double),
        ("neighbor_capacity", ctypes.c_int),
        ("force_block", ctypes.c_int),
        ("mixed_per_pair", ctypes.c_int),
    ]


class Thermo(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in (
        "time", "kinetic_energy", "potential_energy", "total_energy", "virial", "temperature",
        "mean_square_displacement")]


class Stats(ctypes.Structure):
    _fields_ = [
        ("steps", ctypes.c_longlong),
        ("list_builds", ctypes.c_longlong),
        ("neighbor_capacity", ctypes.c_int),
        ("list_cells", ctypes.c_int * 3),
        ("max_neighbors", ctypes.c_int),
        ("small_box", ctypes.c_int),
        ("skin", ctypes.c_double),
        ("kernel_launches", ctypes.c_longlong),
    ]


class PhaseTimes(ctypes.Structure):
    _fields_ = [("kick_drift_ms", ctypes.c_double), ("rebuild_ms", ctypes.c_double),
                ("force_ms", ctypes.c_double), ("finalize_ms", ctypes.c_double),
                ("steps", ctypes.c_longlong), ("rebuilds", ctypes.c_longlong)]


class SimConfig(ctypes.Structure):
    _fields_ = [
        ("temperature", ctypes.c_double), ("density", ctypes.c_double),
        ("particle_count", ctypes.c_int), ("random_seed", ctypes.c_uint),
        ("cutoff_distance", ctypes.c_double), ("time_delta", ctypes.c_double),
        ("eq_name", ctypes.c_char_p), ("eq_tolerance", ctypes.c_double),
        ("eq_sample_size", ctypes.c_int), ("eq_adjustment_interval", ctypes.c_int),
        ("eq_steady_state_time", ctypes.c_int), ("eq_timeout", ctypes.c_int),
        ("ob_name", ctypes.c_char_p), ("ob_tolerance", ctypes.c_double),
        ("ob_sample_size", ctypes.c_int), ("ob_observation_interval", ctypes.c_int),
        ("ob_observation_count", ctypes.c_int),
        ("event_log", ctypes.c_char_p), ("thermodynamic_log", ctypes.c_char_p),
        ("observation_log", ctypes.c_char_p), ("snapshot_log", ctypes.c_char_p),
        ("precision", ctypes.c_int), ("device", ctypes.c_int),
    ]


class SimResult(ctypes.Structure):
    _fields_ = [("time_steps", ctypes.c_longlong), ("outcome", ctypes.c_int),
                ("observations", ctypes.c_int), ("seconds", ctypes.c_double)]


class BatchSystem(ctypes.Structure):
    _fields_ = [("particle_count", ctypes.c_int), ("box", ctypes.c_double * 3),
                ("time_delta", ctypes.c_double), ("skin", ctypes.c_double)]


class AdjParams(ctypes.Structure):
    _fields_ = [("particle_count", ctypes.c_int), ("box", ctypes.c_double * 3),
                ("time_delta", ctypes.c_double), ("steps", ctypes.c_int),
                ("checkpoint_every", ctypes.c_int), ("epsilon", ctypes.c_double),
                ("sigma", ctypes.c_double), ("cutoff_sigma", ctypes.c_double),
                ("device", ctypes.c_int)]


class Observation(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in (
        "temperature", "density", "total_energy", "pressure", "specific_heat", "diffusion_coefficient")]


class BatchTuning(ctypes.Structure):
    _fields_ = [("skin", ctypes.c_double), ("force_block", ctypes.c_int), ("list_cells_per_block", ctypes.c_int),
                ("ms_per_step", ctypes.c_double)]


class LJError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, status, message):
        super().__init__(f"{message} (status {status})")
        self.status = status


_lib = None

# name -> (restype, argtypes); every symbol include/lj_gpu.h declares.
P = ctypes.c_void_p
SIGNATURES = {
    "lj_gpu_default_params": (None, [P]),
    "lj_gpu_create": (ctypes.c_int, [P, P]),
    "lj_gpu_destroy": (ctypes.c_int, [P]),
    "lj_gpu_last_error": (ctypes.c_char_p, [P]),
    "lj_gpu_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "lj_gpu_upload_state": (ctypes.c_int, [P, P, P, P, P, ctypes.c_int, ctypes.c_double,
                                           ctypes.c_double, ctypes.c_double]),
    "lj_gpu_download_state": (ctypes.c_int, [P, P, P, P, P, ctypes.c_int, P, P, P]),
    "lj_gpu_compute_forces": (ctypes.c_int, [P, P, P]),
    "lj_gpu_step": (ctypes.c_int, [P, ctypes.c_int, P]),
    "lj_gpu_measure": (ctypes.c_int, [P, P]),
    "lj_gpu_scale_velocities": (ctypes.c_int, [P, ctypes.c_double]),
    "lj_gpu_set_temperature": (ctypes.c_int, [P, ctypes.c_double, P]),
    "lj_gpu_debug_cells": (ctypes.c_int, [P, P, P, P, P]),
    "lj_gpu_debug_pairs": (ctypes.c_longlong, [P, ctypes.c_longlong, P, P, P, P]),
    "lj_gpu_rdf": (ctypes.c_int, [P, ctypes.c_int, ctypes.c_double, P]),
    "lj_gpu_rdf_accumulate": (ctypes.c_int, [P, ctypes.c_int, ctypes.c_double]),
    "lj_gpu_rdf_read": (ctypes.c_int, [P, P, P]),
    "lj_gpu_rdf_reset": (ctypes.c_int, [P]),
    "lj_gpu_get_stats": (ctypes.c_int, [P, P]),
    "lj_gpu_window_stats": (ctypes.c_int, [P, ctypes.c_int, ctypes.c_double, P]),
    "lj_window_stats_host": (ctypes.c_int, [P, ctypes.c_int, ctypes.c_int, ctypes.c_double, P]),
    "lj_batch_window_stats": (ctypes.c_int, [P, ctypes.c_int, P, P]),
    "lj_gpu_trajectory_open": (ctypes.c_int, [P, ctypes.c_char_p, ctypes.c_int]),
    "lj_gpu_trajectory_close": (ctypes.c_int, [P, P]),
    "lj_gpu_stream": (ctypes.c_void_p, [P]),
    "lj_gpu_step_async": (ctypes.c_int, [P, ctypes.c_int]),
    "lj_gpu_synchronize": (ctypes.c_int, [P]),
    "lj_gpu_step_timed": (ctypes.c_int, [P, ctypes.c_int, P]),
    "lj_gpu_autotune": (ctypes.c_int, [P, P, P, ctypes.c_int, ctypes.c_int, P, P]),
    "lj_gpu_fma_peaks": (ctypes.c_int, [ctypes.c_int, P, P]),
    "lj_gpu_rdf_noalloc": (ctypes.c_int, [P, ctypes.c_int, P, ctypes.c_int, ctypes.c_double, P, P]),
    "lj_sim_run": (ctypes.c_int, [P, ctypes.c_int, P]),
    "lj_sim_run_batch": (ctypes.c_int, [P, ctypes.c_int, ctypes.c_int, P]),
    "lj_format_double": (ctypes.c_int, [ctypes.c_double, ctypes.c_char_p, ctypes.c_int]),
    "lj_pair_along_z": (ctypes.c_int, [ctypes.c_double, ctypes.c_double, P]),
    "lj_batch_create": (ctypes.c_int, [P, ctypes.c_int, ctypes.c_double, ctypes.c_int, P]),
    "lj_batch_destroy": (ctypes.c_int, [P]),
    "lj_batch_last_error": (ctypes.c_char_p, [P]),
    "lj_batch_upload_system": (ctypes.c_int, [P, ctypes.c_int, P, P, ctypes.c_int]),
    "lj_batch_download_system": (ctypes.c_int, [P, ctypes.c_int, P, P, P, ctypes.c_int]),
    "lj_batch_set_active": (ctypes.c_int, [P, ctypes.c_int, ctypes.c_int]),
    "lj_batch_step": (ctypes.c_int, [P, ctypes.c_int, P]),
    "lj_batch_set_iteration_limit": (ctypes.c_int, [P, ctypes.c_int]),
    "lj_batch_set_force_block": (ctypes.c_int, [P, ctypes.c_int]),
    "lj_batch_set_list_tile": (ctypes.c_int, [P, ctypes.c_int]),
    "lj_batch_autotune": (ctypes.c_int, [P, ctypes.c_int, ctypes.c_double, ctypes.c_int, P, P, ctypes.c_int,
                                         ctypes.c_int, P]),
    "lj_batch_measure": (ctypes.c_int, [P, P]),
    "lj_batch_set_temperature": (ctypes.c_int, [P, ctypes.c_int, ctypes.c_double, P]),
    "lj_batch_info": (ctypes.c_int, [P, P, P, P]),
    "lj_adj_create": (ctypes.c_int, [P, P]),
    "lj_adj_destroy": (ctypes.c_int, [P]),
    "lj_adj_last_error": (ctypes.c_char_p, [P]),
    "lj_adj_set_potential": (ctypes.c_int, [P, ctypes.c_double, ctypes.c_double]),
    "lj_adj_forward": (ctypes.c_int, [P, P, P, ctypes.c_int, P, P]),
    "lj_adj_backward": (ctypes.c_int, [P, ctypes.c_double, ctypes.c_double, P, P, ctypes.c_int, P, P]),
    "lj_initial_condition": (ctypes.c_int, [ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                            ctypes.c_uint, P, P, P]),
}


def lib():
    """Load the engine library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python lennard-jonesium_b200/build.py`")
        L = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status, ctx=None):
    if status != LJ_OK:
        L = lib()
        msg = L.lj_gpu_last_error(ctx).decode() if ctx else ""
        if not msg:
            msg = L.lj_gpu_status_string(status).decode()
        raise LJError(status, msg)
