"""Loader of the compiled C ABI (riptide_b200/_riptide_b200.so, declared in
include/riptide_b200.h).

There is no CPU fallback: if the library or a CUDA device is missing, every entry point
raises RuntimeError.
"""
import ctypes
import os
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_riptide_b200.so")

RT_OK, RT_EINVAL, RT_ECUDA, RT_ENOMEM, RT_ETIMEOUT, RT_EINTERNAL, RT_EIO = 0, 1, 2, 3, 4, 5, 6
RT_SAMPLES_F32, RT_SAMPLES_U8, RT_SAMPLES_I8 = 0, 1, 2
RT_FAULT_NONE, RT_FAULT_STAGE_WAIT, RT_FAULT_ALLOC = 0, 1, 2

_sz = ctypes.c_size_t
_vp = ctypes.c_void_p
_d = ctypes.c_double
_u64p = ctypes.POINTER(ctypes.c_uint64)

# name -> (restype, argtypes); mirrors include/riptide_b200.h
SIGNATURES = {
    "rt_last_error": (ctypes.c_char_p, []),
    "rt_version": (ctypes.c_int, []),
    "rt_rollback": (ctypes.c_int, [_vp, _sz, _sz, _vp, _vp]),
    "rt_fused_rollback_add": (ctypes.c_int, [_vp, _vp, _sz, _sz, _vp, _vp]),
    "rt_circular_prefix_sum": (ctypes.c_int, [_vp, _sz, _sz, _vp, _vp]),
    "rt_ffa2": (ctypes.c_int, [_vp, _sz, _sz, _vp, _vp]),
    "rt_ffa2_noalloc": (ctypes.c_int, [_vp, _sz, _sz, _vp, _vp]),
    "rt_benchmark_ffa2": (ctypes.c_int, [_sz, _sz, _sz, ctypes.POINTER(_d)]),
    "rt_snr2": (ctypes.c_int, [_vp, _sz, _sz, _u64p, _sz, ctypes.c_float, _vp, _vp]),
    "rt_downsample": (ctypes.c_int, [_vp, _sz, _d, _vp, _vp]),
    "rt_downsampled_size": (_sz, [_sz, _d]),
    "rt_running_median": (ctypes.c_int, [_vp, _sz, _sz, _vp, _vp]),
    "rt_fast_running_median": (ctypes.c_int, [_vp, _sz, _sz, _sz, _vp, _vp]),
    "rt_deredden": (ctypes.c_int, [_vp, _sz, _d, _d, _sz, _vp, _vp]),
    "rt_normalise": (ctypes.c_int, [_vp, _sz, _vp, _vp]),
    "rt_periodogram_length": (ctypes.c_int, [_sz, _d, _d, _d, _sz, _sz, ctypes.POINTER(_sz)]),
    "rt_periodogram": (ctypes.c_int, [_vp, _sz, _d, _u64p, _sz, _d, _d, _sz, _sz, _vp, _vp, _vp, _vp]),
    "rt_periodogram_plain": (ctypes.c_int, [_vp, _sz, _d, _u64p, _sz, _d, _d, _sz, _sz, _vp, _vp, _vp, _vp]),
    "rt_search_plan_create": (ctypes.c_int, [_u64p, _sz, _vp, _u64p, _sz, ctypes.POINTER(_vp)]),
    "rt_search_plan_rows": (ctypes.c_int, [_vp, _u64p]),
    "rt_search_plan_create_tuned": (ctypes.c_int, [_u64p, _sz, _vp, _u64p, _sz, _vp, ctypes.POINTER(_vp)]),
    "rt_search_plan_create_rules": (ctypes.c_int, [_u64p, _sz, _vp, _u64p, _sz, _vp, _vp, _sz, ctypes.POINTER(_vp)]),
    "rt_search_plan_stats": (ctypes.c_int, [_vp, _vp]),
    "rt_search_run": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "rt_search_check": (ctypes.c_int, [_vp, _vp]),
    "rt_search_set_timing": (ctypes.c_int, [_vp, ctypes.c_int]),
    "rt_search_last_timing": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_int)]),
    "rt_search_set_profiling": (ctypes.c_int, [_vp, ctypes.c_int]),
    "rt_search_phase_cycles": (ctypes.c_int, [_vp, _u64p, ctypes.c_int]),
    "rt_search_plan_destroy": (None, [_vp]),
    "rt_search_set_wait_limit": (ctypes.c_int, [_vp, ctypes.c_longlong]),
    "rt_search_inject_fault": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int]),
    "rt_search_plan_prepare": (ctypes.c_int, [_vp]),
    "rt_search_plan_transforms": (ctypes.c_int, [_vp, _vp]),
    "rt_search_normalisation": (ctypes.c_int, [_vp, ctypes.POINTER(_d), ctypes.POINTER(_d), _vp]),
    "rt_search_backward_rows": (ctypes.c_int, [_vp, _vp, _vp, _vp, _sz, _vp]),
    "rt_peak_segments": (ctypes.c_int, [_vp, _vp, _sz, _u64p, _sz, ctypes.POINTER(_d), _d, _d, _u64p, _vp, _vp, _vp]),
    "rt_peak_select": (ctypes.c_int, [_vp, _vp, _sz, _u64p, _sz, _vp, _sz, _d, _vp, _sz, ctypes.POINTER(_sz), _vp]),
    "rt_snr2_backward": (ctypes.c_int, [_vp, _sz, _sz, _u64p, _sz, ctypes.c_float, _vp, _vp, _vp]),
    "rt_ffa2_transpose": (ctypes.c_int, [_vp, _sz, _sz, _vp, _vp]),
    "rt_downsample_adjoint": (ctypes.c_int, [_vp, _sz, _d, _vp, _vp]),
    "rt_normalise_adjoint": (ctypes.c_int, [_vp, _vp, _sz, _d, _vp, _vp]),
    "rt_search_set_graph": (ctypes.c_int, [_vp, ctypes.c_int]),
    "rt_fold_shape": (ctypes.c_int, [_sz, _d, _d, _sz, ctypes.c_longlong, ctypes.POINTER(_sz), ctypes.POINTER(ctypes.c_int)]),
    "rt_fold": (ctypes.c_int, [_vp, _sz, _d, _d, _sz, ctypes.c_longlong, _vp, _vp]),
    "rt_fold_batched": (ctypes.c_int, [_vp, _sz, _d, _vp, _vp, _vp, _sz, _u64p, _vp, _vp]),
    "rt_file_size": (ctypes.c_int, [ctypes.c_char_p, _u64p]),
    "rt_read_file": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_uint64, ctypes.c_uint64, _vp, ctypes.c_int]),
    "rt_samples_to_f32": (ctypes.c_int, [_vp, ctypes.c_int, _sz, _vp, _vp]),
    "rt_ingest_files": (ctypes.c_int, [ctypes.POINTER(ctypes.c_char_p), _u64p, _u64p, ctypes.POINTER(ctypes.c_int), _sz, _vp, _vp, _sz, ctypes.c_int, _vp]),
    "rt_search_graph_captures": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int)]),
    "rt_search_pipeline_create": (ctypes.c_int, [_u64p, _sz, _vp, _u64p, _sz, _sz, ctypes.POINTER(_vp)]),
    "rt_search_pipeline_rows": (ctypes.c_int, [_vp, _u64p]),
    "rt_search_pipeline_chunks": (ctypes.c_int, [_vp, ctypes.POINTER(_sz)]),
    "rt_search_pipeline_run": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "rt_search_pipeline_check": (ctypes.c_int, [_vp, _vp]),
    "rt_search_pipeline_destroy": (None, [_vp]),
}


class SearchConfig(ctypes.Structure):
    _fields_ = [
        ("tsamp", ctypes.c_double),
        ("period_min", ctypes.c_double),
        ("period_max", ctypes.c_double),
        ("bins_min", ctypes.c_uint64),
        ("bins_max", ctypes.c_uint64),
        ("deredden", ctypes.c_int),
        ("rmed_width", ctypes.c_double),
        ("rmed_minpts", ctypes.c_uint64),
        ("already_normalised", ctypes.c_int),
    ]


class PlanStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in (
        "num_trials", "num_cycles", "num_transforms", "num_work_items", "num_multistage",
        "total_rows", "total_samples", "downsampled_samples", "folded_samples",
        "scrunch_factor")]


class TileRule(ctypes.Structure):
    _fields_ = [("rows_min", ctypes.c_uint32), ("rows_max", ctypes.c_uint32),
                ("bins_min", ctypes.c_uint32), ("bins_max", ctypes.c_uint32),
                ("rows_fraction", ctypes.c_double), ("snr_threads", ctypes.c_int),
                ("max_levels", ctypes.c_int)]


class SearchTuning(ctypes.Structure):
    _fields_ = [("rows_fraction", ctypes.c_double), ("snr_threads", ctypes.c_int),
                ("lag_items", ctypes.c_int), ("rows_fraction_deep", ctypes.c_double)]


class SearchTransform(ctypes.Structure):
    _fields_ = [("trial", ctypes.c_uint32), ("cycle", ctypes.c_uint32), ("bins", ctypes.c_uint32),
                ("rows", ctypes.c_uint32), ("rows_eval", ctypes.c_uint32),
                ("out_row", ctypes.c_uint64), ("factor", ctypes.c_double), ("tau", ctypes.c_double),
                ("stdnoise", ctypes.c_float)]


class RiptideError(RuntimeError):
    """A CUDA or device-side failure reported by the library."""


_lib = None
_lock = threading.Lock()


def load():
    """The loaded C library (ctypes.CDLL). Raises RuntimeError if it cannot be loaded."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"riptide_b200 CUDA library not built ({LIB_PATH} missing); run "
                "`python -c 'import __graft_entry__ as g; g.build()'` or `make -C riptide_b200/csrc`")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def check(status):
    """Raise the Python exception matching a C ABI status code."""
    if status == RT_OK:
        return
    msg = load().rt_last_error().decode(errors="replace")
    if status == RT_EINVAL:
        raise ValueError(msg)
    if status == RT_ENOMEM:
        raise MemoryError(msg)
    if status == RT_EIO:
        raise OSError(msg)
    raise RiptideError(f"[status {status}] {msg}")


def u64_array(values):
    """Contiguous uint64 numpy array and a ctypes pointer to it (keep the array alive)."""
    a = np.ascontiguousarray(np.asarray(values, dtype=np.uint64).ravel())
    return a, a.ctypes.data_as(_u64p)
