"""ctypes binding of libsupertrack_b200.so (the C ABI declared in include/supertrack_b200.h).

The shared library is built in-tree (``make -C supertrack_b200``); importing this module fails
loudly when it is missing, because there is no CPU fallback for the GPU path.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsupertrack_b200.so")

ST_OK = 0
STATUS_NAMES = {
    0: "ST_OK", 1: "ST_ERR_INVALID_ARGUMENT", 2: "ST_ERR_BAD_GEOMETRY",
    3: "ST_ERR_BAD_HISTOGRAM", 4: "ST_ERR_CUDA", 5: "ST_ERR_OUT_OF_MEMORY",
    6: "ST_ERR_CAPACITY", 7: "ST_ERR_NONFINITE_EDEP", 8: "ST_ERR_DEVICE_OVERFLOW",
    9: "ST_ERR_NOT_FOUND", 10: "ST_ERR_STATE", 11: "ST_ERR_IO", 12: "ST_ERR_CONFIG",
    13: "ST_ERR_NO_DEVICE", 14: "ST_ERR_DEVICE_WAIT",
}
for _v, _n in STATUS_NAMES.items():
    globals()[_n] = _v

ST_ZSHIFT_PLUS, ST_ZSHIFT_MINUS, ST_ZSHIFT_NONE = 0, 1, 2
ST_HIST_LIN, ST_HIST_LOG = 0, 1
ST_RUN_BATCHED, ST_RUN_PLAIN = 0, 1


class StError(RuntimeError):
    """A C-ABI call returned a status other than ST_OK."""

    def __init__(self, status: int, what: str, detail: str = ""):
        self.status = status
        name = STATUS_NAMES.get(status, str(status))
        msg = f"{what}: {name}"
        if detail:
            msg += f" ({detail})"
        super().__init__(msg)


class st_geometry(C.Structure):
    _fields_ = [("scoring_region_length", C.c_double), ("scoring_region_half_length", C.c_double),
                ("greatest_sphere_offset", C.c_double), ("num_spheres_linear", C.c_int32),
                ("reserved", C.c_int32), ("sphere_diameter", C.c_double),
                ("sphere_radius", C.c_double)]


class st_track_view(C.Structure):
    _fields_ = [("x", C.c_void_p), ("y", C.c_void_p), ("z", C.c_void_p), ("edep", C.c_void_p),
                ("n", C.c_int64), ("on_device", C.c_int32), ("reserved", C.c_int32)]


class st_job_desc(C.Structure):
    _fields_ = [("half_length", C.c_double), ("sphere_diameter", C.c_double),
                ("zshift", C.c_int32), ("shift_track", C.c_int32),
                ("n_oversamples", C.c_uint32), ("hist_id", C.c_int32),
                ("seed", C.c_uint64), ("track_id", C.c_uint64)]


class st_job_stats(C.Structure):
    _fields_ = [("hits", C.c_uint64), ("spheres", C.c_uint64), ("binned", C.c_uint64),
                ("inbox", C.c_uint64), ("grid_exponent", C.c_int32), ("status", C.c_int32)]


class st_sphere(C.Structure):
    _fields_ = [("key", C.c_uint64), ("y", C.c_double), ("os", C.c_int32), ("job", C.c_int32)]


class st_completion(C.Structure):
    _fields_ = [("tag", C.c_uint64), ("status", C.c_int32), ("batch", C.c_int32),
                ("submit_ns", C.c_int64), ("start_ns", C.c_int64), ("done_ns", C.c_int64)]


class st_tune_result(C.Structure):
    _fields_ = [("default_ms", C.c_double), ("best_ms", C.c_double), ("item_cost", C.c_int64),
                ("chunk_windows", C.c_int32), ("max_helpers", C.c_int32),
                ("share_divisor", C.c_int32), ("table_slots", C.c_int32), ("trials", C.c_int32),
                ("sort_deposits", C.c_int32), ("flag_cells_limit", C.c_int64)]


class st_run_info(C.Structure):
    _fields_ = [("n_tracks", C.c_int64), ("n_oversamples", C.c_int64),
                ("n_effective", C.c_int64), ("random_seed", C.c_int64),
                ("deposits", C.c_int64), ("nbins", C.c_int32), ("reserved", C.c_int32)]


class st_task(C.Structure):
    _fields_ = [("entry", C.c_int64), ("exit", C.c_int64), ("seed", C.c_int64),
                ("thread_id", C.c_int32), ("file_ordinal", C.c_int32),
                ("n_oversamples", C.c_int32), ("track_in_file", C.c_int32)]


# (name, restype, argtypes) of every exported symbol; the CPU tests check each one resolves.
SIGNATURES = [
    ("st_status_string", C.c_char_p, [C.c_int]),
    ("st_version", C.c_char_p, []),
    ("st_geometry_make", C.c_int, [C.c_double, C.c_double, C.POINTER(st_geometry)]),
    ("st_hist_edges", C.c_int, [C.c_int32, C.c_int32, C.c_float, C.c_float, C.c_void_p]),
    ("st_philox4x32_10", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("st_oversample_shifts", C.c_int, [C.POINTER(st_geometry), C.c_int32, C.c_uint64, C.c_uint64,
                                       C.c_uint32, C.c_uint32, C.c_void_p]),
    ("st_grid_exponent", C.c_int32, [C.c_int32, C.c_int32, C.c_int64, C.c_int32]),
    ("st_to_fixed", None, [C.c_double, C.c_int32, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    ("st_from_fixed", C.c_double, [C.c_uint64, C.c_uint64, C.c_int32]),
    ("st_ctx_create", C.c_int, [C.c_int32, C.c_void_p, C.POINTER(C.c_void_p)]),
    ("st_ctx_destroy", C.c_int, [C.c_void_p]),
    ("st_ctx_set_stream", C.c_int, [C.c_void_p, C.c_void_p]),
    ("st_ctx_last_error", C.c_int, [C.c_void_p, C.c_char_p, C.c_size_t]),
    ("st_ctx_sm_count", C.c_int32, [C.c_void_p]),
    ("st_ctx_enable_timing", C.c_int, [C.c_void_p, C.c_int32]),
    ("st_ctx_last_timing", C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                     C.POINTER(C.c_int32)]),
    ("st_ctx_set_tuning", C.c_int, [C.c_void_p, C.c_int64, C.c_int32]),
    ("st_ctx_set_param", C.c_int, [C.c_void_p, C.c_char_p, C.c_int64]),
    ("st_ctx_get_param", C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(C.c_int64)]),
    ("st_ctx_autotune", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(st_tune_result)]),
    ("st_hist_create", C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_float, C.c_float,
                                 C.POINTER(C.c_int32)]),
    ("st_hist_read", C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]),
    ("st_hist_reset", C.c_int, [C.c_void_p, C.c_int32]),
    ("st_hist_read_all", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
                                   C.POINTER(C.c_int64)]),
    ("st_hist_offset", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int64)]),
    ("st_hist_nbins", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int32)]),
    ("st_hist_edges_of", C.c_int, [C.c_void_p, C.c_int32, C.c_void_p]),
    ("st_job_submit", C.c_int, [C.c_void_p, C.POINTER(st_track_view), C.POINTER(st_job_desc),
                                C.POINTER(C.c_int32)]),
    ("st_run", C.c_int, [C.c_void_p, C.c_int32]),
    ("st_job_stats_get", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(st_job_stats)]),
    ("st_jobs_clear", C.c_int, [C.c_void_p]),
    ("st_jobs_reset", C.c_int, [C.c_void_p]),
    ("st_job_submit_many", C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("st_measure_fp64_peak", C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    ("st_measure_smem_atomic_peak", C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    ("st_probe_unit_wait", C.c_int, [C.c_void_p, C.c_int32, C.c_int64, C.POINTER(C.c_int32),
                                     C.POINTER(C.c_int32)]),
    ("st_jobs_count", C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    ("st_run_export", C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.POINTER(C.c_int64)]),
    ("st_run_async", C.c_int, [C.c_void_p]),
    ("st_run_query", C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    ("st_run_finish", C.c_int, [C.c_void_p]),
    ("st_hists_clear", C.c_int, [C.c_void_p]),
    ("st_hist_read_bins_async", C.c_int, [C.c_void_p, C.c_int64, C.c_int64, C.c_void_p,
                                          C.c_void_p]),
    ("st_ctx_order_after", C.c_int, [C.c_void_p, C.c_void_p]),
    ("st_server_create", C.c_int, [C.c_int32, C.c_int64, C.c_int64, C.c_int32,
                                   C.POINTER(C.c_void_p)]),
    ("st_server_destroy", C.c_int, [C.c_void_p]),
    ("st_server_job_footprint", C.c_int, [C.POINTER(st_track_view), C.POINTER(st_job_desc),
                                          C.c_int32, C.POINTER(C.c_int64)]),
    ("st_server_reserve_bytes", C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    ("st_server_submit", C.c_int, [C.c_void_p, C.POINTER(st_track_view), C.POINTER(st_job_desc),
                                   C.c_int32, C.c_int32, C.c_float, C.c_float, C.c_void_p,
                                   C.c_void_p, C.c_uint64]),
    ("st_server_replay", C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_int32, C.c_int32, C.c_float, C.c_float, C.c_void_p,
                                   C.c_void_p]),
    ("st_server_poll", C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.POINTER(C.c_int32)]),
    ("st_server_drain", C.c_int, [C.c_void_p, C.c_int64]),
    ("st_server_batches", C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.POINTER(C.c_int32)]),
    ("st_superimpose_noalloc", C.c_int, [C.POINTER(st_track_view), C.POINTER(st_job_desc),
                                         C.c_int32, C.c_int32, C.c_float, C.c_float,
                                         C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.POINTER(st_job_stats)]),
    ("st_noalloc_scratch_bytes", C.c_int64, []),
    ("st_run_macro", C.c_int, [C.c_char_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p,
                               C.c_int32, C.POINTER(st_run_info), C.c_char_p, C.c_size_t]),
    ("st_track_file_write", C.c_int, [C.c_char_p, C.c_uint64, C.c_void_p, C.c_uint64,
                                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("st_ini_open", C.c_int, [C.c_char_p, C.POINTER(C.c_void_p), C.POINTER(C.c_int32)]),
    ("st_ini_from_string", C.c_int, [C.c_char_p, C.POINTER(C.c_void_p), C.POINTER(C.c_int32)]),
    ("st_ini_close", None, [C.c_void_p]),
    ("st_ini_get", C.c_int, [C.c_void_p, C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p,
                             C.c_size_t]),
    ("st_ini_get_integer", C.c_long, [C.c_void_p, C.c_char_p, C.c_char_p, C.c_long]),
    ("st_ini_get_real", C.c_double, [C.c_void_p, C.c_char_p, C.c_char_p, C.c_double]),
    ("st_ini_get_float", C.c_float, [C.c_void_p, C.c_char_p, C.c_char_p, C.c_float]),
    ("st_ini_get_boolean", C.c_int32, [C.c_void_p, C.c_char_p, C.c_char_p, C.c_int32]),
    ("st_spectrum_bin_log_x", C.c_int, [C.c_int32, C.c_double, C.c_double, C.c_void_p]),
    ("st_spectrum_pmf_to_pdf", C.c_int, [C.c_int32, C.c_void_p, C.c_void_p]),
    ("st_spectrum_prepare_for_semilog", C.c_int, [C.c_int32, C.c_void_p, C.c_void_p]),
    ("st_macro_tasks", C.c_int, [C.c_char_p, C.c_void_p, C.c_int64, C.POINTER(C.c_int64),
                                 C.c_char_p, C.c_size_t]),
]

_lib = None


def lib() -> C.CDLL:
    """Loads libsupertrack_b200.so once and declares every signature."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `make -C supertrack_b200` "
                "(the GPU path has no fallback)")
        handle = C.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def check(status: int, what: str, ctx=None) -> None:
    if status != ST_OK:
        detail = ""
        if ctx is not None:
            buf = C.create_string_buffer(512)
            lib().st_ctx_last_error(ctx, buf, 512)
            detail = buf.value.decode(errors="replace")
        raise StError(status, what, detail)
