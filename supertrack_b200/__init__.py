"""supertrack_b200 — B200-native VoxelConstrainedSphere superimposition (SuperTrack's hot path).

Python surface over the C ABI of ``libsupertrack_b200.so`` (include/supertrack_b200.h):

* host helpers that need no GPU: :func:`geometry`, :func:`hist_edges`, :func:`philox4x32_10`,
  :func:`oversample_shifts`, :class:`INIReader`, :func:`macro_tasks`, :func:`write_track_file`;
* :class:`Context` — device histograms and superimposition jobs (batched or per-track runs);
* reference-named wrappers: :class:`SphericalGeometry`, :class:`Histogram`,
  :class:`VoxelConstrainedSphereMethod`, :class:`SuperTrackManager` (the .ini run loop).
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import _capi
from ._capi import (ST_HIST_LIN, ST_HIST_LOG, ST_OK, ST_RUN_BATCHED, ST_RUN_PLAIN,
                    ST_ZSHIFT_MINUS, ST_ZSHIFT_NONE, ST_ZSHIFT_PLUS, StError, check, lib)

__all__ = [
    "StError", "Context", "geometry", "hist_edges", "philox4x32_10", "oversample_shifts",
    "INIReader", "SphericalGeometry", "Histogram", "VoxelConstrainedSphereMethod",
    "SuperTrackManager", "run_macro", "macro_tasks", "write_track_file", "ZSHIFT",
    "HIST_TYPES", "Server", "CPUHistogramUtils", "to_root_layout",
]

ZSHIFT = {"plus": ST_ZSHIFT_PLUS, "minus": ST_ZSHIFT_MINUS, "none": ST_ZSHIFT_NONE}
HIST_TYPES = {"lin": ST_HIST_LIN, "log": ST_HIST_LOG}

SPHERE_DTYPE = np.dtype([("key", "<u8"), ("y", "<f8"), ("os", "<i4"), ("job", "<i4")])


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


# ------------------------------------------------------------------------------------------------
# host helpers
# ------------------------------------------------------------------------------------------------
def geometry(half_length: float, sphere_diameter: float) -> Dict[str, float]:
    """SphericalGeometry(HL, d) (reference SphericalGeometry.cu:7-32) as a dict."""
    g = _capi.st_geometry()
    check(lib().st_geometry_make(half_length, sphere_diameter, C.byref(g)), "st_geometry_make")
    return {f: getattr(g, f) for f, _ in _capi.st_geometry._fields_ if f != "reserved"}


def _geom_struct(g: Dict[str, float]) -> _capi.st_geometry:
    s = _capi.st_geometry()
    for k, v in g.items():
        setattr(s, k, v)
    return s


def hist_edges(kind: str, nbins: int, lower: float, upper: float) -> np.ndarray:
    """Histogram bin edges (reference utils.cc:8-31; bounds pass through float)."""
    e = np.zeros(nbins + 1, dtype=np.float64)
    check(lib().st_hist_edges(HIST_TYPES[kind], nbins, lower, upper, _ptr(e)), "st_hist_edges")
    return e


def philox4x32_10(ctr: Sequence[int], key: Sequence[int]) -> Tuple[int, int, int, int]:
    c = np.array(ctr, dtype=np.uint32)
    k = np.array(key, dtype=np.uint32)
    o = np.zeros(4, dtype=np.uint32)
    check(lib().st_philox4x32_10(_ptr(c), _ptr(k), _ptr(o)), "st_philox4x32_10")
    return tuple(int(v) for v in o)


def oversample_shifts(half_length: float, sphere_diameter: float, shift_track: bool, seed: int,
                      track_id: int, n_os: int, os_begin: int = 0) -> np.ndarray:
    """(n_os, 2) array of the (sx, sy) shifts the GPU path applies to each oversample."""
    g = _geom_struct(geometry(half_length, sphere_diameter))
    out = np.zeros(2 * max(n_os, 0), dtype=np.float64)
    check(lib().st_oversample_shifts(C.byref(g), int(bool(shift_track)), seed, track_id,
                                     os_begin, n_os, _ptr(out)), "st_oversample_shifts")
    return out.reshape(-1, 2)


class CPUHistogramUtils:
    """Spectrum post-processing of the reference (utils.cc:37-117) on ROOT-layout contents:
    nbins + 2 float64 values, [0] underflow, [1..nbins] the bins, [nbins + 1] overflow (see
    :func:`to_root_layout`). Like the reference's loops, PMF_to_PDF and Prepare_for_Semilog touch
    indices 0..nbins-1 only (the underflow bin and every bin but the last) and sum the
    normalisation in float, so they return the reference's numbers."""

    @staticmethod
    def BinLogX(nbins: int, from_log10: float, to_log10: float) -> np.ndarray:
        e = np.zeros(nbins + 1)
        check(lib().st_spectrum_bin_log_x(nbins, from_log10, to_log10, _ptr(e)),
              "st_spectrum_bin_log_x")
        return e

    @staticmethod
    def PMF_to_PDF(edges: np.ndarray, contents: np.ndarray) -> np.ndarray:
        e = np.ascontiguousarray(edges, dtype=np.float64)
        c = np.array(contents, dtype=np.float64)
        if len(c) != len(e) + 1:
            raise ValueError("contents must have nbins + 2 values (ROOT layout)")
        check(lib().st_spectrum_pmf_to_pdf(len(e) - 1, _ptr(e), _ptr(c)), "st_spectrum_pmf_to_pdf")
        return c

    @staticmethod
    def Prepare_for_Semilog(edges: np.ndarray, contents: np.ndarray) -> np.ndarray:
        e = np.ascontiguousarray(edges, dtype=np.float64)
        c = np.array(contents, dtype=np.float64)
        if len(c) != len(e) + 1:
            raise ValueError("contents must have nbins + 2 values (ROOT layout)")
        check(lib().st_spectrum_prepare_for_semilog(len(e) - 1, _ptr(e), _ptr(c)),
              "st_spectrum_prepare_for_semilog")
        return c


def to_root_layout(counts: np.ndarray) -> np.ndarray:
    """Bin contents (st_hist_read order) as a ROOT TH1 array with empty under/overflow bins,
    as Histogram::AccumulateCPUHistogram fills them (Histogram.cu:177-186)."""
    c = np.zeros(len(counts) + 2)
    c[1:-1] = counts
    return c


def write_track_file(path: str, tracks: Sequence[Tuple[np.ndarray, np.ndarray, np.ndarray,
                                                       np.ndarray]]) -> None:
    """Writes tracks (x, y, z, edep per track) into one track file of the run-loop format."""
    cols = [np.ascontiguousarray(np.concatenate([t[a] for t in tracks]) if tracks else
                                 np.zeros(0), dtype=np.float64) for a in range(4)]
    index = np.cumsum([len(t[0]) for t in tracks]).astype(np.uint64)
    check(lib().st_track_file_write(path.encode(), len(tracks), _ptr(index), len(cols[0]),
                                    *[_ptr(c) for c in cols]), "st_track_file_write")


class INIReader:
    """The .ini reader (inih semantics, reference extern/inih/INIReader.h)."""

    def __init__(self, path: Optional[str] = None, text: Optional[str] = None):
        h = C.c_void_p()
        err = C.c_int32(0)
        if text is not None:
            check(lib().st_ini_from_string(text.encode(), C.byref(h), C.byref(err)), "st_ini")
        else:
            lib().st_ini_open(path.encode(), C.byref(h), C.byref(err))
        self._h = h
        self._error = err.value

    def __del__(self):
        if getattr(self, "_h", None):
            lib().st_ini_close(self._h)
            self._h = None

    def ParseError(self) -> int:
        return self._error

    def Get(self, section: str, name: str, default: str) -> str:
        buf = C.create_string_buffer(1 << 16)
        check(lib().st_ini_get(self._h, section.encode(), name.encode(), default.encode(), buf,
                               1 << 16), "st_ini_get")
        return buf.value.decode()

    def GetInteger(self, section: str, name: str, default: int) -> int:
        return lib().st_ini_get_integer(self._h, section.encode(), name.encode(), default)

    def GetReal(self, section: str, name: str, default: float) -> float:
        return lib().st_ini_get_real(self._h, section.encode(), name.encode(), default)

    def GetFloat(self, section: str, name: str, default: float) -> float:
        return lib().st_ini_get_float(self._h, section.encode(), name.encode(), default)

    def GetBoolean(self, section: str, name: str, default: bool) -> bool:
        return bool(lib().st_ini_get_boolean(self._h, section.encode(), name.encode(),
                                             int(default)))


def macro_tasks(ini_path: str) -> List[Dict[str, int]]:
    """ThreadAllocator::ReturnThreadAllocations of a macro, flattened to one dict per task."""
    n = C.c_int64(0)
    err = C.create_string_buffer(512)
    rc = lib().st_macro_tasks(ini_path.encode(), None, 0, C.byref(n), err, 512)
    if rc != ST_OK:
        raise StError(rc, "st_macro_tasks", err.value.decode())
    arr = (_capi.st_task * max(n.value, 1))()
    rc = lib().st_macro_tasks(ini_path.encode(), arr, n.value, C.byref(n), err, 512)
    if rc != ST_OK:
        raise StError(rc, "st_macro_tasks", err.value.decode())
    return [{f: getattr(arr[i], f) for f, _ in _capi.st_task._fields_} for i in range(n.value)]


def run_macro(ini_path: str, device: int = 0, write_output: bool = True,
              nbins_cap: int = 1 << 22):
    """SuperTrackManager::Initialize + Run on a macro; returns (counts, yfy, info dict)."""
    counts = np.zeros(nbins_cap, dtype=np.int64)
    yfy = np.zeros(nbins_cap, dtype=np.float64)
    info = _capi.st_run_info()
    err = C.create_string_buffer(1024)
    rc = lib().st_run_macro(ini_path.encode(), device, int(write_output), _ptr(counts),
                            _ptr(yfy), nbins_cap, C.byref(info), err, 1024)
    if rc != ST_OK:
        raise StError(rc, "st_run_macro", err.value.decode())
    nb = info.nbins
    return counts[:nb].copy(), yfy[:nb].copy(), {f: getattr(info, f) for f, _ in
                                                  _capi.st_run_info._fields_}


# ------------------------------------------------------------------------------------------------
# GPU context
# ------------------------------------------------------------------------------------------------
class Context:
    """A GPU context: device histograms plus a queue of superimposition jobs.

    Track arrays may be host numpy arrays (float64, contiguous; kept alive by the context until
    :meth:`clear`) or CUDA tensors/pointers (pass ``on_device=True`` with objects exposing
    ``data_ptr()``).
    """

    def __init__(self, device: int = 0, stream: Optional[int] = None):
        h = C.c_void_p()
        check(lib().st_ctx_create(device, C.c_void_p(stream) if stream else None, C.byref(h)),
              "st_ctx_create")
        self._h = h
        self._keep: List[object] = []
        self.device = device

    @property
    def handle(self):
        return self._h

    def close(self) -> None:
        if self._h:
            lib().st_ctx_destroy(self._h)
            self._h = None
            self._keep = []

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int, what: str) -> None:
        check(rc, what, self._h)

    @property
    def sm_count(self) -> int:
        return lib().st_ctx_sm_count(self._h)

    def set_stream(self, stream: Optional[int]) -> None:
        self._check(lib().st_ctx_set_stream(self._h, C.c_void_p(stream) if stream else None),
                    "st_ctx_set_stream")

    def enable_timing(self, on: bool = True) -> None:
        self._check(lib().st_ctx_enable_timing(self._h, int(on)), "st_ctx_enable_timing")

    def last_timing(self) -> Tuple[float, float, int]:
        a, b, n = C.c_float(), C.c_float(), C.c_int32()
        self._check(lib().st_ctx_last_timing(self._h, C.byref(a), C.byref(b), C.byref(n)),
                    "st_ctx_last_timing")
        return a.value, b.value, n.value

    def set_tuning(self, item_cost: int = 0, grid: int = 0) -> None:
        self._check(lib().st_ctx_set_tuning(self._h, item_cost, grid), "st_ctx_set_tuning")

    # histograms ---------------------------------------------------------------------------
    def set_param(self, name: str, value: int) -> None:
        """Sets a named work-planning parameter (st_ctx_set_param)."""
        self._check(lib().st_ctx_set_param(self._h, name.encode(), int(value)), "st_ctx_set_param")

    def get_param(self, name: str) -> int:
        v = C.c_int64(0)
        self._check(lib().st_ctx_get_param(self._h, name.encode(), C.byref(v)), "st_ctx_get_param")
        return v.value

    def autotune(self, max_trials: int = 32) -> Dict[str, float]:
        """Times the queued jobs under candidate planning parameters and keeps the fastest
        (st_ctx_autotune); histograms and job states are unchanged."""
        r = _capi.st_tune_result()
        self._check(lib().st_ctx_autotune(self._h, max_trials, C.byref(r)), "st_ctx_autotune")
        return {f: getattr(r, f) for f, _ in _capi.st_tune_result._fields_}

    def histogram(self, kind: str, nbins: int, lower: float, upper: float) -> int:
        hid = C.c_int32(-1)
        self._check(lib().st_hist_create(self._h, HIST_TYPES[kind], nbins, lower, upper,
                                         C.byref(hid)), "st_hist_create")
        return hid.value

    def nbins(self, hist: int) -> int:
        n = C.c_int32()
        self._check(lib().st_hist_nbins(self._h, hist, C.byref(n)), "st_hist_nbins")
        return n.value

    def edges(self, hist: int) -> np.ndarray:
        e = np.zeros(self.nbins(hist) + 1)
        self._check(lib().st_hist_edges_of(self._h, hist, _ptr(e)), "st_hist_edges_of")
        return e

    def read_histogram(self, hist: int) -> Tuple[np.ndarray, np.ndarray]:
        nb = self.nbins(hist)
        counts = np.zeros(nb, dtype=np.int64)
        yfy = np.zeros(nb, dtype=np.float64)
        self._check(lib().st_hist_read(self._h, hist, _ptr(counts), _ptr(yfy)), "st_hist_read")
        return counts, yfy

    def read_histogram_into(self, hist: int, counts_ptr: int, yfy_ptr: int) -> None:
        self._check(lib().st_hist_read(self._h, hist, counts_ptr, yfy_ptr), "st_hist_read")

    def reset_histogram(self, hist: int = -1) -> None:
        """Zeroes one histogram's counts and y*f(y) (all histograms for -1); ids stay valid."""
        self._check(lib().st_hist_reset(self._h, hist), "st_hist_reset")

    def total_bins(self) -> int:
        n = C.c_int64()
        self._check(lib().st_hist_read_all(self._h, None, None, 0, C.byref(n)), "st_hist_read_all")
        return n.value

    def hist_offset(self, hist: int) -> int:
        o = C.c_int64()
        self._check(lib().st_hist_offset(self._h, hist, C.byref(o)), "st_hist_offset")
        return o.value

    def read_all_into(self, counts_ptr: int, yfy_ptr: int, cap: int) -> None:
        """Copies every histogram into caller buffers (e.g. pinned tensors) in two transfers."""
        n = C.c_int64()
        self._check(lib().st_hist_read_all(self._h, counts_ptr, yfy_ptr, cap, C.byref(n)),
                    "st_hist_read_all")

    def jobs_reset(self) -> None:
        """Marks all queued jobs as not run, so run() repeats the same batch."""
        self._check(lib().st_jobs_reset(self._h), "st_jobs_reset")

    def fp64_peak(self) -> float:
        v = C.c_double()
        self._check(lib().st_measure_fp64_peak(self._h, C.byref(v)), "st_measure_fp64_peak")
        return v.value

    def smem_atomic_peak(self) -> float:
        """Measured conflict-free 64-bit shared-memory atomic additions per second."""
        v = C.c_double()
        self._check(lib().st_measure_smem_atomic_peak(self._h, C.byref(v)),
                    "st_measure_smem_atomic_peak")
        return v.value

    def probe_unit_wait(self, published: int, max_polls: int):
        """The fused kernel's bounded wait for a shared unit's table, against a table that is
        published (>= 0) or never is (< 0): returns (table it got, device error flags)."""
        t, f = C.c_int32(), C.c_int32()
        self._check(lib().st_probe_unit_wait(self._h, published, max_polls, C.byref(t),
                                             C.byref(f)), "st_probe_unit_wait")
        return t.value, f.value

    # jobs -----------------------------------------------------------------------------------
    def submit(self, x, y, z, edep, *, half_length: float, sphere_diameter: float,
               n_oversamples: int, hist: int, seed: int = 0, track_id: int = 0,
               shift_track: bool = True, zshift: str = "plus", on_device: bool = False,
               n: Optional[int] = None) -> int:
        v = _capi.st_track_view()
        if on_device:
            ptrs = [a if isinstance(a, int) else a.data_ptr() for a in (x, y, z, edep)]
            if n is None and isinstance(x, int):
                raise ValueError("n (deposits) is required with raw device pointers")
            nn = n if n is not None else int(x.numel())
            self._keep.extend([x, y, z, edep])
        else:
            if all(hasattr(a, "data_ptr") for a in (x, y, z, edep)):  # pinned host tensors
                ptrs = [a.data_ptr() for a in (x, y, z, edep)]
                nn = n if n is not None else int(x.numel())
                self._keep.extend([x, y, z, edep])
            else:
                arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z, edep)]
                nn = len(arrs[0])
                if any(len(a) != nn for a in arrs):
                    raise ValueError("x, y, z, edep must have the same length")
                ptrs = [_ptr(a) for a in arrs]
                self._keep.extend(arrs)
        v.x, v.y, v.z, v.edep = ptrs
        v.n = nn
        v.on_device = int(bool(on_device))
        d = _capi.st_job_desc()
        d.half_length = half_length
        d.sphere_diameter = sphere_diameter
        d.zshift = ZSHIFT[zshift] if isinstance(zshift, str) else int(zshift)
        d.shift_track = int(bool(shift_track))
        d.n_oversamples = n_oversamples
        d.hist_id = hist
        d.seed = seed & 0xFFFFFFFFFFFFFFFF
        d.track_id = track_id & 0xFFFFFFFFFFFFFFFF
        jid = C.c_int32(-1)
        self._check(lib().st_job_submit(self._h, C.byref(v), C.byref(d), C.byref(jid)),
                    "st_job_submit")
        return jid.value

    def run(self, mode: str = "batched") -> None:
        m = {"batched": ST_RUN_BATCHED, "plain": ST_RUN_PLAIN}[mode]
        self._check(lib().st_run(self._h, m), "st_run")

    def run_async(self) -> None:
        """Enqueues a batched run of the queued jobs and returns at once."""
        self._check(lib().st_run_async(self._h), "st_run_async")

    def query(self) -> bool:
        """True once the run enqueued by :meth:`run_async` has finished (statistics collected)."""
        done = C.c_int32(0)
        self._check(lib().st_run_query(self._h, C.byref(done)), "st_run_query")
        return bool(done.value)

    def finish(self) -> None:
        """Waits for the run enqueued by :meth:`run_async`."""
        self._check(lib().st_run_finish(self._h), "st_run_finish")

    def clear_histograms(self) -> None:
        """Deletes every histogram of the context: their ids become invalid, and a run of jobs
        that still refer to them is refused. To zero the spectra instead, use
        :meth:`reset_histogram`."""
        self._check(lib().st_hists_clear(self._h), "st_hists_clear")

    def run_export(self, cap: int = 1 << 20) -> np.ndarray:
        out = np.zeros(cap, dtype=SPHERE_DTYPE)
        n = C.c_int64(0)
        self._check(lib().st_run_export(self._h, _ptr(out), cap, C.byref(n)), "st_run_export")
        return out[: n.value].copy()

    def stats(self, job: int) -> Dict[str, int]:
        s = _capi.st_job_stats()
        self._check(lib().st_job_stats_get(self._h, job, C.byref(s)), "st_job_stats_get")
        return {f: getattr(s, f) for f, _ in _capi.st_job_stats._fields_}

    def clear(self) -> None:
        self._check(lib().st_jobs_clear(self._h), "st_jobs_clear")
        self._keep = []

    def n_jobs(self) -> int:
        n = C.c_int32()
        self._check(lib().st_jobs_count(self._h, C.byref(n)), "st_jobs_count")
        return n.value


COMPLETION_DTYPE = np.dtype([("tag", "<u8"), ("status", "<i4"), ("batch", "<i4"),
                             ("submit_ns", "<i8"), ("start_ns", "<i8"), ("done_ns", "<i8")])


BATCH_DTYPE = np.dtype([("batch", "<i4"), ("slot", "<i4"), ("n_jobs", "<i4"), ("status", "<i4"),
                        ("units", "<f8"), ("launch_ns", "<i8"), ("launched_ns", "<i8"),
                        ("end_est_ns", "<i8"), ("done_ns", "<i8"), ("prepare_ms", "<f4"),
                        ("fused_ms", "<f4"), ("host_jobs_ms", "<f4"), ("host_run_ms", "<f4"),
                        ("grid", "<i4"), ("host_allocs", "<i4"), ("host_tables_ms", "<f4"),
                        ("host_alloc_ms", "<f4")])


class Server:
    """Continuous-batching server (st_server_*): jobs on device-resident tracks are queued,
    admitted by device footprint against ``budget_bytes`` and run in batches on two alternating
    contexts; each job's spectrum lands in its own host arrays."""

    def __init__(self, device: int = 0, budget_bytes: int = 150_000_000_000,
                 max_track_deposits: int = 2_000_000, max_batch_jobs: int = 4096):
        h = C.c_void_p()
        check(lib().st_server_create(device, int(budget_bytes), int(max_track_deposits),
                                     int(max_batch_jobs), C.byref(h)), "st_server_create")
        self._h = h
        self._keep: List[object] = []

    def close(self) -> None:
        if self._h:
            check(lib().st_server_destroy(self._h), "st_server_destroy")
            self._h = None
            self._keep = []

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _view(x, y, z, edep) -> _capi.st_track_view:
        v = _capi.st_track_view()
        v.x, v.y, v.z, v.edep = [a if isinstance(a, int) else a.data_ptr() for a in (x, y, z, edep)]
        v.n = int(x.numel())
        v.on_device = 1
        return v

    @staticmethod
    def _desc(half_length, sphere_diameter, n_oversamples, seed, track_id, shift_track, zshift):
        d = _capi.st_job_desc()
        d.half_length = half_length
        d.sphere_diameter = sphere_diameter
        d.zshift = ZSHIFT[zshift] if isinstance(zshift, str) else int(zshift)
        d.shift_track = int(bool(shift_track))
        d.n_oversamples = n_oversamples
        d.hist_id = -1
        d.seed = seed & 0xFFFFFFFFFFFFFFFF
        d.track_id = track_id & 0xFFFFFFFFFFFFFFFF
        return d

    def submit(self, x, y, z, edep, *, half_length: float, sphere_diameter: float,
               n_oversamples: int, hist: Tuple[str, int, float, float], counts: np.ndarray,
               yfy: np.ndarray, seed: int = 0, track_id: int = 0, shift_track: bool = True,
               zshift: str = "plus", tag: int = 0) -> None:
        """Queues one job on CUDA tensors x, y, z, edep (float64); ``counts`` (int64) and ``yfy``
        (float64) receive its spectrum and must stay alive until it completes."""
        kind, nb, lo, hi = hist
        if counts.dtype != np.int64 or yfy.dtype != np.float64 or len(counts) < nb or len(yfy) < nb:
            raise ValueError("counts must be int64[nbins] and yfy float64[nbins]")
        v = self._view(x, y, z, edep)
        d = self._desc(half_length, sphere_diameter, n_oversamples, seed, track_id, shift_track,
                       zshift)
        self._keep.extend([x, y, z, edep, counts, yfy])
        check(lib().st_server_submit(self._h, C.byref(v), C.byref(d), HIST_TYPES[kind], nb, lo, hi,
                                     _ptr(counts), _ptr(yfy), tag), "st_server_submit")

    def replay(self, views: np.ndarray, descs: np.ndarray, arrival_ns: np.ndarray,
               hist: Tuple[str, int, float, float], counts: np.ndarray, yfy: np.ndarray) -> None:
        """Releases job i at ``arrival_ns[i]`` after the call (server-side thread); ``views`` and
        ``descs`` are ctypes arrays of st_track_view / st_job_desc, ``counts``/``yfy`` are
        (n, nbins) arrays. Completion tags are the job indices."""
        kind, nb, lo, hi = hist
        n = len(arrival_ns)
        arr = np.ascontiguousarray(arrival_ns, dtype=np.int64)
        if counts.shape != (n, nb) or yfy.shape != (n, nb):
            raise ValueError("counts and yfy must be (n_jobs, nbins)")
        self._keep.extend([views, descs, arr, counts, yfy])
        check(lib().st_server_replay(self._h, n, C.cast(views, C.c_void_p),
                                     C.cast(descs, C.c_void_p), _ptr(arr), HIST_TYPES[kind], nb,
                                     lo, hi, _ptr(counts), _ptr(yfy)), "st_server_replay")

    def reserve_bytes(self) -> int:
        """Budget bytes set aside for the spill tables of the server's two contexts."""
        b = C.c_int64(0)
        check(lib().st_server_reserve_bytes(self._h, C.byref(b)), "st_server_reserve_bytes")
        return b.value

    @staticmethod
    def job_footprint(view: _capi.st_track_view, desc: _capi.st_job_desc, nbins: int) -> int:
        """Device bytes a job is charged against the budget while in flight."""
        b = C.c_int64(0)
        check(lib().st_server_job_footprint(C.byref(view), C.byref(desc), nbins, C.byref(b)),
              "st_server_job_footprint")
        return b.value

    def drain(self, timeout_s: float = 600.0) -> None:
        check(lib().st_server_drain(self._h, int(timeout_s * 1000)), "st_server_drain")

    def batches(self, cap: int = 1 << 14) -> np.ndarray:
        """Records of finished batches (each returned once)."""
        out = np.zeros(cap, dtype=BATCH_DTYPE)
        got = []
        while True:
            n = C.c_int32(0)
            check(lib().st_server_batches(self._h, _ptr(out), cap, C.byref(n)), "st_server_batches")
            got.append(out[: n.value].copy())
            if n.value < cap:
                return np.concatenate(got)

    def poll(self, cap: int = 1 << 16) -> np.ndarray:
        """Completion records of finished jobs (each returned once)."""
        out = np.zeros(cap, dtype=COMPLETION_DTYPE)
        got = []
        while True:
            n = C.c_int32(0)
            check(lib().st_server_poll(self._h, _ptr(out), cap, C.byref(n)), "st_server_poll")
            got.append(out[: n.value].copy())
            if n.value < cap:
                return np.concatenate(got)


# ------------------------------------------------------------------------------------------------
# reference-named wrappers
# ------------------------------------------------------------------------------------------------
class SphericalGeometry:
    """SphericalGeometry (reference SphericalGeometry.cuh:8-23), from (HL, d) or an INIReader."""

    def __init__(self, half_length_or_reader, sphere_diameter: Optional[float] = None):
        if isinstance(half_length_or_reader, INIReader):
            r = half_length_or_reader
            hl = r.GetReal("VoxelConstrainedSphere", "ScoringRegionHalfLength", 0)
            d = r.GetReal("VoxelConstrainedSphere", "ScoringSphereDiameter", 0)
        else:
            hl, d = half_length_or_reader, sphere_diameter
        g = geometry(hl, d)
        self.scoringRegionLength = g["scoring_region_length"]
        self.scoringRegionHalfLength = g["scoring_region_half_length"]
        self.greatestSphereOffset = g["greatest_sphere_offset"]
        self.numSpheresLinear = g["num_spheres_linear"]
        self.sphereDiameter = g["sphere_diameter"]
        self.sphereRadius = g["sphere_radius"]


class Histogram:
    """Histogram(nbins, binLower, binUpper, type) on a Context (reference Histogram.cuh:15-72).

    GetCPUHistogram returns (edges, counts, yfy): int64 f(y) counts and float64 y*f(y) sums.
    """

    def __init__(self, nbins: int, bin_lower: float, bin_upper: float, kind: str,
                 ctx: Context):
        self.ctx = ctx
        self.id = ctx.histogram(kind, nbins, bin_lower, bin_upper)

    @classmethod
    def FromReader(cls, reader: INIReader, ctx: Context) -> "Histogram":
        return cls(reader.GetInteger("Histogram", "NBins", 0),
                   reader.GetFloat("Histogram", "BinLower", 0),
                   reader.GetFloat("Histogram", "BinUpper", 0),
                   reader.Get("Histogram", "Type", ""), ctx)

    def GetCPUHistogram(self):
        counts, yfy = self.ctx.read_histogram(self.id)
        return self.ctx.edges(self.id), counts, yfy


class VoxelConstrainedSphereMethod:
    """VoxelConstrainedSphereMethod: the macro's geometry and shift settings for job submission."""

    def __init__(self, reader: INIReader):
        self.half_length = reader.GetReal("VoxelConstrainedSphere", "ScoringRegionHalfLength", 0)
        self.sphere_diameter = reader.GetReal("VoxelConstrainedSphere", "ScoringSphereDiameter",
                                              0)
        self.shift_track = reader.GetBoolean("VoxelConstrainedSphere", "ShiftTrack", True)
        self.zshift = reader.Get("VoxelConstrainedSphere", "ZOriginShift", "plus").lower()
        if self.zshift not in ZSHIFT:
            self.zshift = "plus"
        self.geometry = SphericalGeometry(self.half_length, self.sphere_diameter)

    @staticmethod
    def Construct(reader: INIReader) -> "VoxelConstrainedSphereMethod":
        return VoxelConstrainedSphereMethod(reader)


class SuperTrackManager:
    """The .ini run loop (reference SuperTrackManager.hh): Initialize(path) then Run()."""

    _instance = None

    @classmethod
    def GetInstance(cls) -> "SuperTrackManager":
        if cls._instance is None:
            cls._instance = cls()
        return cls._instance

    def __init__(self):
        self._path = None
        self._methods: Dict[str, object] = {}
        self.counts = None
        self.yfy = None
        self.info = None
        self.edges = None

    def AddSimulationMethod(self, name: str, ctor) -> None:
        self._methods[name] = ctor

    def Initialize(self, ini_path: str) -> None:
        self._path = ini_path

    def Run(self, device: int = 0, write_output: bool = True) -> None:
        if self._path is None:
            raise StError(_capi.ST_ERR_STATE, "Run", "manager not initialised")
        self.counts, self.yfy, self.info = run_macro(self._path, device, write_output)
        r = INIReader(self._path)
        self.edges = hist_edges(r.Get("Histogram", "Type", ""),
                                r.GetInteger("Histogram", "NBins", 0),
                                r.GetFloat("Histogram", "BinLower", 0),
                                r.GetFloat("Histogram", "BinUpper", 0))

    def GetOutput(self):
        """(edges, counts, yfy) of the last run."""
        return self.edges, self.counts, self.yfy
