"""ctypes wrapper of the CPU oracle (oracle/liboracle.so) — TEST INFRASTRUCTURE ONLY.

Imported by tests/, __graft_entry__.smoke() and bench.py's CPU baseline / reference arm, never
by the supertrack_b200 package. `make -C oracle` builds the library.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

OR_SUM_EXACT = 0
OR_SUM_SEQ = 1

STATS_DTYPE = np.dtype([("hits", "<i8"), ("spheres", "<i8"), ("binned", "<i8"),
                        ("grid_exponent", "<i4"), ("status", "<i4")])
SPHERE_DTYPE = np.dtype([("key", "<u8"), ("y", "<f8"), ("y_seq", "<f8"), ("nhits", "<i8"),
                         ("os", "<i4"), ("bin", "<i4")])


class or_geom(C.Structure):
    _fields_ = [("L", C.c_double), ("HL", C.c_double), ("gSO", C.c_double), ("d", C.c_double),
                ("r", C.c_double), ("N", C.c_int)]


class or_stats(C.Structure):
    _fields_ = [("hits", C.c_int64), ("spheres", C.c_int64), ("binned", C.c_int64),
                ("grid_exponent", C.c_int32), ("status", C.c_int32)]


_lib = None


def build() -> None:
    subprocess.run(["make", "-C", HERE], check=True, capture_output=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        h = C.CDLL(LIB_PATH)
        h.or_geometry.argtypes = [C.c_double, C.c_double, C.POINTER(or_geom)]
        h.or_geometry.restype = C.c_int
        h.or_edges.argtypes = [C.c_int, C.c_int, C.c_float, C.c_float, C.c_void_p]
        h.or_edges.restype = C.c_int
        h.or_philox.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        h.or_philox.restype = None
        h.or_shifts.argtypes = [C.POINTER(or_geom), C.c_int, C.c_uint64, C.c_uint64, C.c_uint32,
                                C.c_uint32, C.c_void_p]
        h.or_shifts.restype = None
        h.or_grid_exponent.argtypes = [C.c_int, C.c_int, C.c_int64, C.c_int]
        h.or_grid_exponent.restype = C.c_int
        h.or_job.argtypes = [C.c_void_p] * 4 + [C.c_int64, C.c_double, C.c_double, C.c_int,
                                                C.c_uint32, C.c_void_p, C.c_void_p, C.c_int,
                                                C.c_int, C.c_void_p, C.c_void_p,
                                                C.POINTER(or_stats), C.c_void_p, C.c_int64,
                                                C.POINTER(C.c_int64)]
        h.or_job.restype = C.c_int
        h.or_job_f32.argtypes = h.or_job.argtypes
        h.or_job_f32.restype = C.c_int
        h.or_run_batch.argtypes = [C.c_int64] + [C.c_void_p] * 22 + [C.c_int32]
        h.or_run_batch.restype = C.c_int
        _lib = h
    return _lib


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


def geometry(hl: float, d: float) -> dict:
    g = or_geom()
    rc = lib().or_geometry(hl, d, C.byref(g))
    if rc:
        raise ValueError(f"bad geometry ({rc})")
    return {f: getattr(g, f) for f, _ in or_geom._fields_}


def edges(kind: str, nbins: int, lo: float, hi: float) -> np.ndarray:
    e = np.zeros(nbins + 1)
    rc = lib().or_edges({"lin": 0, "log": 1}[kind], nbins, lo, hi, _p(e))
    if rc:
        raise ValueError(f"bad histogram ({rc})")
    return e


def philox(ctr, key):
    c = np.array(ctr, dtype=np.uint32)
    k = np.array(key, dtype=np.uint32)
    o = np.zeros(4, dtype=np.uint32)
    lib().or_philox(_p(c), _p(k), _p(o))
    return tuple(int(v) for v in o)


def shifts(hl: float, d: float, shift_track: bool, seed: int, track_id: int, n_os: int,
           os_begin: int = 0) -> np.ndarray:
    g = or_geom()
    if lib().or_geometry(hl, d, C.byref(g)):
        raise ValueError("bad geometry")
    out = np.zeros(2 * max(n_os, 1))
    lib().or_shifts(C.byref(g), int(bool(shift_track)), seed, track_id, os_begin, n_os, _p(out))
    return out[: 2 * n_os].reshape(-1, 2)


def grid_exponent(e_min: int, e_max: int, n: int, anyv: bool) -> int:
    return lib().or_grid_exponent(e_min, e_max, n, int(anyv))


ZS = {"plus": 0, "minus": 1, "none": 2}


def run_job(x, y, z, edep, *, half_length, sphere_diameter, sxsy, edges_arr, zshift="plus",
            sum_mode=OR_SUM_EXACT, spheres_cap=0, counts=None, yfy=None, precision=64):
    """One job through the oracle; returns (counts, yfy, stats dict, spheres array or None).
    precision 32 runs the FP32 geometry variant (or_job_f32)."""
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z, edep)]
    n = len(arrs[0])
    sx = np.ascontiguousarray(sxsy, dtype=np.float64).reshape(-1)
    n_os = len(sx) // 2
    e = np.ascontiguousarray(edges_arr, dtype=np.float64)
    nb = len(e) - 1
    if counts is None:
        counts = np.zeros(nb, dtype=np.int64)
    if yfy is None:
        yfy = np.zeros(nb, dtype=np.float64)
    st = or_stats()
    sph = np.zeros(max(spheres_cap, 1), dtype=SPHERE_DTYPE) if spheres_cap else None
    nsph = C.c_int64(0)
    fn = lib().or_job_f32 if precision == 32 else lib().or_job
    rc = fn(*[_p(a) for a in arrs], n, half_length, sphere_diameter, ZS[zshift],
                      n_os, _p(sx) if n_os else None, _p(e), nb, sum_mode, _p(counts), _p(yfy),
                      C.byref(st), _p(sph) if sph is not None else None, spheres_cap,
                      C.byref(nsph))
    if rc:
        raise RuntimeError(f"oracle job failed ({rc})")
    stats = {f: getattr(st, f) for f, _ in or_stats._fields_}
    if sph is not None:
        if nsph.value > spheres_cap:
            raise RuntimeError("sphere export capacity exceeded")
        sph = sph[: nsph.value]
    return counts, yfy, stats, sph


def run_batch(x, y, z, edep, off, n, hl, d, zshift, shift_track, n_os, seed, track_id, hist,
              edges_list, threads=1, job_stats=False):
    """Many jobs on `threads` host threads, claimed in the given order. edges_list[h] are the
    edges of histogram h. Returns (counts list, yfy list), plus, when job_stats is true, a
    structured array of per-job (hits, spheres, binned, grid_exponent, status) and the thread
    seconds of every job."""
    nb = np.array([len(e) - 1 for e in edges_list], dtype=np.int32)
    eoff = np.concatenate([[0], np.cumsum([len(e) for e in edges_list])[:-1]]).astype(np.int64)
    hoff = np.concatenate([[0], np.cumsum(nb)[:-1]]).astype(np.int64)
    E = np.concatenate(edges_list).astype(np.float64)
    counts = np.zeros(int(nb.sum()), dtype=np.int64)
    yfy = np.zeros(int(nb.sum()), dtype=np.float64)
    a = lambda v, t: np.ascontiguousarray(v, dtype=t)
    args = [a(x, np.float64), a(y, np.float64), a(z, np.float64), a(edep, np.float64),
            a(off, np.int64), a(n, np.int64), a(hl, np.float64), a(d, np.float64),
            a(zshift, np.int32), a(shift_track, np.int32), a(n_os, np.uint32),
            a(seed, np.uint64), a(track_id, np.uint64), a(hist, np.int32), E, eoff, nb, hoff,
            counts, yfy]
    js = np.zeros(len(args[4]), dtype=STATS_DTYPE)
    secs = np.zeros(len(args[4]), dtype=np.float64)
    failed = lib().or_run_batch(len(args[4]), *[_p(v) for v in args], _p(js), _p(secs), threads)
    if failed:
        raise RuntimeError(f"{failed} oracle jobs failed")
    out = ([counts[hoff[h]:hoff[h] + nb[h]] for h in range(len(nb))],
           [yfy[hoff[h]:hoff[h] + nb[h]] for h in range(len(nb))])
    return out + (js, secs) if job_stats else out


# ---------------------------------------------------------------------------------------------
# Spectrum post-processing, restated from utils.cc:37-117 (CPUHistogramUtils) for ROOT-layout
# contents (index 0 underflow, 1..nbins bins, nbins+1 overflow). TAxis::GetBinLowEdge of an
# axis built from explicit edges returns edges[bin-1] for bins 1..nbins+1 and extrapolates with
# the mean width outside. The normalisation accumulates in float (float_t) as in the reference.
# ---------------------------------------------------------------------------------------------
def _root_low_edge(edges, bin_):
    nb = len(edges) - 1
    if bin_ < 1 or bin_ > nb + 1:
        w = (float(edges[nb]) - float(edges[0])) / nb
        return float(edges[0]) + (bin_ - 1) * w
    return float(edges[bin_ - 1])


def bin_log_x(nbins, frm, to):
    """utils.cc:37-57: 10^(from + i*width), width = (to - from) / nbins."""
    width = (frm * 0 + to - frm) / nbins
    return np.array([10.0 ** (frm + i * width) for i in range(nbins + 1)])


def pmf_to_pdf(edges, contents):
    """utils.cc:81-102: loops over indices 0..nbins-1; float normalisation."""
    c = [float(v) for v in contents]
    nb = len(edges) - 1
    norm = np.float32(0.0)
    for i in range(nb):
        value = c[i]
        low = _root_low_edge(edges, i)
        high = _root_low_edge(edges, i + 1)
        with np.errstate(divide="ignore", invalid="ignore"):
            c[i] = float(np.float64(value) / np.float64(high - low))
        norm = np.float32(float(norm) + value)
    with np.errstate(divide="ignore", invalid="ignore"):   # IEEE division, as in C++
        for i in range(nb):
            c[i] = float(np.float64(c[i]) / np.float64(float(norm)))
    return np.array(c)


def prepare_for_semilog(edges, contents):
    """utils.cc:104-117: multiplies indices 0..nbins-1 by their bin midpoints."""
    c = [float(v) for v in contents]
    nb = len(edges) - 1
    for i in range(nb):
        low = _root_low_edge(edges, i)
        high = _root_low_edge(edges, i + 1)
        c[i] = c[i] * ((high + low) / 2)
    return np.array(c)
