"""Served stream: jobs of the uneven batched distribution arriving as a Poisson process.

The server (st_server_*, :class:`supertrack_b200.Server`) takes jobs on device-resident tracks
as they arrive, admits them by device footprint and runs them in continuously formed batches.
This module builds the stream and measures it:

* :func:`served_workload` — the jobs (lognormal sizes, mixed generators, diameters and
  oversample counts, one 200-bin log histogram each), generated on the device;
* :func:`repeated` — the same jobs several times over (a longer stream on the same tracks);
* :func:`poisson_arrivals` — arrival times for an offered load in deposit x oversamples per s;
* :func:`replay` — runs the stream through a server and returns spectra and completion records;
* :func:`latency_summary` — p50/p95/p99 latency and achieved throughput.
"""
from __future__ import annotations

import ctypes as C
import time
from typing import Dict, Tuple

import numpy as np

from . import _capi
from . import workloads as W

HIST = ("log", 200, 0.01, 1e4)


def served_workload(device="cuda", n_jobs: int = 10000, seed: int = 4, size_scale: float = 1.0,
                    max_size: int = 2_000_000) -> W.Workload:
    """The served stream's jobs: the uneven batched distribution drawn with its own seed."""
    w = W.config2(device=device, n_tracks=n_jobs, seed=seed, size_scale=size_scale,
                  max_size=max_size)
    w.name = "served-stream"
    if str(device).startswith("cuda"):
        import torch
        # the generator's temporaries stay in torch's cache otherwise, and the server's contexts
        # size their spill tables from the free device memory
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
    return w


def repeated(w: W.Workload, times: int) -> W.Workload:
    """w's jobs `times` times over, on the same track tensors: repeat r of job j reads job j's
    deposits and has track id j + r * n_jobs, so its oversample shifts are its own."""
    n = w.n_jobs
    tile = lambda a: np.tile(np.asarray(a), times)
    r = W.Workload(name=w.name + f"-x{times}", x=w.x, y=w.y, z=w.z, edep=w.edep,
                   offsets=tile(w.offsets), sizes=tile(w.sizes), half_length=tile(w.half_length),
                   diameter=tile(w.diameter), n_os=tile(w.n_os), seed=tile(w.seed),
                   track_id=(tile(w.track_id) + np.repeat(np.arange(times, dtype=np.uint64),
                                                          n) * np.uint64(n)).astype(np.uint64),
                   hist_of_job=np.arange(n * times, dtype=np.int32),
                   hists=list(w.hists) * times, zshift=w.zshift, shift_track=w.shift_track,
                   generator=None if w.generator is None else tile(w.generator))
    return r


def job_work(w: W.Workload) -> np.ndarray:
    """deposit x oversample count of every job."""
    return w.sizes.astype(np.float64) * w.n_os.astype(np.float64)


def poisson_arrivals(w: W.Workload, offered_dep_os_per_s: float, seed: int = 4) -> np.ndarray:
    """Arrival times (ns from the start) of a Poisson process whose mean rate offers
    ``offered_dep_os_per_s`` of work: rate = offered / mean job work."""
    rate = offered_dep_os_per_s / float(job_work(w).mean())
    gaps = np.random.default_rng(seed).exponential(1.0 / rate, w.n_jobs)
    return np.round(np.cumsum(gaps) * 1e9).astype(np.int64)


def job_arrays(w: W.Workload, zshift: str = "none") -> Tuple[C.Array, C.Array]:
    """ctypes arrays of st_track_view (pointers into the workload's device tensors) and
    st_job_desc for every job."""
    n = w.n_jobs
    views = (_capi.st_track_view * n)()
    descs = (_capi.st_job_desc * n)()
    base = [t.data_ptr() for t in (w.x, w.y, w.z, w.edep)]
    zs = {"plus": 0, "minus": 1, "none": 2}[zshift]
    for j in range(n):
        off = int(w.offsets[j]) * 8
        v = views[j]
        v.x, v.y, v.z, v.edep = [b + off for b in base]
        v.n = int(w.sizes[j])
        v.on_device = 1
        d = descs[j]
        d.half_length = float(w.half_length[j])
        d.sphere_diameter = float(w.diameter[j])
        d.zshift = zs
        d.shift_track = int(bool(w.shift_track))
        d.n_oversamples = int(w.n_os[j])
        d.hist_id = -1
        d.seed = int(w.seed[j])
        d.track_id = int(w.track_id[j])
    return views, descs


def replay(server, w: W.Workload, arrival_ns: np.ndarray, timeout_s: float = 600.0):
    """Releases the jobs at their arrival times, waits for all of them and returns
    (counts [n, bins], yfy [n, bins], completion records sorted by job, wall seconds)."""
    views, descs = job_arrays(w, w.zshift)
    nb = HIST[1]
    counts = np.zeros((w.n_jobs, nb), dtype=np.int64)
    yfy = np.zeros((w.n_jobs, nb), dtype=np.float64)
    t0 = time.perf_counter()
    server.replay(views, descs, arrival_ns, HIST, counts, yfy)
    server.drain(timeout_s)
    wall = time.perf_counter() - t0
    rec = server.poll()
    rec = rec[np.argsort(rec["tag"], kind="stable")]
    return counts, yfy, rec, wall


def latency_summary(rec: np.ndarray, work: np.ndarray) -> Dict[str, float]:
    """p50/p95/p99/max latency (ms, completion minus scheduled arrival), the span from the first
    arrival to the last completion and the throughput over it (deposit x oversamples per s)."""
    lat = (rec["done_ns"] - rec["submit_ns"]) / 1e6
    span = (rec["done_ns"].max() - rec["submit_ns"].min()) / 1e9
    return {
        "p50_ms": float(np.percentile(lat, 50)),
        "p95_ms": float(np.percentile(lat, 95)),
        "p99_ms": float(np.percentile(lat, 99)),
        "max_ms": float(lat.max()),
        "mean_ms": float(lat.mean()),
        "span_s": float(span),
        "throughput": float(work.sum() / span),
        "batches": int(len(np.unique(rec["batch"]))),
        "failed": int(np.count_nonzero(rec["status"] != 0)),
    }
