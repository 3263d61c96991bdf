"""GPU path against the CPU oracle at the benchmark's own sizes.

  * the whole dense-ion configuration (16 tracks x 1e6 deposits, 2 nm spheres, 100 oversamples:
    1.6e9 deposit*oversamples, about ten seconds of the oracle on the host's threads);
  * the first four tracks of the large single-geometry configuration at their full size
    (4e6 deposits each, 10 nm spheres) with 16 of their 1,000 oversamples.

Tracks are generated on the GPU exactly as the benchmark generates them (every track of these
configurations is seeded on its own), submitted device-resident, and run as one batch. Bar: the
histogram counts and every job's hits, spheres and binned spheres bit-exact; y*f(y) within 1e-12
relative (its float64 accumulation order across spheres is not fixed).
"""
import os

import numpy as np
import pytest
import torch

import pyoracle as po
import supertrack_b200 as st
import supertrack_b200.workloads as W

pytestmark = pytest.mark.gpu


def _gpu(w, per_job_hist: bool):
    """Runs every job of w on cuda:0, device-resident; returns (counts, yfy) per histogram and
    the job statistics."""
    with st.Context(0) as ctx:
        if per_job_hist:
            hids = [ctx.histogram(*w.hists[int(w.hist_of_job[j])]) for j in range(w.n_jobs)]
        else:
            all_h = [ctx.histogram(*h) for h in w.hists]
            hids = [all_h[int(w.hist_of_job[j])] for j in range(w.n_jobs)]
        for j in range(w.n_jobs):
            o, n = int(w.offsets[j]), int(w.sizes[j])
            ptrs = [t.data_ptr() + 8 * o for t in (w.x, w.y, w.z, w.edep)]
            ctx.submit(*ptrs, half_length=float(w.half_length[j]),
                       sphere_diameter=float(w.diameter[j]), n_oversamples=int(w.n_os[j]),
                       hist=hids[j], seed=int(w.seed[j]), track_id=int(w.track_id[j]),
                       zshift=w.zshift, on_device=True, n=n)
        torch.cuda.synchronize()
        ctx.run("batched")
        spectra = [ctx.read_histogram(h) for h in sorted(set(hids))]
        stats = [ctx.stats(j) for j in range(w.n_jobs)]
    return spectra, stats


def _oracle(w):
    """Every job through the oracle on all host threads, each into its own histogram."""
    x, y, z, e = [a.cpu().numpy() for a in (w.x, w.y, w.z, w.edep)]
    edges = [po.edges(*w.hists[int(w.hist_of_job[j])]) for j in range(w.n_jobs)]
    counts, yfy, js, _ = po.run_batch(
        x, y, z, e, w.offsets, w.sizes, w.half_length, w.diameter,
        np.full(w.n_jobs, po.ZS[w.zshift]), np.full(w.n_jobs, int(w.shift_track)), w.n_os,
        w.seed, w.track_id, np.arange(w.n_jobs), edges, threads=os.cpu_count() or 1,
        job_stats=True)
    return counts, yfy, js


def _check(w):
    spectra, gs = _gpu(w, per_job_hist=False)
    oc, oy, js = _oracle(w)
    for j in range(w.n_jobs):
        assert gs[j]["hits"] == js["hits"][j], j
        assert gs[j]["spheres"] == js["spheres"][j], j
        assert gs[j]["binned"] == js["binned"][j], j
    # the workload's one shared histogram against the sum of the oracle's per-job spectra
    tot_c = np.sum(oc, axis=0)
    tot_y = np.sum(oy, axis=0)
    gc, gy = spectra[0]
    assert np.array_equal(gc, tot_c), np.nonzero(gc != tot_c)[0][:10]
    nz = tot_y != 0
    assert np.all(gy[~nz] == 0)
    assert np.max(np.abs(gy[nz] - tot_y[nz]) / np.abs(tot_y[nz])) <= 1e-12
    return gc


def test_config1_whole_workload_against_oracle():
    w = W.config1(device="cuda")
    assert w.units == 1_600_000_000
    gc = _check(w)
    assert gc.sum() > 1e8


def test_config4_full_size_tracks_against_oracle():
    w = W.config4(device="cuda", n_tracks=4, n_os=16)
    assert int(w.sizes.min()) == 4_000_000
    gc = _check(w)
    assert gc.sum() > 1e7
