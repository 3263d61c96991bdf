"""Shared drivers for the parity tests: run a workload through the GPU path (C ABI) and through
the CPU oracle with the same shifts."""
import numpy as np

import pyoracle as po
import supertrack_b200 as st


def gpu_run(ctx, w, mode="batched", export_cap=0, jobs=None, zshift=None, hist_ids=None):
    """Submits jobs of workload w (all, or the listed indices) and runs them. Returns
    (counts per hist, yfy per hist, stats per job, exported spheres or None)."""
    ctx.clear()
    if hist_ids is None:
        hist_ids = [ctx.histogram(*h) for h in w.hists]
    jobs = range(w.n_jobs) if jobs is None else jobs
    ids = []
    for j in jobs:
        x, y, z, e = [a.cpu().numpy() for a in w.job_arrays(j)]
        ids.append(ctx.submit(x, y, z, e, half_length=float(w.half_length[j]),
                              sphere_diameter=float(w.diameter[j]), n_oversamples=int(w.n_os[j]),
                              hist=hist_ids[int(w.hist_of_job[j])], seed=int(w.seed[j]),
                              track_id=int(w.track_id[j]), shift_track=w.shift_track,
                              zshift=zshift or w.zshift))
    spheres = None
    if export_cap:
        spheres = ctx.run_export(export_cap)
    else:
        ctx.run(mode)
    stats = [ctx.stats(i) for i in ids]
    out = [ctx.read_histogram(h) for h in hist_ids]
    return [o[0] for o in out], [o[1] for o in out], stats, spheres


def oracle_run(w, jobs=None, zshift=None, spheres_cap=0, sum_mode=po.OR_SUM_EXACT, precision=64):
    edges = [po.edges(*h) for h in w.hists]
    counts = [np.zeros(len(e) - 1, dtype=np.int64) for e in edges]
    yfy = [np.zeros(len(e) - 1) for e in edges]
    stats, spheres = [], []
    jobs = range(w.n_jobs) if jobs is None else jobs
    for j in jobs:
        x, y, z, e = [a.cpu().numpy() for a in w.job_arrays(j)]
        h = int(w.hist_of_job[j])
        sx = st.oversample_shifts(float(w.half_length[j]), float(w.diameter[j]), w.shift_track,
                                  int(w.seed[j]), int(w.track_id[j]), int(w.n_os[j]))
        _, _, s, sph = po.run_job(x, y, z, e, half_length=float(w.half_length[j]),
                                  sphere_diameter=float(w.diameter[j]), sxsy=sx,
                                  edges_arr=edges[h], zshift=zshift or w.zshift,
                                  sum_mode=sum_mode, spheres_cap=spheres_cap, counts=counts[h],
                                  yfy=yfy[h], precision=precision)
        stats.append(s)
        spheres.append(sph)
    return counts, yfy, stats, spheres


def assert_hist_equal(gc, gy, oc, oy, rtol=1e-12):
    for a, b, c, d in zip(gc, gy, oc, oy):
        assert np.array_equal(a, c), np.nonzero(a != c)[0][:10]
        scale = np.maximum(np.abs(d), 1e-300)
        assert np.all(np.abs(b - d) <= rtol * scale), np.max(np.abs(b - d) / scale)


def assert_stats_equal(gs, os_):
    for g, o in zip(gs, os_):
        assert g["hits"] == o["hits"]
        assert g["spheres"] == o["spheres"]
        assert g["binned"] == o["binned"]
        assert g["grid_exponent"] == o["grid_exponent"]
