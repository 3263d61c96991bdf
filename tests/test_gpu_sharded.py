"""The multi-rank path with each rank's jobs run on the GPU through the C ABI: two ranks (spawned
processes, gloo over TCP-free file rendezvous) take their LPT shares of a small workload
(sharding.run_sharded), each runs its share as one batched st_run on cuda:0, and the spectra are
all-reduced. The reduced spectrum must equal the single-process run of all jobs and the CPU
oracle: counts bit-exact, y*f(y) within 1e-12 (the all-reduce adds in its own order). The ranks
share the one GPU here; their kernels never wait on one another, only the host-side collective
joins them, which a short process-group timeout bounds."""
import os

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _workload():
    import supertrack_b200.workloads as W
    return W.config2(n_tracks=48, size_scale=0.05, os_scale=0.1)


def _run_jobs(ctx, w, jobs):
    """Runs the listed jobs of w on the GPU through the C ABI into one spectrum layout (every
    histogram of the workload, in order); returns (counts, yfy) of the whole layout."""
    ctx.clear()
    hids = [ctx.histogram(*h) for h in w.hists]
    for j in jobs:
        x, y, z, e = [a.numpy() for a in w.job_arrays(j)]
        ctx.submit(x, y, z, e, half_length=float(w.half_length[j]),
                   sphere_diameter=float(w.diameter[j]), n_oversamples=int(w.n_os[j]),
                   hist=hids[int(w.hist_of_job[j])], seed=int(w.seed[j]),
                   track_id=int(w.track_id[j]), zshift=w.zshift)
    ctx.run("batched")
    out = [ctx.read_histogram(h) for h in hids]
    return np.concatenate([o[0] for o in out]), np.concatenate([o[1] for o in out])


def _worker(rank, world, store_path, out_path):
    import sys
    from datetime import timedelta
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import supertrack_b200 as st
    from supertrack_b200.sharding import run_sharded
    dist.init_process_group("gloo", init_method="file://" + store_path, rank=rank,
                            world_size=world, timeout=timedelta(seconds=120))
    try:
        w = _workload()
        n_bins = sum(h[1] for h in w.hists)
        with st.Context(0) as ctx:
            c, y, jobs = run_sharded(w.sizes * w.n_os, lambda js: _run_jobs(ctx, w, js),
                                     n_bins, rank, world)
        np.savez(out_path + f".{rank}.npz", counts=c, yfy=y, jobs=np.asarray(jobs, dtype=np.int64))
    finally:
        dist.destroy_process_group()


def test_two_gpu_ranks_reduce_to_the_single_run(tmp_path, ctx):
    import pyoracle as po
    import supertrack_b200 as st
    world = 2
    store = str(tmp_path / "store")
    out = str(tmp_path / "spec")
    mctx = mp.get_context("spawn")
    procs = [mctx.Process(target=_worker, args=(r, world, store, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=600)
    for p in procs:
        if p.is_alive():
            p.kill()
            p.join()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = [np.load(out + f".{r}.npz") for r in range(world)]
    w = _workload()
    # every job ran on exactly one rank, and both ranks hold the same reduced spectrum
    jobs = sorted(np.concatenate([r["jobs"] for r in res]).tolist())
    assert jobs == list(range(w.n_jobs))
    assert np.array_equal(res[0]["counts"], res[1]["counts"])
    assert np.array_equal(res[0]["yfy"], res[1]["yfy"])
    # the single-process run of all jobs
    c1, y1 = _run_jobs(ctx, w, range(w.n_jobs))
    assert np.array_equal(res[0]["counts"], c1)
    np.testing.assert_allclose(res[0]["yfy"], y1, rtol=1e-12, atol=0)
    # and the oracle
    oc, oy = [], []
    for j in range(w.n_jobs):
        x, y, z, e = [a.numpy() for a in w.job_arrays(j)]
        ed = po.edges(*w.hists[int(w.hist_of_job[j])])
        cj = np.zeros(len(ed) - 1, dtype=np.int64)
        yj = np.zeros(len(ed) - 1)
        sx = st.oversample_shifts(float(w.half_length[j]), float(w.diameter[j]), True,
                                  int(w.seed[j]), int(w.track_id[j]), int(w.n_os[j]))
        po.run_job(x, y, z, e, half_length=float(w.half_length[j]),
                   sphere_diameter=float(w.diameter[j]), sxsy=sx, edges_arr=ed,
                   zshift=w.zshift, counts=cj, yfy=yj)
        oc.append(cj)
        oy.append(yj)
    assert np.array_equal(res[0]["counts"], np.concatenate(oc))
    scale = np.maximum(np.abs(np.concatenate(oy)), 1e-300)
    assert np.all(np.abs(res[0]["yfy"] - np.concatenate(oy)) <= 1e-12 * scale)
    ctx.clear()
