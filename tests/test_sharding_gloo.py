"""Multi-rank sharding logic on CPU: gloo ranks run sharding.run_sharded, the same assignment
and reduction the multi-GPU benchmark uses. Each rank takes its LPT share of the jobs and
computes their spectra (the CPU oracle standing in for the rank's GPU, fed the library's own bin
edges and Philox shifts through the C ABI), and the spectra are all-reduced: counts equal the
single-process spectrum of all jobs exactly, y*f(y) within 1e-12 (the all-reduce's order of
addition is the collective's own)."""
import os

import numpy as np
import pytest
import torch.multiprocessing as mp

from supertrack_b200.sharding import lpt_assign, shard


def test_lpt_balances_and_covers():
    rs = np.random.default_rng(0)
    costs = np.exp(rs.normal(10, 1.5, 500))
    for world in (1, 2, 3, 8):
        owner = lpt_assign(costs, world)
        assert set(owner.tolist()) <= set(range(world))
        loads = np.array([costs[owner == r].sum() for r in range(world)])
        assert loads.max() <= costs.sum() / world + costs.max() + 1e-6
        got = sorted(sum((shard(costs, r, world) for r in range(world)), []))
        assert got == list(range(len(costs)))
    assert np.array_equal(lpt_assign(costs, 4), lpt_assign(costs, 4))  # deterministic


def _worker(rank, world, store_path, out_path, n_tracks=12):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "oracle"))
    import torch.distributed as dist
    import pyoracle as po
    import supertrack_b200 as st
    import supertrack_b200.workloads as W
    from supertrack_b200.sharding import run_sharded
    # rendezvous through a file: no port that another process could take in between
    dist.init_process_group("gloo", init_method="file://" + store_path, rank=rank,
                            world_size=world)
    try:
        w = W.config0(n_tracks=n_tracks, n_os=3)
        e = st.hist_edges(*w.hists[0])        # the library's edges (C ABI, host side)

        def runner(jobs):
            counts = np.zeros(len(e) - 1, dtype=np.int64)
            yfy = np.zeros(len(e) - 1)
            for j in jobs:
                x, y, z, ed = [a.numpy() for a in w.job_arrays(j)]
                sx = st.oversample_shifts(2500.0, 10.0, True, int(w.seed[j]), j, int(w.n_os[j]))
                po.run_job(x, y, z, ed, half_length=2500.0, sphere_diameter=10.0, sxsy=sx,
                           edges_arr=e, zshift=w.zshift, counts=counts, yfy=yfy)
            return counts, yfy

        c, y, jobs = run_sharded(w.sizes * w.n_os, runner, len(e) - 1, rank, world)
        np.savez(out_path + f".{rank}.npz", counts=c, yfy=y, jobs=np.asarray(jobs, dtype=np.int64))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,n_tracks", [(2, 12), (3, 2)])
def test_ranks_spectrum_equals_single_process(tmp_path, world, n_tracks):
    """Two ranks sharing 12 tracks, and three ranks with two tracks (one rank has no job but
    still takes part in the reduction)."""
    import pyoracle as po
    import supertrack_b200.workloads as W
    from supertrack_b200.sharding import shard
    w = W.config0(n_tracks=n_tracks, n_os=3)
    owned = [len(shard(w.sizes * w.n_os, r, world)) for r in range(world)]
    assert sum(owned) == w.n_jobs and (n_tracks >= world or 0 in owned)
    out = str(tmp_path / "r")
    ctx = mp.get_context("spawn")
    store = str(tmp_path / "store")
    procs = [ctx.Process(target=_worker, args=(r, world, store, out, n_tracks))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    got = [np.load(out + f".{r}.npz") for r in range(world)]
    owned = sorted(sum((g["jobs"].tolist() for g in got), []))
    assert owned == list(range(w.n_jobs))      # every job on exactly one rank
    e = po.edges(*w.hists[0])
    counts = np.zeros(len(e) - 1, dtype=np.int64)
    yfy = np.zeros(len(e) - 1)
    for j in range(w.n_jobs):
        x, y, z, ed = [a.numpy() for a in w.job_arrays(j)]
        sx = po.shifts(2500.0, 10.0, True, int(w.seed[j]), j, int(w.n_os[j]))
        po.run_job(x, y, z, ed, half_length=2500.0, sphere_diameter=10.0, sxsy=sx, edges_arr=e,
                   zshift=w.zshift, counts=counts, yfy=yfy)
    for g in got:                              # every rank holds the reduced spectrum
        assert np.array_equal(g["counts"], counts)
        np.testing.assert_allclose(g["yfy"], yfy, rtol=1e-12)
