"""Serving (st_server_*): continuous batching of arriving jobs.

The served form must give every job the same spectrum as running it alone: counts bit-exact,
y*f(y) within 1e-12 relative (the per-bin sums of y are float64 atomics, so their order varies).
Also covered: the asynchronous context run it is built on, admission against a small budget
(many batches, same results), rejection of jobs that can never fit, and a direct oracle check.
"""
import numpy as np
import pytest

import supertrack_b200 as st
from supertrack_b200 import _capi, serving

from helpers import oracle_run

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def _alone(w):
    """Spectrum of every job run alone, each in its own batched run."""
    nb = serving.HIST[1]
    counts = np.zeros((w.n_jobs, nb), dtype=np.int64)
    yfy = np.zeros((w.n_jobs, nb))
    with st.Context(0) as c:
        for j in range(w.n_jobs):
            c.clear()
            c.clear_histograms()
            h = c.histogram(*serving.HIST)
            x, y, z, e = w.job_arrays(j)
            c.submit(x, y, z, e, half_length=float(w.half_length[j]),
                     sphere_diameter=float(w.diameter[j]), n_oversamples=int(w.n_os[j]), hist=h,
                     seed=int(w.seed[j]), track_id=int(w.track_id[j]), zshift=w.zshift,
                     on_device=True)
            c.run("batched")
            counts[j], yfy[j] = c.read_histogram(h)
    return counts, yfy


def _assert_same(counts, yfy, ref_counts, ref_yfy):
    assert np.array_equal(counts, ref_counts), np.argwhere(counts != ref_counts)[:5]
    scale = np.maximum(np.abs(ref_yfy), 1e-300)
    assert np.all(np.abs(yfy - ref_yfy) <= RTOL * scale)


@pytest.fixture(scope="module")
def stream():
    w = serving.served_workload("cuda", n_jobs=48, seed=4, size_scale=0.1, max_size=200_000)
    return w, _alone(w)


def test_async_run_matches_sync():
    import torch
    w = serving.served_workload("cuda", n_jobs=8, seed=7, size_scale=0.1, max_size=100_000)
    out = []
    with st.Context(0) as c:
        for mode in ("sync", "async"):
            c.clear()
            c.clear_histograms()
            hs = [c.histogram(*serving.HIST) for _ in range(w.n_jobs)]
            for j in range(w.n_jobs):
                x, y, z, e = w.job_arrays(j)
                c.submit(x, y, z, e, half_length=float(w.half_length[j]),
                         sphere_diameter=float(w.diameter[j]), n_oversamples=int(w.n_os[j]),
                         hist=hs[j], seed=int(w.seed[j]), track_id=int(w.track_id[j]),
                         zshift=w.zshift, on_device=True)
            if mode == "sync":
                c.run("batched")
            else:
                c.run_async()
                with pytest.raises(st.StError):
                    c.run_async()             # one run in flight per context
                while not c.query():
                    pass
                c.finish()                    # nothing left to wait for
            stats = [c.stats(j) for j in range(w.n_jobs)]
            out.append(([c.read_histogram(h) for h in hs], stats))
        torch.cuda.synchronize()
    (h0, s0), (h1, s1) = out
    for (c0, y0), (c1, y1) in zip(h0, h1):
        _assert_same(c1, y1, c0, y0)
    assert s0 == s1


def test_served_equals_alone(stream):
    w, (ref_c, ref_y) = stream
    # arrivals within ~2 ms: most batches hold several jobs
    arr = np.sort(np.random.default_rng(1).integers(0, 2_000_000, w.n_jobs)).astype(np.int64)
    with st.Server(0, budget_bytes=40_000_000_000, max_track_deposits=200_000) as srv:
        counts, yfy, rec, _ = serving.replay(srv, w, arr)
    assert len(rec) == w.n_jobs
    assert np.all(rec["status"] == 0)
    assert np.array_equal(rec["tag"], np.arange(w.n_jobs))
    sizes = np.bincount(rec["batch"])
    assert sizes.max() > 1, "no two jobs shared a batch"
    assert np.all(rec["done_ns"] >= rec["start_ns"])
    _assert_same(counts, yfy, ref_c, ref_y)


def test_submit_one_by_one_equals_alone(stream):
    w, (ref_c, ref_y) = stream
    nb = serving.HIST[1]
    counts = np.zeros((w.n_jobs, nb), dtype=np.int64)
    yfy = np.zeros((w.n_jobs, nb))
    with st.Server(0, budget_bytes=40_000_000_000, max_track_deposits=200_000) as srv:
        for j in range(w.n_jobs):
            x, y, z, e = w.job_arrays(j)
            srv.submit(x, y, z, e, half_length=float(w.half_length[j]),
                       sphere_diameter=float(w.diameter[j]), n_oversamples=int(w.n_os[j]),
                       hist=serving.HIST, counts=counts[j], yfy=yfy[j], seed=int(w.seed[j]),
                       track_id=int(w.track_id[j]), zshift=w.zshift, tag=1000 + j)
        srv.drain(300)
        rec = srv.poll()
    assert sorted(rec["tag"].tolist()) == list(range(1000, 1000 + w.n_jobs))
    assert np.all(rec["status"] == 0)
    _assert_same(counts, yfy, ref_c, ref_y)


def test_small_budget_admits_in_turn(stream):
    w, (ref_c, ref_y) = stream
    views, descs = serving.job_arrays(w, w.zshift)
    foot = np.array([st.Server.job_footprint(views[j], descs[j], serving.HIST[1])
                     for j in range(w.n_jobs)])
    with st.Server(0, budget_bytes=40_000_000_000, max_track_deposits=200_000) as probe:
        reserve = probe.reserve_bytes()
    budget = reserve + int(2.5 * foot.max())
    arr = np.zeros(w.n_jobs, dtype=np.int64)      # everything at once: only the budget limits
    with st.Server(0, budget_bytes=budget, max_track_deposits=200_000) as srv:
        counts, yfy, rec, _ = serving.replay(srv, w, arr)
    # a job that can never fit is refused at submission
    x, y, z, e = w.job_arrays(int(np.argmax(foot)))
    with st.Server(0, budget_bytes=reserve + 1000, max_track_deposits=200_000) as tiny:
        with pytest.raises(st.StError) as ei:
            tiny.submit(x, y, z, e, half_length=2500.0, sphere_diameter=10.0, n_oversamples=10,
                        hist=serving.HIST, counts=np.zeros(200, dtype=np.int64),
                        yfy=np.zeros(200))
        assert ei.value.status == _capi.ST_ERR_CAPACITY
    assert np.all(rec["status"] == 0)
    # every batch stayed within the budget
    for b in np.unique(rec["batch"]):
        assert foot[rec["tag"][rec["batch"] == b].astype(np.int64)].sum() <= budget - reserve
    assert len(np.unique(rec["batch"])) >= int(np.ceil(foot.sum() / (budget - reserve)))
    _assert_same(counts, yfy, ref_c, ref_y)


def test_oversized_track_refused():
    import torch
    x = torch.zeros(1001, dtype=torch.float64, device="cuda")
    with st.Server(0, budget_bytes=40_000_000_000, max_track_deposits=1000) as srv:
        with pytest.raises(st.StError) as ei:
            srv.submit(x, x, x, x, half_length=2500.0, sphere_diameter=10.0, n_oversamples=1,
                       hist=serving.HIST, counts=np.zeros(200, dtype=np.int64),
                       yfy=np.zeros(200))
        assert ei.value.status == _capi.ST_ERR_CAPACITY


def test_served_matches_oracle():
    w = serving.served_workload("cuda", n_jobs=6, seed=12, size_scale=0.02, max_size=20_000)
    w.n_os[:] = np.minimum(w.n_os, 10)
    with st.Server(0, budget_bytes=40_000_000_000, max_track_deposits=20_000) as srv:
        counts, yfy, rec, _ = serving.replay(srv, w, np.zeros(w.n_jobs, dtype=np.int64))
    assert np.all(rec["status"] == 0)
    oc, oy, _, _ = oracle_run(w)      # one histogram per job, as served
    for j in range(w.n_jobs):
        _assert_same(counts[j], yfy[j], oc[j], oy[j])


def test_latency_records_under_load(stream):
    w, _ = stream
    arr = serving.poisson_arrivals(w, offered_dep_os_per_s=5e9, seed=4)
    with st.Server(0, budget_bytes=40_000_000_000, max_track_deposits=200_000) as srv:
        _, _, rec, wall = serving.replay(srv, w, arr)
    s = serving.latency_summary(rec, serving.job_work(w))
    assert s["failed"] == 0
    assert 0 < s["p50_ms"] <= s["p95_ms"] <= s["p99_ms"] <= s["max_ms"]
    assert np.all(rec["submit_ns"][1:] >= rec["submit_ns"][:-1])
    assert wall * 1e3 >= arr[-1] / 1e6
