"""GPU path (through the C ABI) against the CPU oracle on the same seeded inputs and shifts.

Bar: sphere keys, hit counts, sphere counts and histogram counts bit-exact; per-sphere lineal
energies bit-exact against the oracle's exact sum and within 1e-12 relative of its literal
left-to-right FP64 sum; y*f(y) per bin within 1e-12 relative (its float64 accumulation order
across spheres is not fixed).
"""
import numpy as np
import pytest

import pyoracle as po
import supertrack_b200 as st
import supertrack_b200.workloads as W
from helpers import assert_hist_equal, assert_stats_equal, gpu_run, oracle_run

pytestmark = pytest.mark.gpu


def test_config0_full_bit_exact(ctx):
    w = W.config0()
    gc, gy, gs, _ = gpu_run(ctx, w)
    oc, oy, os_, _ = oracle_run(w)
    assert_stats_equal(gs, os_)
    assert_hist_equal(gc, gy, oc, oy)
    assert gc[0].sum() > 10000


def test_config0_spheres_exported(ctx):
    w = W.config0(n_tracks=3, n_os=4)
    _, _, _, sph = gpu_run(ctx, w, export_cap=1 << 20)
    _, _, _, osph = oracle_run(w, spheres_cap=1 << 20)
    for j in range(w.n_jobs):
        g = sph[sph["job"] == j]
        o = osph[j]
        g = np.sort(g, order=["os", "key"])
        o = np.sort(o, order=["os", "key"])
        assert len(g) == len(o)
        assert np.array_equal(g["key"], o["key"])
        assert np.array_equal(g["os"], o["os"])
        assert np.array_equal(g["y"], o["y"])                       # exact sum, bit for bit
        rel = np.abs(g["y"] - o["y_seq"]) / np.abs(o["y_seq"])
        assert rel.max() <= 1e-12                                   # literal FP64 order


@pytest.mark.parametrize("mode", ["batched", "plain"])
def test_config1_scaled(ctx, mode):
    w = W.config1(n_tracks=2, n_dep=200_000, n_os=3)
    gc, gy, gs, _ = gpu_run(ctx, w, mode=mode)
    oc, oy, os_, _ = oracle_run(w)
    assert_stats_equal(gs, os_)
    assert_hist_equal(gc, gy, oc, oy)


def test_config2_scaled_mixed_geometries(ctx):
    w = W.config2(n_tracks=96, size_scale=0.05, os_scale=0.2)
    gc, gy, gs, _ = gpu_run(ctx, w)
    oc, oy, os_, _ = oracle_run(w)
    assert_stats_equal(gs, os_)
    assert_hist_equal(gc, gy, oc, oy)


def test_config4_scaled_dense_spill(ctx):
    """Dense 10 nm spheres with thousands of deposits each, and more spheres per oversample than
    the shared-memory table holds: exercises the HBM spill table."""
    w = W.config4(n_tracks=1, n_dep=600_000, n_os=2)
    gc, gy, gs, _ = gpu_run(ctx, w)
    oc, oy, os_, _ = oracle_run(w)
    assert_stats_equal(gs, os_)
    assert_hist_equal(gc, gy, oc, oy)


def test_sparse_spill_many_spheres(ctx):
    """2 nm spheres over a dense ion track: tens of thousands of distinct spheres per
    oversample, far more than the shared-memory table holds (repeated flushes to HBM)."""
    w = W.config1(n_tracks=1, n_dep=300_000, n_os=2)
    gc, gy, gs, _ = gpu_run(ctx, w)
    oc, oy, os_, _ = oracle_run(w)
    assert_stats_equal(gs, os_)
    assert_hist_equal(gc, gy, oc, oy)
    assert gs[0]["spheres"] > 2 * 40000


def test_batched_plain_and_alone_agree(ctx):
    """Each job's result is the same alone, in a batch and in the per-track loop."""
    w = W.config2(n_tracks=40, size_scale=0.03, os_scale=0.1)
    bc, by, bs, _ = gpu_run(ctx, w, mode="batched")
    pc, py, ps, _ = gpu_run(ctx, w, mode="plain")
    for j in range(0, w.n_jobs, 7):
        hid = ctx.histogram(*w.hists[j])
        ac, ay, as_, _ = gpu_run(ctx, w, jobs=[j], hist_ids=[hid] * len(w.hists))
        assert np.array_equal(ac[0], bc[j])
        assert np.array_equal(as_[0]["hits"], bs[j]["hits"])
        np.testing.assert_allclose(ay[0], by[j], rtol=1e-12, atol=0)
    for j in range(w.n_jobs):
        assert np.array_equal(bc[j], pc[j])
        np.testing.assert_allclose(by[j], py[j], rtol=1e-12, atol=0)


def test_zshift_modes(ctx):
    w = W.config0(n_tracks=3, n_os=2)
    for zs in ("plus", "minus", "none"):
        gc, gy, gs, _ = gpu_run(ctx, w, zshift=zs)
        oc, oy, os_, _ = oracle_run(w, zshift=zs)
        assert_stats_equal(gs, os_)
        assert_hist_equal(gc, gy, oc, oy)


def test_no_shift_oversamples_repeat(ctx):
    w = W.config0(n_tracks=2, n_os=5)
    w.shift_track = False
    gc, _, gs, _ = gpu_run(ctx, w)
    w1 = W.config0(n_tracks=2, n_os=1)
    w1.shift_track = False
    c1, _, s1, _ = gpu_run(ctx, w1)
    assert np.array_equal(gc[0], 5 * c1[0])


@pytest.mark.parametrize("gen,d,n,n_os", [("ion", 2.0, 120_000, 4), ("ion", 10.0, 200_000, 5),
                                          ("proton", 2.0, 60_000, 6), ("ion4", 10.0, 150_000, 4),
                                          ("ion", 2.0, 400_000, 4)])
def test_window_boundary_flags(ctx, gen, d, n, n_os):
    """Multi-window jobs on fine lattices (the prepare stage flags boundary deposits and the fused
    kernel bins complete spheres per window; boundary spheres go through the spill log, whose
    reduction takes several bucketed passes for the 400,000-deposit track): bit-exact with the
    oracle."""
    if gen == "proton":
        w = W.config0(n_tracks=1, n_dep=n, n_os=n_os)
    elif gen == "ion4":
        w = W.config4(n_tracks=1, n_dep=n, n_os=n_os)
    else:
        w = W.config1(n_tracks=1, n_dep=n, n_os=n_os)
    w.diameter[:] = d
    old = ctx.get_param("flag_min_kept")
    ctx.set_param("flag_min_kept", 0)       # flags for every qualifying job, however few kept
    try:
        gc, gy, gs, _ = gpu_run(ctx, w)
    finally:
        ctx.set_param("flag_min_kept", old)
    oc, oy, os_, _ = oracle_run(w)
    assert_stats_equal(gs, os_)
    assert_hist_equal(gc, gy, oc, oy)
