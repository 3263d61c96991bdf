"""The prepare stage's cell grouping (context parameter sort_deposits) at its edges, against the
CPU oracle: every prepare block grouped (mode 2), on ragged track sizes around the 1024-deposit
block, on a block whose deposits all lie in one cell (one group of 1024), with non-finite and
out-of-voxel deposits mixed in, and on a dense multi-window track in every mode. The grouping
only reorders each block's kept deposits, so counts, hits, spheres and binned spheres must be
bit-exact and y*f(y) within 1e-12, as without it."""
import numpy as np
import pytest

import pyoracle as po
import supertrack_b200 as st
import supertrack_b200.workloads as W
from helpers import assert_hist_equal, assert_stats_equal, gpu_run, oracle_run

pytestmark = pytest.mark.gpu


@pytest.fixture
def sorted_ctx(ctx):
    old = ctx.get_param("sort_deposits")
    ctx.set_param("sort_deposits", 2)
    yield ctx
    ctx.set_param("sort_deposits", old)


def _track(n, seed=0, spread=40.0):
    rs = np.random.default_rng(seed)
    pos = np.cumsum(rs.normal(size=(n, 3)) * 1.5, axis=0) + rs.normal(size=3) * spread
    e = np.clip(np.exp(np.log(15) + 0.8 * rs.normal(size=n)), 10, 1000)
    return pos[:, 0].copy(), pos[:, 1].copy(), pos[:, 2].copy(), e


def _both(ctx, tracks, hl=100.0, d=5.0, n_os=3, spec=("lin", 400, 0.01, 100.0), seed=5):
    ctx.clear()
    hid = ctx.histogram(*spec)
    ids = [ctx.submit(*t, half_length=hl, sphere_diameter=d, n_oversamples=n_os, hist=hid,
                      seed=seed, track_id=i, zshift="none") for i, t in enumerate(tracks)]
    ctx.run()
    gc, gy = ctx.read_histogram(hid)
    gs = [ctx.stats(i) for i in ids]
    e = po.edges(*spec)
    oc = np.zeros(len(e) - 1, dtype=np.int64)
    oy = np.zeros(len(e) - 1)
    os_ = []
    for i, t in enumerate(tracks):
        sx = st.oversample_shifts(hl, d, True, seed, i, n_os)
        _, _, s, _ = po.run_job(*t, half_length=hl, sphere_diameter=d, sxsy=sx, edges_arr=e,
                                zshift="none", counts=oc, yfy=oy)
        os_.append(s)
    assert_stats_equal(gs, os_)
    assert_hist_equal([gc], [gy], [oc], [oy])
    return gc


@pytest.mark.parametrize("n", [1, 2, 1023, 1024, 1025, 2047, 2049, 4097])
def test_grouped_blocks_ragged_sizes(sorted_ctx, n):
    _both(sorted_ctx, [_track(n, seed=n)])


def test_grouped_block_with_every_deposit_in_one_cell(sorted_ctx):
    """2,500 deposits at one point (their blocks hold a single group of up to 1024, the largest
    rank the grouping stores), then a scattered tail."""
    x, y, z, e = _track(600, seed=3)
    pt = np.full(2500, 7.25)
    track = (np.concatenate([pt, x]), np.concatenate([pt, y]), np.concatenate([pt, z]),
             np.concatenate([np.full(2500, 20.0), e]))
    gc = _both(sorted_ctx, [track], d=10.0)
    assert gc.sum() > 0


def test_grouped_blocks_with_dropped_and_nonfinite_deposits(sorted_ctx):
    x, y, z, e = _track(3000, seed=9)
    x[::7] = np.nan
    y[1::11] = np.inf
    z[2::13] = 1e6           # outside the voxel for every shift
    _both(sorted_ctx, [(x, y, z, e), _track(1500, seed=10)])


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_dense_windowed_track_in_every_mode(ctx, mode):
    """A dense 10 nm track with window flags (several windows): the grouped layout changes which
    deposits share a window, and the boundary flags follow it."""
    w = W.config4(n_tracks=1, n_dep=150_000, n_os=4)
    old = (ctx.get_param("sort_deposits"), ctx.get_param("flag_min_kept"))
    ctx.set_param("sort_deposits", mode)
    ctx.set_param("flag_min_kept", 0)
    try:
        gc, gy, gs, _ = gpu_run(ctx, w)
    finally:
        ctx.set_param("sort_deposits", old[0])
        ctx.set_param("flag_min_kept", old[1])
    oc, oy, os_, _ = oracle_run(w)
    assert_stats_equal(gs, os_)
    assert_hist_equal(gc, gy, oc, oy)
