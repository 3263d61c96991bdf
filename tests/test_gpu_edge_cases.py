"""Edge cases of the GPU path: empty and ragged tracks, non-finite inputs, capacities,
degenerate geometries, many tiny jobs."""
import numpy as np
import pytest

import pyoracle as po
import supertrack_b200 as st
from supertrack_b200 import _capi

pytestmark = pytest.mark.gpu


def _track(n, seed=0, spread=60.0):
    rs = np.random.default_rng(seed)
    steps = rs.normal(size=(n, 3)) * 1.5
    pos = np.cumsum(steps, axis=0) + rs.normal(size=3) * spread
    e = np.clip(np.exp(np.log(15) + 0.8 * rs.normal(size=n)), 10, 1000)
    return pos[:, 0].copy(), pos[:, 1].copy(), pos[:, 2].copy(), e


def _both(ctx, tracks, hl=100.0, d=5.0, n_os=3, spec=("lin", 400, 0.01, 100.0), zshift="none",
          seed=11):
    ctx.clear()
    hid = ctx.histogram(*spec)
    ids = [ctx.submit(*t, half_length=hl, sphere_diameter=d, n_oversamples=n_os, hist=hid,
                      seed=seed, track_id=i, zshift=zshift) for i, t in enumerate(tracks)]
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
                                zshift=zshift, counts=oc, yfy=oy)
        os_.append(s)
    return gc, gy, gs, oc, oy, os_


@pytest.mark.parametrize("n", [0, 1, 2, 31, 32, 33, 255, 256, 257, 1023, 4097])
def test_ragged_sizes(ctx, n):
    gc, gy, gs, oc, oy, os_ = _both(ctx, [_track(n, seed=n)])
    assert np.array_equal(gc, oc)
    np.testing.assert_allclose(gy, oy, rtol=1e-12, atol=0)
    assert gs[0]["hits"] == os_[0]["hits"]


def test_many_tiny_jobs(ctx):
    tracks = [_track(int(n), seed=i) for i, n in
              enumerate(np.random.default_rng(1).integers(0, 40, 600))]
    gc, gy, gs, oc, oy, os_ = _both(ctx, tracks, n_os=2)
    assert np.array_equal(gc, oc)
    assert [g["hits"] for g in gs] == [o["hits"] for o in os_]


def test_nonfinite_coordinates_are_filtered(ctx):
    x, y, z, e = _track(500, seed=3)
    x[::7] = np.nan
    y[3::11] = np.inf
    z[5::13] = -np.inf
    gc, gy, gs, oc, oy, os_ = _both(ctx, [(x, y, z, e)])
    assert np.array_equal(gc, oc)
    assert gs[0]["hits"] == os_[0]["hits"] and gs[0]["hits"] > 0


def test_nonfinite_edep_rejects_only_that_job(ctx):
    good = _track(300, seed=4)
    bad = list(_track(300, seed=5))
    bad[3] = bad[3].copy()
    bad[3][17] = np.nan
    ctx.clear()
    hid = ctx.histogram("lin", 400, 0.01, 100.0)
    j0 = ctx.submit(*good, half_length=100.0, sphere_diameter=5.0, n_oversamples=2, hist=hid,
                    seed=1, zshift="none")
    j1 = ctx.submit(*bad, half_length=100.0, sphere_diameter=5.0, n_oversamples=2, hist=hid,
                    seed=1, track_id=1, zshift="none")
    with pytest.raises(st.StError) as ex:
        ctx.run()
    assert ex.value.status == _capi.ST_ERR_NONFINITE_EDEP
    assert ctx.stats(j1)["status"] == _capi.ST_ERR_NONFINITE_EDEP
    assert ctx.stats(j0)["status"] == 0
    gc, _ = ctx.read_histogram(hid)
    e = po.edges("lin", 400, 0.01, 100.0)
    oc = np.zeros(400, dtype=np.int64)
    po.run_job(*good, half_length=100.0, sphere_diameter=5.0,
               sxsy=st.oversample_shifts(100.0, 5.0, True, 1, 0, 2), edges_arr=e,
               zshift="none", counts=oc)
    assert np.array_equal(gc, oc)


def test_negative_and_zero_edep(ctx):
    x, y, z, e = _track(800, seed=6)
    e = e.copy()
    e[::3] *= -1
    e[1::5] = 0.0
    gc, gy, gs, oc, oy, os_ = _both(ctx, [(x, y, z, e)], spec=("lin", 400, -100.0, 100.0))
    assert np.array_equal(gc, oc)
    assert gs[0]["spheres"] == os_[0]["spheres"]


def test_zero_oversamples_and_single_sphere_geometry(ctx):
    t = _track(400, seed=7, spread=2.0)
    gc, _, gs, oc, _, _ = _both(ctx, [t], n_os=0)
    assert gc.sum() == 0 and gs[0]["hits"] == 0
    # sphere larger than the voxel: the voxel becomes that one sphere
    gc, gy, gs, oc, oy, os_ = _both(ctx, [t], hl=3.0, d=20.0, n_os=4)
    assert np.array_equal(gc, oc)
    assert gs[0]["hits"] == os_[0]["hits"]


def test_rejected_inputs(ctx):
    hid = ctx.histogram("lin", 10, 0.0, 10.0)
    t = _track(10)
    with pytest.raises(st.StError) as ex:
        ctx.submit(*t, half_length=1.5e6, sphere_diameter=0.5, n_oversamples=1, hist=hid)
    assert ex.value.status == _capi.ST_ERR_BAD_GEOMETRY
    with pytest.raises(st.StError):
        ctx.submit(*t, half_length=10, sphere_diameter=1, n_oversamples=1, hist=hid + 100)
    with pytest.raises(st.StError) as ex:
        ctx.histogram("log", 10, 0.0, 10.0)
    assert ex.value.status == _capi.ST_ERR_BAD_HISTOGRAM


def test_export_capacity_error(ctx):
    ctx.clear()
    hid = ctx.histogram("lin", 400, 0.01, 100.0)
    ctx.submit(*_track(2000, seed=8), half_length=100.0, sphere_diameter=5.0, n_oversamples=4,
               hist=hid, zshift="none")
    with pytest.raises(st.StError) as ex:
        ctx.run_export(3)
    assert ex.value.status == _capi.ST_ERR_CAPACITY


def test_device_resident_tracks(ctx):
    import torch
    t = _track(5000, seed=9)
    dev = [torch.tensor(a, device="cuda") for a in t]
    ctx.clear()
    hid = ctx.histogram("lin", 400, 0.01, 100.0)
    ctx.submit(*dev, half_length=100.0, sphere_diameter=5.0, n_oversamples=3, hist=hid, seed=3,
               zshift="none", on_device=True)
    ctx.run()
    gc, _ = ctx.read_histogram(hid)
    hid2 = ctx.histogram("lin", 400, 0.01, 100.0)
    ctx.clear()
    ctx.submit(*t, half_length=100.0, sphere_diameter=5.0, n_oversamples=3, hist=hid2, seed=3,
               zshift="none")
    ctx.run()
    hc, _ = ctx.read_histogram(hid2)
    assert np.array_equal(gc, hc) and gc.sum() > 0


def test_run_refuses_jobs_of_forgotten_histograms(ctx):
    """st_hists_clear forgets the histograms; queued jobs that still name one make the run fail
    with ST_ERR_STATE instead of adding into a stale table. Zeroing (st_hist_reset) keeps them."""
    ctx.clear()
    hid = ctx.histogram("lin", 50, 0.01, 100.0)
    ctx.submit(*_track(3000, seed=3), half_length=100.0, sphere_diameter=5.0, n_oversamples=2,
               hist=hid, seed=1, track_id=0, zshift="none")
    ctx.run()
    first = ctx.read_histogram(hid)[0].copy()
    assert first.sum() > 0
    ctx.reset_histogram(-1)
    ctx.jobs_reset()
    ctx.run()
    assert np.array_equal(ctx.read_histogram(hid)[0], first)
    ctx.clear_histograms()
    ctx.jobs_reset()
    with pytest.raises(st.StError) as ei:
        ctx.run()
    assert ei.value.status == _capi.ST_ERR_STATE
    ctx.clear()
