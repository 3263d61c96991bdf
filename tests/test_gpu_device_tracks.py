"""Device-resident tracks (st_track_view.on_device) read in place by the prepare stage, against the
CPU oracle: every combination of 16-byte-aligned and 8-byte-offset x, y, z and edep arrays, with
track sizes around the 1024-deposit prepare blocks, must give bit-exact counts, hits, spheres and
binned spheres and y*f(y) within 1e-12. Device arrays that are not 8-byte aligned cannot be read
as doubles and are refused at submit."""
import itertools

import numpy as np
import pytest

import pyoracle as po
import supertrack_b200 as st
from helpers import assert_hist_equal, assert_stats_equal

pytestmark = pytest.mark.gpu

SPEC = ("log", 200, 0.01, 1e4)


def _track(n, seed):
    rs = np.random.default_rng(seed)
    pos = np.cumsum(rs.normal(size=(n, 3)) * 2.0, axis=0) + rs.normal(size=3) * 30.0
    e = np.clip(np.exp(np.log(15) + 0.8 * rs.normal(size=n)), 10, 1000)
    return [pos[:, 0].copy(), pos[:, 1].copy(), pos[:, 2].copy(), e]


def _device_arrays(arrays, offsets):
    """Copies each array into a fresh 16-byte-aligned device buffer at element offset 0 or 1."""
    import torch
    out, keep = [], []
    for a, off in zip(arrays, offsets):
        buf = torch.zeros(len(a) + 2, dtype=torch.float64, device="cuda")
        assert buf.data_ptr() % 16 == 0
        buf[off:off + len(a)] = torch.from_numpy(a)
        keep.append(buf)
        out.append(buf.data_ptr() + 8 * off)
    return out, keep


@pytest.mark.parametrize("n", [1, 2, 3, 1023, 1024, 1025, 2047, 2049, 5000])
def test_device_tracks_every_alignment(ctx, n):
    track = _track(n, seed=n)
    ed = po.edges(*SPEC)
    combos = list(itertools.product([0, 1], repeat=4))
    ctx.clear()
    hid = [ctx.histogram(*SPEC) for _ in combos]
    keep, ids = [], []
    for t, offs in enumerate(combos):
        ptrs, bufs = _device_arrays(track, offs)
        keep.append(bufs)
        ids.append(ctx.submit(*ptrs, half_length=100.0, sphere_diameter=4.0, n_oversamples=3,
                              hist=hid[t], seed=9, track_id=t, zshift="none", on_device=True,
                              n=n))
    ctx.run()
    for t in range(len(combos)):
        gc, gy = ctx.read_histogram(hid[t])
        oc = np.zeros(len(ed) - 1, dtype=np.int64)
        oy = np.zeros(len(ed) - 1)
        sx = st.oversample_shifts(100.0, 4.0, True, 9, t, 3)
        _, _, os_, _ = po.run_job(*track, half_length=100.0, sphere_diameter=4.0, sxsy=sx,
                                  edges_arr=ed, zshift="none", counts=oc, yfy=oy)
        assert_stats_equal([ctx.stats(ids[t])], [os_])
        assert_hist_equal([gc], [gy], [oc], [oy])
    ctx.clear()
    del keep


def test_misaligned_device_arrays_are_refused(ctx):
    import torch
    buf = torch.zeros(64, dtype=torch.float64, device="cuda")
    base = buf.data_ptr()
    ctx.clear()
    hid = ctx.histogram(*SPEC)
    with pytest.raises(st.StError) as err:
        ctx.submit(base + 4, base, base, base, half_length=100.0, sphere_diameter=4.0,
                   n_oversamples=1, hist=hid, on_device=True, n=8)
    assert "INVALID_ARGUMENT" in str(err.value)
    # an 8-byte offset is a valid double array
    ctx.submit(base + 8, base, base, base, half_length=100.0, sphere_diameter=4.0,
               n_oversamples=1, hist=hid, on_device=True, n=8)
    ctx.clear()
