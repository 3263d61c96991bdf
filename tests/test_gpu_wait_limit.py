"""The fused kernel's one cross-CTA wait (a helper of a shared unit waiting for the first helper
to publish the unit's spill table) gives up after its limit instead of hanging: run on the GPU
against a table that is never published, with a short limit, it returns -1 and sets device error
flag 8, which st_run reports as ST_ERR_DEVICE_WAIT. The context stays usable: a run afterwards
is exact. No GPU faults or hangs; the table that is never published stands in for a helper that
died."""
import numpy as np
import pytest

import pyoracle as po
import supertrack_b200 as st
from helpers import assert_hist_equal

pytestmark = pytest.mark.gpu


def test_wait_gives_up_and_reports(ctx):
    table, flags = ctx.probe_unit_wait(-1, 1000)
    assert table == -1 and flags & 8
    table, flags = ctx.probe_unit_wait(-1, 0)
    assert table == -1 and flags & 8


def test_published_table_is_taken_at_once(ctx):
    table, flags = ctx.probe_unit_wait(5, 1000)
    assert table == 5 and flags == 0


def test_limit_is_checked(ctx):
    with pytest.raises(st.StError):
        ctx.probe_unit_wait(-1, (1 << 24) + 1)


def test_context_usable_after_a_wait_ran_out(ctx):
    ctx.probe_unit_wait(-1, 100)
    rs = np.random.default_rng(4)
    n = 3000
    pos = np.cumsum(rs.normal(size=(n, 3)) * 1.5, axis=0)
    e = np.clip(np.exp(np.log(15) + 0.8 * rs.normal(size=n)), 10, 1000)
    x, y, z = pos[:, 0].copy(), pos[:, 1].copy(), pos[:, 2].copy()
    spec = ("lin", 300, 0.01, 100.0)
    ctx.clear()
    hid = ctx.histogram(*spec)
    ctx.submit(x, y, z, e, half_length=100.0, sphere_diameter=5.0, n_oversamples=4, hist=hid,
               seed=2, track_id=0, zshift="none")
    ctx.run()
    gc, gy = ctx.read_histogram(hid)
    ed = po.edges(*spec)
    oc = np.zeros(len(ed) - 1, dtype=np.int64)
    oy = np.zeros(len(ed) - 1)
    sx = st.oversample_shifts(100.0, 5.0, True, 2, 0, 4)
    po.run_job(x, y, z, e, half_length=100.0, sphere_diameter=5.0, sxsy=sx, edges_arr=ed,
               zshift="none", counts=oc, yfy=oy)
    assert_hist_equal([gc], [gy], [oc], [oy])
    assert gc.sum() > 0
    ctx.clear()
