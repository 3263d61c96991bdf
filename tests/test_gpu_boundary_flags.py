"""Window boundary flags under both flag-cell schemes (context parameter flag_cells_limit: cells of
side d probed 27 ways, or of side 2d probed 8 ways by the half of the cell a deposit lies in),
against the CPU oracle. The track is three windows of 8192 kept deposits; half of the second and
third windows sit within d of a deposit of the window before (random directions and lengths up to
d, exactly d on some axes, and deposits placed at the centre and near the edges of the 2d cells),
so that many spheres take hits from two windows. A sphere whose cross-window hits were not
flagged would be binned twice, which changes the sphere count and the spectrum; so hits, spheres,
binned spheres and counts must be bit-exact and y*f(y) within 1e-12, in FP64 and in the FP32
geometry variant."""
import numpy as np
import pytest

import pyoracle as po
import supertrack_b200 as st
from helpers import assert_hist_equal, assert_stats_equal

pytestmark = pytest.mark.gpu

HL, D, N_OS, WIN = 100.0, 1.0, 6, 8192
L2 = 2.0 * D * (1.0 + 2.0 ** -10)     # side of the 2d flag cells


def _partners(rs, base):
    """A partner within distance d of every point of base."""
    n = len(base)
    v = rs.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    length = D * rs.random(n)
    length[: n // 8] = D                       # exactly d
    out = base + v * length[:, None]
    axis = rs.integers(0, 3, n // 8)           # exactly d along one axis
    sign = rs.choice([-1.0, 1.0], n // 8)
    out[n // 8: n // 4] = base[n // 8: n // 4]
    out[np.arange(n // 8, n // 4), axis] += sign * D
    return out


def _track(seed=0):
    rs = np.random.default_rng(seed)
    w0 = rs.uniform(-90, 90, size=(WIN, 3))
    # a quarter of the first window on the centre plane or near the edges of the 2d cells
    k = np.floor(w0[: WIN // 4] / L2)
    frac = rs.choice([0.5, 0.5 - 1e-9, 0.5 + 1e-9, 1e-9, 1.0 - 1e-9, 0.25, 0.75],
                     size=(WIN // 4, 3))
    w0[: WIN // 4] = (k + frac) * L2
    w1 = np.concatenate([_partners(rs, w0[: WIN // 2]), rs.uniform(-90, 90, size=(WIN // 2, 3))])
    w2 = np.concatenate([_partners(rs, w1[WIN // 2:]), rs.uniform(-90, 90, size=(WIN // 2, 3))])
    pos = np.concatenate([w0, w1, w2])
    e = np.clip(np.exp(np.log(20) + 0.8 * rs.normal(size=len(pos))), 10, 1000)
    return pos[:, 0].copy(), pos[:, 1].copy(), pos[:, 2].copy(), e


@pytest.mark.parametrize("precision", [64, 32])
@pytest.mark.parametrize("limit", [0, 1 << 50])
def test_cross_window_spheres_under_both_flag_cell_schemes(ctx, limit, precision):
    x, y, z, e = _track()
    spec = ("log", 300, 0.01, 1e4)
    old = (ctx.get_param("flag_cells_limit"), ctx.get_param("precision"))
    ctx.set_param("flag_cells_limit", limit)
    ctx.set_param("precision", precision)
    try:
        ctx.clear()
        hid = ctx.histogram(*spec)
        jid = ctx.submit(x, y, z, e, half_length=HL, sphere_diameter=D, n_oversamples=N_OS,
                         hist=hid, seed=11, track_id=3, zshift="none")
        ctx.run()
        gc, gy = ctx.read_histogram(hid)
        gs = ctx.stats(jid)
    finally:
        ctx.set_param("flag_cells_limit", old[0])
        ctx.set_param("precision", old[1])
    ed = po.edges(*spec)
    oc = np.zeros(len(ed) - 1, dtype=np.int64)
    oy = np.zeros(len(ed) - 1)
    sx = st.oversample_shifts(HL, D, True, 11, 3, N_OS)
    _, _, os_, _ = po.run_job(x, y, z, e, half_length=HL, sphere_diameter=D, sxsy=sx,
                              edges_arr=ed, zshift="none", counts=oc, yfy=oy,
                              precision=precision)
    assert_stats_equal([gs], [os_])
    assert_hist_equal([gc], [gy], [oc], [oy])
    assert gs["spheres"] > 0
