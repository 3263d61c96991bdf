"""Contribution ranges at the edges of the exact accumulators, against the CPU oracle, on dense
multi-window tracks with window flags on: a wide edep range (about 40 bits between the smallest
and largest contribution on the job's fixed-point grid, values past 64 bits), a narrow range with
negative energies (two's-complement sums whose spheres can total below zero and fall out of the
spectrum), and all-zero energies (no grid at all). Counts, hits, spheres and binned spheres
bit-exact; y*f(y) within 1e-12."""
import numpy as np
import pytest
import torch

import supertrack_b200.workloads as W
from helpers import assert_hist_equal, assert_stats_equal, gpu_run, oracle_run

pytestmark = pytest.mark.gpu


def _workload(edep_fn):
    w = W.config4(n_tracks=2, n_dep=60_000, n_os=4)
    rs = np.random.default_rng(17)
    e = edep_fn(rs, int(w.sizes.sum()))
    w.edep = torch.from_numpy(e)
    return w


@pytest.mark.parametrize("form", ["wide", "negative", "zero"])
def test_contribution_ranges(ctx, form):
    if form == "wide":       # 1e-6 .. 1e6 eV: about 40 bits of range on the grid
        fn = lambda rs, n: np.exp(rs.uniform(np.log(1e-6), np.log(1e6), n))
    elif form == "negative":  # 10 .. 1000 eV with every seventh deposit negative
        fn = lambda rs, n: np.where(np.arange(n) % 7 == 3, -1.0, 1.0) * rs.uniform(10, 1000, n)
    else:
        fn = lambda rs, n: np.zeros(n)
    w = _workload(fn)
    old = ctx.get_param("flag_min_kept")
    ctx.set_param("flag_min_kept", 0)
    try:
        gc, gy, gs, _ = gpu_run(ctx, w)
    finally:
        ctx.set_param("flag_min_kept", old)
    oc, oy, os_, _ = oracle_run(w)
    assert_stats_equal(gs, os_)
    assert_hist_equal(gc, gy, oc, oy)
    if form != "zero":
        assert sum(s["binned"] for s in gs) > 0
