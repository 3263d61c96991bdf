"""FP32 geometry variant on the GPU (context parameter precision = 32) against its CPU
restatement (or_job_f32) on the same seeded inputs and shifts.

Every float operation of the variant is rounded on its own on both sides, so the bar is the FP64
path's: hit, sphere and histogram counts and sphere keys bit-exact, per-sphere energies exact
(the same integer accumulation), y*f(y) per bin within 1e-12 relative.
"""
import numpy as np
import pytest

import supertrack_b200.workloads as W
from helpers import assert_hist_equal, assert_stats_equal, gpu_run, oracle_run

pytestmark = pytest.mark.gpu


@pytest.fixture
def ctx32(ctx):
    old = ctx.get_param("precision")
    ctx.set_param("precision", 32)
    assert ctx.get_param("precision") == 32
    yield ctx
    ctx.set_param("precision", old)


def _check(ctx, w, mode="batched", zshift=None):
    gc, gy, gs, _ = gpu_run(ctx, w, mode=mode, zshift=zshift)
    oc, oy, os_, _ = oracle_run(w, zshift=zshift, precision=32)
    assert_stats_equal(gs, os_)
    assert_hist_equal(gc, gy, oc, oy)
    return gs, os_


def test_config0_full(ctx32):
    _check(ctx32, W.config0())


@pytest.mark.parametrize("mode", ["batched", "plain"])
def test_config1_scaled(ctx32, mode):
    _check(ctx32, W.config1(n_tracks=2, n_dep=200_000, n_os=3), mode=mode)


def test_config2_scaled_mixed_geometries(ctx32):
    _check(ctx32, W.config2(n_tracks=96, size_scale=0.05, os_scale=0.2))


def test_config4_scaled_dense_spill(ctx32):
    _check(ctx32, W.config4(n_tracks=1, n_dep=600_000, n_os=2))


@pytest.mark.parametrize("gen,d,n,n_os", [("ion", 2.0, 120_000, 4), ("ion", 10.0, 200_000, 5),
                                          ("proton", 2.0, 60_000, 6)])
def test_window_boundary_flags(ctx32, gen, d, n, n_os):
    """Multi-window jobs on fine lattices: the boundary flags use cells widened by HL' 2^-16 so
    that two float hits of one sphere still lie in neighbouring cells."""
    if gen == "proton":
        w = W.config0(n_tracks=1, n_dep=n, n_os=n_os)
    else:
        w = W.config1(n_tracks=1, n_dep=n, n_os=n_os)
    w.diameter[:] = d
    _check(ctx32, w)


def test_zshift_modes_and_no_shift(ctx32):
    w = W.config0(n_tracks=3, n_os=2)
    for zs in ("plus", "minus", "none"):
        _check(ctx32, w, zshift=zs)
    w.shift_track = False
    _check(ctx32, w)


def test_spheres_exported(ctx32):
    w = W.config0(n_tracks=3, n_os=4)
    _, _, _, sph = gpu_run(ctx32, w, export_cap=1 << 20)
    _, _, _, osph = oracle_run(w, spheres_cap=1 << 20, precision=32)
    for j in range(w.n_jobs):
        g = np.sort(sph[sph["job"] == j], order=["os", "key"])
        o = np.sort(osph[j], order=["os", "key"])
        assert len(g) == len(o)
        assert np.array_equal(g["key"], o["key"])
        assert np.array_equal(g["y"], o["y"])


def test_midpoint_deposit_key_follows_precision(ctx):
    """x = 10 + 5e-9 (HL 2500, d 10, no shift, z at a centre) scores in sphere 251 in FP64 and
    in sphere 250 in the FP32 form, on the GPU as in the oracle."""
    import torch
    n = 500
    want = {64: 251 + 250 * n + 250 * n * n, 32: 250 + 250 * n + 250 * n * n}
    old = ctx.get_param("precision")
    try:
        for prec in (64, 32):
            ctx.set_param("precision", prec)
            ctx.clear()
            h = ctx.histogram("lin", 10, 0.0, 100.0)
            x = np.array([10.0 + 5e-9]); y = np.array([5.0]); z = np.array([5.0])
            e = np.array([100.0])
            ctx.submit(x, y, z, e, half_length=2500.0, sphere_diameter=10.0, n_oversamples=1,
                       hist=h, seed=1, track_id=0, shift_track=False, zshift="none")
            sph = ctx.run_export(16)
            assert len(sph) == 1
            assert int(sph["key"][0]) == want[prec]
    finally:
        ctx.set_param("precision", old)
        torch.cuda.synchronize()
