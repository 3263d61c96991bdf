"""st_superimpose_noalloc: the superimposition entry point that allocates no device memory.

Callers that cannot allocate on their path use it: cudaFree synchronises the whole device (a
serving thread sharing the GPU cannot stall every other stream), and frameworks that own all
device memory through their own pool leave no room for, or forbid, a plug-in's cudaMalloc. The
entry point runs in a fixed scratch array compiled into the library. These tests call it through
the C ABI and compare it with the regular entry points (st_job_submit + st_run + st_hist_read)
and with the CPU oracle fed the same shifts, on the same tracks: histogram counts, hits and
spheres must be identical and y*f(y) within 1e-12 relative, on two calls in a row (the second
call reuses the scratch the first one left behind), on the default stream and on a created
stream. This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import pyoracle as po
import supertrack_b200 as st
import supertrack_b200.workloads as W
from supertrack_b200 import _capi

pytestmark = pytest.mark.gpu


def _regular(track, hl, d, n_os, seed, tid, zshift, spec):
    with st.Context(0) as ctx:
        hid = ctx.histogram(*spec)
        j = ctx.submit(*track, half_length=hl, sphere_diameter=d, n_oversamples=n_os, hist=hid,
                       seed=seed, track_id=tid, zshift=zshift)
        ctx.run()
        counts, yfy = ctx.read_histogram(hid)
        return counts, yfy, ctx.stats(j)


def _noalloc(track, hl, d, n_os, seed, tid, zshift, spec, stream=None):
    dev = [torch.tensor(a, device="cuda", dtype=torch.float64) for a in track]
    v = _capi.st_track_view()
    v.x, v.y, v.z, v.edep = [t.data_ptr() for t in dev]
    v.n = int(dev[0].numel())
    v.on_device = 1
    desc = _capi.st_job_desc()
    desc.half_length = hl
    desc.sphere_diameter = d
    desc.zshift = st.ZSHIFT[zshift]
    desc.shift_track = 1
    desc.n_oversamples = n_os
    desc.hist_id = -1
    desc.seed = seed
    desc.track_id = tid
    kind, nb, lo, hi = spec
    counts = torch.zeros(nb, dtype=torch.int64, device="cuda")
    yfy = torch.zeros(nb, dtype=torch.float64, device="cuda")
    stats = _capi.st_job_stats()
    # the inputs were filled on torch's stream; a created stream does not wait for it
    torch.cuda.synchronize()
    rc = _capi.lib().st_superimpose_noalloc(C.byref(v), C.byref(desc), st.HIST_TYPES[kind], nb,
                                            lo, hi, counts.data_ptr(), yfy.data_ptr(), stream,
                                            C.byref(stats))
    return rc, counts.cpu().numpy(), yfy.cpu().numpy(), stats


def _oracle(track, hl, d, n_os, seed, tid, zshift, spec):
    sx = st.oversample_shifts(hl, d, True, seed, tid, n_os)
    counts, yfy, stats, _ = po.run_job(*track, half_length=hl, sphere_diameter=d, sxsy=sx,
                                       edges_arr=po.edges(*spec), zshift=zshift)
    return counts, yfy, stats


CASES = [
    # (generator, tracks, d, oversamples, histogram, stream): 10 nm spheres on proton-like tracks,
    # and a dense 2 nm ion track of the maximum size (several windows of kept deposits), each on
    # the legacy default stream and on a created stream
    ("proton", 2, 10.0, 10, ("lin", 3000, 0.01, 300.0), "default"),
    ("ion", 1, 2.0, 5, ("log", 500, 0.1, 1e4), "default"),
    ("proton", 1, 100.0, 20, ("log", 200, 0.01, 1e4), "created"),
    ("ion", 1, 10.0, 3, ("lin", 3000, 0.01, 300.0), "created"),
]


@pytest.mark.parametrize("gen,ntracks,d,n_os,spec,stream_kind", CASES)
def test_noalloc_matches_regular_entry_point_and_oracle(gen, ntracks, d, n_os, spec, stream_kind):
    if gen == "proton":
        w = W.config0(n_tracks=ntracks, n_dep=4000, n_os=n_os)
    else:
        w = W.config1(n_tracks=ntracks, n_dep=16384, n_os=n_os)
    hl = float(w.half_length[0])
    stream = torch.cuda.Stream() if stream_kind == "created" else None
    handle = stream.cuda_stream if stream is not None else None
    for j in range(w.n_jobs):
        track = [a.cpu().numpy() for a in w.job_arrays(j)]
        rc_, ry, rs = _regular(track, hl, d, n_os, 7, j, "none", spec)
        oc, oy, os_ = _oracle(track, hl, d, n_os, 7, j, "none", spec)
        assert rc_.sum() > 0
        assert np.array_equal(rc_, oc)
        for call in range(2):  # two calls in a row share the scratch array
            rc, counts, yfy, stats = _noalloc(track, hl, d, n_os, 7, j, "none", spec, handle)
            assert rc == 0, _capi.STATUS_NAMES.get(rc, rc)
            assert np.array_equal(counts, rc_), call
            assert np.array_equal(counts, oc), call
            np.testing.assert_allclose(yfy, ry, rtol=1e-12, atol=0)
            np.testing.assert_allclose(yfy, oy, rtol=1e-12, atol=0)
            assert stats.hits == rs["hits"] == os_["hits"]
            assert stats.spheres == rs["spheres"] == os_["spheres"]
            assert stats.binned == os_["binned"]
            assert stats.grid_exponent == os_["grid_exponent"]


def test_noalloc_rejects_requests_beyond_its_scratch():
    track = [np.zeros(16385) for _ in range(4)]
    rc, *_ = _noalloc(track, 2500.0, 10.0, 1, 1, 0, "none", ("lin", 10, 0.0, 10.0))
    assert rc == _capi.ST_ERR_CAPACITY
    small = [np.zeros(10) for _ in range(4)]
    rc, *_ = _noalloc(small, 2500.0, 10.0, 1, 1, 0, "none", ("lin", 4097, 0.0, 10.0))
    assert rc == _capi.ST_ERR_CAPACITY
    rc, *_ = _noalloc(small, 2500.0, 10.0, 65537, 1, 0, "none", ("lin", 10, 0.0, 10.0))
    assert rc == _capi.ST_ERR_CAPACITY
    assert _capi.lib().st_noalloc_scratch_bytes() < 8 * 1024 * 1024
