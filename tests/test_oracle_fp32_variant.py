"""The FP32 geometry variant in the CPU oracle (or_job_f32).

The reference computes in FP64 throughout; its readme asks for a float form (readme.md:29). In
the FP32 variant x, y, the shifts, the x/y box test, the x/y lattice index and the sphere
distance are float (every operation rounded on its own); z, keys and energies are as in the FP64
form. It is not a reference algorithm, so nothing pins it bit for bit against the reference.
These tests pin it three ways instead:
  * the reference's own known answers (A1-A8, H1-H8), whose coordinates are float-exact, come out
    the same as in the FP64 form;
  * on seeded tracks it stays within a small distance of the FP64 form;
  * a deposit 5e-9 nm past the midpoint of two sphere centres scores in a different sphere than
    in FP64 (the float rounding of x is really applied).
The GPU form is checked against this restatement bit for bit in test_gpu_fp32_variant.py.
"""
import numpy as np
import pytest

import make_golden as mg
import pyoracle as po
import supertrack_b200.workloads as W
from test_oracle_known_answers import assert_single_bin, run_oracle_case


@pytest.mark.parametrize("name", ["A1", "A2", "A8"])
def test_known_answers_single_oversample(name):
    c = mg.a_case(name)
    e, counts, _, _, _ = run_oracle_case(c, precision=32)
    assert_single_bin(e, counts, c["expect"]["value"], c["expect"]["count"])


def test_known_answers_lines_and_box_edges():
    c = mg.a_case("A4")
    e, counts, _, _, _ = run_oracle_case(c, n_os=5, precision=32)
    assert_single_bin(e, counts, 1.0, 3000 * 5 * 5)
    c = mg.a_case("A6")
    _, counts, _, _, _ = run_oracle_case(c, precision=32)
    assert counts.sum() == 0
    e, counts, _, _, _ = run_oracle_case(c, zshift="minus", precision=32)
    assert_single_bin(e, counts, 1.0, mg.A6_MINUS_EXPECT["count"])


def test_known_answers_64bit_keys():
    c = mg.a_case("A8")
    _, _, _, _, sph = run_oracle_case(c, spheres_cap=16, precision=32)
    assert sorted(int(k) for k in sph[0]["key"]) == sorted(c["keys"])


@pytest.mark.parametrize("name", list(mg.H_CASES))
def test_histogram_known_answers(name):
    h = mg.H_CASES[name]
    spec = h["restated"] if h.get("invalid") else h["hist"]
    tracks = mg.h_track(h["n"], h["value"], h["same"])
    c = dict(half_length=mg.H_GEOM["half_length"], diameter=mg.H_GEOM["diameter"],
             shift_track=False, n_os=1, seed=1, zshift="none", hist=spec, tracks=tracks)
    e, counts, yfy, stats, _ = run_oracle_case(c, precision=32)
    target = h.get("sum_value", h["value"])
    assert_single_bin(e, counts, target, h["expect_count"])
    assert yfy.sum() == target * h["expect_count"]
    assert stats[0]["hits"] == h["n"]


def _run(w, j, precision):
    x, y, z, e = [a.numpy() for a in w.job_arrays(j)]
    sx = po.shifts(float(w.half_length[j]), float(w.diameter[j]), w.shift_track, int(w.seed[j]),
                   int(w.track_id[j]), int(w.n_os[j]))
    return po.run_job(x, y, z, e, half_length=float(w.half_length[j]),
                      sphere_diameter=float(w.diameter[j]), sxsy=sx,
                      edges_arr=po.edges(*w.hists[int(w.hist_of_job[j])]), zshift=w.zshift,
                      precision=precision)


@pytest.mark.parametrize("gen,d", [("proton", 10.0), ("ion", 2.0)])
def test_close_to_fp64_on_seeded_tracks(gen, d):
    if gen == "proton":
        w = W.config0(n_tracks=2, n_dep=20_000, n_os=20)
    else:
        w = W.config1(n_tracks=1, n_dep=40_000, n_os=10)
    w.diameter[:] = d
    for j in range(w.n_jobs):
        c64, y64, s64, _ = _run(w, j, 64)
        c32, y32, s32, _ = _run(w, j, 32)
        assert s64["hits"] > 1000
        # membership decisions differ only for deposits within float rounding of a sphere
        # surface or a box face
        assert abs(s32["hits"] - s64["hits"]) <= 1e-4 * s64["hits"] + 2
        assert abs(s32["spheres"] - s64["spheres"]) <= 1e-4 * s64["spheres"] + 2
        assert np.abs(c32 - c64).sum() <= 1e-3 * c64.sum() + 4


def test_float_rounding_moves_a_midpoint_deposit():
    """HL 2500, d 10 (gSO = -2495), no shift, z at a sphere centre: x = 10 + 5e-9 lies just past
    the midpoint of the centres 5 and 15. In FP64 the deposit scores in sphere 251 (distance
    4.999999995 < r); in float x rounds to 10, the quotient to 250.5 and rint to the even 250."""
    x = np.array([10.0 + 5e-9])
    y = np.array([5.0])
    z = np.array([5.0])
    e = np.array([100.0])
    sx = np.zeros((1, 2))
    edges = po.edges("lin", 10, 0.0, 100.0)
    keys = {}
    for prec in (64, 32):
        _, _, st, sph = po.run_job(x, y, z, e, half_length=2500.0, sphere_diameter=10.0, sxsy=sx,
                                   edges_arr=edges, zshift="none", spheres_cap=4,
                                   precision=prec)
        assert st["hits"] == 1
        keys[prec] = int(sph["key"][0])
    n = 500
    assert keys[64] == 251 + 250 * n + 250 * n * n
    assert keys[32] == 250 + 250 * n + 250 * n * n
