"""Pins the CPU oracle against the reference's own known-answer tests (A1-A8, H1-H8).

Expected answers come from tst/tests/SuperTrackVoxelConstrainedTests.cu and
tst/tests/HistogramTests.cu (recorded in tests/golden/known_answers.json); the tracks are rebuilt
from tst/testTracks/tstTrackGenerator.cc's loops (tests/golden/make_golden.py). Oversample counts
of the slowest cases are reduced here and the expectation scaled: with ShiftTrack = false every
oversample of a track is identical, so the count is proportional to the oversamples.
"""
import json
import os

import numpy as np
import pytest

import make_golden as mg
import pyoracle as po

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = json.load(open(os.path.join(HERE, "golden", "known_answers.json")))


def run_oracle_case(c, n_os=None, zshift=None, tracks=None, sum_mode=po.OR_SUM_EXACT,
                    spheres_cap=0, precision=64):
    kind, nb, lo, hi = c["hist"]
    e = po.edges(kind, nb, lo, hi)
    counts = np.zeros(nb, dtype=np.int64)
    yfy = np.zeros(nb)
    n_os = c["n_os"] if n_os is None else n_os
    stats = []
    spheres = []
    for ti, t in enumerate(tracks if tracks is not None else c["tracks"]):
        seed = c["seed"] if c.get("seed", -1) != -1 else 1
        sx = po.shifts(c["half_length"], c["diameter"], c["shift_track"], seed, ti, n_os)
        _, _, s, sph = po.run_job(*t, half_length=c["half_length"],
                                  sphere_diameter=c["diameter"], sxsy=sx, edges_arr=e,
                                  zshift=zshift or c["zshift"], sum_mode=sum_mode,
                                  spheres_cap=spheres_cap, counts=counts, yfy=yfy,
                                  precision=precision)
        stats.append(s)
        spheres.append(sph)
    return e, counts, yfy, stats, spheres


def assert_single_bin(e, counts, value, count):
    b = int(np.searchsorted(e, value, side="right") - 1)
    assert counts[b] == count, (counts[b], count)
    assert counts.sum() == count


def test_golden_record_is_current():
    """known_answers.json is what make_golden.py writes (fixtures and script agree)."""
    for k, c in mg.A_CASES.items():
        assert GOLDEN["A"][k]["expect"] == c["expect"]
        assert GOLDEN["A"][k]["zshift"] == c["zshift"]
    for k, c in mg.H_CASES.items():
        assert GOLDEN["H"][k]["expect_count"] == c["expect_count"]


@pytest.mark.parametrize("name", ["A1", "A2", "A3", "A8"])
def test_single_oversample_cases(name):
    c = mg.a_case(name)
    e, counts, _, stats, _ = run_oracle_case(c)
    assert_single_bin(e, counts, c["expect"]["value"], c["expect"]["count"])


def test_a1_value_is_0999():
    # edep = 2000/3 in integer arithmetic = 666 eV -> y = 666/666.67 = 0.999 keV/um, same bin as 1
    c = mg.a_case("A1")
    _, _, _, _, sph = run_oracle_case(c, spheres_cap=4)
    assert sph[0]["y"][0] == 666 / ((2. / 3.) * 1000)


def test_a4_lines_times_oversamples():
    c = mg.a_case("A4")
    e, counts, _, _, _ = run_oracle_case(c, n_os=20)
    assert_single_bin(e, counts, 1.0, 3000 * 20 * 5)


def test_a5_thousand_deposits_per_sphere():
    c = mg.a_case("A5")
    tracks = mg.track_a5(copies=1000, n_tracks=1)
    e, counts, _, stats, _ = run_oracle_case(c, n_os=2, tracks=tracks)
    assert_single_bin(e, counts, 1000.0, 1 * 2 * 3000)
    # the literal left-to-right FP64 sum lands in the same bin
    e2, counts2, _, _, _ = run_oracle_case(c, n_os=1, tracks=tracks, sum_mode=po.OR_SUM_SEQ)
    assert_single_bin(e2, counts2, 1000.0, 3000)


def test_a6_edges_of_the_box():
    c = mg.a_case("A6")
    e, counts, _, _, _ = run_oracle_case(c)                       # literal +HL': all zero
    assert counts.sum() == 0
    e, counts, _, _, _ = run_oracle_case(c, zshift="minus")       # face 1 inside under -HL'
    assert_single_bin(e, counts, 1.0, mg.A6_MINUS_EXPECT["count"])


def test_a7_pi_estimate():
    c = mg.a_case("A7")
    for seed in (1, 2):
        c["seed"] = seed
        e, counts, _, _, _ = run_oracle_case(c, n_os=2000)
        mid = (e[1:] + e[:-1]) / 2
        pi_hat = 6 * float((mid * counts).sum()) / (20000 * 2000)
        assert 3.05 < pi_hat < 3.3, pi_hat
    # with the literal +HL' the line sits outside the voxel and nothing is scored
    e, counts, _, _, _ = run_oracle_case(c, n_os=10, zshift="plus")
    assert counts.sum() == 0


def test_a8_64bit_keys():
    c = mg.a_case("A8")
    e, counts, _, _, sph = run_oracle_case(c, spheres_cap=16)
    assert_single_bin(e, counts, 1.0, 7)
    assert sorted(int(k) for k in sph[0]["key"]) == sorted(c["keys"])


@pytest.mark.parametrize("name", list(mg.H_CASES))
def test_histogram_cases(name):
    h = mg.H_CASES[name]
    if h.get("invalid"):
        with pytest.raises(ValueError):
            po.edges(*h["hist"])
        spec = h["restated"]
    else:
        spec = h["hist"]
    tracks = mg.h_track(h["n"], h["value"], h["same"])
    c = dict(half_length=mg.H_GEOM["half_length"], diameter=mg.H_GEOM["diameter"],
             shift_track=False, n_os=1, seed=1, zshift="none", hist=spec, tracks=tracks)
    e, counts, yfy, stats, _ = run_oracle_case(c)
    target = h.get("sum_value", h["value"])
    assert_single_bin(e, counts, target, h["expect_count"])
    assert yfy.sum() == target * h["expect_count"]
    assert stats[0]["hits"] == h["n"]


def test_sequential_sum_within_tolerance_of_exact():
    """Per-sphere energies: the exact sum and the left-to-right FP64 sum agree to 1e-12."""
    import supertrack_b200.workloads as W
    w = W.config0(n_tracks=4, n_os=3)
    e = po.edges("lin", 3000, 0.01, 300.0)
    for j in range(w.n_jobs):
        x, y, z, ed = [a.numpy() for a in w.job_arrays(j)]
        sx = po.shifts(2500, 10, True, 1, j, 3)
        _, _, _, sph = po.run_job(x, y, z, ed, half_length=2500, sphere_diameter=10, sxsy=sx,
                                  edges_arr=e, zshift="none", spheres_cap=100000)
        assert len(sph) > 100
        rel = np.abs(sph["y"] - sph["y_seq"]) / np.abs(sph["y"])
        assert rel.max() <= 1e-12
