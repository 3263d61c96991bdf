"""Known-answer fixtures of the reference's own tests, restated.

The reference's end-to-end tests A1-A8 (tst/tests/SuperTrackVoxelConstrainedTests.cu) read
ROOT track files made by tst/testTracks/tstTrackGenerator.cc, which are not shipped; the
Histogram tests H1-H8 (tst/tests/HistogramTests.cu) fill (volume, edep) pairs directly. This
module rebuilds every track from the generator's loops (cited per function) and records the
macro settings and expected answers of every test. Running it writes known_answers.json, the
committed record of those expectations; the tests import the track builders from here.

Expected answers in the reference assume the z-origin shift that its tests were written for:
A1-A5, A7 and A8 place deposits at z in [0, 3e6) nm and pass only with z shifted by -HL'
(or not at all); A6 passes only with the literal +HL' of VoxelConstrainedSphereMethod.cu:45.
Each case records the z-shift it is checked with.
"""
from __future__ import annotations

import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

# Macro values shared by testA1..testA8.ini (tst/testMacros/testA1.ini:17-29)
BASE = dict(half_length=1.5e6, diameter=1e3, shift_track=False, n_os=1, seed=1234,
            hist=("lin", 256, 0.1, 100.0))


def _col(v, n):
    return np.full(n, v, dtype=np.float64)


def track_a1():
    """tstTrackGenerator.cc:37-88: one deposit at (500, 500, 500), edep = 2000/3 in integer
    arithmetic (666 eV)."""
    z = []
    v = 0.5e3
    while v < 0.5e3 + 1e3:
        z.append(v)
        v += 1e3
    n = len(z)
    return [(_col(0.5e3, n), _col(0.5e3, n), np.array(z), _col(float(2000 // 3), n))]


def _line_z():
    z = []
    v = 0.5e3
    while v <= 3e6 - 0.5e3:
        z.append(v)
        v += 1e3
    return np.array(z)


def track_a2():
    """tstTrackGenerator.cc:90-141: 3000 deposits along z at sphere centres."""
    z = _line_z()
    n = len(z)
    return [(_col(0.5e3, n), _col(0.5e3, n), z, _col(2000.0 / 3, n))]


def track_a3():
    """tstTrackGenerator.cc:143-195: a 3000 x 3000 plane at x = 500 (y outer, z inner loop)."""
    ys = []
    v = 0.5e3 - 1.5e6
    while v <= 3e6 - 0.5e3 - 1.5e6:
        ys.append(v)
        v += 1e3
    zs = _line_z()
    y = np.repeat(np.array(ys), len(zs))
    z = np.tile(zs, len(ys))
    n = len(y)
    return [(_col(0.5e3, n), y, z, _col(2000.0 / 3, n))]


def track_a4():
    """tstTrackGenerator.cc:197-248: five copies of the A2 line, one track each."""
    return track_a2() * 5


def track_a5(copies=1000, n_tracks=5):
    """tstTrackGenerator.cc:250-311: per track, 1000 coincident deposits at each of the 3000
    sphere centres of the A2 line; five tracks."""
    z = np.repeat(_line_z(), copies)
    n = len(z)
    t = (_col(0.5e3, n), _col(0.5e3, n), z, _col(2000.0 / 3, n))
    return [t] * n_tracks


def track_a6():
    """tstTrackGenerator.cc:313-405: four 'faces'. The loop variables leak between faces: face 3
    keeps z at the value that ended face 2's loop (3000500) and overwrites its y = 500 with the
    inner loop; face 4 keeps y = 2999500."""
    start, stop, step = 0.5e3, 3e6 - 0.5e3, 1e3
    inner = []
    v = start - 1.5e6
    while v <= stop - 1.5e6:
        inner.append(v)
        v += step
    outer = []
    v = start
    while v <= stop:
        outer.append(v)
        v += step
    inner = np.array(inner)
    outer = np.array(outer)
    z_end = outer[-1] + step          # value of z after face 2's loop ends
    X, Y, Z = [], [], []
    # face 1: x = start; z outer, y inner
    X.append(np.full(len(outer) * len(inner), start)); Z.append(np.repeat(outer, len(inner)))
    Y.append(np.tile(inner, len(outer)))
    # face 2: x = stop
    X.append(np.full(len(outer) * len(inner), stop)); Z.append(np.repeat(outer, len(inner)))
    Y.append(np.tile(inner, len(outer)))
    # face 3: x outer, y inner, z = z_end
    X.append(np.repeat(outer, len(inner))); Y.append(np.tile(inner, len(outer)))
    Z.append(np.full(len(outer) * len(inner), z_end))
    # face 4: y = stop; x outer, z inner
    X.append(np.repeat(outer, len(inner))); Z.append(np.tile(inner, len(outer)))
    Y.append(np.full(len(outer) * len(inner), stop))
    x, y, z = (np.concatenate(a) for a in (X, Y, Z))
    return [(x, y, z, _col(2000.0 / 3, len(x)))]


def track_a7():
    """tstTrackGenerator.cc:407-461: x = y = 0, z in [0, 2e5) every 10 nm (20000 deposits)."""
    z = []
    v = 0.0
    while v < 0.2e6:
        z.append(v)
        v += 10
    z = np.array(z)
    n = len(z)
    return [(_col(0.0, n), _col(0.0, n), z, _col(2000.0 / 3, n))]


def track_a8():
    """tstTrackGenerator.cc:463-536: seven deposits placed to land on 64-bit sphere keys
    (d = 10 nm, N = 300000)."""
    b = 1.5e6
    pts = [(5 - b, 5 - b, 5.0), (836465 - b, 71585 - b, 5.0), (836475 - b, 71585 - b, 5.0),
           (836485 - b, 71585 - b, 5.0), (1672955 - b, 143166 - b, 5.0),
           (1672965 - b, 143166 - b, 5.0), (5 - b, 5 - b, 1.5e6 - 5)]
    a = np.array(pts, dtype=np.float64)
    return [(a[:, 0].copy(), a[:, 1].copy(), a[:, 2].copy(), _col(20.0 / 3, len(a)))]


# Macro deltas per test (tst/testMacros/testA*.ini) and the reference's expectations
# (tst/tests/SuperTrackVoxelConstrainedTests.cu). "value" is the lineal energy whose bin must
# hold "count"; every other bin must be empty.
A_CASES = {
    "A1": dict(track="track_a1", zshift="minus", expect=dict(value=1.0, count=1),
               source="SuperTrackVoxelConstrainedTests.cu:11-48"),
    "A2": dict(track="track_a2", zshift="minus", expect=dict(value=1.0, count=3000),
               source="SuperTrackVoxelConstrainedTests.cu:50-87"),
    "A3": dict(track="track_a3", zshift="minus", expect=dict(value=1.0, count=9000000),
               source="SuperTrackVoxelConstrainedTests.cu:89-126"),
    "A4": dict(track="track_a4", zshift="minus", n_os=1000,
               expect=dict(value=1.0, count=3000 * 1000 * 5),
               source="SuperTrackVoxelConstrainedTests.cu:128-165"),
    "A5": dict(track="track_a5", zshift="minus", n_os=1000, hist=("lin", 30000, 0.1, 1e4),
               expect=dict(value=1000.0, count=5 * 1000 * 3000),
               source="SuperTrackVoxelConstrainedTests.cu:167-208"),
    "A6": dict(track="track_a6", zshift="plus", hist=("lin", 30000, 0.1, 1e4),
               expect=dict(all_zero=True), source="SuperTrackVoxelConstrainedTests.cu:210-238",
               note="with -HL' face 1 (x = 500) lies inside the voxel: 9e6 hits at y = 1"),
    "A7": dict(track="track_a7", zshift="minus", n_os=10000, shift_track=True,
               hist=("lin", 10000, 1.0, 1e4), expect=dict(pi_range=[3.05, 3.3]),
               source="SuperTrackVoxelConstrainedTests.cu:240-278"),
    "A8": dict(track="track_a8", zshift="minus", diameter=10.0,
               hist=("lin", 10000, 0.01, 1e3), expect=dict(value=1.0, count=7),
               keys=[0, 2**31 - 2, 2**31 - 1, 2**31, 2**32 - 1, 2**32, 149999 * 300000**2],
               source="SuperTrackVoxelConstrainedTests.cu:280-317"),
}
A6_MINUS_EXPECT = dict(value=1.0, count=9000000)


def a_case(name):
    c = dict(BASE)
    c.update({k: v for k, v in A_CASES[name].items()})
    c["tracks"] = globals()[c["track"]]()
    return c


# Histogram unit tests (tst/tests/HistogramTests.cu). The reference fills (volume, edep) pairs
# directly; here the same pairs come out of the geometry: d = 1.5 nm makes the lineal
# denominator (2/3)*d exactly 1, so each deposit at a sphere centre contributes exactly its edep.
H_GEOM = dict(half_length=150.0, diameter=1.5)   # N = 200 spheres per side


def h_track(n_pairs: int, value: float, same_sphere: bool):
    """n_pairs deposits of lineal energy `value`, each in its own sphere or all in one."""
    g_so = -150.0 + 0.75
    if same_sphere:
        ix = np.zeros(n_pairs, dtype=np.int64)
    else:
        ix = np.arange(n_pairs, dtype=np.int64)
    x = g_so + 1.5 * (ix % 200)
    y = g_so + 1.5 * (ix // 200)
    z = np.full(n_pairs, g_so)
    return [(x.astype(np.float64), y.astype(np.float64), z, np.full(n_pairs, float(value)))]


H_CASES = {
    "H1": dict(n=100, value=1.0, same=False, hist=("lin", 500, 0.0, 500.0), expect_count=100,
               source="HistogramTests.cu:36-84"),
    "H2": dict(n=100, value=5.0, same=False, hist=("lin", 500, 0.0, 500.0), expect_count=100,
               source="HistogramTests.cu:86-134"),
    "H3": dict(n=100, value=5.0, same=True, hist=("lin", 500, 0.0, 1000.0), expect_count=1,
               sum_value=500.0, source="HistogramTests.cu:136-184"),
    "H4": dict(n=1000, value=1000.0, same=True, hist=("lin", 30000, 0.1, 1e7), expect_count=1,
               sum_value=1e6, source="HistogramTests.cu:186-234"),
    # log variants: a lower bound of 0 makes LogSpace take log10(0) = -inf and every edge NaN;
    # those specifications are rejected, and the cases are also run with a positive lower bound.
    "H5": dict(n=100, value=1.0, same=False, hist=("log", 500, 0.0, 500.0), invalid=True,
               restated=("log", 500, 0.1, 500.0), expect_count=100,
               source="HistogramTests.cu:236-284"),
    "H6": dict(n=100, value=5.0, same=False, hist=("log", 500, 0.0, 500.0), invalid=True,
               restated=("log", 500, 0.1, 500.0), expect_count=100,
               source="HistogramTests.cu:286-334"),
    "H7": dict(n=100, value=5.0, same=True, hist=("log", 500, 0.0, 1000.0), invalid=True,
               restated=("log", 500, 0.1, 1000.0), expect_count=1, sum_value=500.0,
               source="HistogramTests.cu:336-384"),
    "H8": dict(n=1000, value=1000.0, same=True, hist=("log", 30000, 0.1, 1e7), expect_count=1,
               sum_value=1e6, source="HistogramTests.cu:386-433"),
}


def main():
    out = {"base_macro": {k: (list(v) if isinstance(v, tuple) else v) for k, v in BASE.items()},
           "A": {}, "H": {}}
    for k, c in A_CASES.items():
        tr = globals()[c["track"]]()
        rec = {kk: (list(v) if isinstance(v, tuple) else v) for kk, v in c.items()}
        rec["n_tracks"] = len(tr)
        rec["deposits_per_track"] = [int(len(t[0])) for t in tr]
        out["A"][k] = rec
    out["A"]["A6"]["expect_minus"] = A6_MINUS_EXPECT
    for k, c in H_CASES.items():
        out["H"][k] = {kk: (list(v) if isinstance(v, tuple) else v) for kk, v in c.items()}
    with open(os.path.join(HERE, "known_answers.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
