"""Host-side logic that needs no GPU: Philox, geometry, bin edges, shifts, the exact-sum grid,
the .ini reader, task/seed allocation and the track file format."""
import math
import os
import random
import re
from fractions import Fraction

import numpy as np
import pytest

import pyoracle as po
import supertrack_b200 as st
from supertrack_b200 import _capi

# Philox4x32-10 known-answer vectors published with the Random123 library (kat_vectors).
PHILOX_KAT = [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


@pytest.mark.parametrize("ctr,key,out", PHILOX_KAT)
def test_philox_known_answers(ctr, key, out):
    assert st.philox4x32_10(ctr, key) == out
    assert po.philox(ctr, key) == out


def test_geometry_matches_oracle_and_reference_rules():
    rs = random.Random(7)
    cases = [(1.5e6, 1e3), (2500, 10), (5000, 2), (2500, 1000), (2500, 2), (5, 100), (0, 1),
             (1.5e6, 10), (7.3, 2.2), (-3, 1)]
    cases += [(rs.uniform(1, 1e4), rs.choice([0.5, 1, 2, 3.3, 10, 77.7, 1000])) for _ in range(200)]
    for hl, d in cases:
        g = st.geometry(hl, d)
        o = po.geometry(hl, d)
        assert g["num_spheres_linear"] == o["N"]
        assert g["scoring_region_length"] == o["L"]
        assert g["scoring_region_half_length"] == o["HL"]
        assert g["greatest_sphere_offset"] == o["gSO"]
        assert g["sphere_radius"] == o["r"]
    g = st.geometry(1.5e6, 1e3)
    assert g["num_spheres_linear"] == 3000 and g["greatest_sphere_offset"] == -1499500.0
    g = st.geometry(5, 100)  # sphere larger than the voxel: one sphere, gSO = 0
    assert g["num_spheres_linear"] == 1 and g["scoring_region_half_length"] == 50.0
    assert g["greatest_sphere_offset"] == 0.0


@pytest.mark.parametrize("hl,d", [(1, 0), (1, -2), (float("nan"), 1), (1, float("inf")),
                                  (1e13, 1)])
def test_geometry_rejects(hl, d):
    with pytest.raises(st.StError) as e:
        st.geometry(hl, d)
    assert e.value.status == _capi.ST_ERR_BAD_GEOMETRY


@pytest.mark.parametrize("kind,nb,lo,hi", [("lin", 3000, 0.01, 300.0), ("log", 500, 0.1, 1e4),
                                           ("log", 200, 0.01, 1e4), ("lin", 256, 0.1, 100.0),
                                           ("lin", 30000, 0.1, 1e4), ("lin", 10000, 1.0, 1e4),
                                           ("lin", 500, 0.0, 500.0), ("log", 30000, 0.1, 1e7)])
def test_edges_match_oracle(kind, nb, lo, hi):
    a = st.hist_edges(kind, nb, lo, hi)
    b = po.edges(kind, nb, lo, hi)
    assert np.array_equal(a, b)
    assert np.all(np.diff(a) > 0)


def test_edges_float_typing():
    # bounds pass through float: 0.1 becomes 0.100000001490116...
    e = st.hist_edges("lin", 256, 0.1, 100.0)
    assert e[0] == float(np.float32(0.1))
    w = np.float32(np.float32(100.0) - np.float32(0.1)) / np.float32(256)
    assert e[1] == float(np.float32(0.1)) + 1 * float(np.float32(w))


@pytest.mark.parametrize("kind,nb,lo,hi", [("log", 500, 0.0, 500.0), ("lin", 0, 0, 1),
                                           ("lin", 10, 5.0, 1.0), ("log", 10, -1.0, 10.0)])
def test_edges_rejects_ill_defined(kind, nb, lo, hi):
    with pytest.raises(st.StError) as e:
        st.hist_edges(kind, nb, lo, hi)
    assert e.value.status == _capi.ST_ERR_BAD_HISTOGRAM


def test_shift_export_matches_oracle_contract():
    for hl, d, seed, tid in [(2500, 10, 1, 0), (5000, 2, 2, 15), (1.5e6, 1e3, 123400, 0),
                             (2500, 1000, 2**63 + 5, 2**40 + 3)]:
        a = st.oversample_shifts(hl, d, True, seed, tid, 257)
        b = po.shifts(hl, d, True, seed, tid, 257)
        assert np.array_equal(a, b)
        g = st.geometry(hl, d)
        L, HL = g["scoring_region_length"], g["scoring_region_half_length"]
        assert np.all(a > -HL) and np.all(a <= HL)
        # an oversample block starting mid-way equals the tail of the full sequence
        assert np.array_equal(st.oversample_shifts(hl, d, True, seed, tid, 7, os_begin=250),
                              a[250:])
    z = st.oversample_shifts(2500, 10, False, 1, 0, 5)
    assert np.all(z == 0.0)  # u = 0.5 gives 0.5*L - HL' = 0 exactly


def test_shift_uniformity():
    s = st.oversample_shifts(2500, 10, True, 99, 0, 20000)
    g = st.geometry(2500, 10)
    u = (s + g["scoring_region_half_length"]) / g["scoring_region_length"]
    for col in (u[:, 0], u[:, 1]):
        assert abs(col.mean() - 0.5) < 0.01
        assert abs(col.var() - 1 / 12) < 0.005
    assert abs(np.corrcoef(u[:, 0], u[:, 1])[0, 1]) < 0.03


def _fx(v, e0):
    lo = _capi.C.c_uint64()
    hi = _capi.C.c_uint64()
    _capi.lib().st_to_fixed(v, e0, _capi.C.byref(lo), _capi.C.byref(hi))
    val = (hi.value << 64) | lo.value
    return val - (1 << 128) if val >> 127 else val


def test_fixed_point_exact_and_round_trip():
    rs = np.random.default_rng(3)
    vals = np.exp(rs.uniform(np.log(1e-3), np.log(1e4), 2000))
    vals[::7] *= -1
    e = [int(math.frexp(abs(v))[1]) - 53 for v in vals]
    e0 = st_grid = _capi.lib().st_grid_exponent(min(e), max(e), len(vals), 1)
    assert st_grid == po.grid_exponent(min(e), max(e), len(vals), True)
    total = 0
    for v in vals:
        f = _fx(float(v), e0)
        assert Fraction(f) * Fraction(2) ** e0 == Fraction(float(v))   # exact representation
        total += f
    # the sum rounded once equals the correctly rounded exact sum
    hi, lo = (total >> 64) & ((1 << 64) - 1), total & ((1 << 64) - 1)
    got = _capi.lib().st_from_fixed(lo, hi, e0)
    exact = sum(Fraction(float(v)) for v in vals)
    assert got == float(exact)


def test_from_fixed_ties_to_even():
    # 2^53 + 1 is halfway between 2^53 and 2^53 + 2: rounds to the even 2^53
    assert _capi.lib().st_from_fixed((1 << 53) + 1, 0, 0) == float(2**53)
    assert _capi.lib().st_from_fixed((1 << 53) + 3, 0, 0) == float(2**53 + 4)
    big = (1 << 100) + (1 << 47)  # halfway above 2^100 at 53 bits -> even (down)
    assert _capi.lib().st_from_fixed(big & ((1 << 64) - 1), big >> 64, 0) == float(2**100)
    big = (1 << 100) + (1 << 47) + 1  # just above halfway -> up
    assert _capi.lib().st_from_fixed(big & ((1 << 64) - 1), big >> 64, 0) == float(2**100 + 2**48)


# ---------------------------------------------------------------------------------------------
# .ini reader (semantics of inih's INIReader)
# ---------------------------------------------------------------------------------------------
INI_TEXT = """; comment
# another comment
[Run]
Type = Folder
Path = /tmp/tracks/ ; inline comment after whitespace
FirstFile = -1 ;
Threads = 0x10
Oversamples=10
Odd = a;b
[VoxelConstrainedSphere]
ScoringRegionHalfLength = 2.5e3    ; nm
ShiftTrack = false\t\t\t   ; turn off
Multi = first
  second
[Histogram]
Type = lin
BinLower = 1e-1
Bad = abc
"""


def test_ini_reader_semantics():
    r = st.INIReader(text=INI_TEXT)
    assert r.ParseError() == 0
    assert r.Get("Run", "Type", "") == "Folder"
    assert r.Get("run", "PATH", "") == "/tmp/tracks/"         # case-insensitive, comment cut
    assert r.GetInteger("Run", "FirstFile", 5) == -1
    assert r.GetInteger("Run", "Threads", 1) == 16            # strtol base 0
    assert r.GetInteger("Run", "Oversamples", 1) == 10
    assert r.Get("Run", "Odd", "") == "a;b"                   # ';' without whitespace kept
    assert r.GetReal("VoxelConstrainedSphere", "ScoringRegionHalfLength", 0) == 2500.0
    assert r.GetBoolean("VoxelConstrainedSphere", "ShiftTrack", True) is False
    assert r.Get("VoxelConstrainedSphere", "Multi", "") == "first\nsecond"
    assert r.Get("Histogram", "Type", "") == "lin"
    assert r.GetFloat("Histogram", "BinLower", 0) == float(np.float32(0.1))
    assert r.GetReal("Histogram", "Bad", 7.5) == 7.5            # unparsable -> default
    assert r.GetInteger("Histogram", "Missing", 3) == 3
    assert r.GetBoolean("Histogram", "Type", True) is True      # not a boolean -> default


def test_ini_reader_errors():
    assert st.INIReader(text="[Run\nx=1\n").ParseError() == 1
    assert st.INIReader(text="[Run]\nno separator here\n").ParseError() == 2
    assert st.INIReader(path="/nonexistent/file.ini").ParseError() == -1


def test_reference_macros_parse():
    # the reference's own macro layout (macros/default.ini keys)
    text = """[Run]
Type = Folder
Path = /x/
FirstFile = -1 ; #-1 is the default case
LastFile = -1 ;
Threads = 10
Oversamples = 10

[Simulation]
Method = VoxelConstrainedSphere

[VoxelConstrainedSphere]
;Geometry parameters
ScoringRegionHalfLength = 2.5e3    ; side length in nanometers
ScoringSphereDiameter = 10        ; sphere diameter in nanometers
SuggestedCudaBlocks = 256
SuggestedCudaThreads = 32

[Histogram]
Type = lin
NBins = 3000
BinLower = 0.01
BinUpper = 300.0
"""
    r = st.INIReader(text=text)
    assert r.GetInteger("Run", "LastFile", 0) == -1
    assert r.Get("Simulation", "Method", "") == "VoxelConstrainedSphere"
    assert r.GetReal("VoxelConstrainedSphere", "ScoringSphereDiameter", 0) == 10.0
    assert r.GetInteger("Histogram", "NBins", 0) == 3000


# ---------------------------------------------------------------------------------------------
# task allocation, seeds and track files
# ---------------------------------------------------------------------------------------------
def _write_folder(tmp_path, tracks_per_file):
    rs = np.random.default_rng(0)
    for fi, nt in enumerate(tracks_per_file):
        tracks = []
        for t in range(nt):
            n = int(rs.integers(1, 50))
            tracks.append(tuple(rs.normal(size=n) for _ in range(4)))
        st.write_track_file(str(tmp_path / f"f{fi:02d}.strk"), tracks)


def _macro(tmp_path, **run):
    keys = dict(Type="Folder", Path=str(tmp_path) + "/", Threads=1, Oversamples=3,
                RandomSeed=1234)
    keys.update(run)
    lines = ["[Run]"] + [f"{k} = {v}" for k, v in keys.items()]
    lines += ["[Simulation]", "Method = VoxelConstrainedSphere", "[VoxelConstrainedSphere]",
              "ScoringRegionHalfLength = 100", "ScoringSphereDiameter = 10",
              "[Histogram]", "Type = lin", "NBins = 10", "BinLower = 0", "BinUpper = 10"]
    p = tmp_path / "m.ini"
    p.write_text("\n".join(lines) + "\n")
    return str(p)


def test_thread_allocation_split_and_seeds(tmp_path):
    _write_folder(tmp_path, [3, 4, 2])
    tasks = st.macro_tasks(_macro(tmp_path, Threads=4))
    assert len(tasks) == 9
    # 9 tasks over 4 threads: 3, 2, 2, 2 (ThreadAllocator.cc:134-159)
    per = [sum(1 for t in tasks if t["thread_id"] == i) for i in range(4)]
    assert per == [3, 2, 2, 2]
    # seed = concat(RandomSeed, threadID, task index in the thread)
    k = 0
    for i, cnt in enumerate(per):
        for j in range(cnt):
            assert tasks[k]["seed"] == int(f"1234{i}{j}")
            assert tasks[k]["n_oversamples"] == 3
            k += 1
    # entry/exit points are cumulative within each file
    assert tasks[0]["entry"] == 0 and tasks[1]["entry"] == tasks[0]["exit"]
    assert [t["file_ordinal"] for t in tasks] == [1, 1, 1, 2, 2, 2, 2, 3, 3]


def test_thread_allocation_file_limits(tmp_path):
    _write_folder(tmp_path, [1, 2, 3])
    assert len(st.macro_tasks(_macro(tmp_path, FirstFile=2, LastFile=3))) == 5
    assert len(st.macro_tasks(_macro(tmp_path, FirstFile=2, LastFile=2))) == 2
    for bad in (dict(FirstFile=3, LastFile=2), dict(FirstFile=1, LastFile=4),
                dict(FirstFile=0, LastFile=2)):
        with pytest.raises(st.StError) as e:
            st.macro_tasks(_macro(tmp_path, **bad))
        assert e.value.status == _capi.ST_ERR_CONFIG
    # more threads than tracks: threads drop to the track count
    tasks = st.macro_tasks(_macro(tmp_path, Threads=50))
    assert sorted({t["thread_id"] for t in tasks}) == list(range(6))


def test_track_file_layout(tmp_path):
    """A track file is the magic STRKv001, the deposit and track counts (u64), the cumulative end
    index of every track (u64, the reference's "Track index" tree), then float64 x, y, z and edep
    over all deposits (the "Tracks" tree), little-endian."""
    rs = np.random.default_rng(5)
    sizes = [3, 0, 7, 1]                      # an empty track included
    tracks = [tuple(rs.normal(size=n) for _ in range(4)) for n in sizes]
    p = tmp_path / "t.strk"
    st.write_track_file(str(p), tracks)
    raw = p.read_bytes()
    nd, nt = (int(v) for v in np.frombuffer(raw[8:24], dtype="<u8"))
    assert raw[:8] == b"STRKv001" and nd == sum(sizes) and nt == len(sizes)
    assert len(raw) == 24 + 8 * nt + 32 * nd
    index = np.frombuffer(raw[24:24 + 8 * nt], dtype="<u8")
    assert index.tolist() == np.cumsum(sizes).tolist()
    soa = np.frombuffer(raw[24 + 8 * nt:], dtype="<f8").reshape(4, nd)
    for a in range(4):
        assert np.array_equal(soa[a], np.concatenate([t[a] for t in tracks]))
    # the folder loop makes one task per track, empty ones included, with cumulative entry points
    tasks = st.macro_tasks(_macro(tmp_path))
    assert [(t["entry"], t["exit"]) for t in tasks] == [(0, 3), (3, 3), (3, 10), (10, 11)]


def test_corrupt_track_files_are_config_errors(tmp_path):
    rs = np.random.default_rng(6)
    st.write_track_file(str(tmp_path / "f00.strk"),
                        [tuple(rs.normal(size=n) for _ in range(4)) for n in (4, 6)])
    good = (tmp_path / "f00.strk").read_bytes()
    bad_files = [b"XXXXv001" + good[8:],                                    # wrong magic
                 good[:20],                                                 # short header
                 good[:24] + np.array([6, 4], "<u8").tobytes() + good[40:],  # index decreases
                 good[:24] + np.array([4, 11], "<u8").tobytes() + good[40:]]  # index past the end
    for bad in bad_files:
        (tmp_path / "f00.strk").write_bytes(bad)
        with pytest.raises(st.StError) as e:
            st.macro_tasks(_macro(tmp_path))
        assert e.value.status == _capi.ST_ERR_CONFIG


CXX_PROGRAM = r"""
#include <cstdio>
#include <string>
#include "supertrack.h"

// The reference's C++ route up to the GPU launch, linked against libsupertrack_b200.so.
int main(int argc, char** argv) {
  st::SphericalGeometry g(2500.0, 10.0);
  st_geometry c;
  if (st_geometry_make(2500.0, 10.0, &c) != ST_OK) return 2;
  std::printf("geometry %d %.17g %.17g %d\n", g.numSpheresLinear, g.greatestSphereOffset,
              g.scoringRegionHalfLength, c.num_spheres_linear == g.numSpheresLinear);
  st::INIReader r = st::INIReader::FromString("[Histogram]\nNBins = 3000 ; bins\n");
  std::printf("nbins %ld\n", r.GetInteger("Histogram", "NBins", 0));
  st::SuperTrackManager& mgr = st::SuperTrackManager::GetInstance();
  mgr.AddSimulationMethod("VoxelConstrainedSphere", &st::VoxelConstrainedSphereMethod::Construct);
  const std::string e = mgr.Initialize(argv[1]);
  if (!e.empty()) {
    std::printf("error %s\n", e.c_str());
    return 3;
  }
  st::INIReader macro(argv[1]);
  st::SimulationMethodFactory& f = st::SimulationMethodFactory::GetInstance();
  f.AddSimulationMethod("VoxelConstrainedSphere", &st::VoxelConstrainedSphereMethod::Construct);
  st::SimulationMethod* m = f.Construct(macro);
  auto* vcs = dynamic_cast<st::VoxelConstrainedSphereMethod*>(m);
  if (!vcs) return 4;
  std::printf("method %d %d\n", vcs->Geometry().numSpheresLinear, (int)vcs->ShiftTrack());
  long tasks = 0;
  double sum = 0;
  for (const auto& a : mgr.Allocations())
    for (const auto& t : a.tasks) {
      st::Track track;
      if (!track.AllocateAndLoadTrack(t)) return 5;
      for (int64_t i = 0; i < track.Size(); ++i) sum += track.edep[i];
      ++tasks;
    }
  std::printf("tasks %ld %.17g\n", tasks, sum);
  delete m;
  return 0;
}
"""


def test_cpp_surface_links_and_runs_the_host_side(tmp_path):
    """A C++ caller of the reference's classes (SphericalGeometry, INIReader,
    SimulationMethodFactory, VoxelConstrainedSphereMethod, SuperTrackManager, Track) compiles
    against the shipped headers, links libsupertrack_b200.so alone, and gets the same geometry,
    tasks and deposits as the Python surface (everything before the GPU launch)."""
    import shutil
    import subprocess
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    libdir = os.path.join(root, "supertrack_b200")
    src = tmp_path / "route.cc"
    src.write_text(CXX_PROGRAM)
    exe = tmp_path / "route"
    subprocess.run(["g++", "-std=c++17", "-O1", "-o", str(exe), str(src),
                    "-I", os.path.join(root, "supertrack_b200", "csrc"),
                    "-L", libdir, "-lsupertrack_b200", "-Wl,-rpath," + libdir],
                   check=True, capture_output=True, text=True)
    folder = tmp_path / "tracks"
    folder.mkdir()
    _write_folder(folder, [3, 2])
    out = subprocess.run([str(exe), _macro(folder, Threads=2)], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    lines = dict(l.split(" ", 1) for l in out.stdout.strip().splitlines())
    g = st.geometry(2500.0, 10.0)
    n, gso, hl, same = lines["geometry"].split()
    assert int(n) == g["num_spheres_linear"] and float(gso) == g["greatest_sphere_offset"]
    assert float(hl) == g["scoring_region_half_length"] and same == "1"
    assert lines["nbins"] == "3000"
    assert lines["method"].split() == [str(st.geometry(100.0, 10.0)["num_spheres_linear"]), "1"]
    tasks = st.macro_tasks(_macro(folder, Threads=2))
    total = 0.0
    rs = np.random.default_rng(0)                 # the deposits _write_folder generated
    for nt in (3, 2):
        for _ in range(nt):
            m = int(rs.integers(1, 50))
            arrs = [rs.normal(size=m) for _ in range(4)]
            for v in arrs[3]:
                total += v
    nt_out, s_out = lines["tasks"].split()
    assert int(nt_out) == len(tasks) == 5
    assert float(s_out) == total


def test_cli_reports_unusable_macros(tmp_path):
    """`supertrack macro.ini` (SuperTrack.cu:9-36) exits 1 with the reason when the macro cannot
    be used, before any GPU work."""
    import subprocess
    exe = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                       "supertrack_b200", "supertrack")
    if not os.path.exists(exe):
        pytest.skip("the supertrack command is not built")
    r = subprocess.run([exe, str(tmp_path / "none.ini")], capture_output=True, text=True)
    assert r.returncode == 1 and "Cannot open macro file" in r.stderr
    bad = tmp_path / "bad.ini"
    bad.write_text("[Run]\nType = Folder\n")
    r = subprocess.run([exe, str(bad)], capture_output=True, text=True)
    assert r.returncode == 1 and "configuration error" in r.stderr


def test_run_macro_without_device_reports_no_device(tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    _write_folder(tmp_path, [2])
    with pytest.raises(st.StError) as e:
        st.run_macro(_macro(tmp_path), write_output=False)
    assert e.value.status == _capi.ST_ERR_NO_DEVICE


def test_macro_errors(tmp_path):
    p = tmp_path / "bad.ini"
    p.write_text("[Run]\nType = File\nPath = /x\n")
    with pytest.raises(st.StError):
        st.macro_tasks(str(p))
    p.write_text("[Run]\nType = Folder\n")
    with pytest.raises(st.StError):
        st.macro_tasks(str(p))
    p.write_text("[Run]\nType = Folder\nPath = /nonexistent_dir_st/\n")
    with pytest.raises(st.StError):
        st.macro_tasks(str(p))


def test_header_declares_what_the_library_exports():
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    hdr = open(os.path.join(root, "include", "supertrack_b200.h")).read()
    declared = set(re.findall(r"ST_API\s+[^;()]*?\b(st_\w+)\s*\(", hdr))
    assert len(declared) >= 39
    lib = _capi.lib()
    for name in declared:
        assert hasattr(lib, name), name
    bound = {n for n, _, _ in _capi.SIGNATURES}
    assert declared == bound


def test_no_device_is_reported_not_crashed():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(st.StError) as e:
        st.Context(0)
    assert e.value.status == _capi.ST_ERR_NO_DEVICE


def test_server_job_footprint():
    """The admission charge of a served job: grows with deposits, oversamples and bins; the
    boundary-cell hash of window-flagged jobs (fine lattice, >8192 deposits, >=4 oversamples)
    is charged on top; bad geometry is refused."""
    def foot(n, d=10.0, os_=10, nbins=200, hl=2500.0):
        v = _capi.st_track_view()
        v.n = n
        v.on_device = 1
        q = _capi.st_job_desc()
        q.half_length = hl
        q.sphere_diameter = d
        q.n_oversamples = os_
        b = _capi.C.c_int64(0)
        rc = _capi.lib().st_server_job_footprint(_capi.C.byref(v), _capi.C.byref(q), nbins,
                                                 _capi.C.byref(b))
        return rc, b.value
    rc, b0 = foot(1000)
    assert rc == 0 and b0 >= 80 * 1000
    assert foot(2000)[1] > b0 and foot(1000, os_=100)[1] > b0 and foot(1000, nbins=3000)[1] > b0
    # 1e5 deposits: flagged for d = 10 nm (N = 500), not for d = 1000 nm (N = 5)
    assert foot(100_000, d=10.0)[1] - foot(100_000, d=1000.0)[1] >= 16 * 2 * 100_000
    assert foot(1000, d=-1.0)[0] == _capi.ST_ERR_BAD_GEOMETRY


@pytest.mark.parametrize("kind,nb,lo,hi", [("log", 200, 0.01, 1e4), ("lin", 3000, 0.01, 300.0),
                                          ("log", 7, 0.5, 2.0), ("lin", 1, 0.0, 1.0)])
def test_spectrum_post_processing_matches_oracle(kind, nb, lo, hi):
    """PMF_to_PDF and Prepare_for_Semilog (utils.cc:81-117) on ROOT-layout contents: bit-equal
    to the oracle's restatement, including the reference's index range (underflow bin in, last
    bin untouched) and its float normalisation."""
    rs = np.random.default_rng(nb)
    edges = po.edges(kind, nb, lo, hi)
    counts = rs.integers(0, 10_000, nb).astype(np.float64)
    c = st.to_root_layout(counts)
    assert c[0] == 0 and c[-1] == 0 and np.array_equal(c[1:-1], counts)
    pdf = st.CPUHistogramUtils.PMF_to_PDF(edges, c)
    assert np.array_equal(pdf, po.pmf_to_pdf(edges, c), equal_nan=True)
    semi = st.CPUHistogramUtils.Prepare_for_Semilog(edges, pdf)
    assert np.array_equal(semi, po.prepare_for_semilog(edges, pdf), equal_nan=True)
    # the last bin keeps its raw count in both steps (the reference's loops stop before it)
    assert pdf[nb] == counts[-1] and semi[nb] == counts[-1]
    if nb > 1:
        # every other bin: count / width / (float sum of all counts but the last)
        norm = np.float32(0.0)
        for v in c[:nb]:
            norm = np.float32(float(norm) + v)
        b = nb // 2
        assert pdf[b] == counts[b - 1] / (edges[b] - edges[b - 1]) / float(norm)


def test_spectrum_bin_log_x():
    e = st.CPUHistogramUtils.BinLogX(60, -2.0, 4.0)
    assert np.array_equal(e, po.bin_log_x(60, -2.0, 4.0))
    assert abs(e[0] - 0.01) < 1e-15 and abs(e[-1] / 1e4 - 1) < 1e-14
    assert np.all(np.diff(e) > 0)
    rc = _capi.lib().st_spectrum_bin_log_x(0, 0.0, 1.0, None)
    assert rc == _capi.ST_ERR_INVALID_ARGUMENT
