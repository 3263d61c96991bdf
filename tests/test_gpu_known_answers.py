"""The reference's known-answer tests (A1-A8, H1-H8) run through the GPU path, at full size.

A1-A8 run through the C ABI job interface and, for a subset, through the SuperTrackManager
macro loop (st_run_macro) reading track files, which reads like the reference's gtest cases.
"""
import json
import os

import numpy as np
import pytest

import make_golden as mg
import supertrack_b200 as st

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def run_case(ctx, c, zshift=None, n_os=None, export_cap=0, seed=None):
    ctx.clear()
    hid = ctx.histogram(*c["hist"])
    for ti, t in enumerate(c["tracks"]):
        ctx.submit(*t, half_length=c["half_length"], sphere_diameter=c["diameter"],
                   n_oversamples=c["n_os"] if n_os is None else n_os, hist=hid,
                   seed=c["seed"] if seed is None else seed, track_id=ti,
                   shift_track=c["shift_track"], zshift=zshift or c["zshift"])
    sph = ctx.run_export(export_cap) if export_cap else ctx.run("batched")
    counts, yfy = ctx.read_histogram(hid)
    return ctx.edges(hid), counts, yfy, sph


def assert_single_bin(e, counts, value, count):
    b = int(np.searchsorted(e, value, side="right") - 1)
    assert counts[b] == count, (counts[b], count)
    assert counts.sum() == count


@pytest.mark.parametrize("name", ["A1", "A2", "A3", "A4", "A5", "A8"])
def test_a_cases(ctx, name):
    c = mg.a_case(name)
    e, counts, _, _ = run_case(ctx, c)
    assert_single_bin(e, counts, c["expect"]["value"], c["expect"]["count"])


def test_a6_box_edges(ctx):
    c = mg.a_case("A6")
    e, counts, _, _ = run_case(ctx, c)
    assert counts.sum() == 0
    e, counts, _, _ = run_case(ctx, c, zshift="minus")
    assert_single_bin(e, counts, 1.0, mg.A6_MINUS_EXPECT["count"])


@pytest.mark.parametrize("seed", [1234, 1, 987654321])
def test_a7_pi(ctx, seed):
    c = mg.a_case("A7")
    e, counts, _, _ = run_case(ctx, c, seed=seed)
    mid = (e[1:] + e[:-1]) / 2
    pi_hat = 6 * float((mid * counts).sum()) / (20000 * 10000)
    assert 3.05 < pi_hat < 3.3, pi_hat


def test_a8_keys(ctx):
    c = mg.a_case("A8")
    _, counts, _, sph = run_case(ctx, c, export_cap=64)
    assert sorted(int(k) for k in sph["key"]) == sorted(c["keys"])
    assert counts.sum() == 7


@pytest.mark.parametrize("name", list(mg.H_CASES))
def test_h_cases(ctx, name):
    h = mg.H_CASES[name]
    spec = h["restated"] if h.get("invalid") else h["hist"]
    if h.get("invalid"):
        with pytest.raises(st.StError):
            ctx.histogram(*h["hist"])
    c = dict(half_length=mg.H_GEOM["half_length"], diameter=mg.H_GEOM["diameter"],
             shift_track=False, n_os=1, seed=1, zshift="none", hist=spec,
             tracks=mg.h_track(h["n"], h["value"], h["same"]))
    e, counts, yfy, _ = run_case(ctx, c)
    target = h.get("sum_value", h["value"])
    assert_single_bin(e, counts, target, h["expect_count"])
    assert yfy.sum() == target * h["expect_count"]


def _write_macro(tmp_path, name, c, zshift):
    folder = tmp_path / name
    folder.mkdir()
    st.write_track_file(str(folder / f"{name}.strk"), c["tracks"])
    out = tmp_path / "out"
    out.mkdir(exist_ok=True)
    kind, nb, lo, hi = c["hist"]
    text = f"""; {name} restated from tst/testMacros/test{name}.ini
[Run]
Type = Folder
Path = {folder}/
FirstFile = -1 ; #-1 is the default case, will analyze whole folder
LastFile = -1 ;
Threads = 1
Oversamples = {c['n_os']}
RandomSeed = {c['seed']} ; set to -1, or don't set at all to take the current time as seed

[Simulation]
Method = VoxelConstrainedSphere

[VoxelConstrainedSphere]
ScoringRegionHalfLength = {c['half_length']}    ; side length in nanometers
ScoringSphereDiameter = {c['diameter']}        ; sphere diameter in nanometers
ShiftTrack = {'true' if c['shift_track'] else 'false'}				   ; track shifting
ZOriginShift = {zshift}
SuggestedCudaBlocks = 256
SuggestedCudaThreads = 32

[Histogram]
Type = {kind}
NBins = {nb}
BinLower = {lo}
BinUpper = {hi}
SuggestedCudaAccumulateBlocks = 4
SuggestedCudaAccumulateThreads = 32

[Output]
Path = {out}/
NamePrefix = test_{name}_
"""
    p = tmp_path / f"test{name}.ini"
    p.write_text(text)
    return str(p), out


@pytest.mark.parametrize("name", ["A2", "A4", "A8"])
def test_manager_macro_run(tmp_path, name):
    """SuperTrackManager: AddSimulationMethod, Initialize(INIReader(path)), Run, GetOutput."""
    c = mg.a_case(name)
    path, out = _write_macro(tmp_path, name, c, c["zshift"])
    manager = st.SuperTrackManager.GetInstance()
    manager.AddSimulationMethod("VoxelConstrainedSphere", st.VoxelConstrainedSphereMethod.Construct)
    manager.Initialize(path)
    manager.Run()
    edges, counts, yfy = manager.GetOutput()
    assert_single_bin(edges, counts, c["expect"]["value"], c["expect"]["count"])
    side = json.load(open(out / f"test_{name}_{c['seed']}.json"))
    assert side["Number of Tracks"] == len(c["tracks"])
    assert side["Effective Number of Tracks"] == len(c["tracks"]) * c["n_os"]
    csv = np.loadtxt(out / f"test_{name}_{c['seed']}.csv", delimiter=",", skiprows=1)
    assert np.array_equal(csv[:, 2].astype(np.int64), counts)
