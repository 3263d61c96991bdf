"""The bench line's figures from the committed ncu capture of the fused kernel: DRAM traffic
scaled by the workload's units and the shared-memory roofline term (CPU only)."""
import json
import os

import bench

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_figures_of_the_captured_workload():
    p = json.load(open(os.path.join(ROOT, "profiles", "fused_traffic.json")))
    traffic, smem = bench.profile_figures(p["config"], 1e9)
    assert traffic == p["bytes_per_unit"] * 1e9
    assert smem["bound"] == "smem"
    assert 0.0 < smem["frac"] <= 1.0
    assert smem["frac"] == p["smem_wavefront_frac"]
    assert 0.0 <= smem["bank_conflict_share"] <= 1.0


def test_no_figures_for_other_workloads():
    p = json.load(open(os.path.join(ROOT, "profiles", "fused_traffic.json")))
    assert bench.profile_figures(p["config"] + 100, 1e9) == (None, None)
