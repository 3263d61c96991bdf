"""The bench line's CPU-side pieces (CPU only): DRAM traffic from the committed ncu capture, the
stratified CPU-baseline sample and its whole-workload estimate, the job-by-job parity block,
and the config dict that both arms print."""
import json
import os

import numpy as np

import bench
import supertrack_b200.workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_traffic_of_the_captured_workload():
    p = json.load(open(os.path.join(ROOT, "profiles", "fused_traffic.json")))
    assert bench.profile_figures(p["config"], 1e9) == p["bytes_per_unit"] * 1e9
    assert bench.profile_figures(p["config"] + 100, 1e9) is None


def _sizes_only(n=4096):
    """A config-2 workload description without tracks (sizes, classes and settings only)."""
    sizes, kind, d, os_ = W.config2_sizes(n, 3)
    nj = len(sizes)
    return W.Workload(name="sizes", x=None, y=None, z=None, edep=None,
                      offsets=np.concatenate([[0], np.cumsum(sizes)[:-1]]), sizes=sizes,
                      half_length=np.full(nj, 2500.0), diameter=d, n_os=os_,
                      seed=np.full(nj, 3, dtype=np.uint64), track_id=np.arange(nj, dtype=np.uint64),
                      hist_of_job=np.arange(nj), hists=[("log", 200, 0.01, 1e4)] * nj,
                      generator=np.where(kind, 0, 1).astype(np.int8))


def test_stratified_sample_covers_every_class_in_proportion():
    w = _sizes_only()
    cls = w.job_classes()
    assert len(np.unique(cls)) == 24          # 2 generators x 4 diameters x 3 oversample counts
    units = w.sizes * w.n_os.astype(np.int64)
    for frac in (0.05, 0.2):
        jobs, os_run = bench.stratified_sample(w, frac, seed=1)
        assert len(set(jobs.tolist())) == len(jobs)
        assert np.array_equal(os_run, w.n_os[jobs].astype(np.int64))
        assert set(np.unique(cls[jobs]).tolist()) == set(np.unique(cls).tolist())
        total = units[jobs].sum() / units.sum()
        assert 0.5 * frac < total < 1.6 * frac, total
    # deterministic for a seed, different for another
    a, _ = bench.stratified_sample(w, 0.1, seed=3)
    b, _ = bench.stratified_sample(w, 0.1, seed=3)
    c, _ = bench.stratified_sample(w, 0.1, seed=4)
    assert np.array_equal(a, b) and not np.array_equal(a, c)


def test_stratified_sample_caps_oversamples():
    w = W.config4(n_tracks=4, n_dep=1000, n_os=1000)
    jobs, os_run = bench.stratified_sample(w, 0.5, os_cap=16)
    assert np.all(os_run == 16) and len(jobs) >= 1


def test_cpu_estimate_weights_classes_by_their_share_of_the_workload():
    """Thread seconds proportional to units within each class, with a class-dependent cost per
    unit: the estimate must equal the workload's units over its exact thread time / threads,
    whatever the sample's own mix."""
    w = _sizes_only(512)
    cls = w.job_classes()
    cost = {c: 1e-8 * (1 + (i % 5)) for i, c in enumerate(np.unique(cls))}
    jobs, os_run = bench.stratified_sample(w, 0.3, seed=2)
    secs = np.array([cost[cls[j]] * w.sizes[j] * r for j, r in zip(jobs, os_run)])
    est = bench.cpu_estimate(w, jobs, os_run, secs, wall=1.0, threads=8)
    full = w.sizes * w.n_os.astype(np.int64)
    exact_time = sum(cost[cls[j]] * full[j] for j in range(w.n_jobs)) / 8
    assert abs(est["value"] - full.sum() / exact_time) <= 1e-9 * est["value"]
    assert est["cores"] == 8 and est["kind"] == "port"


def test_parity_block_flags_count_stats_and_energy_mismatches():
    oc = [np.array([1, 2, 3]), np.array([0, 5, 0])]
    oy = [np.array([1.0, 2.0, 3.0]), np.array([0.0, 7.5, 0.0])]
    js = np.zeros(2, dtype=[("hits", "<i8"), ("spheres", "<i8"), ("binned", "<i8")])
    js["hits"] = [10, 20]
    js["spheres"] = [6, 5]
    js["binned"] = [6, 5]
    sample = (np.array([3, 9]), np.array([10, 100]), oc, oy, js)
    gs = [{"hits": 10, "spheres": 6, "binned": 6, "n": 100},
          {"hits": 20, "spheres": 5, "binned": 5, "n": 50}]
    ok = bench.parity_block([c.copy() for c in oc], [y * (1 + 1e-14) for y in oy], gs, sample, "t")
    assert ok["pass"] and ok["counts_equal"] and ok["stats_equal"]
    assert ok["jobs_checked"] == 2 and ok["units_checked"] == 100 * 10 + 50 * 100
    bad_c = [oc[0].copy(), oc[1] + np.array([0, 1, 0])]
    r = bench.parity_block(bad_c, oy, gs, sample, "t")
    assert not r["pass"] and not r["counts_equal"] and r["first_mismatch_job"] == 9
    bad_s = [dict(g) for g in gs]
    bad_s[0]["spheres"] += 1
    r = bench.parity_block(oc, oy, bad_s, sample, "t")
    assert not r["pass"] and not r["stats_equal"] and r["first_mismatch_job"] == 3
    r = bench.parity_block(oc, [oy[0] * (1 + 1e-9), oy[1]], gs, sample, "t")
    assert not r["pass"] and r["max_rel_yfy"] > 1e-12


def test_both_arms_print_the_same_config():
    w = W.config0(n_tracks=2, n_dep=100)
    a = bench.config_dict(0, w, 1, 1.0)
    b = bench.config_dict(0, w, 1, 1.0)
    assert a == b and a["units_per_step"] == w.units
    assert "flushed" in a["l2"]       # a tiny workload fits L2: the GPU arm flushes it
    assert bench.config_dict(2, _sizes_only(), 1, 1.0)["l2"].startswith("inputs larger")


def test_reference_arm_prints_the_contract_line():
    """`bench.py --impl reference` (the CPU restatement, no GPU needed) on the small proton
    workload prints one JSON line with the contract's keys and the same config as the GPU arm."""
    import subprocess
    import sys
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--config", "0", "--steps", "2", "--warmup", "1"],
                         capture_output=True, text=True, timeout=600, check=True).stdout
    line = json.loads(out.strip().splitlines()[-1])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "higher_is_better",
              "scaling", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["value"] == line["value"]
    assert line["config"] == bench.config_dict(0, W.config0(), 1, 1.0)
    assert len(line["cpu_baseline"]["per_step_values"]) == 2
