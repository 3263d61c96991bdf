"""Benchmark of the VoxelConstrainedSphere superimposition path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config 2|0|1|4] [--also 0,1,4] [--scale S]

One step = one pass of the hot path over the whole synthetic workload: every track's prepare
pass plus the fused superimposition of all its oversamples into its histogram. The headline
workload is the batched uneven configuration (4,096 tracks, lognormal sizes with median 2e4
deposits, d in {2,10,100,1000} nm, oversamples in {1,10,100}, one 200-bin log histogram per
track), the one the batched-versus-plain metric is quoted on. The other configurations that fit
one GPU (--also: the 64-track proton set, the 16 dense ion tracks, and the 256 x 4e6-deposit
single-geometry run at full size) are measured in the same run and reported under
"per_config".

Metric: deposit*oversamples per second (higher is better).
  value : inputs resident in HBM, one batched run per step, device time (CUDA events on the
          stream the kernels run on), max over ranks;
  e2e   : the same through the public API with host (pinned) tracks: every step copies the
          tracks host->device (in groups on a second stream, overlapped with the kernels of
          earlier groups) and reads every histogram back device->host.
Parity: the jobs the CPU baseline runs through the oracle are compared job by job with the GPU's
own results (histogram counts, hits, spheres and binned spheres bit-exact; y*f(y) within 1e-12
relative) and reported as "parity".
Multi-GPU (torchrun, or --gpus N, which starts its own N ranks): the headline workload's jobs are
partitioned across ranks by longest-processing-time first on their deposit*oversamples; each
rank runs its share as one batched launch, and every step ends with one NCCL all-reduce of the
spectra (the reference's TH1::Add of the workers' histograms). The total work is fixed (strong
scaling); value = the workload's units / the slowest rank's time. --scaling weak gives every
rank its own replica of the workload instead (seed offset by 1000 x rank, the same spectrum
all-reduce); value = all ranks' units / the slowest rank's time.

--impl reference: the reference cannot be built here (CERN ROOT is absent and its histogram
stage needs device-side cudaDeviceSynchronize, which CUDA 12 rejects), so this arm times the
CPU restatement of the reference algorithm (oracle/) on all host threads, on the same workload
and config as the GPU arm: each step a stratified sample of its jobs, scaled to the whole
workload by job class. Rank 0 alone runs it.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "deposit*oversamples/s on 1 B200 (batched persistent form)"
UNIT = "deposit*oversamples/s"
# FP64 operations of the literal reference arithmetic per deposit*oversample: 2 shift adds for
# every deposit, and for deposits inside the voxel 3 subtractions, 3 divisions, 3 multiplies
# (k*d), 3 subtractions, 3 squares and 2 additions (VoxelConstrainedSphereMethod.cu:183-258).
FP64_OPS_ALL = 2
FP64_OPS_INBOX = 17
# Algorithmic HBM bytes of one fused launch: the prepared record of every deposit read once
# (36 B: x, y, dz^2 and the 12-byte share of value and key a deposit needs on average) and the
# histograms written once (16 B per bin).
BYTES_PREP = 36
# Oversamples of a config-4 job that the CPU baseline and the parity check run (its 1,000
# oversamples would take the host minutes per job).
CFG4_OS_SAMPLE = 16
# Tracks of the 256-track configuration that its plain per-track loop runs.
CFG4_PLAIN_TRACKS = 32


def profile_figures(config: int, units: float):
    """Figures of the committed k_fused ncu capture, for the bench line: DRAM traffic scaled to
    `units` deposit*oversamples (bytes per unit x units). None when no capture of this workload
    exists."""
    prof = os.path.join(ROOT, "profiles", "fused_traffic.json")
    try:
        p = json.load(open(prof))
    except (OSError, ValueError):
        return None
    if p.get("config") != config:
        return None
    return float(p["bytes_per_unit"]) * units if "bytes_per_unit" in p else None


def parse(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--config", type=int, default=2, choices=[0, 1, 2, 4])
    p.add_argument("--also", default="0,1,4",
                   help="other configurations measured in the same run (comma list, '' for none)")
    p.add_argument("--scale", type=float, default=1.0,
                   help="track-count scale of the headline workload (1.0 = as specified)")
    p.add_argument("--scaling", default="strong", choices=["strong", "weak"],
                   help="several GPUs: strong = the one headline workload LPT-sharded over the "
                        "ranks; weak = every rank runs its own replica of it (seed offset by "
                        "1000 x rank)")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-plain", action="store_true")
    p.add_argument("--no-fp32", action="store_true",
                   help="skip the FP32 geometry variant's leg (reported beside the FP64 value)")
    p.add_argument("--cpu-seconds", type=float, default=15.0,
                   help="host seconds of the CPU baseline's sample (all threads)")
    p.add_argument("--no-tune", action="store_true",
                   help="skip the autotuner (default planning parameters)")
    p.add_argument("--tune-trials", type=int, default=24)
    p.add_argument("--no-serve", action="store_true",
                   help="skip the served-stream leg (10,000 arriving jobs at four loads)")
    p.add_argument("--serve-jobs", type=int, default=10000)
    return p.parse_args(argv)


# ---------------------------------------------------------------------------------------------
# Workloads and the config dict both arms print
# ---------------------------------------------------------------------------------------------
DESC = {
    0: "config0: 64 proton-like tracks x 4000 deposits, HL 2500 nm, d 10 nm, 10 OS, lin 3000 bins",
    1: "config1: 16 ion tracks x 1e6 deposits, HL 5000 nm, d 2 nm, 100 OS, log 500 bins",
    2: ("config2: 4096 uneven tracks (lognormal sizes median 2e4, sigma 1.5, clipped [500, 2e6]), "
        "half proton-like, half ion-like, d in {2,10,100,1000} nm, OS in {1,10,100}, HL 2500 nm, "
        "one log 200-bin histogram per track"),
    4: ("config4: 256 ion tracks x 4e6 deposits (core sigma 3 nm, penumbra to 1000 nm), "
        "HL 5000 nm, d 10 nm, 1000 OS, lin 3000 bins, f(y) and y*f(y)"),
}
SEED = {0: 1, 1: 2, 2: 3, 4: 5}


def make_workload(cfg: int, device, scale: float = 1.0, replica: int = 0):
    """The configuration's workload; replica r > 0 (weak scaling) draws it with seed + 1000 r."""
    import supertrack_b200.workloads as W
    n = {0: 64, 1: 16, 2: 4096, 4: 256}[cfg]
    n = max(1, int(round(n * scale)))
    gen = {0: W.config0, 1: W.config1, 2: W.config2, 4: W.config4}[cfg]
    return gen(device=device, n_tracks=n, seed=SEED[cfg] + 1000 * replica)


L2_BYTES = 126 * 2**20


def fits_l2(w) -> bool:
    """Whether the tracks and prepared records (32 + 56 bytes per deposit) could stay in L2."""
    return w.deposits * 88 <= 2 * L2_BYTES


def config_dict(cfg: int, w, world: int, scale: float, scaling: str = "strong") -> dict:
    """The workload description both arms print (identical for the same arguments). Under weak
    scaling every one of the `world` ranks runs its own replica of w."""
    desc = DESC[cfg] if scale == 1.0 else DESC[cfg] + f" (track count x{scale})"
    reps = world if scaling == "weak" else 1
    if world == 1:
        par = "1 GPU"
    elif scaling == "weak":
        par = (f"{world} GPUs: one replica of the workload per rank (seed + 1000 x rank), "
               "one spectrum all-reduce per step")
    else:
        par = f"{world} GPUs: LPT job shards, one spectrum all-reduce per step"
    return {"workload": desc, "seed": SEED[cfg], "jobs": w.n_jobs * reps,
            "deposits": w.deposits * reps, "units_per_step": w.units * reps,
            "l2": ("L2 flushed before every timed step (a 512 MB write outside the timed events)"
                   if fits_l2(w) else
                   "inputs larger than L2 (tracks + prepared records > 126 MB), no flush"),
            "parallelism": par}


def cpu_model() -> str:
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, mx, reasons, power = [], None, set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
                power.append(float(f[3]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm),
                "power_w_max": max(power) if power else None}


# ---------------------------------------------------------------------------------------------
# CPU baseline (the oracle port) on a stratified sample, and the parity check of that sample
# ---------------------------------------------------------------------------------------------
def stratified_sample(w, frac: float, seed: int = 0, os_cap=None):
    """Jobs of w in every class (generator x sphere diameter x oversamples), each class sampled
    to about `frac` of its deposit*oversamples (at least one job per class). os_cap limits the
    oversamples a sampled job runs. Returns (job indices, oversamples each job runs)."""
    cls = w.job_classes()
    n_os = w.n_os.astype(np.int64)
    os_eff = np.minimum(n_os, os_cap) if os_cap else n_os
    units = w.sizes.astype(np.int64) * os_eff
    rs = np.random.default_rng(seed)
    chosen = []
    for c in np.unique(cls):
        jobs = np.nonzero(cls == c)[0]
        target = frac * float(units[jobs].sum())
        got = 0
        for j in jobs[rs.permutation(len(jobs))]:
            if got >= target:
                break
            if got == 0 or got + units[j] / 2 <= target:
                chosen.append(int(j))
                got += int(units[j])
    chosen = np.array(sorted(chosen), dtype=np.int64)
    return chosen, os_eff[chosen]


def oracle_sample(w, jobs, os_run, threads):
    """Runs the listed jobs (oversamples 0..os_run-1 each) through the oracle, each into its own
    histogram, largest first across `threads` host threads. Returns per-job counts, y*f(y),
    stats, thread seconds, and the wall seconds of the run."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    x, y, z, e = [a.cpu().numpy() for a in (w.x, w.y, w.z, w.edep)]
    units = w.sizes[jobs].astype(np.int64) * os_run
    order = np.argsort(-units, kind="stable")
    sel = jobs[order]
    edges = [po.edges(*w.hists[int(w.hist_of_job[j])]) for j in sel]
    t0 = time.perf_counter()
    counts, yfy, js, secs = po.run_batch(
        x, y, z, e, w.offsets[sel], w.sizes[sel], w.half_length[sel], w.diameter[sel],
        np.full(len(sel), {"plus": 0, "minus": 1, "none": 2}[w.zshift]),
        np.full(len(sel), int(w.shift_track)), os_run[order], w.seed[sel], w.track_id[sel],
        np.arange(len(sel)), edges, threads=threads, job_stats=True)
    wall = time.perf_counter() - t0
    inv = np.empty_like(order)
    inv[order] = np.arange(len(order))
    return ([counts[i] for i in inv], [yfy[i] for i in inv], js[inv], secs[inv], wall)


def cpu_estimate(w, jobs, os_run, secs, wall, threads, kind="port"):
    """Whole-workload CPU rate from a sample: thread seconds per deposit*oversample of each job
    class, scaled to the class's units in the full workload, spread over the host threads (as if
    the full workload balanced perfectly over them)."""
    cls = w.job_classes()
    full_units = w.sizes.astype(np.int64) * w.n_os.astype(np.int64)
    s_units = w.sizes[jobs].astype(np.int64) * os_run
    t_full = 0.0
    for c in np.unique(cls):
        m = cls[jobs] == c
        t_full += float(secs[m].sum()) * float(full_units[cls == c].sum()) / float(s_units[m].sum())
    value = float(full_units.sum()) / (t_full / threads)
    return {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
            "cpu_model": cpu_model(),
            "sample": (f"{len(jobs)} of {w.n_jobs} jobs in {len(np.unique(cls))} classes "
                       f"(generator x d x oversamples), {int(s_units.sum()):.3e} "
                       f"deposit*oversamples, {wall:.1f} s on {threads} threads; thread seconds "
                       "per unit of each class scaled to the class's share of the workload"),
            "sample_rate": float(s_units.sum()) / wall}


def cpu_baseline(w, seconds: float, threads: int, seed: int = 0, os_cap=None):
    """Times the oracle on a stratified sample sized for about `seconds` of host time; returns
    (cpu_baseline dict, (jobs, os_run, counts, yfy, stats) of the sample for the parity check)."""
    n_os = w.n_os.astype(np.int64)
    full_units = float((w.sizes * (np.minimum(n_os, os_cap) if os_cap else n_os)).sum())
    # a first small sample calibrates the rate per thread (thread seconds: a small sample keeps
    # only a few threads busy), the second is sized from it
    frac0 = min(1.0, 4e6 * threads / full_units)
    jobs, os_run = stratified_sample(w, frac0, seed, os_cap)
    c, y, js, secs, wall = oracle_sample(w, jobs, os_run, threads)
    rate = float((w.sizes[jobs] * os_run).sum()) / max(float(secs.sum()), 1e-6) * threads
    frac = min(1.0, rate * seconds / full_units)
    if frac > 1.5 * frac0:
        jobs, os_run = stratified_sample(w, frac, seed, os_cap)
        c, y, js, secs, wall = oracle_sample(w, jobs, os_run, threads)
    return cpu_estimate(w, jobs, os_run, secs, wall, threads), (jobs, os_run, c, y, js)


def parity_block(gpu_counts, gpu_yfy, gpu_stats, sample, where: str) -> dict:
    """Job-by-job comparison of GPU results with the oracle's for the sampled jobs."""
    jobs, os_run, oc, oy, js = sample
    counts_equal = stats_equal = True
    max_rel = 0.0
    first_bad = None
    for k, j in enumerate(jobs):
        gc, gy, gs = gpu_counts[k], gpu_yfy[k], gpu_stats[k]
        ce = bool(np.array_equal(gc, oc[k]))
        se = (gs["hits"] == js["hits"][k] and gs["spheres"] == js["spheres"][k]
              and gs["binned"] == js["binned"][k])
        if (not ce or not se) and first_bad is None:
            first_bad = int(j)
        counts_equal &= ce
        stats_equal &= bool(se)
        scale = np.maximum(np.abs(oy[k]), 1e-300)
        if len(gy):
            max_rel = max(max_rel, float(np.max(np.abs(gy - oy[k]) / scale)))
    return {"jobs_checked": int(len(jobs)),
            "units_checked": int((np.asarray(os_run, dtype=np.int64) *
                                  np.asarray([gs["n"] for gs in gpu_stats], dtype=np.int64)).sum()),
            "counts_equal": counts_equal, "stats_equal": stats_equal,
            "max_rel_yfy": max_rel, "yfy_tolerance": 1e-12,
            "pass": bool(counts_equal and stats_equal and max_rel <= 1e-12),
            "first_mismatch_job": first_bad, "where": where}


def reference_arm(args, rank, world):
    if rank != 0:
        return
    import torch
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    w = make_workload(args.config, dev, args.scale).to("cpu")
    threads = os.cpu_count() or 1
    per_step = max(2.0, min(20.0, 150.0 / max(1, args.steps + args.warmup)))
    os_cap = CFG4_OS_SAMPLE if args.config == 4 else None
    res = []
    for k in range(args.warmup + args.steps):
        r, _ = cpu_baseline(w, per_step, threads, seed=k, os_cap=os_cap)
        if k >= args.warmup:
            res.append(r)
    value = statistics.median([r["value"] for r in res])
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": args.scaling, "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": config_dict(args.config, w, world, args.scale, args.scaling),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "cpu_model": cpu_model(), "sample": res[-1]["sample"],
                             "per_step_values": [r["value"] for r in res]},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "ms_per_step": None}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------------------------
def submit_jobs(ctx, w, jobs, hist_ids, on_device: bool, tensors, os_run=None):
    """Submits the listed jobs of w; tensors = (x, y, z, edep) flat (device or pinned host);
    hist_ids[k] is the histogram of the k-th listed job."""
    import supertrack_b200 as st
    from supertrack_b200 import _capi
    import ctypes as C
    n = len(jobs)
    if n == 0:
        return
    tv = (_capi.st_track_view * n)()
    jd = (_capi.st_job_desc * n)()
    base = [t.data_ptr() for t in tensors]
    for k, j in enumerate(jobs):
        o = int(w.offsets[j]) * 8
        tv[k].x, tv[k].y, tv[k].z, tv[k].edep = [b + o for b in base]
        tv[k].n = int(w.sizes[j])
        tv[k].on_device = int(on_device)
        jd[k].half_length = float(w.half_length[j])
        jd[k].sphere_diameter = float(w.diameter[j])
        jd[k].zshift = st.ZSHIFT[w.zshift]
        jd[k].shift_track = int(w.shift_track)
        jd[k].n_oversamples = int(w.n_os[j] if os_run is None else os_run[k])
        jd[k].hist_id = hist_ids[k]
        jd[k].seed = int(w.seed[j])
        jd[k].track_id = int(w.track_id[j])
    st.check(_capi.lib().st_job_submit_many(ctx.handle, n, tv, jd, None), "submit", ctx.handle)


def read_spectra(ctx, hids):
    """(counts, y*f(y)) of the listed histograms, read with one copy of every bin."""
    import torch
    nb = ctx.total_bins()
    c = torch.empty(nb, dtype=torch.int64)
    y = torch.empty(nb, dtype=torch.float64)
    ctx.read_all_into(c.data_ptr(), y.data_ptr(), nb)
    c, y = c.numpy(), y.numpy()
    out_c, out_y = [], []
    for h in hids:
        o, n = ctx.hist_offset(h), ctx.nbins(h)
        out_c.append(c[o:o + n].copy())
        out_y.append(y[o:o + n].copy())
    return out_c, out_y


def job_stats(ctx, n_jobs_in_ctx, w, jobs):
    out = []
    for k in range(n_jobs_in_ctx):
        s = dict(ctx.stats(k))
        s["n"] = int(w.sizes[jobs[k]])
        out.append(s)
    return out


class Timer:
    """CUDA-event timing of a region on the bench's stream, max over ranks."""

    def __init__(self, stream, world, dev):
        import torch
        self.torch, self.stream, self.world, self.dev = torch, stream, world, dev

    def __enter__(self):
        torch = self.torch
        if self.world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        self.e0 = torch.cuda.Event(enable_timing=True)
        self.e1 = torch.cuda.Event(enable_timing=True)
        self.e0.record(self.stream)
        return self

    def __exit__(self, *exc):
        torch = self.torch
        self.e1.record(self.stream)
        torch.cuda.synchronize()
        if self.world > 1:
            torch.distributed.barrier()
        t = torch.tensor([self.e0.elapsed_time(self.e1)], device=self.dev)
        if self.world > 1:
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        self.ms = float(t.item())


def hbm_peak():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"], \
            "MEASURED_PEAKS.json"
    except Exception:
        return 6650.0, "fallback"


def serve_leg(dev, batched_value: float, n_jobs: int):
    """Served stream: n_jobs of the uneven distribution (seed 4) arrive as a Poisson process
    offering 25/50/80/100% of the measured batched throughput; the server admits them against a
    150 GB budget and batches them continuously. Latency = completion (spectrum in the caller's
    host arrays) minus scheduled arrival."""
    import torch
    import supertrack_b200 as st
    from supertrack_b200 import serving
    w = serving.served_workload(dev, n_jobs=n_jobs, seed=4)
    torch.cuda.synchronize()
    work = serving.job_work(w)
    out = {"jobs": n_jobs, "deposits": w.deposits, "units": float(work.sum()),
           "budget_bytes": 150_000_000_000, "offered_basis": batched_value,
           "workload": "served stream: 10,000 jobs of the uneven batched distribution, seed 4",
           "latency": "completion (spectrum copied to host) minus scheduled Poisson arrival",
           "loads": []}
    with st.Server(dev.index, budget_bytes=150_000_000_000, max_track_deposits=2_000_000,
                   max_batch_jobs=4096) as srv:
        # warm-up: one burst of every job sizes the contexts' device arenas, so that no
        # allocation (cudaFree waits for the whole device) happens while latencies are measured
        _, _, rec, _ = serving.replay(srv, w, np.zeros(w.n_jobs, dtype=np.int64))
        if np.any(rec["status"] != 0):
            raise RuntimeError("served warm-up failed")
        for load in (0.25, 0.5, 0.8, 1.0):
            arr = serving.poisson_arrivals(w, load * batched_value, seed=4)
            _, _, rec, wall = serving.replay(srv, w, arr)
            summ = serving.latency_summary(rec, work)
            summ.update({"load": load, "offered": load * batched_value,
                         "arrival_span_s": float(arr[-1] / 1e9)})
            out["loads"].append(summ)
        # a longer window at 80 % load: the same tracks replayed five times over (50,000 jobs,
        # each repeat with its own track ids and so its own shifts)
        wl = serving.repeated(w, 5)
        arr = serving.poisson_arrivals(wl, 0.8 * batched_value, seed=5)
        _, _, rec, wall = serving.replay(srv, wl, arr)
        summ = serving.latency_summary(rec, serving.job_work(wl))
        summ.update({"load": 0.8, "offered": 0.8 * batched_value, "jobs": wl.n_jobs,
                     "arrival_span_s": float(arr[-1] / 1e9),
                     "workload": "the 10,000 jobs replayed five times at 80 % load"})
        out["long_stream_80pct"] = summ
    out["p99_ms_at_80pct"] = next(l["p99_ms"] for l in out["loads"] if l["load"] == 0.8)
    return out


def headline(args, rank, world, dev, stream):
    """The headline configuration: value, e2e, plain, FP32 leg, rooflines, CPU baseline and the
    parity of the CPU sample against this run's own per-job spectra."""
    import torch
    import supertrack_b200 as st
    from supertrack_b200.sharding import reduce_spectra_device, shard
    weak = world > 1 and args.scaling == "weak"
    w = make_workload(args.config, dev, args.scale, replica=rank if weak else 0)
    torch.cuda.synchronize()
    torch.cuda.empty_cache()   # the generator's temporaries: the context sizes from free memory
    costs = w.sizes.astype(np.float64) * w.n_os.astype(np.float64)
    mine = np.array(shard(costs, rank, world) if world > 1 and not weak else range(w.n_jobs),
                    dtype=np.int64)
    ctx = st.Context(dev.index, stream=stream.cuda_stream)
    # every rank holds every histogram of the workload (the same bin layout on all ranks, which
    # the all-reduce needs) and submits its own jobs into theirs
    all_hids = [ctx.histogram(*h) for h in w.hists]
    hids = [all_hids[int(w.hist_of_job[j])] for j in mine]
    submit_jobs(ctx, w, mine, hids, True, (w.x, w.y, w.z, w.edep))
    ctx.enable_timing(True)
    # spectra of the whole workload on this device, all-reduced over the ranks every step
    spec_bins = ctx.total_bins()
    spec_c = torch.zeros(spec_bins, dtype=torch.int64, device=dev)
    spec_y = torch.zeros(spec_bins, dtype=torch.float64, device=dev)

    def step():
        ctx.jobs_reset()
        ctx.run("batched")
        if world > 1:
            ctx.read_all_into(spec_c.data_ptr(), spec_y.data_ptr(), spec_bins)
            reduce_spectra_device(spec_c, spec_y)

    # ---- autotuned planning parameters (untimed; histograms and job states are restored),
    # then warm-up: the first rerun captures the CUDA graph the timed steps replay
    ctx.run("batched")
    tune = None if args.no_tune else ctx.autotune(args.tune_trials)
    for _ in range(args.warmup):
        step()
    stats = [ctx.stats(k) for k in range(len(mine))]
    inbox = sum(s["inbox"] for s in stats)
    hits = sum(s["hits"] for s in stats)
    spheres = sum(s["spheres"] for s in stats)
    tot = torch.tensor([inbox, hits, spheres], dtype=torch.float64, device=dev)
    if world > 1:
        torch.distributed.all_reduce(tot)
    inbox, hits, spheres = (int(v) for v in tot.tolist())

    # ---- timed region: inputs resident in HBM (9+ GB of tracks and prepared records, well
    # above the 126 MB L2, so no flush is needed between steps)
    sampler = ClockSampler(dev.index)
    sampler.start()
    g_before = ctx.get_param("graph_launches")
    t_prep = t_fused = 0.0
    launches = 0
    with Timer(stream, world, dev) as T:
        for _ in range(args.steps):
            step()
            a, b, n = ctx.last_timing()
            t_prep += a
            t_fused += b
            launches += n
    clocks = sampler.stop()
    graph_steps = ctx.get_param("graph_launches") - g_before
    units = w.units * (world if weak else 1)   # the whole job's units over all ranks
    value = units * args.steps / (T.ms * 1e-3)

    # ---- parity of this run's per-job results against the oracle on the CPU sample (rank 0
    # checks the jobs it owns; the others only run the clean pass)
    ctx.reset_histogram(-1)
    ctx.jobs_reset()
    ctx.run("batched")
    gc, gy = read_spectra(ctx, hids)
    gs = job_stats(ctx, len(mine), w, mine)

    # ---- e2e through the public API with pinned host tracks and histogram read-back
    e2e = None
    if not args.no_e2e:
        hx = [t.to("cpu").pin_memory() for t in (w.x, w.y, w.z, w.edep)]
        ctx2 = st.Context(dev.index, stream=stream.cuda_stream)
        all2 = [ctx2.histogram(*h) for h in w.hists]
        hid2 = [all2[int(w.hist_of_job[j])] for j in mine]
        submit_jobs(ctx2, w, mine, hid2, False, hx)
        nb = ctx2.total_bins()
        out_c = torch.empty(nb, dtype=torch.int64, pin_memory=True)
        out_y = torch.empty(nb, dtype=torch.float64, pin_memory=True)
        for _ in range(max(1, args.warmup)):
            ctx2.jobs_reset()
            ctx2.run("batched")
            ctx2.read_all_into(out_c.data_ptr(), out_y.data_ptr(), nb)
        e2e_steps = max(1, min(args.steps, 5))
        with Timer(stream, world, dev) as E:
            for _ in range(e2e_steps):
                ctx2.jobs_reset()
                ctx2.run("batched")
                ctx2.read_all_into(out_c.data_ptr(), out_y.data_ptr(), nb)
        # bytes of the whole job: every rank uploads its own tracks and reads its spectra back
        h2d = int(w.deposits) * 32 * (world if weak else 1)
        e2e = {"value": units * e2e_steps / (E.ms * 1e-3), "unit": UNIT,
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": int(nb * 16) * world,
               "steps": e2e_steps}
        # the upload's roofline (untimed): this rank's track bytes per step over the e2e step
        # time, against one plain pinned host-to-device copy of its x array on the same link
        mine_bytes = int(w.sizes[mine].sum()) * 32
        dst = torch.empty(hx[0].shape, dtype=hx[0].dtype, device=dev)
        best = None
        with torch.cuda.stream(stream):
            for _ in range(3):
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
                dst.copy_(hx[0], non_blocking=True)
                b.record(stream)
                b.synchronize()
                t = a.elapsed_time(b)
                best = t if best is None else min(best, t)
        copy_gbs = hx[0].numel() * 8 / (best * 1e-3) / 1e9
        achieved = mine_bytes / (E.ms / e2e_steps * 1e-3) / 1e9
        e2e["pcie"] = {"achieved_gbs": achieved, "copy_gbs": copy_gbs, "frac": achieved / copy_gbs,
                       "copy": "one pinned cudaMemcpyAsync of this rank's x array "
                               f"({hx[0].numel() * 8 / 1e9:.2f} GB), best of 3",
                       "rank_bytes_per_step": mine_bytes}
        del dst
        ctx2.close()
        del hx

    # ---- plain per-track form on the same workload (one pass), for the batched/plain ratio
    plain = None
    if not args.no_plain:
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        ctx.jobs_reset()
        t0 = time.perf_counter()
        ctx.run("plain")
        torch.cuda.synchronize()
        pt = torch.tensor([time.perf_counter() - t0], device=dev)
        if world > 1:
            torch.distributed.all_reduce(pt, op=torch.distributed.ReduceOp.MAX)
        pval = units / float(pt.item())
        plain = {"value": pval, "unit": UNIT, "batched_over_plain": value / pval,
                 "timing": "host wall clock around the per-track loop (one sync per track)"}

    # ---- FP32 geometry variant on the same jobs (not the headline: it is not bound to the
    # reference's FP64 results); its spectra are compared with one FP64 run of the same jobs
    fp32 = None
    if not args.no_fp32:
        nb = ctx.total_bins()
        spectra = {}
        for prec in (64, 32):
            ctx.set_param("precision", prec)
            ctx.reset_histogram(-1)        # zero every histogram (they stay in place)
            ctx.jobs_reset()
            ctx.run("batched")
            c_ = torch.empty(nb, dtype=torch.int64)
            y_ = torch.empty(nb, dtype=torch.float64)
            ctx.read_all_into(c_.data_ptr(), y_.data_ptr(), nb)
            st_ = [ctx.stats(k) for k in range(len(mine))]
            spectra[prec] = (c_.numpy().copy(), sum(s["hits"] for s in st_),
                             sum(s["spheres"] for s in st_), sum(s["binned"] for s in st_))
        ctx.set_param("precision", 32)
        for _ in range(args.warmup):
            ctx.jobs_reset()
            ctx.run("batched")
        f_prep = f_fused = 0.0
        with Timer(stream, world, dev) as F:
            for _ in range(args.steps):
                ctx.jobs_reset()
                ctx.run("batched")
                a, b, _n = ctx.last_timing()
                f_prep += a
                f_fused += b
        ctx.set_param("precision", 64)
        c64, h64, s64, b64 = spectra[64]
        c32, h32, s32, b32 = spectra[32]
        fp32 = {"value": units * args.steps / (F.ms * 1e-3), "unit": UNIT,
                "ms_per_step": F.ms / args.steps,
                "kernel_ms": {"prepare": f_prep / args.steps, "fused": f_fused / args.steps},
                "fp64_run": {"hits": h64, "spheres": s64, "binned": b64},
                "diff_vs_fp64": {"hits": h32 - h64, "spheres": s32 - s64, "binned": b32 - b64,
                                 "counts_l1": int(np.abs(c32 - c64).sum())},
                "hits_rel_diff": (h32 - h64) / max(h64, 1),
                "spheres_rel_diff": (s32 - s64) / max(s64, 1),
                "counts_l1_rel": float(np.abs(c32 - c64).sum()) / max(float(c64.sum()), 1.0),
                "note": "FP32 geometry variant (x/y geometry in float; z, keys and energies as "
                        "FP64): reported beside the FP64 value, not bound to reference parity"}

    fp64_peak = ctx.fp64_peak()
    smem_peak = ctx.smem_atomic_peak()
    nbins_total = ctx.total_bins()
    ctx.close()
    if rank != 0:
        return None, w
    fused_ms = t_fused / args.steps
    prep_ms = t_prep / args.steps
    peak, peak_src = hbm_peak()
    fused_bytes = BYTES_PREP * w.deposits + 16 * nbins_total
    fp64_ops = FP64_OPS_ALL * units + FP64_OPS_INBOX * inbox
    smem_ops = hits + spheres
    traffic = profile_figures(args.config, units) if world == 1 else None
    cpu, sample = cpu_baseline(w.to("cpu") if w.x.is_cuda else w, args.cpu_seconds,
                               os.cpu_count() or 1)
    pos = {int(j): k for k, j in enumerate(mine)}
    keep = [k for k, j in enumerate(sample[0]) if int(j) in pos]
    sub = (sample[0][keep], sample[1][keep], [sample[2][k] for k in keep],
           [sample[3][k] for k in keep], sample[4][keep])
    idx = [pos[int(j)] for j in sub[0]]
    parity = parity_block([gc[i] for i in idx], [gy[i] for i in idx], [gs[i] for i in idx], sub,
                          "the headline batch's own per-job spectra and job statistics (a clean "
                          "rerun of the timed batch)")
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": T.ms / args.steps, "higher_is_better": True,
        "scaling": args.scaling, "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_dict(args.config, w, world, args.scale, args.scaling),
        "work_per_step": {"inbox_units": inbox, "hits": hits, "spheres": spheres},
        "gpu_launches": launches,
        "graph_steps": graph_steps,
        "autotune": tune,
        "kernel_ms": {"prepare": prep_ms, "fused": fused_ms},
        "roofline": {"bound": "hbm", "achieved": fused_bytes / (fused_ms * 1e-3) / 1e9,
                     "peak": peak, "unit": "GB/s",
                     "frac": fused_bytes / (fused_ms * 1e-3) / 1e9 / peak,
                     "traffic": traffic, "peak_source": peak_src,
                     "kernel": "k_fused (dominant)", "bytes_per_launch": fused_bytes},
        "roofline_fp64": {"bound": "fp64", "achieved": fp64_ops / (fused_ms * 1e-3) / 1e12,
                          "peak": fp64_peak / 1e12, "unit": "TFLOP/s (fp64 add/mul/div)",
                          "frac": fp64_ops / (fused_ms * 1e-3) / fp64_peak,
                          "ops_per_launch": fp64_ops,
                          "peak_source": "measured live (dependent add+mul chains)"},
        "roofline_smem": {"bound": "smem", "achieved": smem_ops / (fused_ms * 1e-3),
                          "peak": smem_peak, "unit": "shared-memory 64-bit atomic updates/s",
                          "frac": smem_ops / (fused_ms * 1e-3) / smem_peak,
                          "ops_per_launch": smem_ops,
                          "ops": "one accumulator update per hit + one histogram update per "
                                 "sphere (algorithmic counts of the launch)",
                          "peak_source": "measured live (conflict-free 64-bit shared atomics, "
                                         "one 1024-thread CTA per SM)"},
        "clocks": clocks,
        "e2e": e2e,
        "plain": plain,
        "fp32": fp32,
        "cpu_baseline": cpu,
        "parity": parity,
        "serving": None,
        "per_config": {},
    }
    return line, w


def other_config(cfg, args, dev, stream):
    """One more configuration on this GPU: value (device-resident, batched), plain, e2e where the
    host holds its tracks comfortably, rooflines, CPU baseline and parity."""
    import torch
    import supertrack_b200 as st
    t_gen = time.perf_counter()
    w = make_workload(cfg, dev)
    torch.cuda.synchronize()
    t_gen = time.perf_counter() - t_gen
    torch.cuda.empty_cache()
    jobs = np.arange(w.n_jobs)
    ctx = st.Context(dev.index, stream=stream.cuda_stream)
    hids_all = [ctx.histogram(*h) for h in w.hists]
    submit_jobs(ctx, w, jobs, [hids_all[int(w.hist_of_job[j])] for j in jobs], True,
                (w.x, w.y, w.z, w.edep))
    ctx.enable_timing(True)
    t0 = time.perf_counter()
    ctx.run("batched")
    torch.cuda.synchronize()
    first_s = time.perf_counter() - t0
    warm = 3
    for _ in range(warm):
        ctx.jobs_reset()
        ctx.run("batched")
    a, b, _n = ctx.last_timing()
    steps = int(min(max(args.steps, 1), max(2, math.ceil(10000.0 / max(a + b, 1e-3)))))
    t_prep = t_fused = 0.0
    # every step timed by its own events; a workload that fits L2 gets it flushed before each
    flush = torch.empty(512 * 2**20, dtype=torch.uint8, device=dev) if fits_l2(w) else None
    step_ms = 0.0
    for _ in range(steps):
        if flush is not None:
            flush.fill_(1)
        with Timer(stream, 1, dev) as T:
            ctx.jobs_reset()
            ctx.run("batched")
        step_ms += T.ms
        a, b, _n = ctx.last_timing()
        t_prep += a
        t_fused += b
    del flush
    stats = [ctx.stats(k) for k in range(w.n_jobs)]
    inbox = sum(s["inbox"] for s in stats)
    units = w.units
    value = units * steps / (step_ms * 1e-3)
    # the shared histogram of one clean run, for a whole-workload comparison
    ctx.reset_histogram(-1)
    ctx.jobs_reset()
    ctx.run("batched")
    whole_c, whole_y = read_spectra(ctx, hids_all)
    plain = None
    nbins_total = ctx.total_bins()
    if not args.no_plain:
        # the per-track loop over every job; for the 256 equal 4e6-deposit tracks, over the
        # first CFG4_PLAIN_TRACKS of them (a track's loop iteration costs the same whatever the
        # number of tracks, and the whole loop would take as long as several batched steps)
        pj = jobs[:CFG4_PLAIN_TRACKS] if cfg == 4 else jobs
        if len(pj) < len(jobs):
            ctx.close()
            ctx = st.Context(dev.index, stream=stream.cuda_stream)
            hp = [ctx.histogram(*h) for h in w.hists]
            submit_jobs(ctx, w, pj, [hp[int(w.hist_of_job[j])] for j in pj], True,
                        (w.x, w.y, w.z, w.edep))
            ctx.run("plain")                  # untimed: sizes the context's arenas
        p_units = int((w.sizes[pj].astype(np.int64) * w.n_os[pj].astype(np.int64)).sum())
        torch.cuda.synchronize()
        ctx.jobs_reset()
        t0 = time.perf_counter()
        ctx.run("plain")
        torch.cuda.synchronize()
        pval = p_units / (time.perf_counter() - t0)
        plain = {"value": pval, "batched_over_plain": value / pval, "jobs": len(pj),
                 "timing": "host wall clock around the per-track loop (one sync per track)"}
    ctx.close()
    e2e = None
    if cfg in (0, 1) and not args.no_e2e:
        hx = [t.to("cpu").pin_memory() for t in (w.x, w.y, w.z, w.edep)]
        ctx2 = st.Context(dev.index, stream=stream.cuda_stream)
        h2 = [ctx2.histogram(*h) for h in w.hists]
        submit_jobs(ctx2, w, jobs, [h2[int(w.hist_of_job[j])] for j in jobs], False, hx)
        nb = ctx2.total_bins()
        oc_ = torch.empty(nb, dtype=torch.int64, pin_memory=True)
        oy_ = torch.empty(nb, dtype=torch.float64, pin_memory=True)
        for _ in range(3):
            ctx2.jobs_reset()
            ctx2.run("batched")
            ctx2.read_all_into(oc_.data_ptr(), oy_.data_ptr(), nb)
        e_steps = max(2, min(steps, 5))
        with Timer(stream, 1, dev) as E:
            for _ in range(e_steps):
                ctx2.jobs_reset()
                ctx2.run("batched")
                ctx2.read_all_into(oc_.data_ptr(), oy_.data_ptr(), nb)
        e2e = {"value": units * e_steps / (E.ms * 1e-3), "unit": UNIT,
               "h2d_bytes_per_step": int(w.deposits * 32), "d2h_bytes_per_step": int(nb * 16),
               "steps": e_steps}
        ctx2.close()
        del hx
    # CPU baseline and parity: the sampled jobs again on the GPU, each into its own histogram,
    # with the oversamples the oracle ran (config 4: the first CFG4_OS_SAMPLE of each job)
    os_cap = CFG4_OS_SAMPLE if cfg == 4 else None
    wc = w.to("cpu")
    cpu, sample = cpu_baseline(wc, args.cpu_seconds, os.cpu_count() or 1, os_cap=os_cap)
    sj, so = sample[0], sample[1]
    pctx = st.Context(dev.index, stream=stream.cuda_stream)
    ph = [pctx.histogram(*w.hists[int(w.hist_of_job[j])]) for j in sj]
    submit_jobs(pctx, w, sj, ph, True, (w.x, w.y, w.z, w.edep), os_run=so)
    pctx.run("batched")
    gc, gy = read_spectra(pctx, ph)
    gs = job_stats(pctx, len(sj), w, sj)
    pctx.close()
    parity = parity_block(gc, gy, gs, sample,
                          "the sampled jobs rerun as one batch with a histogram each"
                          + (f" ({CFG4_OS_SAMPLE} oversamples per job)" if os_cap else ""))
    # when the sample is the whole workload, the timed batch's shared spectrum is checked too
    if len(sj) == w.n_jobs and not os_cap:
        tot_c = [np.zeros_like(c) for c in whole_c]
        tot_y = [np.zeros_like(y) for y in whole_y]
        for k, j in enumerate(sj):
            h = int(w.hist_of_job[j])
            tot_c[h] += sample[2][k]
            tot_y[h] += sample[3][k]
        parity["whole_workload_counts_equal"] = all(
            bool(np.array_equal(a, b)) for a, b in zip(whole_c, tot_c))
        parity["whole_workload_max_rel_yfy"] = max(
            float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300))) for a, b in
            zip(whole_y, tot_y))
    fused_ms = t_fused / steps
    peak, peak_src = hbm_peak()
    fused_bytes = BYTES_PREP * w.deposits + 16 * nbins_total
    out = {"config": config_dict(cfg, w, 1, 1.0), "value": value, "unit": UNIT,
           "steps": steps, "warmup": warm, "ms_per_step": step_ms / steps,
           "kernel_ms": {"prepare": t_prep / steps, "fused": fused_ms},
           "first_run_s": first_s, "generation_s": t_gen,
           "roofline": {"bound": "hbm", "achieved": fused_bytes / (fused_ms * 1e-3) / 1e9,
                        "peak": peak, "unit": "GB/s", "peak_source": peak_src,
                        "frac": fused_bytes / (fused_ms * 1e-3) / 1e9 / peak},
           "inbox_units_per_step": inbox,
           "plain": plain, "e2e": e2e, "cpu_baseline": cpu, "parity": parity}
    if e2e is None and cfg == 4:
        out["e2e_note"] = ("not measured: the 32.8 GB of tracks would have to be pinned in host "
                           "memory")
    del w, wc
    torch.cuda.empty_cache()
    return out


def ours(args, rank, world):
    import torch
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    # a dedicated stream: the context enqueues every copy and kernel on it, and the CUDA events
    # are recorded on it
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    line, w = headline(args, rank, world, dev, stream)
    del w
    torch.cuda.empty_cache()
    if rank != 0:
        return
    if not args.no_serve and args.config == 2 and world == 1:
        line["serving"] = serve_leg(dev, line["value"], args.serve_jobs)
        torch.cuda.empty_cache()
    if world == 1:
        for cfg in [int(c) for c in args.also.split(",") if c.strip()]:
            if cfg != args.config:
                line["per_config"][str(cfg)] = other_config(cfg, args, dev, stream)
    print(json.dumps(line), flush=True)


def spawn_ranks(args) -> int:
    """--gpus N without a launcher: runs this script under torch.distributed.run with N ranks."""
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={args.gpus}", "--master-addr", "127.0.0.1",
           "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "0"))
    if world == 0:
        if args.gpus > 1:
            sys.exit(spawn_ranks(args))
        world = 1
    rank = int(os.environ.get("RANK", "0"))
    if world > 1:
        import torch
        import datetime
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        if args.impl == "reference":
            reference_arm(args, rank, world)
        else:
            ours(args, rank, world)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
