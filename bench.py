"""Benchmark of the VoxelConstrainedSphere superimposition path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config 2|0|1|4] [--scale S]

One step = one pass of the hot path over the whole synthetic workload: every track's prepare
pass plus the fused superimposition of all its oversamples into its histogram. The default
workload is the batched uneven configuration (4,096 tracks, lognormal sizes with median 2e4
deposits, d in {2,10,100,1000} nm, oversamples in {1,10,100}, one 200-bin log histogram per
track), the one the batched-versus-plain metric is quoted on.

Metric: deposit*oversamples per second (higher is better).
  value : inputs resident in HBM, one batched run per step, device time (CUDA events on the
          stream the kernels run on), max over ranks;
  e2e   : the same through the public API with host (pinned) tracks: every step copies the
          tracks host->device (in groups on a second stream, overlapped with the kernels of
          earlier groups) and reads every histogram back device->host.
Multi-GPU (torchrun): every rank runs its own full workload (seed offset by rank), no
collective on the data path (weak scaling); value = all ranks' units / max rank time.

--impl reference: the reference cannot be built here (CERN ROOT is absent and its histogram
stage needs device-side cudaDeviceSynchronize, which CUDA 12 rejects), so this arm times the
CPU restatement of the reference algorithm (oracle/) on all host threads, each step a bounded
sample of the same workload. Rank 0 alone runs it.
"""
from __future__ import annotations

import argparse
import json
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
# Algorithmic HBM bytes: each track's float64 x, y, z, edep read once (32 B per deposit), the
# prepared record written once and read once per launch (36 B per deposit each way), and the
# histograms written once (16 B per bin).
BYTES_TRACK = 32
BYTES_PREP = 36


def profile_figures(config: int, units: float):
    """Figures of the committed k_fused ncu capture, for the bench line: DRAM traffic scaled to
    `units` deposit*oversamples (bytes per unit x units), and the shared-memory roofline term
    (wavefronts as a fraction of their peak). (None, None) when no capture of this workload
    exists."""
    prof = os.path.join(ROOT, "profiles", "fused_traffic.json")
    try:
        p = json.load(open(prof))
    except (OSError, ValueError):
        return None, None
    if p.get("config") != config:
        return None, None
    traffic = float(p["bytes_per_unit"]) * units if "bytes_per_unit" in p else None
    smem = None
    if "smem_wavefront_frac" in p:
        smem = {"bound": "smem", "frac": float(p["smem_wavefront_frac"]),
                "unit": "shared-memory wavefronts / peak",
                "bank_conflict_share": p.get("smem_bank_conflict_share"),
                "source": p.get("source"),
                "note": "measured by ncu on a 256-track batch of the same workload (not live)"}
    return traffic, smem


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--config", type=int, default=2, choices=[0, 1, 2, 4])
    p.add_argument("--scale", type=float, default=1.0,
                   help="track-count scale of the workload (1.0 = as specified)")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-plain", action="store_true")
    p.add_argument("--no-fp32", action="store_true",
                   help="skip the FP32 geometry variant's leg (reported beside the FP64 value)")
    p.add_argument("--cpu-seconds", type=float, default=15.0)
    p.add_argument("--no-tune", action="store_true",
                   help="skip the autotuner (default planning parameters)")
    p.add_argument("--tune-trials", type=int, default=24)
    p.add_argument("--no-serve", action="store_true",
                   help="skip the served-stream leg (10,000 arriving jobs at four loads)")
    p.add_argument("--serve-jobs", type=int, default=10000)
    return p.parse_args()


def make_workload(cfg: int, device, seed_offset: int, scale: float):
    import supertrack_b200.workloads as W
    if cfg == 0:
        w = W.config0(device=device, n_tracks=max(1, int(64 * scale)), seed=1 + seed_offset)
        desc = "config0: 64 proton-like tracks x 4000 deposits, HL 2500 nm, d 10 nm, 10 OS, lin 3000 bins"
    elif cfg == 1:
        w = W.config1(device=device, n_tracks=max(1, int(16 * scale)), seed=2 + seed_offset)
        desc = "config1: 16 ion tracks x 1e6 deposits, HL 5000 nm, d 2 nm, 100 OS, log 500 bins"
    elif cfg == 4:
        w = W.config4(device=device, n_tracks=max(1, int(256 * scale)), seed=5 + seed_offset)
        desc = "config4: 256 ion tracks x 4e6 deposits, HL 5000 nm, d 10 nm, 1000 OS, lin 3000 bins"
    else:
        w = W.config2(device=device, n_tracks=max(1, int(4096 * scale)), seed=3 + seed_offset)
        desc = ("config2: 4096 uneven tracks (lognormal sizes median 2e4, sigma 1.5, clipped "
                "[500, 2e6]), half proton-like, half ion-like, d in {2,10,100,1000} nm, "
                "OS in {1,10,100}, HL 2500 nm, one log 200-bin histogram per track")
    return w, desc


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


def cpu_sample_jobs(w, target_units):
    """A deterministic sample of jobs (every k-th by index) with about target_units units."""
    units = w.sizes.astype(np.int64) * w.n_os.astype(np.int64)
    order = np.argsort(np.random.default_rng(0).random(w.n_jobs))
    chosen, tot = [], 0
    for j in order:
        if tot >= target_units:
            break
        chosen.append(int(j))
        tot += int(units[j])
    return sorted(chosen), tot


def run_cpu_baseline(w, seconds: float, threads: int):
    """Times the CPU restatement (oracle) on a bounded sample of w; returns dict."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    x, y, z, e = [a.cpu().numpy() for a in (w.x, w.y, w.z, w.edep)]
    edges = [po.edges(*h) for h in w.hists]

    def run(jobs):
        sel = np.array(jobs, dtype=np.int64)
        t0 = time.perf_counter()
        po.run_batch(x, y, z, e, w.offsets[sel], w.sizes[sel], w.half_length[sel],
                     w.diameter[sel], np.full(len(sel), {"plus": 0, "minus": 1, "none": 2}[w.zshift]),
                     np.full(len(sel), int(w.shift_track)), w.n_os[sel], w.seed[sel],
                     w.track_id[sel], np.arange(len(sel)) if len(w.hists) > 1 else np.zeros(len(sel)),
                     [edges[w.hist_of_job[j]] for j in sel] if len(w.hists) > 1 else edges[:1],
                     threads=threads)
        return time.perf_counter() - t0

    jobs, units = cpu_sample_jobs(w, 2e6 * threads)
    dt = run(jobs)
    rate = units / max(dt, 1e-9)
    jobs, units = cpu_sample_jobs(w, rate * seconds)
    dt = run(jobs)
    return {"value": units / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{len(jobs)} of {w.n_jobs} jobs ({units:.3e} deposit*oversamples, "
                      f"{dt:.1f} s on {threads} threads)"}


def reference_arm(args, rank):
    import torch
    if rank != 0:
        return
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    w, desc = make_workload(args.config, dev, 0, args.scale)
    w = w.to("cpu")
    threads = os.cpu_count() or 1
    per_step = max(2.0, min(20.0, 150.0 / max(1, args.steps + args.warmup)))
    res = []
    for k in range(args.warmup + args.steps):
        r = run_cpu_baseline(w, per_step, threads)
        if k >= args.warmup:
            res.append(r)
    value = statistics.median([r["value"] for r in res])
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": desc, "jobs": w.n_jobs, "deposits": w.deposits,
                       "units_per_step": w.units},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": res[-1]["sample"]},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "ms_per_step": None}
    print(json.dumps(line), flush=True)


def submit_all(ctx, w, hist_ids, on_device: bool, tensors):
    """Submits every job of w; tensors = (x, y, z, edep) flat (device or pinned host)."""
    import supertrack_b200 as st
    from supertrack_b200 import _capi
    import ctypes as C
    n = w.n_jobs
    tv = (_capi.st_track_view * n)()
    jd = (_capi.st_job_desc * n)()
    base = [t.data_ptr() for t in tensors]
    for j in range(n):
        o = int(w.offsets[j]) * 8
        tv[j].x, tv[j].y, tv[j].z, tv[j].edep = [b + o for b in base]
        tv[j].n = int(w.sizes[j])
        tv[j].on_device = int(on_device)
        jd[j].half_length = float(w.half_length[j])
        jd[j].sphere_diameter = float(w.diameter[j])
        jd[j].zshift = st.ZSHIFT[w.zshift]
        jd[j].shift_track = int(w.shift_track)
        jd[j].n_oversamples = int(w.n_os[j])
        jd[j].hist_id = hist_ids[int(w.hist_of_job[j])]
        jd[j].seed = int(w.seed[j])
        jd[j].track_id = int(w.track_id[j])
    st.check(_capi.lib().st_job_submit_many(ctx.handle, n, tv, jd, None), "submit", ctx.handle)


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
    out["p99_ms_at_80pct"] = next(l["p99_ms"] for l in out["loads"] if l["load"] == 0.8)
    return out


def ours(args, rank, world):
    import torch
    import supertrack_b200 as st
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    # a dedicated stream: the context enqueues every copy and kernel on it, and the CUDA events
    # below are recorded on it
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    w, desc = make_workload(args.config, dev, 1000 * rank, args.scale)
    torch.cuda.synchronize()
    torch.cuda.empty_cache()   # the generator's temporaries: the context sizes from free memory
    ctx = st.Context(dev.index, stream=stream.cuda_stream)
    hist_ids = [ctx.histogram(*h) for h in w.hists]
    submit_all(ctx, w, hist_ids, True, (w.x, w.y, w.z, w.edep))
    ctx.enable_timing(True)

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    # ---- autotuned planning parameters (untimed; histograms and job states are restored),
    # then warm-up: the first rerun captures the CUDA graph the timed steps replay
    ctx.run("batched")
    tune = None if args.no_tune else ctx.autotune(args.tune_trials)
    for _ in range(args.warmup):
        ctx.jobs_reset()
        ctx.run("batched")
    stats = [ctx.stats(j) for j in range(w.n_jobs)]
    inbox = sum(s["inbox"] for s in stats)
    hits = sum(s["hits"] for s in stats)

    # ---- timed region: inputs resident in HBM (9+ GB of tracks and prepared records, well
    # above the 126 MB L2, so no flush is needed between steps)
    sampler = ClockSampler(dev.index)
    sampler.start()
    barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    g_before = ctx.get_param("graph_launches")
    ev0.record(stream)
    t_prep = t_fused = 0.0
    launches = 0
    for _ in range(args.steps):
        ctx.jobs_reset()
        ctx.run("batched")
        a, b, n = ctx.last_timing()
        t_prep += a
        t_fused += b
        launches += n
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clocks = sampler.stop()
    graph_steps = ctx.get_param("graph_launches") - g_before
    ms = ev0.elapsed_time(ev1)
    ms_t = torch.tensor([ms], device=dev)
    if world > 1:
        torch.distributed.all_reduce(ms_t, op=torch.distributed.ReduceOp.MAX)
    ms_max = float(ms_t.item())
    units = w.units
    value = units * world * args.steps / (ms_max * 1e-3)

    # ---- e2e through the public API with pinned host tracks and histogram read-back
    e2e = None
    if not args.no_e2e:
        hx = [t.to("cpu").pin_memory() for t in (w.x, w.y, w.z, w.edep)]
        ctx2 = st.Context(dev.index, stream=stream.cuda_stream)
        hid2 = [ctx2.histogram(*h) for h in w.hists]
        submit_all(ctx2, w, hid2, False, hx)
        nb = ctx2.total_bins()
        out_c = torch.empty(nb, dtype=torch.int64, pin_memory=True)
        out_y = torch.empty(nb, dtype=torch.float64, pin_memory=True)
        for _ in range(max(1, args.warmup)):
            ctx2.jobs_reset()
            ctx2.run("batched")
            ctx2.read_all_into(out_c.data_ptr(), out_y.data_ptr(), nb)
        e2e_steps = max(1, min(args.steps, 5))
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(e2e_steps):
            ctx2.jobs_reset()
            ctx2.run("batched")
            ctx2.read_all_into(out_c.data_ptr(), out_y.data_ptr(), nb)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        ems = torch.tensor([e0.elapsed_time(e1)], device=dev)
        if world > 1:
            torch.distributed.all_reduce(ems, op=torch.distributed.ReduceOp.MAX)
        e2e = {"value": units * world * e2e_steps / (float(ems.item()) * 1e-3), "unit": UNIT,
               "h2d_bytes_per_step": int(w.deposits * 32), "d2h_bytes_per_step": int(nb * 16),
               "steps": e2e_steps}
        ctx2.close()

    # ---- plain per-track form on the same workload (one pass), for the batched/plain ratio
    plain = None
    if not args.no_plain:
        barrier()
        torch.cuda.synchronize()
        ctx.jobs_reset()
        t0 = time.perf_counter()
        ctx.run("plain")
        torch.cuda.synchronize()
        pdt = time.perf_counter() - t0
        pt = torch.tensor([pdt], device=dev)
        if world > 1:
            torch.distributed.all_reduce(pt, op=torch.distributed.ReduceOp.MAX)
        pval = units * world / float(pt.item())
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
            st_ = [ctx.stats(j) for j in range(w.n_jobs)]
            spectra[prec] = (c_.numpy().copy(), sum(s["hits"] for s in st_),
                             sum(s["spheres"] for s in st_), sum(s["binned"] for s in st_))
        for _ in range(args.warmup):
            ctx.jobs_reset()
            ctx.run("batched")
        barrier()
        torch.cuda.synchronize()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        f_prep = f_fused = 0.0
        for _ in range(args.steps):
            ctx.jobs_reset()
            ctx.run("batched")
            a, b, _n = ctx.last_timing()
            f_prep += a
            f_fused += b
        f1.record(stream)
        torch.cuda.synchronize()
        barrier()
        fms = torch.tensor([f0.elapsed_time(f1)], device=dev)
        if world > 1:
            torch.distributed.all_reduce(fms, op=torch.distributed.ReduceOp.MAX)
        ctx.set_param("precision", 64)
        c64, h64, s64, b64 = spectra[64]
        c32, h32, s32, b32 = spectra[32]
        fp32 = {"value": units * world * args.steps / (float(fms.item()) * 1e-3), "unit": UNIT,
                "ms_per_step": float(fms.item()) / args.steps,
                "kernel_ms": {"prepare": f_prep / args.steps, "fused": f_fused / args.steps},
                "fp64_run": {"hits": h64, "spheres": s64, "binned": b64},
                "diff_vs_fp64": {"hits": h32 - h64, "spheres": s32 - s64, "binned": b32 - b64,
                                 "counts_l1": int(np.abs(c32 - c64).sum())},
                "hits_rel_diff": (h32 - h64) / max(h64, 1),
                "spheres_rel_diff": (s32 - s64) / max(s64, 1),
                "counts_l1_rel": float(np.abs(c32 - c64).sum()) / max(float(c64.sum()), 1.0),
                "note": "FP32 geometry variant (x/y geometry in float; z, keys and energies as "
                        "FP64): reported beside the FP64 value, not bound to reference parity"}

    if rank != 0:
        ctx.close()
        return

    fp64_peak = ctx.fp64_peak()
    fused_ms = t_fused / args.steps
    prep_ms = t_prep / args.steps
    hbm_peak = None
    try:
        hbm_peak = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]
        peak_src = "MEASURED_PEAKS.json"
    except Exception:
        hbm_peak, peak_src = 6650.0, "fallback"
    nbins_total = ctx.total_bins()
    fused_bytes = BYTES_PREP * w.deposits + 16 * nbins_total
    fp64_ops = FP64_OPS_ALL * units + FP64_OPS_INBOX * inbox
    traffic, roofline_smem = profile_figures(args.config, units)
    cpu = run_cpu_baseline(w, args.cpu_seconds, os.cpu_count() or 1)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": desc, "jobs": w.n_jobs, "deposits": w.deposits,
                   "units_per_step": units, "inbox_units_per_step": inbox,
                   "hits_per_step": hits, "mode": "batched persistent launch",
                   "l2": "inputs larger than L2 (tracks + prepared records > 126 MB), no flush",
                   "parallelism": f"{world} independent replica(s), one per GPU"},
        "gpu_launches": launches,
        "graph_steps": graph_steps,
        "autotune": tune,
        "kernel_ms": {"prepare": prep_ms, "fused": fused_ms},
        "roofline": {"bound": "hbm", "achieved": fused_bytes / (fused_ms * 1e-3) / 1e9,
                     "peak": hbm_peak, "unit": "GB/s",
                     "frac": fused_bytes / (fused_ms * 1e-3) / 1e9 / hbm_peak,
                     "traffic": traffic, "peak_source": peak_src,
                     "kernel": "k_fused (dominant)", "bytes_per_launch": fused_bytes},
        "roofline_fp64": {"bound": "fp64", "achieved": fp64_ops / (fused_ms * 1e-3) / 1e12,
                          "peak": fp64_peak / 1e12, "unit": "TFLOP/s (fp64 add/mul/div)",
                          "frac": fp64_ops / (fused_ms * 1e-3) / fp64_peak,
                          "ops_per_launch": fp64_ops,
                          "peak_source": "measured live (dependent add+mul chains)"},
        "roofline_smem": roofline_smem,
        "clocks": clocks,
        "e2e": e2e,
        "plain": plain,
        "fp32": fp32,
        "cpu_baseline": cpu,
        "serving": None,
    }
    ctx.close()
    if not args.no_serve and args.config == 2 and world == 1:
        del w
        torch.cuda.empty_cache()
        line["serving"] = serve_leg(dev, value, args.serve_jobs)
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1:
        import torch
        import datetime
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        if args.impl == "reference":
            reference_arm(args, rank)
        else:
            ours(args, rank, world)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
