"""Small profiling case: the batched path on a scaled workload (default: 256 tracks of the uneven
4,096-track workload).

    python -m supertrack_b200.profile_case [n_tracks] [--config 2|1|4] [--os N] [--grid G]
                                           [--class ion:2] [--max-size N] [--runs R]
                                           [--param NAME=VALUE ...]

Runs the batch R times (default 2) on cuda:0, so that a profiler can skip the first fused
launch, and prints the prepare and fused times of the fastest run (CUDA events around the
launches). ``--config`` picks the workload: 2 the uneven batch, 1 the dense 2 nm ion tracks,
4 the 4e6-deposit 10 nm tracks; ``--os`` overrides the oversample count of configs 1 and 4.
``--class`` keeps only the config-2 tracks of one generator and sphere diameter (``ion:2`` =
ion-like tracks with d = 2 nm, ``proton:10`` ...), or of one generator (``proton``);
``--max-size`` caps the config-2 track sizes; ``--grid`` sets the fused kernel's CTA count
(every CTA holds a spill table sized for the largest track: a capture of 4e6-deposit tracks on
a few CTAs stays at a few GB of device memory); ``--param`` sets context parameters
(st_ctx_set_param). Used to produce the fused-kernel captures
summarised under profiles/.
"""
import argparse

import numpy as np
import torch

import supertrack_b200 as st
import supertrack_b200.workloads as W


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("n_tracks", nargs="?", type=int, default=256)
    ap.add_argument("--config", type=int, default=2, choices=[1, 2, 4])
    ap.add_argument("--os", type=int, default=0)
    ap.add_argument("--class", dest="cls", default="")
    ap.add_argument("--max-size", type=int, default=2_000_000)
    ap.add_argument("--runs", type=int, default=2)
    ap.add_argument("--grid", type=int, default=0)
    ap.add_argument("--param", action="append", default=[])
    args = ap.parse_args()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    if args.config == 2:
        w = W.config2(device=dev, n_tracks=args.n_tracks, max_size=args.max_size)
    else:
        gen = W.config1 if args.config == 1 else W.config4
        kw = {"n_os": args.os} if args.os > 0 else {}
        w = gen(device=dev, n_tracks=args.n_tracks, **kw)
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    jobs = np.arange(w.n_jobs)
    if args.cls and args.config == 2:
        kind, _, dd = args.cls.partition(":")
        _, is_proton, _, _ = W.config2_sizes(args.n_tracks, 3, 1.0, args.max_size)
        keep = is_proton == (kind == "proton")
        if dd:
            keep &= w.diameter == float(dd)
        jobs = np.nonzero(keep)[0]
    ctx = st.Context(0, stream=stream.cuda_stream)
    if args.grid > 0:
        ctx.set_tuning(grid=args.grid)
    for kv in args.param:
        name, _, value = kv.partition("=")
        ctx.set_param(name, int(value))
    hist = [ctx.histogram(*h) for h in w.hists]
    units = 0
    for j in jobs:
        o, n = int(w.offsets[j]), int(w.sizes[j])
        ptrs = [t.data_ptr() + 8 * o for t in (w.x, w.y, w.z, w.edep)]
        ctx.submit(*ptrs, half_length=float(w.half_length[j]), sphere_diameter=float(w.diameter[j]),
                   n_oversamples=int(w.n_os[j]), hist=hist[int(w.hist_of_job[j])],
                   seed=int(w.seed[j]), track_id=int(w.track_id[j]), zshift=w.zshift,
                   on_device=True, n=n)
        units += n * int(w.n_os[j])
    best = None
    for _ in range(max(1, args.runs)):
        ctx.jobs_reset()
        ctx.run("batched")
        prep_ms, fused_ms, _ = ctx.last_timing()
        if best is None or fused_ms < best[1]:
            best = (prep_ms, fused_ms)
    stats = [ctx.stats(k) for k in range(len(jobs))]
    print("jobs", len(jobs), "units", units, "deposits", int(w.sizes[jobs].sum()),
          "hits", sum(s["hits"] for s in stats), "spheres", sum(s["spheres"] for s in stats),
          f"prepare_ms {best[0]:.2f} fused_ms {best[1]:.2f}")
    ctx.close()


if __name__ == "__main__":
    main()
