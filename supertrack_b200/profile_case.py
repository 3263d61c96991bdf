"""Small profiling case: the batched path on a scaled config-2 workload (default 256 tracks).

    python -m supertrack_b200.profile_case [n_tracks] [--class ion:2] [--max-size N] [--runs R]

Runs the batch R times (default 2) on cuda:0, so that a profiler can skip the first fused
launch, and prints the prepare and fused times of the fastest run (CUDA events around the
launches). ``--class`` keeps only the tracks of one generator and sphere diameter (``ion:2`` =
ion-like tracks with d = 2 nm, ``proton:10`` ...), or of one generator (``proton``);
``--max-size`` caps the track sizes. Used to produce the fused-kernel captures summarised under
profiles/.
"""
import argparse
import copy

import numpy as np
import torch

import supertrack_b200 as st
import supertrack_b200.workloads as W


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("n_tracks", nargs="?", type=int, default=256)
    ap.add_argument("--class", dest="cls", default="")
    ap.add_argument("--max-size", type=int, default=2_000_000)
    ap.add_argument("--runs", type=int, default=2)
    args = ap.parse_args()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    w = W.config2(device=dev, n_tracks=args.n_tracks, max_size=args.max_size)
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    jobs = np.arange(w.n_jobs)
    if args.cls:
        kind, _, dd = args.cls.partition(":")
        _, is_proton, _, _ = W.config2_sizes(args.n_tracks, 3, 1.0, args.max_size)
        keep = is_proton == (kind == "proton")
        if dd:
            keep &= w.diameter == float(dd)
        jobs = np.nonzero(keep)[0]
    ctx = st.Context(0, stream=stream.cuda_stream)
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
    print("jobs", len(jobs), "units", units, "deposits", int(w.sizes[jobs].sum()),
          f"prepare_ms {best[0]:.2f} fused_ms {best[1]:.2f}")
    ctx.close()


if __name__ == "__main__":
    main()
