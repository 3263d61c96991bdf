"""Multi-GPU sharding of superimposition jobs (one process per GPU).

Tracks are independent (reference SuperTrackManager.cu:53-89); the only step that crosses units
is summing the spectra (Histogram.cu:188-199, TH1::Add). So jobs are partitioned across ranks
by longest-processing-time first on their cost (deposits x oversamples), every rank runs its
share with one batched launch, and the spectra are reduced once at the end: int64 counts exactly
(integer sums), float64 y*f(y) by value. The order in which the all-reduce adds the ranks'
y*f(y) is the collective's own and not fixed, so reduced y*f(y) values agree with a one-process
run within rounding (1e-12 relative), while counts are identical.

run_sharded is the whole multi-rank path with the per-rank runner as an argument: the GPU
benchmark passes a runner that submits the rank's jobs to a context, the multi-rank CPU tests
pass one that runs them through the CPU oracle, and both share the assignment and the reduction.
"""
from __future__ import annotations

import heapq
from typing import List, Sequence

import numpy as np


def lpt_assign(costs: Sequence[float], world: int) -> np.ndarray:
    """Rank of every job: jobs in decreasing cost go to the currently least-loaded rank
    (ties to the lower rank), a deterministic function of (costs, world)."""
    costs = np.asarray(costs, dtype=np.float64)
    order = np.lexsort((np.arange(len(costs)), -costs))
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    owner = np.empty(len(costs), dtype=np.int64)
    for j in order:
        load, r = heapq.heappop(heap)
        owner[j] = r
        heapq.heappush(heap, (load + costs[j], r))
    return owner


def shard(costs: Sequence[float], rank: int, world: int) -> List[int]:
    """Indices of the jobs this rank runs, in their original order."""
    return [int(j) for j in np.nonzero(lpt_assign(costs, world) == rank)[0]]


def reduce_spectra_device(counts, yfy, group=None) -> None:
    """In-place all-reduce (sum) of spectra already held in torch tensors on this rank's
    device (NCCL) or in host memory (gloo)."""
    import torch.distributed as dist
    dist.all_reduce(counts, group=group)
    dist.all_reduce(yfy, group=group)


def run_sharded(costs: Sequence[float], runner, n_bins: int, rank: int, world: int, group=None):
    """The multi-rank path: this rank's LPT share of the jobs (costs[j] = deposits x
    oversamples of job j) is run by runner(jobs) -> (counts, yfy), arrays of the workload's
    whole spectrum layout (n_bins bins, zero outside the rank's jobs); the spectra are summed
    over the ranks. Every rank returns the reduced (counts, yfy) and its job list."""
    jobs = shard(costs, rank, world)
    counts, yfy = runner(jobs)
    counts = np.asarray(counts, dtype=np.int64)
    yfy = np.asarray(yfy, dtype=np.float64)
    if counts.shape != (n_bins,) or yfy.shape != (n_bins,):
        raise ValueError("runner returned spectra of the wrong size")
    if world > 1:
        counts, yfy = reduce_spectra(counts, yfy, group)
    return counts, yfy, jobs


def reduce_spectra(counts: np.ndarray, yfy: np.ndarray, group=None):
    """All-reduce of one rank's spectra (int64 counts, float64 y*f(y)); returns the sums.

    Works with any torch.distributed backend (nccl with CUDA tensors, gloo with CPU tensors).
    """
    import torch
    import torch.distributed as dist
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else "cpu"
    c = torch.as_tensor(np.ascontiguousarray(counts, dtype=np.int64), device=dev)
    y = torch.as_tensor(np.ascontiguousarray(yfy, dtype=np.float64), device=dev)
    dist.all_reduce(c, group=group)
    dist.all_reduce(y, group=group)
    return c.cpu().numpy(), y.cpu().numpy()
