"""Multi-GPU sharding of superimposition jobs (one process per GPU).

Tracks are independent (reference SuperTrackManager.cu:53-89); the only step that crosses units
is summing the spectra (Histogram.cu:188-199, TH1::Add). So jobs are partitioned across ranks
by longest-processing-time first on their cost (deposits x oversamples), every rank runs its
share with one batched launch, and the spectra are reduced once at the end: int64 counts exactly
(integer sums), float64 y*f(y) by value.
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
