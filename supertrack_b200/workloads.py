"""Seeded synthetic track workloads of the shapes the benchmark configurations name.

The reference measures on track libraries from its sister project (MicroTrackGenerator) that are
not available here; these generators stand in with the stated shapes, sizes and value
distributions. Tracks are centred on the voxel centre, so jobs built from them use the
z-origin shift "none".

Generators (all lengths in nm, energies in eV, float64):
  proton : a straight primary line through the voxel centre along a uniform random direction,
           exponential spacing (mean 1.2 nm); 5% of the points are delta-ray random walks of 20
           isotropic 2 nm steps that branch from random primary points; edep lognormal
           (median 15 eV, sigma 0.8) clipped to [10, 1000].
  ion    : 70% of the points in a Gaussian core (sigma `core_sigma`) around a random straight
           line through the centre, 30% in a penumbra with areal density ~ 1/r^2 for r in
           [5, `pen_max`] (log-uniform radius, uniform angle); positions along the line uniform
           over [-HL, HL] and sorted; edep lognormal (median 20 eV, sigma 0.9) clipped to
           [10, 5000].

Everything is vectorised with torch so that the large configurations can be generated on the
GPU in seconds; the same seed on the same device type gives the same tracks. The single-geometry
configurations (1 and 4) seed every track on its own (track t of seed s uses the generator
seeded s * 1_000_003 + t), so a subset of their tracks is generated exactly as in the full
workload, and the generator's temporaries stay at one track's size.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional, Tuple

import numpy as np
import torch


@dataclass
class Workload:
    name: str
    x: torch.Tensor
    y: torch.Tensor
    z: torch.Tensor
    edep: torch.Tensor
    offsets: np.ndarray          # int64 [n_jobs]
    sizes: np.ndarray            # int64 [n_jobs]
    half_length: np.ndarray      # float64 [n_jobs]
    diameter: np.ndarray         # float64 [n_jobs]
    n_os: np.ndarray             # uint32 [n_jobs]
    seed: np.ndarray             # uint64 [n_jobs]
    track_id: np.ndarray         # uint64 [n_jobs]
    hist_of_job: np.ndarray      # int32 [n_jobs]
    hists: List[Tuple[str, int, float, float]] = field(default_factory=list)
    zshift: str = "none"
    shift_track: bool = True
    generator: Optional[np.ndarray] = None   # int8 [n_jobs]: 0 proton-like, 1 ion-like

    @property
    def n_jobs(self) -> int:
        return len(self.sizes)

    @property
    def deposits(self) -> int:
        return int(self.sizes.sum())

    @property
    def units(self) -> int:
        """deposit*oversamples of one pass over the workload."""
        return int((self.sizes.astype(np.int64) * self.n_os.astype(np.int64)).sum())

    def to(self, device) -> "Workload":
        w = Workload(**{k: getattr(self, k) for k in self.__dataclass_fields__})
        for k in ("x", "y", "z", "edep"):
            setattr(w, k, getattr(self, k).to(device))
        return w

    def job_classes(self) -> np.ndarray:
        """Class of every job, (generator, sphere diameter, oversamples) as one integer: jobs of
        a class cost about the same per deposit*oversample."""
        gen = self.generator if self.generator is not None else np.zeros(self.n_jobs, np.int8)
        d_code = np.searchsorted(np.unique(self.diameter), self.diameter)
        os_code = np.searchsorted(np.unique(self.n_os), self.n_os)
        return (gen.astype(np.int64) * 64 + d_code) * 64 + os_code

    def job_arrays(self, j: int):
        o, n = int(self.offsets[j]), int(self.sizes[j])
        return (self.x[o:o + n], self.y[o:o + n], self.z[o:o + n], self.edep[o:o + n])


def _unit_vectors(g: torch.Generator, n: int, device) -> torch.Tensor:
    v = torch.randn(n, 3, generator=g, device=device, dtype=torch.float64)
    return v / v.norm(dim=1, keepdim=True).clamp_min(1e-300)


def _orthonormal(u: torch.Tensor) -> Tuple[torch.Tensor, torch.Tensor]:
    ref = torch.zeros_like(u)
    ref[:, 0] = 1.0
    swap = u[:, 0].abs() > 0.9
    ref[swap, 0] = 0.0
    ref[swap, 1] = 1.0
    a = torch.cross(u, ref, dim=1)
    a = a / a.norm(dim=1, keepdim=True)
    b = torch.cross(u, a, dim=1)
    return a, b


def _lognormal_clipped(g, n, median, sigma, lo, hi, device) -> torch.Tensor:
    e = torch.randn(n, generator=g, device=device, dtype=torch.float64)
    return torch.exp(math.log(median) + sigma * e).clamp_(lo, hi)


def _segment_starts(sizes: torch.Tensor) -> torch.Tensor:
    return torch.cumsum(sizes, 0) - sizes


def gen_proton(g, sizes: torch.Tensor, device) -> Tuple[torch.Tensor, ...]:
    """Proton-like tracks of the given sizes, concatenated."""
    T = len(sizes)
    total = int(sizes.sum())
    tid = torch.repeat_interleave(torch.arange(T, device=device), sizes)
    start = _segment_starts(sizes)
    local = torch.arange(total, device=device) - start[tid]
    n_delta = torch.round(0.05 * sizes.double()).long()
    n_prim = sizes - n_delta
    is_prim = local < n_prim[tid]
    u = _unit_vectors(g, T, device)
    # primary line: exponential spacing, centred on the track's middle primary point
    step = -1.2 * torch.log1p(-torch.rand(total, generator=g, device=device, dtype=torch.float64))
    step = torch.where(is_prim, step, torch.zeros_like(step))
    csum = torch.cumsum(step, 0)
    seg0 = csum[start] - step[start]
    t = csum - seg0[tid]
    mid_idx = start + torch.clamp(n_prim // 2, min=0)
    t = t - t[mid_idx.clamp(max=total - 1)][tid]
    pos = t[:, None] * u[tid]
    # delta rays: walks of 20 isotropic 2 nm steps from random primary points of the track
    dl = local - n_prim[tid]                       # index inside the delta part (>= 0)
    walk = torch.div(dl, 20, rounding_mode="floor")
    dsteps = 2.0 * _unit_vectors(g, total, device)
    dsteps[is_prim] = 0.0
    wid = torch.where(is_prim, torch.full_like(local, -1), walk)
    # per-deposit walk key (track, walk) to find walk starts
    key = tid * (1 << 20) + wid
    first_of_walk = torch.ones(total, dtype=torch.bool, device=device)
    first_of_walk[1:] = key[1:] != key[:-1]
    cs = torch.stack([torch.cumsum(dsteps[:, k].contiguous(), 0) for k in range(3)], 1)
    walk_begin_idx = torch.cummax(torch.where(first_of_walk, torch.arange(total, device=device),
                                              torch.zeros_like(local)), 0).values
    within = cs - cs[walk_begin_idx] + dsteps[walk_begin_idx]
    # origin: a random primary point of the same track
    r = torch.rand(total, generator=g, device=device, dtype=torch.float64)
    pick = start[tid] + (r * n_prim[tid].double()).long()
    pick = torch.minimum(pick, start[tid] + torch.clamp(n_prim[tid] - 1, min=0))
    origin = pos[pick[walk_begin_idx]]
    dpos = origin + within
    pos = torch.where(is_prim[:, None], pos, dpos)
    edep = _lognormal_clipped(g, total, 15.0, 0.8, 10.0, 1000.0, device)
    return pos[:, 0].contiguous(), pos[:, 1].contiguous(), pos[:, 2].contiguous(), edep


def gen_ion(g, sizes: torch.Tensor, half_length: float, core_sigma: float, pen_max: float,
            device) -> Tuple[torch.Tensor, ...]:
    """Dense ion tracks (Gaussian core + 1/r^2 penumbra) of the given sizes, concatenated."""
    T = len(sizes)
    total = int(sizes.sum())
    tid = torch.repeat_interleave(torch.arange(T, device=device), sizes)
    u = _unit_vectors(g, T, device)
    a, b = _orthonormal(u)
    t = (2 * torch.rand(total, generator=g, device=device, dtype=torch.float64) - 1) * half_length
    # sort along the line inside each track (track order)
    t, _ = torch.sort(t + tid.double() * (4 * half_length + 1))
    t = t - tid.double() * (4 * half_length + 1)
    core = torch.rand(total, generator=g, device=device, dtype=torch.float64) < 0.7
    gc = core_sigma * torch.randn(total, 2, generator=g, device=device, dtype=torch.float64)
    rr = 5.0 * torch.pow(pen_max / 5.0, torch.rand(total, generator=g, device=device,
                                                   dtype=torch.float64))
    ph = 2 * math.pi * torch.rand(total, generator=g, device=device, dtype=torch.float64)
    o1 = torch.where(core, gc[:, 0], rr * torch.cos(ph))
    o2 = torch.where(core, gc[:, 1], rr * torch.sin(ph))
    pos = t[:, None] * u[tid] + o1[:, None] * a[tid] + o2[:, None] * b[tid]
    edep = _lognormal_clipped(g, total, 20.0, 0.9, 10.0, 5000.0, device)
    return pos[:, 0].contiguous(), pos[:, 1].contiguous(), pos[:, 2].contiguous(), edep


def _per_track(device, n_tracks, n_dep, seed, gen_one) -> Tuple[torch.Tensor, ...]:
    """n_tracks tracks of n_dep deposits, track t generated by gen_one(generator, sizes) with a
    generator seeded seed * 1_000_003 + t, written into preallocated arrays."""
    total = n_tracks * n_dep
    out = [torch.empty(total, dtype=torch.float64, device=device) for _ in range(4)]
    sizes = torch.full((1,), n_dep, dtype=torch.long, device=device)
    for t in range(n_tracks):
        g = torch.Generator(device=device).manual_seed(seed * 1_000_003 + t)
        part = gen_one(g, sizes)
        for k in range(4):
            out[k][t * n_dep:(t + 1) * n_dep] = part[k]
        del part
    return tuple(out)


def _assemble(name, parts, sizes, hl, d, n_os, seed, hists, hist_of_job, generator=0) -> Workload:
    x = torch.cat([p[0] for p in parts])
    y = torch.cat([p[1] for p in parts])
    z = torch.cat([p[2] for p in parts])
    e = torch.cat([p[3] for p in parts])
    sizes = np.asarray(sizes, dtype=np.int64)
    offsets = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
    nj = len(sizes)
    return Workload(name=name, x=x, y=y, z=z, edep=e, offsets=offsets, sizes=sizes,
                    half_length=np.broadcast_to(np.asarray(hl, dtype=np.float64), (nj,)).copy(),
                    diameter=np.broadcast_to(np.asarray(d, dtype=np.float64), (nj,)).copy(),
                    n_os=np.broadcast_to(np.asarray(n_os, dtype=np.uint32), (nj,)).copy(),
                    seed=np.full(nj, seed, dtype=np.uint64),
                    track_id=np.arange(nj, dtype=np.uint64), hists=hists,
                    hist_of_job=np.asarray(hist_of_job, dtype=np.int32),
                    generator=np.full(nj, generator, dtype=np.int8))


def config0(device="cpu", n_tracks=64, n_dep=4000, n_os=10, seed=1) -> Workload:
    """64 proton-like tracks x 4000 deposits, HL 2500 nm, d 10 nm, 10 oversamples,
    lin 3000 bins over 0.01-300 keV/um."""
    g = torch.Generator(device=device).manual_seed(seed)
    sizes = torch.full((n_tracks,), n_dep, dtype=torch.long, device=device)
    part = gen_proton(g, sizes, device)
    return _assemble("config0-plain-small", [part], [n_dep] * n_tracks, 2500.0, 10.0, n_os,
                     seed, [("lin", 3000, 0.01, 300.0)], [0] * n_tracks)


def config1(device="cpu", n_tracks=16, n_dep=1_000_000, n_os=100, seed=2) -> Workload:
    """16 dense ion tracks x 1e6 deposits, HL 5000 nm, d 2 nm, 100 oversamples,
    log 500 bins over 0.1-1e4 keV/um."""
    part = _per_track(device, n_tracks, n_dep, seed,
                      lambda g, sz: gen_ion(g, sz, 5000.0, 5.0, 500.0, device))
    return _assemble("config1-dense-ion", [part], [n_dep] * n_tracks, 5000.0, 2.0, n_os, seed,
                     [("log", 500, 0.1, 1e4)], [0] * n_tracks, generator=1)


def config2_sizes(n_tracks=4096, seed=3, size_scale=1.0, max_size=2_000_000):
    rs = np.random.default_rng(seed)
    sizes = np.clip(np.round(np.exp(math.log(20000) + 1.5 * rs.standard_normal(n_tracks))),
                    500, 2_000_000)
    sizes = np.maximum(np.round(sizes * size_scale), 1).astype(np.int64)
    sizes = np.minimum(sizes, max_size)
    kind = rs.random(n_tracks) < 0.5                   # True: proton-like generator
    d = rs.choice(np.array([2.0, 10.0, 100.0, 1000.0]), n_tracks)
    os_ = rs.choice(np.array([1, 10, 100], dtype=np.uint32), n_tracks)
    return sizes, kind, d, os_


def config2(device="cpu", n_tracks=4096, seed=3, size_scale=1.0, os_scale=1.0,
            max_size=2_000_000) -> Workload:
    """4096 uneven tracks (lognormal sizes, median 2e4, sigma 1.5, clipped to [500, 2e6]),
    half proton-like and half ion-like, d in {2,10,100,1000} nm, oversamples in {1,10,100},
    HL 2500 nm, each job with its own log histogram of 200 bins over 0.01-1e4 keV/um."""
    sizes, kind, d, os_ = config2_sizes(n_tracks, seed, size_scale, max_size)
    os_ = np.maximum(np.round(os_ * os_scale), 1).astype(np.uint32)
    g = torch.Generator(device=device).manual_seed(seed)
    sz = torch.as_tensor(sizes, device=device)
    kt = torch.as_tensor(kind, device=device)
    xs = [None] * 4
    px = gen_proton(g, sz[kt], device) if bool(kt.any()) else None
    ix = gen_ion(g, sz[~kt], 2500.0, 5.0, 500.0, device) if bool((~kt).any()) else None
    # interleave back into track order
    total = int(sizes.sum())
    out = [torch.empty(total, dtype=torch.float64, device=device) for _ in range(4)]
    offs = torch.as_tensor(np.concatenate([[0], np.cumsum(sizes)[:-1]]), device=device)
    tid = torch.repeat_interleave(torch.arange(n_tracks, device=device), sz)
    local = torch.arange(total, device=device) - offs[tid]
    mask = kt[tid]
    for k in range(4):
        if px is not None:
            out[k][mask] = px[k]
        if ix is not None:
            out[k][~mask] = ix[k]
    del xs, local
    nj = n_tracks
    return Workload(name="config2-batched-uneven", x=out[0], y=out[1], z=out[2], edep=out[3],
                    offsets=np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64),
                    sizes=sizes, half_length=np.full(nj, 2500.0), diameter=d.astype(np.float64),
                    n_os=os_.astype(np.uint32), seed=np.full(nj, seed, dtype=np.uint64),
                    track_id=np.arange(nj, dtype=np.uint64),
                    hists=[("log", 200, 0.01, 1e4)] * nj,
                    hist_of_job=np.arange(nj, dtype=np.int32),
                    generator=np.where(kind, 0, 1).astype(np.int8))


def config4(device="cpu", n_tracks=256, n_dep=4_000_000, n_os=1000, seed=5) -> Workload:
    """256 ion tracks x 4e6 deposits (core sigma 3 nm, penumbra to 1000 nm), HL 5000 nm,
    d 10 nm, 1000 oversamples, lin 3000 bins over 0.01-300 keV/um with f(y) and y*f(y)."""
    part = _per_track(device, n_tracks, n_dep, seed,
                      lambda g, sz: gen_ion(g, sz, 5000.0, 3.0, 1000.0, device))
    return _assemble("config4-large", [part], [n_dep] * n_tracks, 5000.0, 10.0, n_os, seed,
                     [("lin", 3000, 0.01, 300.0)], [0] * n_tracks, generator=1)


def served_stream(n_jobs=10000, seed=4):
    """Job shapes of the served stream: config 2's distribution with seed 4."""
    return config2_sizes(n_jobs, seed)
