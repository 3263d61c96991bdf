// sm_100a kernels of the VoxelConstrainedSphere superimposition path.
//
//   prepare   : once per track (k_prep_count/scan/write/pad). z-origin shift, the deposits that
//               can be in the voxel for some shift, the z part of the lattice test (k_z and
//               (k_z*d - a_z)^2, which do not depend on the oversample), the lineal energy
//               contribution v = edep/((2/3)d), the job's fixed-point exponent range, and the
//               ordered compaction of the kept deposits into the pair-blocked prepared arena.
//               Follows VoxelConstrainedSphereMethod.cu:138-154 (z shift), :198 (|z| test),
//               :249-258 (z axis of the membership test), :302/:322 (lineal denominator).
//   k_fused   : persistent work-stealing kernel over (job, oversample block) items. Per
//               oversample: Philox shift, x/y shift + strict box test (:176-198), x/y lattice
//               indices and the inclusive sphere test (:249-271), the 64-bit key (:313-318),
//               exact reduce-by-key of the contributions (Histogram.cu:150-153) in registers,
//               shared memory and, when a job's spheres overflow shared memory, the CTA's spill
//               table in HBM, and the HistogramRange binning of each sphere's lineal energy
//               (Histogram.cu:158) plus its y*f(y) weight, accumulated over oversamples
//               (Histogram.cu:161-171).
#include <cuda_runtime.h>
#include <limits.h>
#include "st_device.cuh"

namespace st {

__device__ __forceinline__ uint32_t slot_hash(uint64_t key, uint32_t mask) {
  return (uint32_t)((key * 0x9E3779B97F4A7C15ull) >> 40) & mask;
}

// Slot of a sphere key in the shared-memory table: Fibonacci hashing proper, the top
// log2(mask + 1) bits of key * 2^64/phi (mask + 1 a power of two of at least 2). The middle bits
// that slot_hash takes map the regular lattice keys of a straight track into long runs of
// neighbouring slots, which at a quarter load already exceeded the 32-slot probe limit.
__device__ __forceinline__ uint32_t table_hash(uint64_t key, uint32_t mask) {
  return (uint32_t)((key * 0x9E3779B97F4A7C15ull) >> 32) >> __clz((int)mask);
}

// ---------------------------------------------------------------------------------------------
// Lattice index along one axis, k = llrint(a / d), bit-exact with the IEEE quotient. The fused
// kernel forms q = RN(a * RN(1/d)), whose distance to RN(a/d) is below |q| * 2^-51.2; it takes
// k = rint(q) (adding and subtracting 1.5 * 2^52 rounds to the nearest integer, ties to even)
// unless q lies within 2^-20 of a half-integer, where the correctly rounded division decides.
// ---------------------------------------------------------------------------------------------
constexpr double kMagic = 0x1.8p52;             // adding it rounds |q| < 2^51 to an integer
constexpr double kRiskBand = 0.5 - 0x1p-20;     // |q - rint(q)| at or above it: decide exactly
constexpr int kGeoBlock = 2;                     // deposits per straight-line geometry block

// The same, for one value: k = llrint(a / d) for |a / d| < 2^21.
__device__ __forceinline__ double lattice_index(double a, double d, double inv_d) {
  const double q = st_dmul(a, inv_d);
  const double k = st_dsub(st_dadd(q, kMagic), kMagic);
  return fabs(st_dsub(q, k)) >= kRiskBand ? rint(__ddiv_rn(a, d)) : k;
}

// ---------------------------------------------------------------------------------------------
// Prepare stage (once per track): four launches.
//   k_prep_count : per block of kPrepSlotsPerBlock source deposits, the number of deposits that
//                  can lie inside the voxel for some oversample (z after the z-origin shift
//                  strictly inside; |x|, |y| below xy_keep), plus the job's exponent range of
//                  the contributions v = edep/((2/3)d) over all its deposits;
//   k_prep_scan  : per job, exclusive scan of its block counts -> block offsets, kept total;
//   k_prep_write : ordered compaction of the kept deposits into the pair-blocked arena with
//                  the oversample-independent z part of the lattice test;
//   k_prep_pad   : padding of each job's last warp tile (NaN x so the box test rejects it).
// A dropped deposit can be inside the box for no shift, so dropping it changes no result.
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ int find_job(const int64_t* blk_prefix, int n_jobs, int64_t b) {
  int lo = 0, hi = n_jobs;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (blk_prefix[mid] <= b) lo = mid; else hi = mid;
  }
  return lo;
}

// The job of prepare block b: one load from the block table, which saves the short prepare
// blocks a dozen dependent loads of the binary search before their first track load.
__device__ __forceinline__ int prep_job(const PrepareParams& p, int64_t b) {
  return p.blk_job ? __ldg(&p.blk_job[b]) - p.job_base : find_job(p.blk_prefix, p.n_jobs, b);
}

// Slot of kept deposit k of a job in the prepared arena: warp tiles of kWarpTile deposits in
// which lane l owns deposits 4l..4l+3, stored "pair-blocked": the pair (4l, 4l+1) at tile slots
// 2l, 2l+1 and the pair (4l+2, 4l+3) at 64 + 2l, 64 + 2l + 1. A warp reads a geometry block
// (one pair per lane) with one 16-byte load per lane, 512 contiguous bytes per warp.
__device__ __forceinline__ int64_t prep_slot(const JobDev& J, int64_t k) {
  const int64_t w = k / kWarpTile;
  const int rem = (int)(k - w * kWarpTile);
  const int l = rem / kDepPerLane, pp = rem % kDepPerLane;
  return J.prep_off + w * kWarpTile + (pp >> 1) * 64 + 2 * l + (pp & 1);
}

// A windowed job whose kept deposits share cells (fewer than half as many occupied flag cells
// of side d as deposits, or a quarter as many of side 2d: several hits per sphere) runs with
// coarse windows of kCoarseTiles warp tiles per warp; others with kWinTiles. Its cells record
// windows of kWindow deposits, a coarse window is two of them.
__device__ __forceinline__ bool coarse_windows(const JobDev& J, const JobAux& A) {
  return A.windowed && (J.cell_nbr8 ? 4 : 2) * (long long)A.cells < A.kept;
}

__device__ __forceinline__ bool keep_deposit(const JobDev& J, double x, double y, double z) {
  const double z1 = st_dadd(z, J.zsh);
  return fabs(z1) < J.HL && fabs(x) < J.xy_keep && fabs(y) < J.xy_keep;
}

// Flag cell of side cell_size containing (x, y, z): integer cell coordinates, offset to be
// non-negative, from u = RN(c * RN(1/cell_size)) per axis (within |u| 2^-51 of the exact
// quotient, below 2^-31 for the coordinates of a flagged job, |u| < 2^20). A job's flag cells
// have a side slightly above d or slightly above 2d (JobDev::cell_nbr8). With side d, two
// deposits within distance d of each other lie in the same or in adjacent cells: 27 cells around
// a point hold every deposit within d of it. With side 2d, a deposit within d of a point lies in
// the point's cell or in the neighbour cell on the side of the half of the cell the point is in:
// per axis, |u' - u| < 1/2 - 2^-12 for the other deposit's u', so floor(u') is floor(u) - 1 or
// floor(u) when u - floor(u) < 1/2, and floor(u) or floor(u) + 1 otherwise (the rounding errors
// are far below the margin): eight cells hold every deposit within d.
struct CellCoord {
  long long x, y, z;
};

__device__ __forceinline__ CellCoord cell_of(double x, double y, double z, double inv_cs) {
  const long long off = 1ll << (kCellBits - 1);
  return {(long long)floor(st_dmul(x, inv_cs)) + off, (long long)floor(st_dmul(y, inv_cs)) + off,
          (long long)floor(st_dmul(z, inv_cs)) + off};
}

// The cell of a point (as cell_of) and, per axis, the side of its neighbour cells (-1: the point
// is in the lower half of its cell).
struct CellNbr {
  CellCoord c;
  int sx, sy, sz;
};

__device__ __forceinline__ int half_side(double u) {
  return st_dsub(u, floor(u)) < 0.5 ? -1 : 1;
}

__device__ __forceinline__ CellNbr cell_nbr(double x, double y, double z, double inv_cs) {
  const long long off = 1ll << (kCellBits - 1);
  const double u = st_dmul(x, inv_cs), v = st_dmul(y, inv_cs), w = st_dmul(z, inv_cs);
  return {{(long long)floor(u) + off, (long long)floor(v) + off, (long long)floor(w) + off},
          half_side(u), half_side(v), half_side(w)};
}

// Key of the cell at offset (dx, dy, dz) from c.
__device__ __forceinline__ uint64_t cell_key(const CellCoord& c, int dx, int dy, int dz) {
  return ((uint64_t)(c.z + dz) << (2 * kCellBits)) | ((uint64_t)(c.y + dy) << kCellBits) |
         (uint64_t)(c.x + dx);
}

// Records window `win` in the cell `key`; true when this call created the cell.
__device__ __forceinline__ bool cell_insert(const PrepareParams& p, const JobDev& J,
                                            uint64_t key, uint32_t win) {
  const uint32_t mask = J.cell_cap - 1;
  uint32_t h = slot_hash(key, mask);
  for (uint32_t probe = 0; probe < J.cell_cap; ++probe) {
    CellSlot* slot = p.cells + J.cell_off + h;
    const uint64_t k = __ldcg(&slot->key);
    bool mine = k == key, created = false;
    if (!mine && k == kEmptyKey) {
      const uint64_t old = atomicCAS(&slot->key, kEmptyKey, key);
      created = old == kEmptyKey;
      mine = created || old == key;
    }
    if (mine) {
      atomicMin(&slot->wmin, win);
      atomicMin(&slot->nwmax, ~win);
      return created;
    }
    h = (h + 1) & mask;
  }
  return false;
}

// True when the cell slot v holds a deposit of a window other than `win`; windows are compared
// after a right shift by `shift` (1: coarse windows of two recorded windows each).
__device__ __forceinline__ bool slot_foreign(const ulonglong2& v, uint32_t win, int shift) {
  return ((uint32_t)v.y >> shift) != (win >> shift) ||
         (~(uint32_t)(v.y >> 32) >> shift) != (win >> shift);
}

// Neighbour keys as offsets from a cell's key: the coordinate fields of every cell a flagged job
// probes stay inside [0, 2^kCellBits), so a key of the cell at (dx, dy, dz) from c is c's key plus
// dz 2^(2 kCellBits) + dy 2^kCellBits + dx in two's complement. Neighbour c (0..26) of the 27
// around a side-d cell has (c % 3 - 1, c / 3 % 3 - 1, c / 9 - 1); neighbour c (0..7) of the eight
// around a point in a side-2d cell adds n.sx on x when bit 0 of c is set, n.sy on y for bit 1 and
// n.sz on z for bit 2.
__host__ __device__ constexpr int64_t cell_offset(int dx, int dy, int dz) {
  return (int64_t)dz * ((int64_t)1 << (2 * kCellBits)) + (int64_t)dy * ((int64_t)1 << kCellBits) + dx;
}
__device__ __forceinline__ uint64_t nbr_key27(uint64_t base, int c) {
  return base + (uint64_t)cell_offset(c % 3 - 1, (c / 3) % 3 - 1, c / 9 - 1);
}
struct NbrOffsets {
  uint64_t base;
  int64_t ox, oy, oz;
};
__device__ __forceinline__ NbrOffsets nbr_offsets8(const CellNbr& n) {
  return {cell_key(n.c, 0, 0, 0), cell_offset(n.sx, 0, 0), cell_offset(0, n.sy, 0),
          cell_offset(0, 0, n.sz)};
}
__device__ __forceinline__ uint64_t nbr_key8(const NbrOffsets& o, int c) {
  return o.base + (uint64_t)(((c & 1) ? o.ox : 0) + ((c & 2) ? o.oy : 0) + ((c & 4) ? o.oz : 0));
}

// True when one of the neighbour cells c0 .. c0 + BATCH - 1 (keys from key_of) holds a deposit
// of another window. Their first hash slots are loaded together, so a lane has several L2
// round trips in flight instead of one; a cell whose first slot holds another key continues
// probing alone. The hash is read-only here (k_prep_write filled it), and the neighbourhoods of
// a block's deposits overlap, so cached loads serve many probes from L1.
template <int BATCH, typename KeyOf>
__device__ __forceinline__ bool cells_foreign(const PrepareParams& p, const JobDev& J,
                                              const KeyOf& key_of, int c0, uint32_t win,
                                              int shift) {
  const uint32_t mask = J.cell_cap - 1;
  const CellSlot* base = p.cells + J.cell_off;
  ulonglong2 v[BATCH];
  uint32_t h[BATCH];
#pragma unroll
  for (int t = 0; t < BATCH; ++t) {
    h[t] = slot_hash(key_of(c0 + t), mask);
    v[t] = __ldg(reinterpret_cast<const ulonglong2*>(base + h[t]));
  }
  bool foreign = false;
#pragma unroll
  for (int t = 0; t < BATCH; ++t) {
    const uint64_t key = key_of(c0 + t);
    if (v[t].x == key) {
      foreign |= slot_foreign(v[t], win, shift);
    } else if (v[t].x != kEmptyKey) {
      uint32_t hh = h[t];
#pragma unroll 1
      for (uint32_t probe = 1; probe < J.cell_cap; ++probe) {
        hh = (hh + 1) & mask;
        const ulonglong2 w = __ldg(reinterpret_cast<const ulonglong2*>(base + hh));
        if (w.x == key) {
          foreign |= slot_foreign(w, win, shift);
          break;
        }
        if (w.x == kEmptyKey) break;
        if (probe == J.cell_cap - 1) foreign = true;  // a full table: conservative
      }
    }
  }
  return foreign;
}

// Eight blocks per SM (32 registers): more track loads in flight.
__global__ void __launch_bounds__(kPrepThreads, 8) k_prep_count(PrepareParams p) {
  const int64_t b = p.blk_base + blockIdx.x;
  const int j = prep_job(p, b);
  const JobDev J = p.jobs[j];
  const int64_t i0 = (b - p.blk_prefix[j]) * (int64_t)kPrepSlotsPerBlock;
  int emin = INT_MAX, emax = INT_MIN, flags = 0, kept = 0;
  // a guard rather than a break, so that the loads of all rounds can be in flight together
#pragma unroll
  for (int s = threadIdx.x; s < kPrepSlotsPerBlock; s += kPrepThreads) {
    const int64_t i = i0 + s;
    if (i >= J.n) continue;
    kept += keep_deposit(J, J.x[i], J.y[i], J.z[i]) ? 1 : 0;
    const double v = __ddiv_rn(J.edep[i], J.denom);
    if (!isfinite(v)) {
      flags |= kAuxNonfinite;
    } else if (v != 0.0) {
      flags |= kAuxNonzero;
      const int ex = ulp_exponent(v);
      emin = min(emin, ex);
      emax = max(emax, ex);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    emin = min(emin, __shfl_xor_sync(0xffffffffu, emin, o));
    emax = max(emax, __shfl_xor_sync(0xffffffffu, emax, o));
    flags |= __shfl_xor_sync(0xffffffffu, flags, o);
    kept += __shfl_xor_sync(0xffffffffu, kept, o);
  }
  // the block's warps meet in shared memory; one thread updates the job's record, whose
  // address every block of the job shares
  __shared__ int s_kept, s_flags, s_emin, s_emax;
  if (threadIdx.x == 0) {
    s_kept = 0;
    s_flags = 0;
    s_emin = INT_MAX;
    s_emax = INT_MIN;
  }
  __syncthreads();
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&s_kept, kept);
    if (flags) {
      atomicOr(&s_flags, flags);
      atomicMin(&s_emin, emin);
      atomicMax(&s_emax, emax);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    p.blk_count[b] = s_kept;
    if (s_flags) {
      atomicOr(&p.aux[j].flags, s_flags);
      if (s_flags & kAuxNonzero) {
        atomicMin(&p.aux[j].e_min, s_emin);
        atomicMax(&p.aux[j].e_max, s_emax);
      }
    }
  }
}

// One CTA per job: exclusive scan of the job's block counts.
__global__ void __launch_bounds__(1024) k_prep_scan(PrepareParams p) {
  const int j = blockIdx.x;
  const int64_t b0 = p.blk_prefix[j], nb = p.blk_prefix[j + 1] - b0;
  __shared__ long long s_warp[32];
  __shared__ long long s_carry;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int64_t base = 0; base < nb; base += 1024) {
    const int64_t k = base + threadIdx.x;
    long long v = k < nb ? p.blk_count[b0 + k] : 0;
    long long incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const long long t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      long long w = s_warp[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const long long t = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += t;
      }
      s_warp[lane] = w;  // inclusive over warps
    }
    __syncthreads();
    const long long warp_base = warp ? s_warp[warp - 1] : 0;
    if (k < nb) p.blk_offset[b0 + k] = s_carry + warp_base + incl - v;
    __syncthreads();
    if (threadIdx.x == 0) s_carry += s_warp[31];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    p.aux[j].kept = s_carry;
    p.aux[j].windowed = p.jobs[j].flagged && s_carry > p.flag_min_kept;
  }
}

// In-block grouping of kept deposits by cell (sorted prepare blocks): a block writes its kept
// deposits grouped by d-cell (x, y and z after the z-origin shift, each divided by d and rounded
// down), the groups in the order of their cells' first deposit in the block. Deposits of one cell
// mostly share a sphere for any shift, so the fused kernel sums them as runs in registers and
// across lanes instead of one shared-memory insert each; line-ordered tracks keep their order
// apart from the deposits pulled forward to their cell's first one. Cells are told apart by a
// kCellHashBins-way hash (a collision only merges two groups). Sort mode 1 groups the blocks of
// window-flagged jobs (multi-window jobs on fine lattices: the dense tracks whose spheres take
// several hits that the source order scatters), mode 2 every block.
constexpr int kCellHashBins = 1024;
__device__ __forceinline__ unsigned cell_hash_bin(const JobDev& J, double x, double y, double z1) {
  const unsigned cx = (unsigned)__double2int_rd(st_dmul(x, J.inv_d));
  const unsigned cy = (unsigned)__double2int_rd(st_dmul(y, J.inv_d));
  const unsigned cz = (unsigned)__double2int_rd(st_dmul(z1, J.inv_d));
  return ((cx * 73856093u) ^ (cy * 19349663u) ^ (cz * 83492791u)) & (kCellHashBins - 1);
}

// Four blocks per SM (64 registers, a few bytes of spills): the stage is memory-bound, and the
// fourth block's loads in flight are worth more than the spills cost.
__global__ void __launch_bounds__(kPrepThreads, 4) k_prep_write(PrepareParams p) {
  const int64_t b = p.blk_base + blockIdx.x;
  const int j = prep_job(p, b);
  const JobDev J = p.jobs[j];
  const int64_t i0 = (b - p.blk_prefix[j]) * (int64_t)kPrepSlotsPerBlock;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int kWarpsPerBlock = kPrepThreads / 32;
  constexpr int kRounds = kPrepSlotsPerBlock / kPrepThreads;
  constexpr int kGroupsPerThread = kPrepSlotsPerBlock / kPrepThreads;
  constexpr int kHashPerThread = kCellHashBins / kPrepThreads;
  __shared__ int s_warp[kRounds][kWarpsPerBlock];
  // sorted blocks: the first deposit (block-local index) of every cell-hash bin, and per group
  // (named by that first deposit) its size, then its offset
  __shared__ unsigned s_first[kCellHashBins];
  __shared__ unsigned s_group[kPrepSlotsPerBlock];
  __shared__ unsigned s_part[kWarpsPerBlock];
  int64_t run = p.blk_offset[b];  // kept index of the next kept deposit of this block
  const bool sorted = p.sort == 2 || (p.sort == 1 && J.flagged);
  if (sorted) {
#pragma unroll
    for (int t = 0; t < kHashPerThread; ++t) s_first[threadIdx.x * kHashPerThread + t] = ~0u;
#pragma unroll
    for (int t = 0; t < kGroupsPerThread; ++t) s_group[threadIdx.x * kGroupsPerThread + t] = 0;
  }
  const JobAux A = p.aux[j];
  const int E0 = choose_grid_exponent(A.e_min, A.e_max, J.n, A.flags & kAuxNonzero);
  unsigned created_cells = 0;  // cells this thread created (windowed jobs)
  // the loads of all rounds are issued before the block's one barrier, so each thread has all
  // of its source deposits in flight at once
  double x[kRounds], y[kRounds], z1[kRounds], e[kRounds];
#pragma unroll
  for (int r = 0; r < kRounds; ++r) {
    const int64_t i = i0 + r * kPrepThreads + threadIdx.x;
    x[r] = 0; y[r] = 0; z1[r] = 0;
    if (i < J.n) {
      x[r] = J.x[i];
      y[r] = J.y[i];
      z1[r] = J.z[i];
    }
  }
  unsigned keep = 0, m[kRounds];
  unsigned slot_of[kRounds];  // sorted blocks: cell-hash bin, then group (high 16 bits) and rank
  if (sorted) __syncthreads();  // tables initialised
#pragma unroll
  for (int r = 0; r < kRounds; ++r) {
    const int64_t i = i0 + r * kPrepThreads + threadIdx.x;
    z1[r] = st_dadd(z1[r], J.zsh);
    const bool k = i < J.n && fabs(z1[r]) < J.HL && fabs(x[r]) < J.xy_keep && fabs(y[r]) < J.xy_keep;
    keep |= k ? 1u << r : 0u;
    m[r] = __ballot_sync(0xffffffffu, k);
    if (lane == 0) s_warp[r][warp] = __popc(m[r]);
    e[r] = k ? J.edep[i] : 0.0;
    slot_of[r] = 0;
    if (sorted && k) {
      slot_of[r] = cell_hash_bin(J, x[r], y[r], z1[r]);
      atomicMin(&s_first[slot_of[r]], (unsigned)(r * kPrepThreads + threadIdx.x));
    }
  }
  __syncthreads();
  if (sorted) {
#pragma unroll
    for (int r = 0; r < kRounds; ++r) {
      if (keep & (1u << r)) {
        const unsigned g = s_first[slot_of[r]];
        slot_of[r] = (g << 16) | atomicAdd(&s_group[g], 1u);
      }
    }
    __syncthreads();
    // exclusive scan of the group sizes: each thread sums its kGroupsPerThread groups, the warps
    // scan the thread sums, and the warp totals are scanned in shared memory
    unsigned v[kGroupsPerThread], tsum = 0;
#pragma unroll
    for (int t = 0; t < kGroupsPerThread; ++t) {
      v[t] = s_group[threadIdx.x * kGroupsPerThread + t];
      tsum += v[t];
    }
    unsigned incl = tsum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned u = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += u;
    }
    if (lane == 31) s_part[warp] = incl;
    __syncthreads();
    unsigned base = incl - tsum;
    for (int w = 0; w < warp; ++w) base += s_part[w];
#pragma unroll
    for (int t = 0; t < kGroupsPerThread; ++t) {
      s_group[threadIdx.x * kGroupsPerThread + t] = base;
      base += v[t];
    }
    __syncthreads();
  }
#pragma unroll
  for (int r = 0; r < kRounds; ++r) {
    int before = 0, total = 0;
#pragma unroll
    for (int w = 0; w < kWarpsPerBlock; ++w) {
      const int c = s_warp[r][w];
      before += (w < warp) ? c : 0;
      total += c;
    }
    uint64_t ckey = kEmptyKey;  // windowed jobs: the kept deposit's flag cell and window
    uint32_t cwin = 0;
    if (keep & (1u << r)) {
      // kept index: block order, or the position of the deposit's group and rank in sorted
      // blocks
      const int64_t k = sorted ? p.blk_offset[b] + s_group[slot_of[r] >> 16] + (slot_of[r] & 0xFFFFu)
                               : run + before + __popc(m[r] & ((1u << lane) - 1u));
      const double az = st_dsub(z1[r], J.gSO);
      const double kd = lattice_index(az, J.d, J.inv_d);
      const double dz = st_dsub(st_dmul(kd, J.d), az);
      const int64_t dst = prep_slot(J, k);
      if (p.fp32) {
        reinterpret_cast<float2*>(p.PXY)[dst] = make_float2(__double2float_rn(x[r]), __double2float_rn(y[r]));
        reinterpret_cast<float*>(p.PDZ2)[dst] = __double2float_rn(st_dmul(dz, dz));
      } else {
        p.PXY[dst] = make_double2(x[r], y[r]);
        p.PDZ2[dst] = st_dmul(dz, dz);
      }
      uint64_t lo, hi;
      to_fixed(__ddiv_rn(e[r], J.denom), E0, &lo, &hi);
      p.PV[dst] = make_ulonglong2(lo, hi);
      p.PKEY[dst] = (uint64_t)(long long)kd * J.N2;
      if (A.windowed) {
        p.PZ[dst] = z1[r];
        ckey = cell_key(cell_of(x[r], y[r], z1[r], J.inv_cell), 0, 0, 0);
        cwin = (uint32_t)(k / kWindow);
      }
    }
    if (A.windowed) {
      // adjacent lanes hold adjacent source deposits, which on dense tracks share a cell and a
      // window: an insert equal to the previous lane's changes nothing and is skipped, which
      // spares the cell's slot most of its same-address atomics
      const uint64_t pkey = __shfl_up_sync(0xffffffffu, ckey, 1);
      const uint32_t pwin = __shfl_up_sync(0xffffffffu, cwin, 1);
      if (ckey != kEmptyKey && !(lane > 0 && pkey == ckey && pwin == cwin))
        created_cells += cell_insert(p, J, ckey, cwin);
    }
    run += total;
  }
  if (A.windowed) {  // occupied cells, one addition per block (the window size depends on them)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) created_cells += __shfl_xor_sync(0xffffffffu, created_cells, o);
    __shared__ unsigned s_cells;
    if (threadIdx.x == 0) s_cells = 0;
    __syncthreads();
    if (lane == 0 && created_cells) atomicAdd(&s_cells, created_cells);
    __syncthreads();
    if (threadIdx.x == 0 && s_cells) atomicAdd(&p.aux[j].cells, (unsigned long long)s_cells);
  }
}

// One block per job: padding slots [kept, kept rounded up to a warp tile).
__global__ void __launch_bounds__(kWarpTile) k_prep_pad(PrepareParams p) {
  const int j = blockIdx.x;
  const JobDev J = p.jobs[j];
  const long long kept = p.aux[j].kept;
  if ((kept % kWarpTile) == 0) return;
  const long long k = kept + threadIdx.x;
  if (k >= (kept / kWarpTile + 1) * kWarpTile) return;
  const int64_t dst = prep_slot(J, k);
  if (p.fp32) {
    reinterpret_cast<float2*>(p.PXY)[dst] = make_float2(__int_as_float(0x7FC00000), __int_as_float(0x7FC00000));
    reinterpret_cast<float*>(p.PDZ2)[dst] = __int_as_float(0x7F800000);
  } else {
    p.PXY[dst] = make_double2(__longlong_as_double(0x7FF8000000000000ll),
                              __longlong_as_double(0x7FF8000000000000ll));
    p.PDZ2[dst] = __longlong_as_double(0x7FF0000000000000ll);
  }
  p.PV[dst] = make_ulonglong2(0, 0);
  p.PKEY[dst] = 0;
}

// Boundary flags of the kept deposits of flagged jobs: a deposit is a boundary deposit when one of
// the flag cells around it (27 of side d, or eight of side 2d chosen by cell_nbr) holds a
// deposit of another window. A sphere whose hits in a window are
// all non-boundary has no hit in any other window (its hits are within distance d of each other),
// so the fused kernel can bin it as soon as the window is done.
// Eight blocks per SM (32 registers): the cell probes are L2 latency, which more warps hide.
__global__ void __launch_bounds__(kPrepThreads, 8) k_prep_flag(PrepareParams p) {
  const int64_t b = p.blk_base + blockIdx.x;
  const int j = prep_job(p, b);
  const JobDev J = p.jobs[j];
  const JobAux A = p.aux[j];
  if (!A.windowed) return;
  const int shift = coarse_windows(J, A) ? 1 : 0;
  const int64_t k0 = p.blk_offset[b];
  const int cnt = p.blk_count[b];
  for (int q = threadIdx.x; q < cnt; q += kPrepThreads) {
    const int64_t k = k0 + q;
    const int64_t dst = prep_slot(J, k);
    double x, y;
    if (p.fp32) {  // float-rounded x, y: the FP32 jobs' cell size covers the rounding
      const float2 xy = reinterpret_cast<const float2*>(p.PXY)[dst];
      x = xy.x;
      y = xy.y;
    } else {
      const double2 xy = p.PXY[dst];
      x = xy.x;
      y = xy.y;
    }
    const double z = p.PZ[dst];
    const uint32_t win = (uint32_t)(k / kWindow);
    bool boundary = false;
    // batches unrolled, so that the neighbour offsets are constants
    if (J.cell_nbr8) {
      const NbrOffsets o = nbr_offsets8(cell_nbr(x, y, z, J.inv_cell));
      const auto key_of = [&](int c) { return nbr_key8(o, c); };
#pragma unroll
      for (int c0 = 0; c0 < 8; c0 += 2)
        if (!boundary) boundary = cells_foreign<2>(p, J, key_of, c0, win, shift);
    } else {
      const uint64_t base = cell_key(cell_of(x, y, z, J.inv_cell), 0, 0, 0);
      const auto key_of = [&](int c) { return nbr_key27(base, c); };
#pragma unroll
      for (int c0 = 0; c0 < 27; c0 += 3)
        if (!boundary) boundary = cells_foreign<3>(p, J, key_of, c0, win, shift);
    }
    if (boundary) p.PKEY[dst] |= kBoundaryBit;
  }
}

// ---------------------------------------------------------------------------------------------
// Exact 128-bit accumulators
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ void acc_add(unsigned long long* lo_p, unsigned long long* hi_p,
                                        uint64_t lo, uint64_t hi) {
  const unsigned long long old = atomicAdd(lo_p, (unsigned long long)lo);
  const unsigned long long h = hi + ((old + lo < old) ? 1ull : 0ull);
  if (h) atomicAdd(hi_p, h);
}

__device__ __forceinline__ void add128(uint64_t& alo, uint64_t& ahi, uint64_t lo, uint64_t hi) {
  const uint64_t s = alo + lo;
  ahi += hi + (s < alo ? 1ull : 0ull);
  alo = s;
}

// Spill-table insert (HBM). Returns false when the table has no free slot.
__device__ __forceinline__ bool gtable_add(uint64_t* gk, unsigned long long* glo,
                                           unsigned long long* ghi, uint32_t* gused,
                                           unsigned int* gcnt, uint32_t gcap, uint64_t key,
                                           uint64_t lo, uint64_t hi) {
  const uint32_t mask = gcap - 1;
  uint32_t h = slot_hash(key, mask);
  for (uint32_t probe = 0; probe < gcap; ++probe) {
    const uint64_t k = __ldcg((const unsigned long long*)&gk[h]);
    if (k == key) { acc_add(&glo[h], &ghi[h], lo, hi); return true; }
    if (k == kEmptyKey) {
      const uint64_t old = atomicCAS((unsigned long long*)&gk[h], kEmptyKey, key);
      if (old == kEmptyKey) {
        const unsigned idx = atomicAdd(gcnt, 1u);
        gused[idx] = h;
        acc_add(&glo[h], &ghi[h], lo, hi);
        return true;
      }
      if (old == key) { acc_add(&glo[h], &ghi[h], lo, hi); return true; }
    }
    h = (h + 1) & mask;
  }
  return false;
}

// {x, y} of two consecutive slots (32 bytes, 32-byte aligned: a lane's pair in a pair-blocked
// tile) with one 256-bit read-only load.
__device__ __forceinline__ void ldg_xy_pair(const double2* p, double* v) {
  asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
      : "=d"(v[0]), "=d"(v[1]), "=d"(v[2]), "=d"(v[3])
      : "l"(p));
}

// Dynamic shared memory of the fused kernel. The sphere table sits at fixed offsets (so that its
// addresses cost no registers): keys, low and high accumulator words, the used-slot list and the
// boundary bitmap; the shared-memory histogram (y*f(y), edges, counts) follows it.
extern __shared__ __align__(16) unsigned char smem_raw[];

template <int CAP>
struct SmemTable {
  __device__ __forceinline__ static uint64_t* keys() { return reinterpret_cast<uint64_t*>(smem_raw); }
  __device__ __forceinline__ static unsigned long long* lo() {
    return reinterpret_cast<unsigned long long*>(smem_raw + 8 * CAP);
  }
  __device__ __forceinline__ static unsigned long long* hi() {
    return reinterpret_cast<unsigned long long*>(smem_raw + 16 * CAP);
  }
  __device__ __forceinline__ static uint16_t* used() {
    return reinterpret_cast<uint16_t*>(smem_raw + 24 * CAP);
  }
  // CAP bits: the entry holds a boundary deposit's contribution
  __device__ __forceinline__ static unsigned int* flags() {
    return reinterpret_cast<unsigned int*>(smem_raw + 26 * CAP);
  }
  __device__ __forceinline__ static double* hist() {
    return reinterpret_cast<double*>(smem_raw + 26 * CAP + CAP / 8);
  }
};

// Occupancy and overflow of the sphere table are counted per window in one of three rotating
// slots (window i uses slot i % 3; a job without window flags always uses slot 0): the slot of the
// next window can then be cleared while the current window's is still being read, which saves a
// CTA barrier per window.
struct CtaState {
  int item;
  int tc[3];        // used slots of the table (the used-list length) in this window
  int spilled;      // some sphere of this oversample has a partial sum in the spill table
  int ovf[3];       // this window sent a contribution to the spill table directly
  int edges_hist;   // histogram whose edges are in shared memory (-1: none)
  int log_mode;     // private item: table overflows, flushes and window-end spills go to the log
  int logn;         // records in the spill log of this oversample
};

// Spill table of the current item: the CTA's table restricted to a power-of-two prefix sized
// for the item's job, so that small jobs touch a small, cache-friendly region.
struct Spill {
  uint64_t* keys;
  unsigned long long* lo;
  unsigned long long* hi;
  uint32_t* used;
  unsigned int* count;
  uint32_t cap;
};

// Appends a sphere's partial sum to the CTA's spill log: the first half of the item's spill table
// holds (key, lo, hi) records in arrival order, written with plain stores, so a window end does
// not wait for global atomics. A log takes at most one record per hit of its oversample, and the
// table has at least two slots per kept deposit, so it cannot run out.
__device__ __forceinline__ void log_append(CtaState* cs, const FusedParams& P, const Spill& G,
                                           uint64_t key, uint64_t lo, uint64_t hi) {
  const unsigned idx = (unsigned)atomicAdd(&cs->logn, 1);
  if (idx < G.cap / 2) {
    G.keys[idx] = key;
    G.lo[idx] = lo;
    G.hi[idx] = hi;
  } else {
    atomicOr(P.error_flags, 1);
  }
}

// Adds a contribution to the CTA's shared-memory table. A sphere already in the table is always
// found there; a new one is refused (false) when the table is three quarters full or its probe
// sequence is too long.
template <int CAP>
__device__ __forceinline__ bool table_insert(const SmemTable<CAP>& T, CtaState* cs, uint64_t key,
                                             uint64_t lo, uint64_t hi, bool boundary, int slot) {
  constexpr int kHardLimit = (CAP * 3) / 4;
  uint32_t h = table_hash(key, CAP - 1);
#pragma unroll 1
  for (int probe = 0; probe < 32; ++probe) {
    const uint64_t k = ((volatile uint64_t*)T.keys())[h];
    bool mine = k == key;
    if (!mine && k == kEmptyKey) {
      if (*(volatile int*)&cs->tc[slot] >= kHardLimit) return false;
      const uint64_t old = atomicCAS((unsigned long long*)&T.keys()[h], kEmptyKey, key);
      if (old == kEmptyKey) {
        const int idx = atomicAdd(&cs->tc[slot], 1);
        T.used()[idx] = (uint16_t)h;
      }
      mine = old == kEmptyKey || old == key;
    }
    if (mine) {
      acc_add(&T.lo()[h], &T.hi()[h], lo, hi);
      if (boundary) atomicOr(&T.flags()[h >> 5], 1u << (h & 31));
      return true;
    }
    h = (h + 1) & (CAP - 1);
  }
  return false;
}

// Adds one sphere contribution to the shared-memory table, or, when the table refuses it, to the
// spill log (window-flagged private items) or the spill table. Jobs with window flags empty the
// table at every window end; other jobs keep their spheres for the whole oversample, and on the
// 4096-slot table are also flushed at window ends once it is half full (window_checks).
template <int CAP>
__device__ __forceinline__ void sphere_add(const SmemTable<CAP>& T, CtaState* cs,
                                           const FusedParams& P, const Spill& G, uint64_t key,
                                           uint64_t lo, uint64_t hi, bool boundary, int slot) {
  if (table_insert<CAP>(T, cs, key, lo, hi, boundary, slot)) return;
  *(volatile int*)&cs->ovf[slot] = 1;
  if (*(volatile int*)&cs->log_mode) {
    log_append(cs, P, G, key, lo, hi);
    return;
  }
  *(volatile int*)&cs->spilled = 1;
  if (!gtable_add(G.keys, G.lo, G.hi, G.used, G.count, G.cap, key, lo, hi))
    atomicOr(P.error_flags, 1);
}

constexpr int kHistCopies = 4;   // at most this many shared-memory copies of a histogram

struct BinContext {
  const double* edges;    // shared-memory copy when the histogram fits, else HBM
  unsigned long long* gcounts;
  double* gyfy;
  unsigned int* hcount;   // null: accumulate straight into HBM
  unsigned long long* hylo;  // y*f(y) per bin: 128-bit sum on the bin's grid (see bin_sphere)
  unsigned long long* hyhi;
  int copies;             // shared-memory copies of the histogram, used by warp % copies
  int nbins;
  int mode;               // 0: linear candidate, 1: log2 candidate
  double ca, cb;          // candidate bin = (y - ca) * cb, or (log2 y - ca) * cb
  int E0;
  int job;
};

// HistogramRange bin of y (edges[b] <= y < edges[b+1], else -1). An arithmetic guess of the
// bin is corrected against the exact edges, so the result is the same as a binary search.
__device__ __forceinline__ int find_bin_fast(const BinContext& B, double y) {
  const double* e = B.edges;
  const int nb = B.nbins;
  if (!(y >= e[0]) || !(y < e[nb])) return -1;
  const float t = B.mode ? (__log2f((float)y) - (float)B.ca) * (float)B.cb
                         : (float)((y - B.ca) * B.cb);
  int b = (t >= 0.f) ? (t < (float)nb ? (int)t : nb - 1) : 0;
#pragma unroll 1
  for (int it = 0; it < 8; ++it) {
    if (y < e[b]) { --b; continue; }
    if (y >= e[b + 1]) { ++b; continue; }
    return b;
  }
  int l = 0, h = nb;  // far-off guess: binary search
  while (h - l > 1) {
    const int m = (l + h) >> 1;
    if (e[m] <= y) l = m; else h = m;
  }
  return l;
}

__device__ __forceinline__ void bin_sphere(const BinContext& B, const FusedParams& P,
                                           uint64_t key, uint64_t lo, uint64_t hi,
                                           unsigned int& spheres, unsigned int& binned, int os) {
  const double y = from_fixed(lo, hi, B.E0);
  ++spheres;
  const int b = find_bin_fast(B, y);
  if (b >= 0) {
    ++binned;
    if (B.hcount) {
      // warps spread over the copies, so that fewer of them contend for a bin's 64-bit add
      const int c = B.copies > 1 ? (int)((threadIdx.x >> 5) % (unsigned)B.copies) * B.nbins : 0;
      atomicAdd(&B.hcount[c + b], 1u);
      // y >= edge_b > 0 is a whole multiple of ulp(edge_b): its sum is kept exactly as a 128-bit
      // integer on that grid, with integer atomics (a double atomic add is a retry loop under
      // contention). A bin whose lower edge is not a positive normal number keeps a double sum
      // in the low word instead.
      const uint64_t eb = (uint64_t)__double_as_longlong(B.edges[b]);
      if ((int64_t)eb > 0 && (eb >> 52) != 0) {
        uint64_t lo, hi;
        to_fixed(y, (int)(eb >> 52) - 1075, &lo, &hi);
        acc_add(&B.hylo[c + b], &B.hyhi[c + b], lo, hi);
      } else {
        atomicAdd(reinterpret_cast<double*>(&B.hylo[c + b]), y);
      }
    } else {
      atomicAdd(&B.gcounts[b], 1ull);
      atomicAdd(&B.gyfy[b], y);
    }
  }
  if (P.export_buf) {
    const unsigned long long idx = atomicAdd(P.export_count, 1ull);
    if (idx < P.export_cap) {
      SphereRecord r;
      r.key = key;
      r.y = y;
      r.os = os;
      r.job = B.job;
      P.export_buf[idx] = r;
    } else {
      atomicOr(P.error_flags, 2);
    }
  }
}

// Appends every shared-memory entry to the spill log and empties the shared table.
template <int CAP, int THREADS>
__device__ __forceinline__ void flush_to_log(const SmemTable<CAP>& T, int cnt, CtaState* cs,
                                             const FusedParams& P, const Spill& G) {
  for (int i = threadIdx.x; i < cnt; i += THREADS) {
    const uint32_t h = T.used()[i];
    log_append(cs, P, G, T.keys()[h], T.lo()[h], T.hi()[h]);
    T.keys()[h] = kEmptyKey; T.lo()[h] = 0; T.hi()[h] = 0;
  }
}

// Moves every shared-memory entry into the spill table and empties the shared table.
template <int CAP, int THREADS>
__device__ __forceinline__ void flush_to_spill(const SmemTable<CAP>& T, int cnt,
                                               const FusedParams& P, const Spill& G) {
  for (int i = threadIdx.x; i < cnt; i += THREADS) {
    const uint32_t h = T.used()[i];
    if (!gtable_add(G.keys, G.lo, G.hi, G.used, G.count, G.cap, T.keys()[h], T.lo()[h], T.hi()[h]))
      atomicOr(P.error_flags, 1);
    T.keys()[h] = kEmptyKey;
    T.lo()[h] = 0;
    T.hi()[h] = 0;
  }
}

// ---------------------------------------------------------------------------------------------
// Spill-table pool: one table per CTA of the launch. A CTA holds at most one table at a time
// (for its private item, or for the shared unit it works on until the unit is binned), so a free
// table always exists; the bounded scan only guards against a logic error.
// ---------------------------------------------------------------------------------------------
__device__ int pool_acquire(unsigned int* bits, int n_tables, int* err) {
  const int words = (n_tables + 31) / 32;
  for (int attempt = 0; attempt < 64; ++attempt) {
    for (int w = 0; w < words; ++w) {
      const unsigned valid = (w == words - 1 && (n_tables & 31)) ? ((1u << (n_tables & 31)) - 1u) : ~0u;
      unsigned freeb = ~__ldcg(&bits[w]) & valid;
      while (freeb) {
        const int b = __ffs(freeb) - 1;
        const unsigned old = atomicOr(&bits[w], 1u << b);
        if (!(old & (1u << b))) return w * 32 + b;
        freeb &= ~(1u << b);
      }
    }
  }
  atomicOr(err, 4);
  return -1;
}

__device__ __forceinline__ void pool_release(unsigned int* bits, int t) {
  atomicAnd(&bits[t >> 5], ~(1u << (t & 31)));
}

// Table of shared unit u: the first helper acquires it, the others wait (bounded: max_polls
// sleeps of at least 64 ns) until it is published. A wait that runs out sets error flag 8 and
// returns -1, and the item is given up; the host reports the run as ST_ERR_DEVICE_WAIT.
constexpr long long kUnitWaitPolls = 1ll << 24;
__device__ int unit_table_get(const FusedParams& P, int u, long long max_polls = kUnitWaitPolls) {
  int t = atomicCAS(&P.unit_table[u], -1, -2);
  if (t == -1) {
    t = pool_acquire(P.pool_bits, gridDim.x, P.error_flags);
    atomicExch(&P.unit_table[u], t < 0 ? -3 : t);
    return t;
  }
  for (long long spin = 0; t == -2 && spin < max_polls; ++spin) {
    __nanosleep(64);
    t = *(volatile int*)&P.unit_table[u];
  }
  if (t < 0) { atomicOr(P.error_flags, 8); return -1; }
  return t;
}

__device__ __forceinline__ Spill spill_of(const FusedParams& P, int t, long long kept) {
  Spill G;
  G.keys = P.gkeys + (size_t)t * P.gcap;
  G.lo = P.glo + (size_t)t * P.gcap;
  G.hi = P.ghi + (size_t)t * P.gcap;
  G.used = P.gused + (size_t)t * P.gcap;
  G.count = P.gcount + t;
  uint32_t cap = 1024;
  while (cap < P.gcap && (long long)cap < 2 * kept) cap <<= 1;
  G.cap = cap;
  return G;
}

// Bins and clears every entry of a spill table (all threads of the CTA).
template <int THREADS>
__device__ __forceinline__ void bin_spill(const Spill& G, const BinContext& B, const FusedParams& P,
                                          unsigned int& spheres, unsigned int& binned, int os) {
  const unsigned gc = __ldcg(G.count);
  for (unsigned i = threadIdx.x; i < gc; i += THREADS) {
    const uint32_t h = __ldcg(&G.used[i]);
    const uint64_t key = __ldcg((const unsigned long long*)&G.keys[h]);
    const uint64_t lo = __ldcg(&G.lo[h]);
    const uint64_t hi = __ldcg(&G.hi[h]);
    bin_sphere(B, P, key, lo, hi, spheres, binned, os);
    G.keys[h] = kEmptyKey; G.lo[h] = 0; G.hi[h] = 0;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    *G.count = 0;
    __threadfence();
  }
}

// Partition of a spill-log record: a hash of the key independent of the table's slot hash.
__device__ __forceinline__ int log_part(uint64_t key, int parts) {
  return (int)(((uint64_t)(uint32_t)((key * 0xD6E8FEB86659FD93ull) >> 32) * (uint64_t)parts) >> 32);
}

// One reduction pass: the records [r0, r1) of R whose partition is `part` (all of them when
// parts is 1) are summed in the empty shared table and binned. If the table refused any record,
// the pass's spheres go whole to the hash table F instead (binned last), so that no sphere is
// split between the two. Returns whether F received anything (the same in every thread).
template <int CAP, int THREADS>
__device__ __forceinline__ int log_pass(const SmemTable<CAP>& T, CtaState& cs,
                                        const FusedParams& P, const Spill& R, int r0, int r1,
                                        int part, int parts, const Spill& F, int slot,
                                        const BinContext& B, unsigned int& spheres,
                                        unsigned int& binned, int os) {
  const int tid = threadIdx.x;
  int refused = 0;
  // four records in flight per thread before any is inserted
  for (int i0 = r0 + tid; i0 < r1; i0 += 4 * THREADS) {
    uint64_t kk[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int i = i0 + u * THREADS;
      kk[u] = i < r1 ? __ldcg((const unsigned long long*)&R.keys[i]) : kEmptyKey;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int i = i0 + u * THREADS;
      if (i >= r1 || (parts > 1 && log_part(kk[u], parts) != part)) continue;
      const uint64_t lo = __ldcg(&R.lo[i]), hi = __ldcg(&R.hi[i]);
      if (!table_insert<CAP>(T, &cs, kk[u], lo, hi, false, slot)) {
        if (!gtable_add(F.keys, F.lo, F.hi, F.used, F.count, F.cap, kk[u], lo, hi))
          atomicOr(P.error_flags, 1);
        refused = 1;
      }
    }
  }
  refused = __syncthreads_or(refused);
  const int cnt = cs.tc[slot];
  if (tid == 0) cs.tc[(slot + 1) % 3] = 0;  // the next pass's slot: last read two passes ago
  for (int i = tid; i < cnt; i += THREADS) {
    const uint32_t h = T.used()[i];
    if (refused) {
      if (!gtable_add(F.keys, F.lo, F.hi, F.used, F.count, F.cap, T.keys()[h], T.lo()[h], T.hi()[h]))
        atomicOr(P.error_flags, 1);
    } else {
      bin_sphere(B, P, T.keys()[h], T.lo()[h], T.hi()[h], spheres, binned, os);
    }
    T.keys()[h] = kEmptyKey; T.lo()[h] = 0; T.hi()[h] = 0;
  }
  __syncthreads();
  return refused;
}

// End of a window-flagged private oversample: sums the spill log (the first half of the spill
// table, records [0, L)) per sphere and bins it, in passes of at most CAP / 2 records (a pass has
// no more distinct keys than records, so the table stays at most half full).
//  - Bucketed (more than one pass, and the per-pass counts fit the table's used-slot list, free at
//    this point): the records are counted per hash partition, scattered into buckets in the second
//    half of the spill table, and each bucket is summed in one pass; the emptied first half is the
//    fallback table, and the bucket bounds sit in the spill table's used list beyond its reach.
//  - Otherwise every pass scans the whole log for its partition, with the second half of the
//    spill table as the fallback.
// Every record is cleared again for the pool's next user.
template <int CAP, int THREADS>
__device__ __forceinline__ void log_reduce(const SmemTable<CAP>& T, CtaState& cs,
                                           const FusedParams& P, const Spill& G,
                                           const BinContext& B, unsigned int& spheres,
                                           unsigned int& binned, int os) {
  const int tid = threadIdx.x;
  const int L = cs.logn;  // read after superimpose's closing barrier: the same in every thread
  if (L == 0) return;
  constexpr int kPart = CAP / 2;  // records per pass
  const int parts = (L + kPart - 1) / kPart;
  Spill lo_half = G, hi_half = G;
  lo_half.cap = G.cap / 2;
  hi_half.keys += G.cap / 2;
  hi_half.lo += G.cap / 2;
  hi_half.hi += G.cap / 2;
  hi_half.cap = G.cap / 2;
  if (tid == 0) for (int k = 0; k < 3; ++k) cs.tc[k] = 0;
  __syncthreads();
  int any_out = 0;
  if (parts == 1 || 2 * parts > CAP / 2) {
    for (int q = 0; q < parts; ++q)
      any_out |= log_pass<CAP, THREADS>(T, cs, P, lo_half, 0, L, q, parts, hi_half, q % 3, B,
                                        spheres, binned, os);
    for (int i = tid; i < L; i += THREADS) { G.keys[i] = kEmptyKey; G.lo[i] = 0; G.hi[i] = 0; }
    if (any_out) bin_spill<THREADS>(hi_half, B, P, spheres, binned, os);
  } else {
    unsigned int* cnt = reinterpret_cast<unsigned int*>(T.used());  // parts counts, parts cursors
    uint32_t* bounds = G.used + G.cap / 2;                              // parts + 1 bucket bounds
    for (int i = tid; i < 2 * parts; i += THREADS) cnt[i] = 0;
    __syncthreads();
    for (int i = tid; i < L; i += THREADS)
      atomicAdd(&cnt[log_part(__ldcg((const unsigned long long*)&G.keys[i]), parts)], 1u);
    __syncthreads();
    if (tid == 0) {
      unsigned run = 0;
      for (int q = 0; q < parts; ++q) {
        bounds[q] = run;
        cnt[parts + q] = run;
        run += cnt[q];
      }
      bounds[parts] = run;
    }
    __syncthreads();
    for (int i = tid; i < L; i += THREADS) {
      const uint64_t key = __ldcg((const unsigned long long*)&G.keys[i]);
      const uint64_t lo = __ldcg(&G.lo[i]), hi = __ldcg(&G.hi[i]);
      const unsigned pos = atomicAdd(&cnt[parts + log_part(key, parts)], 1u);
      hi_half.keys[pos] = key; hi_half.lo[pos] = lo; hi_half.hi[pos] = hi;
      G.keys[i] = kEmptyKey; G.lo[i] = 0; G.hi[i] = 0;
    }
    __syncthreads();  // buckets written, the first half empty again (the fallback from here on)
    for (int q = 0; q < parts; ++q) {
      const int r0 = (int)__ldcg(&bounds[q]), r1 = (int)__ldcg(&bounds[q + 1]);
      any_out |= log_pass<CAP, THREADS>(T, cs, P, hi_half, r0, r1, q, 1, lo_half, q % 3, B,
                                        spheres, binned, os);
    }
    for (int i = tid; i < L; i += THREADS) {
      hi_half.keys[i] = kEmptyKey; hi_half.lo[i] = 0; hi_half.hi[i] = 0;
    }
    if (any_out) bin_spill<THREADS>(lo_half, B, P, spheres, binned, os);
  }
  __syncthreads();
  if (tid == 0) {
    for (int k = 0; k < 3; ++k) cs.tc[k] = 0;
    cs.logn = 0;
  }
  __syncthreads();
}

struct FusedJob {
  JobDev J;
  int E0;
  int win_tiles;    // warp tiles per warp in a window: kWinTiles, or kCoarseTiles
  int64_t n_wt;     // warp tiles of kept deposits
};

// Warp tiles of a shared unit's chunk: chunk_windows windows of kWinTiles tiles per warp,
// rounded up to whole coarse windows, so that no window is ever split between two chunks.
__host__ __device__ __forceinline__ int64_t chunk_tiles(int chunk_windows) {
  constexpr int64_t kCoarse = (int64_t)kFusedWarps * kCoarseTiles;
  const int64_t t = (int64_t)chunk_windows * kFusedWarps * kWinTiles;
  return (t + kCoarse - 1) / kCoarse * kCoarse;
}

// Superimposes oversample `os` of a job over warp tiles [wt_begin, wt_end) (whole windows):
// shift, box test, lattice test, key, exact run / warp / shared-memory reduction. For flagged jobs
// every window ends by binning its complete spheres and moving boundary spheres to G; otherwise
// spheres accumulate across windows and the shared table spills to G when it fills up.
// F32: the FP32 geometry variant (x, y, shifts, lattice index and distance in float; z part of
// the distance, keys and energies as in the FP64 form).
template <int CAP, int THREADS, bool F32>
__device__ __forceinline__ void superimpose(const FusedParams& P, const FusedJob& F,
                                            const SmemTable<CAP>& T, CtaState& cs,
                                            const Spill& G, const BinContext& B, int os,
                                            int64_t wt_begin, int64_t wt_end,
                                            unsigned int& hits, unsigned int& inbox,
                                            unsigned int& spheres, unsigned int& binned) {
  constexpr int kWarps = THREADS / 32;
  const JobDev& J = F.J;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  float ux, uy;
  shift_uniforms(J.seed, J.track_id, (uint32_t)os, J.shift_track, &ux, &uy);
  const double sx = shift_from_uniform(ux, J.L, J.HL);
  const double sy = shift_from_uniform(uy, J.L, J.HL);
  const float sxf = __double2float_rn(sx), syf = __double2float_rn(sy);

  // Jobs without window flags on the 8192-slot table run their windows without a barrier (a CTA
  // barrier per window cost more than the occasional new sphere sent to the spill table by a
  // full table); on the 4096-slot table, a job whose whole lattice (N^3 spheres) exceeds the flush
  // threshold checks the table at every window end and flushes it to the spill table
  const bool log_mode = cs.log_mode != 0;
  const bool window_checks = CAP < 2 * kCtaTile && !J.flagged &&
                             (uint64_t)J.N * J.N2 > (uint64_t)P.flush_threshold;
  int wi = 0;  // window index within this call
  const int wtiles = F.win_tiles;
  for (int64_t wt0 = wt_begin; wt0 < wt_end; wt0 += kWarps * wtiles) {
    const int slot = J.flagged ? wi % 3 : 0;
    // a window is wtiles warp tiles per warp
#pragma unroll 1
    for (int tt = 0; tt < wtiles; ++tt) {
      const int64_t w = wt0 + tt * kWarps + warp;
      if (w < wt_end) {
        // pair-blocked tile (prep_slot): this lane's deposits p = 0, 1 are the slots tb, tb + 1
        // and p = 2, 3 the slots tb + 64, tb + 65
        const int64_t tb = J.prep_off + w * kWarpTile + 2 * lane;
        uint32_t kxv[kDepPerLane], kyv[kDepPerLane];
        unsigned hitmask = 0, boxmask = 0;
        if constexpr (F32) {
          // x' = x + sx, box |x'| < HL', a = x' - gSO, k = rint(a * (1/d)), dx = k*d - a,
          // hit iff (dx^2 + dy^2) + dz^2 <= r^2, every step rounded to float
          const float2* pxy = reinterpret_cast<const float2*>(P.PXY) + tb;
          const float* pdz = reinterpret_cast<const float*>(P.PDZ2) + tb;
          const float4 xy01 = __ldg(reinterpret_cast<const float4*>(pxy));
          const float4 xy23 = __ldg(reinterpret_cast<const float4*>(pxy + 64));
          const float2 dz01 = __ldg(reinterpret_cast<const float2*>(pdz));
          const float2 dz23 = __ldg(reinterpret_cast<const float2*>(pdz + 64));
  #pragma unroll
          for (int p = 0; p < kDepPerLane; ++p) {
            const float2 xy = p == 0 ? make_float2(xy01.x, xy01.y) : p == 1 ? make_float2(xy01.z, xy01.w)
                            : p == 2 ? make_float2(xy23.x, xy23.y) : make_float2(xy23.z, xy23.w);
            const float dzp = p == 0 ? dz01.x : p == 1 ? dz01.y : p == 2 ? dz23.x : dz23.y;
            const float x1 = __fadd_rn(xy.x, sxf);
            const float y1 = __fadd_rn(xy.y, syf);
            const bool inb = fabsf(x1) < J.f_HL && fabsf(y1) < J.f_HL;
            boxmask |= (unsigned)inb << p;
            const float ax = __fsub_rn(x1, J.f_gSO);
            const float ay = __fsub_rn(y1, J.f_gSO);
            const int ix = __float2int_rn(__fmul_rn(ax, J.f_inv_d));
            const int iy = __float2int_rn(__fmul_rn(ay, J.f_inv_d));
            const float ddx = __fsub_rn(__fmul_rn((float)ix, J.f_d), ax);
            const float ddy = __fsub_rn(__fmul_rn((float)iy, J.f_d), ay);
            const float dist = __fadd_rn(__fadd_rn(__fmul_rn(ddx, ddx), __fmul_rn(ddy, ddy)), dzp);
            hitmask |= (unsigned)(inb && dist <= J.f_r2) << p;
            kxv[p] = (uint32_t)ix;
            kyv[p] = (uint32_t)iy;
          }
        } else {
        // geometry in straight-line blocks of kGeoBlock deposits, so their FP64 chains interleave
  #pragma unroll
        for (int h4 = 0; h4 < kDepPerLane; h4 += kGeoBlock) {
          static_assert(kGeoBlock == 2, "a geometry block is a lane's pair of slots");
          double ax[kGeoBlock], ay[kGeoBlock], kdx[kGeoBlock], kdy[kGeoBlock];
          unsigned risk = 0;
          double xy[4];  // x0, y0, x1, y1 of the pair: one 32-byte load
          ldg_xy_pair(P.PXY + tb + h4 * 32, xy);
  #pragma unroll
          for (int p = 0; p < kGeoBlock; ++p) {
            const double x1 = st_dadd(xy[2 * p], sx);
            const double y1 = st_dadd(xy[2 * p + 1], sy);
            const bool inb = fabs(x1) < J.HL && fabs(y1) < J.HL;
            boxmask |= (unsigned)inb << (h4 + p);
            ax[p] = st_dsub(x1, J.gSO);
            ay[p] = st_dsub(y1, J.gSO);
            const double qx = st_dmul(ax[p], J.inv_d);
            const double qy = st_dmul(ay[p], J.inv_d);
            kdx[p] = st_dsub(st_dadd(qx, kMagic), kMagic);
            kdy[p] = st_dsub(st_dadd(qy, kMagic), kMagic);
            const bool near_half = fabs(st_dsub(qx, kdx[p])) >= kRiskBand ||
                                   fabs(st_dsub(qy, kdy[p])) >= kRiskBand;
            risk |= (unsigned)(near_half && inb) << p;
          }
          if (risk) {
            // q = RN(a * RN(1/d)) is within |q| 2^-51.2 of RN(a/d), far below 2^-20 for in-box
            // quotients (|q| < 2^21); only a quotient this close to a half-integer can round
            // differently, and then the IEEE division decides (rare: lattice-aligned inputs)
  #pragma unroll
            for (int p = 0; p < kGeoBlock; ++p) {
              if (risk & (1u << p)) {
                kdx[p] = rint(__ddiv_rn(ax[p], J.d));
                kdy[p] = rint(__ddiv_rn(ay[p], J.d));
              }
            }
          }
          const double2 zb = __ldg(reinterpret_cast<const double2*>(P.PDZ2 + tb + h4 * 32));
  #pragma unroll
          for (int p = 0; p < kGeoBlock; ++p) {
            const double ddx = st_dsub(st_dmul(kdx[p], J.d), ax[p]);
            const double ddy = st_dsub(st_dmul(kdy[p], J.d), ay[p]);
            const double dz2 = p == 0 ? zb.x : zb.y;
            const double dist = st_dadd(st_dadd(st_dmul(ddx, ddx), st_dmul(ddy, ddy)), dz2);
            const bool hit = ((boxmask >> (h4 + p)) & 1u) && dist <= J.r2;
            hitmask |= (unsigned)hit << (h4 + p);
            kxv[h4 + p] = (uint32_t)__double2loint(st_dadd(kdx[p], kMagic));
            kyv[h4 + p] = (uint32_t)__double2loint(st_dadd(kdy[p], kMagic));
          }
        }
        }
        hits += __popc(hitmask);
        inbox += __popc(boxmask);
        // runs of equal keys inside the lane's consecutive deposits are summed in registers
        uint64_t rkey = kEmptyKey, rlo = 0, rhi = 0;
        bool rflag = false;
  #pragma unroll
        for (int p = 0; p < kDepPerLane; ++p) {
          if (hitmask & (1u << p)) {
            const int64_t idx = tb + (p >> 1) * 64 + (p & 1);
            const ulonglong2 v = __ldg(&P.PV[idx]);
            const uint64_t lo = v.x;
            const uint64_t hi = v.y;
            const uint64_t kzw = __ldg(&P.PKEY[idx]);
            // (the FP32 form converts a lattice index like the reference's llrint: sign-extended)
            const uint64_t key =
                (F32 ? (uint64_t)(int64_t)(int32_t)kxv[p] + (uint64_t)(int64_t)(int32_t)kyv[p] * J.N
                     : (uint64_t)kxv[p] + (uint64_t)kyv[p] * J.N) + (kzw & ~kBoundaryBit);
            const bool bflag = (kzw & kBoundaryBit) != 0;
            if (key == rkey) {
              add128(rlo, rhi, lo, hi);
              rflag |= bflag;
            } else {
              if (rkey != kEmptyKey) sphere_add<CAP>(T, &cs, P, G, rkey, rlo, rhi, rflag, slot);
              rkey = key; rlo = lo; rhi = hi; rflag = bflag;
            }
          }
        }
        // the lanes' last runs: segmented sum over consecutive lanes with the same key, so a
        // sphere spanning several lanes costs one shared-memory update
        {
          const uint64_t kprev = __shfl_up_sync(0xffffffffu, rkey, 1);
          const uint64_t knext = __shfl_down_sync(0xffffffffu, rkey, 1);
          bool head = lane == 0 || kprev != rkey;
          const bool tail = lane == 31 || knext != rkey;
          const bool any_run = __any_sync(0xffffffffu, !head && rkey != kEmptyKey);
  #pragma unroll
          for (int o = 1; any_run && o < 32; o <<= 1) {
            const uint64_t olo = __shfl_up_sync(0xffffffffu, rlo, o);
            const uint64_t ohi = __shfl_up_sync(0xffffffffu, rhi, o);
            const bool ohead = __shfl_up_sync(0xffffffffu, head, o);
            const bool oflag = __shfl_up_sync(0xffffffffu, rflag, o);
            if (lane >= o && !head) {
              add128(rlo, rhi, olo, ohi);
              rflag |= oflag;
              head = ohead;
            }
          }
          if (tail && rkey != kEmptyKey) sphere_add<CAP>(T, &cs, P, G, rkey, rlo, rhi, rflag, slot);
        }
      }
    }
    if (J.flagged) {
      // window done: spheres without boundary contributions are complete -> bin them now;
      // the others (or all, if the window overflowed) go to the spill table
      __syncthreads();
      const int cnt = cs.tc[slot];
      const bool all_out = cs.ovf[slot] != 0;
      if (tid == 0) {  // the next window's slot: last read two windows ago
        cs.tc[(wi + 1) % 3] = 0;
        cs.ovf[(wi + 1) % 3] = 0;
      }
      int sent = 0;
      for (int i = tid; i < cnt; i += THREADS) {
        const uint32_t h = T.used()[i];
        const unsigned bit = 1u << (h & 31);
        const bool flagged = (T.flags()[h >> 5] & bit) != 0;
        if (flagged) atomicAnd(&T.flags()[h >> 5], ~bit);
        const bool out = all_out || flagged;
        if (out && log_mode) {
          log_append(&cs, P, G, T.keys()[h], T.lo()[h], T.hi()[h]);
        } else if (out) {
          if (!gtable_add(G.keys, G.lo, G.hi, G.used, G.count, G.cap, T.keys()[h], T.lo()[h], T.hi()[h]))
            atomicOr(P.error_flags, 1);
          sent = 1;
        } else {
          bin_sphere(B, P, T.keys()[h], T.lo()[h], T.hi()[h], spheres, binned, os);
        }
        T.keys()[h] = kEmptyKey; T.lo()[h] = 0; T.hi()[h] = 0;
      }
      // the table and its boundary bits are clear again once every thread is past this point
      sent = __syncthreads_or(sent);
      if (sent && tid == 0) cs.spilled = 1;
    } else if (window_checks && wt0 + kWarps * wtiles < wt_end) {
      __syncthreads();
      if (cs.tc[0] > P.flush_threshold) {
        if (log_mode) flush_to_log<CAP, THREADS>(T, cs.tc[0], &cs, P, G);
        else flush_to_spill<CAP, THREADS>(T, cs.tc[0], P, G);
        __syncthreads();
        if (tid == 0) { cs.tc[0] = 0; cs.spilled |= !log_mode; }
        __syncthreads();
      }
    }
    ++wi;
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------------------------
// k_fused: persistent work-stealing kernel. Items are either private (every window of a block of
// oversamples of a small or medium job, one CTA) or helpers of a shared unit (one oversample of
// a large job, whose window chunks are claimed dynamically by every helper that arrives).
// ---------------------------------------------------------------------------------------------
template <int CAP, int THREADS, bool F32>
__global__ void __launch_bounds__(THREADS, 1) k_fused(FusedParams P) {
  static_assert(CAP <= 65536, "used-slot list stores 16-bit slot indices");
  static_assert(THREADS / 32 == kFusedWarps, "a window is one CTA tile of warp tiles");
  __shared__ CtaState cs;
  __shared__ int s_bcast[2];
  __shared__ BinContext sB;   // the item's binning context and spill table, uniform over the
  __shared__ Spill sG;        // CTA: kept in shared memory rather than in every thread's registers

  const int HB = P.smem_hist_bins;
  const SmemTable<CAP> T;
  unsigned long long* hylo = reinterpret_cast<unsigned long long*>(SmemTable<CAP>::hist());
  unsigned long long* hyhi = hylo + HB;
  double* sedges = reinterpret_cast<double*>(hyhi + HB);         // HB + 1 edges
  unsigned int* hcount = reinterpret_cast<unsigned int*>(sedges + HB + 1);

  const int tid = threadIdx.x;
  const int lane = tid & 31;

  for (int i = tid; i < CAP; i += THREADS) { T.keys()[i] = kEmptyKey; T.lo()[i] = 0; T.hi()[i] = 0; }
  for (int i = tid; i < HB; i += THREADS) { hcount[i] = 0; hylo[i] = 0; hyhi[i] = 0; }
  for (int i = tid; i < CAP / 32; i += THREADS) T.flags()[i] = 0;
  if (tid == 0) {
    for (int k = 0; k < 3; ++k) { cs.tc[k] = 0; cs.ovf[k] = 0; }
    cs.spilled = 0;
    cs.log_mode = 0;
    cs.logn = 0;
    cs.edges_hist = -1;
  }
  __syncthreads();

  for (;;) {
    if (tid == 0) cs.item = (int)atomicAdd(P.work_counter, 1u);
    __syncthreads();
    const int it = cs.item;
    const int cached_hist = cs.edges_hist;
    __syncthreads();
    if (it >= *P.n_items) break;

    const WorkItem W = P.items[it];
    const JobAux A = P.aux[W.job];
    if (A.flags & kAuxNonfinite) continue;  // rejected job: contributes nothing, host reports it
    FusedJob F;
    F.J = P.jobs[W.job];
    F.J.flagged = A.windowed;  // window flags were computed only for these jobs
    F.win_tiles = coarse_windows(F.J, A) ? kCoarseTiles : kWinTiles;
    F.E0 = choose_grid_exponent(A.e_min, A.e_max, F.J.n, A.flags & kAuxNonzero);
    F.n_wt = (A.kept + kWarpTile - 1) / kWarpTile;
    const HistDev H = P.hists[F.J.hist];
    const bool smem_hist = H.nbins <= HB;

    // histogram edges into shared memory (kept while consecutive items use the same histogram)
    if (smem_hist && cached_hist != F.J.hist) {
      for (int i = tid; i <= H.nbins; i += THREADS) sedges[i] = H.edges[i];
      __syncthreads();
      if (tid == 0) cs.edges_hist = F.J.hist;
    }

    if (tid == 0) {
      sB.edges = smem_hist ? sedges : H.edges;
      sB.gcounts = H.counts;
      sB.gyfy = H.yfy;
      sB.nbins = H.nbins;
      sB.mode = H.mode;
      sB.ca = H.ca;
      sB.cb = H.cb;
      sB.E0 = F.E0;
      sB.job = W.job;
      sB.hcount = smem_hist ? hcount : nullptr;
      sB.hylo = smem_hist ? hylo : nullptr;
      sB.hyhi = smem_hist ? hyhi : nullptr;
      sB.copies = smem_hist ? min(kHistCopies, HB / H.nbins) : 1;
    }
    __syncthreads();
    const BinContext& B = sB;

    // per-thread counts of one item (an item covers at most a few million deposit*oversamples)
    unsigned int hits = 0, spheres = 0, binned = 0, inbox = 0;

    // Segments: a private item walks its oversamples (all windows each) with one pool table; a
    // helper claims window chunks of its shared unit until none is left.
    const bool shared = W.unit >= 0;
    const int64_t wpc = chunk_tiles(P.chunk_windows);  // warp tiles per chunk
    const int64_t n_chunks = (F.n_wt + wpc - 1) / wpc;
    int private_table = -1;
    if (!shared) {
      if (tid == 0) s_bcast[0] = pool_acquire(P.pool_bits, gridDim.x, P.error_flags);
      __syncthreads();
      private_table = s_bcast[0];
      __syncthreads();
    }
    for (int seg = 0;; ++seg) {
      int os, t;
      int64_t wb, we;
      if (!shared) {
        if (private_table < 0 || seg >= W.os_count) break;
        os = W.os_begin + seg;
        t = private_table;
        wb = 0;
        we = F.n_wt;
      } else {
        if (tid == 0) {
          const unsigned c = atomicAdd(&P.unit_next[W.unit], 1u);
          s_bcast[0] = (int64_t)c < n_chunks ? (int)c : -1;
          s_bcast[1] = s_bcast[0] >= 0 ? unit_table_get(P, W.unit) : -1;
        }
        __syncthreads();
        const int c = s_bcast[0];
        t = s_bcast[1];
        __syncthreads();
        if (c < 0 || t < 0) break;
        os = W.os_begin;
        wb = (int64_t)c * wpc;
        we = wb + wpc < F.n_wt ? wb + wpc : F.n_wt;
      }
      if (tid == 0) {
        sG = spill_of(P, t, A.kept);
        cs.log_mode = !shared;  // a single CTA sees every window of the oversample
      }
      __syncthreads();
      const Spill& G = sG;
      superimpose<CAP, THREADS, F32>(P, F, T, cs, G, B, os, wb, we, hits, inbox, spheres, binned);
      if (cs.log_mode) {
        if (!F.J.flagged && cs.logn > 0) {
          // the table's spheres may have parts in the log: they join it
          flush_to_log<CAP, THREADS>(T, cs.tc[0], &cs, P, G);
          __syncthreads();
          if (tid == 0) cs.tc[0] = 0;
          __syncthreads();
        }
        log_reduce<CAP, THREADS>(T, cs, P, G, B, spheres, binned, os);
      }
      const int cnt = F.J.flagged ? 0 : cs.tc[0];  // flagged windows leave the table empty
      bool bin_table;
      if (!shared) {
        bin_table = cs.spilled != 0;
        if (bin_table) {
          flush_to_spill<CAP, THREADS>(T, cnt, P, G);
        } else {
          for (int i = tid; i < cnt; i += THREADS) {
            const uint32_t h = T.used()[i];
            bin_sphere(B, P, T.keys()[h], T.lo()[h], T.hi()[h], spheres, binned, os);
            T.keys()[h] = kEmptyKey; T.lo()[h] = 0; T.hi()[h] = 0;
          }
        }
        __syncthreads();
      } else {
        // everything left in shared memory may meet contributions of other chunks
        flush_to_spill<CAP, THREADS>(T, cnt, P, G);
        __threadfence();
        __syncthreads();
        if (tid == 0) {
          const unsigned done = atomicAdd(&P.unit_done[W.unit], 1u) + 1u;
          s_bcast[0] = (int64_t)done == n_chunks ? 1 : 0;
        }
        __syncthreads();
        bin_table = s_bcast[0] != 0;  // last chunk of the unit: every contribution is in G
        if (bin_table) __threadfence();
      }
      if (bin_table) {
        bin_spill<THREADS>(G, B, P, spheres, binned, os);
        if (shared && tid == 0) pool_release(P.pool_bits, t);
      }
      if (tid == 0) {
        for (int k = 0; k < 3; ++k) { cs.tc[k] = 0; cs.ovf[k] = 0; }
        cs.spilled = 0;
        cs.log_mode = 0;
      }
      __syncthreads();
    }
    if (private_table >= 0) {
      __threadfence();
      __syncthreads();
      if (tid == 0) pool_release(P.pool_bits, private_table);
    }

    // ---- per-item flush of the shared-memory histogram and the job statistics
    if (smem_hist) {
      const int copies = B.copies;
      for (int b = tid; b < H.nbins; b += THREADS) {
        const uint64_t eb = (uint64_t)__double_as_longlong(sedges[b]);
        const bool exact = (int64_t)eb > 0 && (eb >> 52) != 0;  // as in bin_sphere
        unsigned cnt = 0;
        uint64_t lo = 0, hi = 0;
        double ys = 0.0;
        for (int c = 0; c < copies; ++c) {
          const int i = c * H.nbins + b;
          cnt += hcount[i];
          if (exact) add128(lo, hi, hylo[i], hyhi[i]);
          else ys += __longlong_as_double((long long)hylo[i]);
          hcount[i] = 0;
          hylo[i] = 0;
          hyhi[i] = 0;
        }
        if (cnt) {
          atomicAdd(&H.counts[b], (unsigned long long)cnt);
          atomicAdd(&H.yfy[b], exact ? from_fixed(lo, hi, (int)(eb >> 52) - 1075) : ys);
        }
      }
    }
    unsigned long long w_hits = hits, w_spheres = spheres, w_binned = binned, w_inbox = inbox;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      w_hits += __shfl_xor_sync(0xffffffffu, w_hits, o);
      w_spheres += __shfl_xor_sync(0xffffffffu, w_spheres, o);
      w_binned += __shfl_xor_sync(0xffffffffu, w_binned, o);
      w_inbox += __shfl_xor_sync(0xffffffffu, w_inbox, o);
    }
    if (lane == 0) {
      if (w_hits) atomicAdd(&P.aux[W.job].hits, w_hits);
      if (w_spheres) atomicAdd(&P.aux[W.job].spheres, w_spheres);
      if (w_binned) atomicAdd(&P.aux[W.job].binned, w_binned);
      if (w_inbox) atomicAdd(&P.aux[W.job].inbox, w_inbox);
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------------------------
// Planner (after the prepare stage, before k_fused): work items from the kept deposit counts.
// A job whose kept deposits per oversample exceed both min_chunks chunks (4) and 1/share_divisor
// (1/8) of one CTA's share of the batch runs as shared units (one per oversample, `helpers` helper items each);
// every other job runs as private items of about item_cost deposit*oversamples. Items are
// bucketed by cost, largest first (longest-processing-time order at bucket granularity).
// ---------------------------------------------------------------------------------------------
__global__ void k_plan_total(PlanParams q) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long v = 0;
  if (j < q.n_jobs) v = (unsigned long long)q.aux[j].kept * (unsigned long long)q.jobs[j].n_os;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0 && v) atomicAdd(q.total_units, v);
}

__device__ __forceinline__ int cost_bucket(long long cost) {
  int l = 0;
  while (cost > 1 && l < 62) { cost >>= 1; ++l; }
  return kPlanBuckets - 1 - l;  // larger cost -> smaller bucket -> earlier
}

__global__ void k_plan_size(PlanParams q) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= q.n_jobs) return;
  const long long kept = q.aux[j].kept;
  const long long nos = q.jobs[j].n_os;
  JobPlan pl;
  pl.items = 0;
  pl.bucket = kPlanBuckets - 1;
  pl.unit_base = -1;
  pl.blk_os = 1;
  if (kept > 0 && nos > 0 && !(q.aux[j].flags & kAuxNonfinite)) {
    const long long chunk = chunk_tiles(q.chunk_windows) * kWarpTile;
    const long long share =
        q.share_divisor > 0 ? (long long)(*q.total_units / ((unsigned long long)q.share_divisor * q.grid)) : 0;
    if (q.share_divisor > 0 && kept > (long long)q.min_chunks * chunk && kept > share) {
      const long long chunks = (kept + chunk - 1) / chunk;
      const int helpers = (int)(chunks < q.max_helpers ? chunks : q.max_helpers);
      pl.blk_os = helpers;
      pl.items = (int)(nos * helpers);
      pl.unit_base = (int)atomicAdd(q.unit_counter, (unsigned)nos);
      pl.bucket = cost_bucket(kept);
    } else {
      const long long pad = ((kept + kWarpTile - 1) / kWarpTile) * kWarpTile;
      long long b = q.item_cost / pad;
      b = b < 1 ? 1 : (b > nos ? nos : b);
      pl.blk_os = (int)b;
      pl.items = (int)((nos + b - 1) / b);
      pl.bucket = cost_bucket(pad * b);
    }
    atomicAdd(&q.bucket_count[pl.bucket], (unsigned)pl.items);
  }
  q.plan[j] = pl;
}

__global__ void k_plan_scan(PlanParams q) {
  if (threadIdx.x != 0) return;
  unsigned run = 0;
  for (int b = 0; b < kPlanBuckets; ++b) {
    q.bucket_start[b] = run;
    q.bucket_cursor[b] = 0;
    run += q.bucket_count[b];
  }
  *q.n_items = (long long)run <= q.item_cap ? (int)run : (int)q.item_cap;
}

__global__ void __launch_bounds__(128) k_plan_write(PlanParams q) {
  const int j = blockIdx.x;
  const JobPlan pl = q.plan[j];
  if (pl.items == 0) return;
  __shared__ unsigned s_pos;
  if (threadIdx.x == 0)
    s_pos = q.bucket_start[pl.bucket] + atomicAdd(&q.bucket_cursor[pl.bucket], (unsigned)pl.items);
  __syncthreads();
  const int nos = q.jobs[j].n_os;
  for (int k = threadIdx.x; k < pl.items; k += blockDim.x) {
    const long long pos = (long long)s_pos + k;
    if (pos >= q.item_cap) break;
    WorkItem w;
    w.job = j;
    if (pl.unit_base >= 0) {
      const int u = k / pl.blk_os;
      w.os_begin = u;
      w.os_count = 1;
      w.unit = pl.unit_base + u;
    } else {
      w.os_begin = k * pl.blk_os;
      w.os_count = (w.os_begin + pl.blk_os <= nos) ? pl.blk_os : nos - w.os_begin;
      w.unit = -1;
    }
    q.items[pos] = w;
  }
}

// Job counters of a run to their initial values (exponent range empty, everything else zero).
// A kernel rather than a copy from the host: a host-to-device copy on the run's stream would queue
// on a copy engine behind any track upload in flight and hold the run's kernels back.
__global__ void k_reset_aux(JobAux* aux, int n) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  JobAux a;
  a.e_min = INT_MAX;
  a.e_max = INT_MIN;
  a.flags = 0;
  a.windowed = 0;
  a.kept = 0;
  a.hits = 0;
  a.spheres = 0;
  a.binned = 0;
  a.inbox = 0;
  a.cells = 0;
  aux[j] = a;
}

cudaError_t launch_reset_aux(JobAux* aux, int n, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_reset_aux<<<(n + 255) / 256, 256, 0, s>>>(aux, n);
  return cudaGetLastError();
}

cudaError_t launch_plan(const PlanParams& q, cudaStream_t s) {
  if (q.n_jobs <= 0) return cudaSuccess;
  const int blocks = (q.n_jobs + 255) / 256;
  k_plan_total<<<blocks, 256, 0, s>>>(q);
  k_plan_size<<<blocks, 256, 0, s>>>(q);
  k_plan_scan<<<1, 32, 0, s>>>(q);
  k_plan_write<<<q.n_jobs, 128, 0, s>>>(q);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------
// FP64 issue-rate probe: independent chains of dependent double additions and multiplications
// (8 chains per thread), used to measure the FP64 pipe throughput the fused kernel is bound by.
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_fp64_probe(double* out, int iters, double a, double b) {
  double v[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) v[k] = (double)(threadIdx.x + k) * 1e-3;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = __dadd_rn(__dmul_rn(v[k], a), b);
  }
  double s = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += v[k];
  if (s == 12345.678) out[blockIdx.x] = s;  // keeps the chains alive
}

// One helper's wait for the table of shared unit 0 (unit_table_get), with max_polls sleeps;
// out[0] receives the table it got (-1: the wait ran out).
__global__ void k_unit_wait_probe(FusedParams p, long long max_polls, int* out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) out[0] = unit_table_get(p, 0, max_polls);
}

cudaError_t launch_unit_wait_probe(int* table, int* error_flags, int* out, long long max_polls,
                                   cudaStream_t s) {
  FusedParams p{};
  p.unit_table = table;
  p.error_flags = error_flags;
  k_unit_wait_probe<<<1, 32, 0, s>>>(p, max_polls, out);
  return cudaGetLastError();
}

cudaError_t launch_fp64_probe(double* out, int blocks, int iters, cudaStream_t s) {
  k_fp64_probe<<<blocks, 256, 0, s>>>(out, iters, 0.999999999, 1e-9);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------
// Shared-memory atomic probe: 64-bit atomic additions on a 4096-slot shared array, one CTA of
// 1024 threads per SM (the fused kernel's shape). The lanes of a warp update consecutive slots
// (no bank conflict beyond the two wavefronts a 64-bit warp access needs), so the rate is the
// peak the fused kernel's per-hit and per-sphere shared-memory updates are set against.
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(1024, 1) k_smem_atomic_probe(unsigned long long* out, int iters) {
  __shared__ unsigned long long s[4096];
  for (int i = threadIdx.x; i < 4096; i += blockDim.x) s[i] = 0;
  __syncthreads();
  const unsigned idx = threadIdx.x;  // 1024 distinct slots: lanes of a warp are consecutive
  for (int i = 0; i < iters; ++i) atomicAdd(&s[(idx + (unsigned)i * 1024u) & 4095u], 1ull);
  __syncthreads();
  if (threadIdx.x == 0) out[blockIdx.x] = s[0] + s[4095];
}

cudaError_t launch_smem_atomic_probe(unsigned long long* out, int blocks, int iters, cudaStream_t s) {
  k_smem_atomic_probe<<<blocks, 1024, 0, s>>>(out, iters);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------
// Host-side launch wrappers
// ---------------------------------------------------------------------------------------------
// 32 warps (64 registers each): the kernel is latency-bound, and more resident warps hide more
// of it than longer per-thread blocks would.
constexpr int kFusedThreads = 1024;

// Two shapes of the fused kernel: a 4096-slot sphere table with room for histograms of up to
// 4096 bins in shared memory, or an 8192-slot table when every histogram of the batch has at
// most kSmallHistBins bins.
constexpr int kSmallHistBins = 600;
constexpr int kBigHistBins = 4096;

size_t fused_smem_bytes(int cap, int hist_bins) {
  return (size_t)cap * 26 + (size_t)cap / 8 + (size_t)hist_bins * 28 + 8;
}

cudaError_t launch_prepare(const PrepareParams& p, int64_t n_blocks, bool any_flagged,
                           cudaStream_t s) {
  if (n_blocks <= 0) return cudaSuccess;
  k_prep_count<<<(unsigned)n_blocks, kPrepThreads, 0, s>>>(p);
  k_prep_scan<<<p.n_jobs, 1024, 0, s>>>(p);
  k_prep_write<<<(unsigned)n_blocks, kPrepThreads, 0, s>>>(p);
  k_prep_pad<<<p.n_jobs, kWarpTile, 0, s>>>(p);
  if (any_flagged) k_prep_flag<<<(unsigned)n_blocks, kPrepThreads, 0, s>>>(p);
  return cudaGetLastError();
}

template <bool F32>
static cudaError_t configure_fused_form() {
  cudaError_t e = cudaFuncSetAttribute(k_fused<4096, kFusedThreads, F32>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)fused_smem_bytes(4096, kBigHistBins));
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_fused<8192, kFusedThreads, F32>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)fused_smem_bytes(8192, kSmallHistBins));
}

cudaError_t configure_fused() {
  const cudaError_t e = configure_fused_form<false>();
  return e != cudaSuccess ? e : configure_fused_form<true>();
}

template <bool F32>
static void launch_fused_form(const FusedParams& p, int grid, bool big_table, cudaStream_t s) {
  if (big_table)
    k_fused<8192, kFusedThreads, F32>
        <<<grid, kFusedThreads, fused_smem_bytes(8192, kSmallHistBins), s>>>(p);
  else
    k_fused<4096, kFusedThreads, F32>
        <<<grid, kFusedThreads, fused_smem_bytes(4096, kBigHistBins), s>>>(p);
}

// Picks the kernel shape: the 8192-slot sphere table when the largest histogram of the batch
// fits the remaining shared memory (and table_slots does not ask for 4096), else 4096 slots with
// room for 4096 bins; fills P.smem_hist_bins and P.flush_threshold. P.fp32 picks the FP32
// geometry form.
cudaError_t launch_fused(FusedParams p, int max_nbins, int grid, int table_slots, cudaStream_t s) {
  if (grid <= 0) return cudaSuccess;
  const bool big_table = max_nbins <= kSmallHistBins && table_slots != 4096;
  if (big_table) {
    p.smem_hist_bins = kSmallHistBins;
    p.flush_threshold = 8192 - 4096 - 8192 / 4;  // unused: no window checks on this table
  } else {
    p.smem_hist_bins = kBigHistBins;
    p.flush_threshold = 4096 / 2;
  }
  if (p.fp32) launch_fused_form<true>(p, grid, big_table, s);
  else launch_fused_form<false>(p, grid, big_table, s);
  return cudaGetLastError();
}

int fused_threads() { return kFusedThreads; }

}  // namespace st
