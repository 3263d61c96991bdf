// sm_100a kernels of the VoxelConstrainedSphere superimposition path.
//
//   k_prepare : once per track. z-origin shift, z-box test, the z part of the lattice test
//               (k_z and (k_z*d - a_z)^2, which do not depend on the oversample), the lineal
//               energy contribution v = edep/((2/3)d), the job's fixed-point exponent range, and
//               the lane-blocked relayout of the deposits into the prepared arena.
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

// ---------------------------------------------------------------------------------------------
// Lattice index along one axis: k = llrint(a / d) and k as a double, bit-exact with the IEEE
// quotient. The quotient is first formed as RN(a * RN(1/d)), whose distance to RN(a/d) is below
// |q| * 2^-51.2; only when q lies within |q| * 2^-50 of a half-integer can the two round to
// different integers, and then the correctly rounded division decides.
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ void lattice_index(double a, double d, double inv_d, uint32_t& k,
                                              double& kd) {
  const double kMagic = 0x1.8p52;  // adding it rounds |q| < 2^51 to an integer (ties to even)
  const double q = st_dmul(a, inv_d);
  double t = st_dadd(q, kMagic);
  kd = st_dsub(t, kMagic);
  const double f = st_dsub(q, kd);  // exact: q minus its nearest integer
  if (fabs(st_dsub(fabs(f), 0.5)) <= st_dmul(fabs(q), 0x1p-50)) {
    kd = rint(__ddiv_rn(a, d));
    t = st_dadd(kd, kMagic);
  }
  k = (uint32_t)__double2loint(t);
}

// ---------------------------------------------------------------------------------------------
// k_prepare
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kPrepThreads) k_prepare(PrepareParams p) {
  const int64_t b = blockIdx.x;
  int lo = 0, hi = p.n_jobs;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (p.blk_prefix[mid] <= b) lo = mid; else hi = mid;
  }
  const int j = lo;
  const JobDev J = p.jobs[j];
  const int64_t local0 = (b - p.blk_prefix[j]) * (int64_t)kPrepSlotsPerBlock;
  int emin = INT_MAX, emax = INT_MIN, flags = 0;
  const double nan = __longlong_as_double(0x7FF8000000000000ll);
  const double inf = __longlong_as_double(0x7FF0000000000000ll);
  for (int s = threadIdx.x; s < kPrepSlotsPerBlock; s += kPrepThreads) {
    const int64_t t = local0 + s;
    if (t >= J.n_pad) break;
    const int64_t w = t / kWarpTile;
    const int rem = (int)(t - w * kWarpTile);
    const int pp = rem >> 5, lane = rem & 31;
    const int64_t i = w * kWarpTile + lane * kDepPerLane + pp;
    double px = nan, py = nan, dz2 = inf, v = 0.0;
    uint32_t kz = 0;
    if (i < J.n) {
      px = J.x[i];
      py = J.y[i];
      const double z1 = st_dadd(J.z[i], J.zsh);
      if (fabs(z1) < J.HL) {
        const double az = st_dsub(z1, J.gSO);
        const double kd = rint(__ddiv_rn(az, J.d));
        const double dz = st_dsub(st_dmul(kd, J.d), az);
        dz2 = st_dmul(dz, dz);
        kz = (uint32_t)(long long)kd;
      }
      v = __ddiv_rn(J.edep[i], J.denom);
      if (!isfinite(v)) {
        flags |= kAuxNonfinite;
      } else if (v != 0.0) {
        flags |= kAuxNonzero;
        const int ex = ulp_exponent(v);
        emin = min(emin, ex);
        emax = max(emax, ex);
      }
    }
    const int64_t dst = J.prep_off + t;
    p.PX[dst] = px;
    p.PY[dst] = py;
    p.PDZ2[dst] = dz2;
    p.PV[dst] = v;
    p.PKZ[dst] = kz;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    emin = min(emin, __shfl_xor_sync(0xffffffffu, emin, o));
    emax = max(emax, __shfl_xor_sync(0xffffffffu, emax, o));
    flags |= __shfl_xor_sync(0xffffffffu, flags, o);
  }
  if ((threadIdx.x & 31) == 0 && flags) {
    atomicOr(&p.aux[j].flags, flags);
    if (flags & kAuxNonzero) {
      atomicMin(&p.aux[j].e_min, emin);
      atomicMax(&p.aux[j].e_max, emax);
    }
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

template <int CAP>
struct SmemTable {
  uint64_t* keys;
  unsigned long long* lo;
  unsigned long long* hi;
  uint16_t* used;
};

struct CtaState {
  int item;
  int tcount;
  int spilled;
};

// Adds one sphere contribution to the CTA's shared-memory table, or to the spill table when the
// shared table is at its load limit.
template <int CAP>
__device__ __forceinline__ void sphere_add(const SmemTable<CAP>& T, CtaState* cs,
                                           const FusedParams& P, uint64_t* gk,
                                           unsigned long long* glo, unsigned long long* ghi,
                                           uint32_t* gused, unsigned int* gcnt, uint64_t key,
                                           uint64_t lo, uint64_t hi) {
  constexpr int kHardLimit = (CAP * 3) / 4;
  if (*(volatile int*)&cs->tcount < kHardLimit) {
    uint32_t h = slot_hash(key, CAP - 1);
#pragma unroll 1
    for (int probe = 0; probe < 32; ++probe) {
      const uint64_t k = ((volatile uint64_t*)T.keys)[h];
      if (k == key) { acc_add(&T.lo[h], &T.hi[h], lo, hi); return; }
      if (k == kEmptyKey) {
        const uint64_t old = atomicCAS((unsigned long long*)&T.keys[h], kEmptyKey, key);
        if (old == kEmptyKey) {
          const int idx = atomicAdd(&cs->tcount, 1);
          T.used[idx] = (uint16_t)h;
          acc_add(&T.lo[h], &T.hi[h], lo, hi);
          return;
        }
        if (old == key) { acc_add(&T.lo[h], &T.hi[h], lo, hi); return; }
      }
      h = (h + 1) & (CAP - 1);
    }
  }
  *(volatile int*)&cs->spilled = 1;
  if (!gtable_add(gk, glo, ghi, gused, gcnt, P.gcap, key, lo, hi)) atomicOr(P.error_flags, 1);
}

struct BinContext {
  const double* edges;
  unsigned long long* gcounts;
  double* gyfy;
  unsigned int* hcount;   // null: accumulate straight into HBM
  double* hyfy;
  int nbins;
  int E0;
  int os;
  int job;
};

__device__ __forceinline__ void bin_sphere(const BinContext& B, const FusedParams& P,
                                           uint64_t key, uint64_t lo, uint64_t hi,
                                           unsigned long long& spheres,
                                           unsigned long long& binned) {
  const double y = from_fixed(lo, hi, B.E0);
  ++spheres;
  int b;
  {
    // HistogramRange: edges[b] <= y < edges[b+1]
    const double* e = B.edges;
    if (!(y >= __ldg(&e[0])) || !(y < __ldg(&e[B.nbins]))) {
      b = -1;
    } else {
      int l = 0, h = B.nbins;
      while (h - l > 1) {
        const int m = (l + h) >> 1;
        if (__ldg(&e[m]) <= y) l = m; else h = m;
      }
      b = l;
    }
  }
  if (b >= 0) {
    ++binned;
    if (B.hcount) {
      atomicAdd(&B.hcount[b], 1u);
      atomicAdd(&B.hyfy[b], y);
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
      r.os = B.os;
      r.job = B.job;
      P.export_buf[idx] = r;
    } else {
      atomicOr(P.error_flags, 2);
    }
  }
}

// ---------------------------------------------------------------------------------------------
// k_fused
// ---------------------------------------------------------------------------------------------
template <int CAP, int THREADS>
__global__ void __launch_bounds__(THREADS, 1) k_fused(FusedParams P) {
  static_assert(CAP <= 65536, "used-slot list stores 16-bit slot indices");
  constexpr int kWarps = THREADS / 32;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ CtaState cs;

  SmemTable<CAP> T;
  T.keys = reinterpret_cast<uint64_t*>(smem_raw);
  T.lo = reinterpret_cast<unsigned long long*>(T.keys + CAP);
  T.hi = T.lo + CAP;
  double* hyfy = reinterpret_cast<double*>(T.hi + CAP);
  unsigned int* hcount = reinterpret_cast<unsigned int*>(hyfy + P.smem_hist_bins);
  T.used = reinterpret_cast<uint16_t*>(hcount + P.smem_hist_bins);

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  uint64_t* gk = P.gkeys + (size_t)blockIdx.x * P.gcap;
  unsigned long long* glo = P.glo + (size_t)blockIdx.x * P.gcap;
  unsigned long long* ghi = P.ghi + (size_t)blockIdx.x * P.gcap;
  uint32_t* gused = P.gused + (size_t)blockIdx.x * P.gcap;
  unsigned int* gcnt = P.gcount + blockIdx.x;

  for (int i = tid; i < CAP; i += THREADS) { T.keys[i] = kEmptyKey; T.lo[i] = 0; T.hi[i] = 0; }
  for (int i = tid; i < P.smem_hist_bins; i += THREADS) { hcount[i] = 0; hyfy[i] = 0.0; }
  if (tid == 0) { cs.tcount = 0; cs.spilled = 0; }
  __syncthreads();

  for (;;) {
    if (tid == 0) cs.item = (int)atomicAdd(P.work_counter, 1u);
    __syncthreads();
    const int it = cs.item;
    __syncthreads();
    if (it >= P.n_items) break;

    const WorkItem W = P.items[it];
    const JobDev J = P.jobs[W.job];
    const JobAux A = P.aux[W.job];
    if (A.flags & kAuxNonfinite) continue;  // rejected job: contributes nothing, host reports it
    const HistDev H = P.hists[J.hist];
    const int E0 = choose_grid_exponent(A.e_min, A.e_max, J.n, A.flags & kAuxNonzero);

    BinContext B;
    B.edges = H.edges;
    B.gcounts = H.counts;
    B.gyfy = H.yfy;
    B.nbins = H.nbins;
    B.E0 = E0;
    B.job = W.job;
    const bool smem_hist = H.nbins <= P.smem_hist_bins;
    B.hcount = smem_hist ? hcount : nullptr;
    B.hyfy = smem_hist ? hyfy : nullptr;

    const int64_t n_wt = J.n_pad / kWarpTile;
    unsigned long long hits = 0, spheres = 0, binned = 0, inbox = 0;
    const double kInf = __longlong_as_double(0x7FF0000000000000ll);

    for (int os = W.os_begin; os < W.os_begin + W.os_count; ++os) {
      float ux, uy;
      shift_uniforms(J.seed, J.track_id, (uint32_t)os, J.shift_track, &ux, &uy);
      const double sx = shift_from_uniform(ux, J.L, J.HL);
      const double sy = shift_from_uniform(uy, J.L, J.HL);
      B.os = os;

      for (int64_t wt0 = 0; wt0 < n_wt; wt0 += kWarps) {
        const int64_t w = wt0 + warp;
        if (w < n_wt) {
          const int64_t tb = J.prep_off + w * kWarpTile + lane;
          double xv[kDepPerLane], yv[kDepPerLane], dv[kDepPerLane];
#pragma unroll
          for (int p = 0; p < kDepPerLane; ++p) {
            xv[p] = __ldg(&P.PX[tb + p * 32]);
            yv[p] = __ldg(&P.PY[tb + p * 32]);
            dv[p] = __ldg(&P.PDZ2[tb + p * 32]);
          }
          uint32_t kxv[kDepPerLane], kyv[kDepPerLane];
          unsigned hitmask = 0, boxmask = 0;
#pragma unroll
          for (int p = 0; p < kDepPerLane; ++p) {
            const double x1 = st_dadd(xv[p], sx);
            const double y1 = st_dadd(yv[p], sy);
            const double ax = st_dsub(x1, J.gSO);
            const double ay = st_dsub(y1, J.gSO);
            double kdx, kdy;
            lattice_index(ax, J.d, J.inv_d, kxv[p], kdx);
            lattice_index(ay, J.d, J.inv_d, kyv[p], kdy);
            const double ddx = st_dsub(st_dmul(kdx, J.d), ax);
            const double ddy = st_dsub(st_dmul(kdy, J.d), ay);
            const double dist = st_dadd(st_dadd(st_dmul(ddx, ddx), st_dmul(ddy, ddy)), dv[p]);
            const bool inbox = fabs(x1) < J.HL && fabs(y1) < J.HL && dv[p] != kInf;
            if (inbox) boxmask |= 1u << p;
            if (inbox && dist <= J.r2) hitmask |= 1u << p;
          }
          hits += __popc(hitmask);
          inbox += __popc(boxmask);
          uint64_t rkey = kEmptyKey, rlo = 0, rhi = 0;
#pragma unroll
          for (int p = 0; p < kDepPerLane; ++p) {
            if (hitmask & (1u << p)) {
              const int64_t idx = tb + p * 32;
              const double v = __ldg(&P.PV[idx]);
              const uint32_t kz = __ldg(&P.PKZ[idx]);
              const uint64_t key =
                  (uint64_t)kxv[p] + (uint64_t)kyv[p] * J.N + (uint64_t)kz * J.N2;
              uint64_t lo, hi;
              to_fixed(v, E0, &lo, &hi);
              if (key == rkey) {
                add128(rlo, rhi, lo, hi);
              } else {
                if (rkey != kEmptyKey) sphere_add<CAP>(T, &cs, P, gk, glo, ghi, gused, gcnt, rkey, rlo, rhi);
                rkey = key; rlo = lo; rhi = hi;
              }
            }
          }
          if (rkey != kEmptyKey) sphere_add<CAP>(T, &cs, P, gk, glo, ghi, gused, gcnt, rkey, rlo, rhi);
        }
        if (wt0 + kWarps < n_wt) {
          __syncthreads();
          if (cs.tcount > P.flush_threshold) {
            const int cnt = cs.tcount;
            for (int i = tid; i < cnt; i += THREADS) {
              const uint32_t h = T.used[i];
              if (!gtable_add(gk, glo, ghi, gused, gcnt, P.gcap, T.keys[h], T.lo[h], T.hi[h]))
                atomicOr(P.error_flags, 1);
              T.keys[h] = kEmptyKey; T.lo[h] = 0; T.hi[h] = 0;
            }
            __syncthreads();
            if (tid == 0) { cs.tcount = 0; cs.spilled = 1; }
            __syncthreads();
          }
        }
      }
      __syncthreads();

      // ---- reduce-by-key complete for this oversample: bin every sphere
      const int cnt = cs.tcount;
      if (cs.spilled) {
        for (int i = tid; i < cnt; i += THREADS) {
          const uint32_t h = T.used[i];
          if (!gtable_add(gk, glo, ghi, gused, gcnt, P.gcap, T.keys[h], T.lo[h], T.hi[h]))
            atomicOr(P.error_flags, 1);
          T.keys[h] = kEmptyKey; T.lo[h] = 0; T.hi[h] = 0;
        }
        __syncthreads();
        const unsigned gc = __ldcg(gcnt);
        for (unsigned i = tid; i < gc; i += THREADS) {
          const uint32_t h = __ldcg(&gused[i]);
          const uint64_t key = __ldcg((const unsigned long long*)&gk[h]);
          const uint64_t lo = __ldcg(&glo[h]);
          const uint64_t hi = __ldcg(&ghi[h]);
          bin_sphere(B, P, key, lo, hi, spheres, binned);
          gk[h] = kEmptyKey; glo[h] = 0; ghi[h] = 0;
        }
        __syncthreads();
        if (tid == 0) *gcnt = 0;
      } else {
        for (int i = tid; i < cnt; i += THREADS) {
          const uint32_t h = T.used[i];
          bin_sphere(B, P, T.keys[h], T.lo[h], T.hi[h], spheres, binned);
          T.keys[h] = kEmptyKey; T.lo[h] = 0; T.hi[h] = 0;
        }
      }
      __syncthreads();
      if (tid == 0) { cs.tcount = 0; cs.spilled = 0; }
      __syncthreads();
    }

    // ---- per-item flush of the shared-memory histogram and the job statistics
    if (smem_hist) {
      for (int b = tid; b < H.nbins; b += THREADS) {
        const unsigned c = hcount[b];
        if (c) {
          atomicAdd(&H.counts[b], (unsigned long long)c);
          atomicAdd(&H.yfy[b], hyfy[b]);
          hcount[b] = 0;
          hyfy[b] = 0.0;
        }
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      hits += __shfl_xor_sync(0xffffffffu, hits, o);
      spheres += __shfl_xor_sync(0xffffffffu, spheres, o);
      binned += __shfl_xor_sync(0xffffffffu, binned, o);
      inbox += __shfl_xor_sync(0xffffffffu, inbox, o);
    }
    if (lane == 0) {
      if (hits) atomicAdd(&P.aux[W.job].hits, hits);
      if (spheres) atomicAdd(&P.aux[W.job].spheres, spheres);
      if (binned) atomicAdd(&P.aux[W.job].binned, binned);
      if (inbox) atomicAdd(&P.aux[W.job].inbox, inbox);
    }
    __syncthreads();
  }
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

cudaError_t launch_fp64_probe(double* out, int blocks, int iters, cudaStream_t s) {
  k_fp64_probe<<<blocks, 256, 0, s>>>(out, iters, 0.999999999, 1e-9);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------
// Host-side launch wrappers
// ---------------------------------------------------------------------------------------------
constexpr int kFusedThreads = 512;
constexpr int kSmemCap = 4096;

size_t fused_smem_bytes(int smem_hist_bins) {
  return (size_t)kSmemCap * 24 + (size_t)smem_hist_bins * 12 + (size_t)kSmemCap * 2;
}

cudaError_t launch_prepare(const PrepareParams& p, int64_t n_blocks, cudaStream_t s) {
  if (n_blocks <= 0) return cudaSuccess;
  k_prepare<<<(unsigned)n_blocks, kPrepThreads, 0, s>>>(p);
  return cudaGetLastError();
}

cudaError_t configure_fused(int smem_hist_bins) {
  return cudaFuncSetAttribute(k_fused<kSmemCap, kFusedThreads>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)fused_smem_bytes(smem_hist_bins));
}

cudaError_t launch_fused(const FusedParams& p, int grid, cudaStream_t s) {
  if (grid <= 0) return cudaSuccess;
  k_fused<kSmemCap, kFusedThreads>
      <<<grid, kFusedThreads, fused_smem_bytes(p.smem_hist_bins), s>>>(p);
  return cudaGetLastError();
}

int fused_threads() { return kFusedThreads; }

}  // namespace st
