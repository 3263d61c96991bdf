// Host/device building blocks of the VoxelConstrainedSphere superimposition path.
//
// Everything here is compiled twice by nvcc (host and sm_100a device) so that the host-side
// exports (geometry, shift export, fixed-point helpers) and the kernels share one definition.
// Floating-point expressions that decide hit membership or bin placement are written with
// explicitly rounded operations (st_dadd/st_dsub/st_dmul); the host side is compiled with
// -ffp-contract=off and the device side with --fmad=false, so no a*b+c is ever fused.
#pragma once
#include <stdint.h>
#include <math.h>

#ifdef __CUDACC__
#define ST_HD __host__ __device__ __forceinline__
#else
#define ST_HD inline
#endif

namespace st {

// ---------------------------------------------------------------------------------------------
// Correctly rounded (round-to-nearest-even) primitive operations, never contracted.
// ---------------------------------------------------------------------------------------------
ST_HD double st_dadd(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dadd_rn(a, b);
#else
  return a + b;
#endif
}
ST_HD double st_dsub(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dsub_rn(a, b);
#else
  return a - b;
#endif
}
ST_HD double st_dmul(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dmul_rn(a, b);
#else
  return a * b;
#endif
}

// ---------------------------------------------------------------------------------------------
// Lattice geometry. Field meaning follows SphericalGeometry (reference
// include/Simulation_method/VoxelConstrainedSphereMethod/SphericalGeometry.cuh:8-23); the
// construction rule is SphericalGeometry.cu:7-32: N = floor(2*HL/d), the voxel shrinks to N*d,
// gSO = -HL' + r, and a sphere larger than the voxel turns the voxel into that one sphere.
// ---------------------------------------------------------------------------------------------
struct Geometry {
  double scoringRegionLength;      // L  = N*d
  double scoringRegionHalfLength;  // HL' = L/2
  double greatestSphereOffset;     // gSO = -HL' + r
  int32_t numSpheresLinear;        // N
  int32_t reserved;
  double sphereDiameter;           // d
  double sphereRadius;             // r = d/2
};

// Largest lattice side accepted: keeps N^3 < 2^63 so the 64-bit sphere key never wraps and the
// all-ones key stays free as the empty-slot marker of the hash tables.
constexpr int32_t kMaxSpheresLinear = 2097151;  // 2^21 - 1

// Returns 0 on success, nonzero when the inputs cannot form a lattice (d <= 0, non-finite
// values, or a lattice side beyond kMaxSpheresLinear).
inline int make_geometry(double half_length, double sphere_diameter, Geometry* g) {
  if (!(sphere_diameter > 0.0) || !isfinite(sphere_diameter) || !isfinite(half_length)) return 1;
  g->scoringRegionHalfLength = half_length;
  g->sphereDiameter = sphere_diameter;
  g->sphereRadius = sphere_diameter / 2;
  double nd = floor((half_length * 2) / sphere_diameter);
  if (nd > (double)kMaxSpheresLinear) return 2;
  if (nd < -2147483648.0) nd = -2147483648.0;  // only reached for negative half lengths
  g->numSpheresLinear = (int32_t)nd;
  g->scoringRegionLength = g->numSpheresLinear * sphere_diameter;
  g->scoringRegionHalfLength = g->scoringRegionLength / 2;
  g->greatestSphereOffset = -g->scoringRegionHalfLength + g->sphereRadius;
  if (g->sphereRadius > g->scoringRegionHalfLength) {
    g->scoringRegionHalfLength = g->sphereRadius;
    g->numSpheresLinear = 1;
    g->scoringRegionLength = g->scoringRegionHalfLength * 2;
    g->greatestSphereOffset = -g->scoringRegionHalfLength + g->sphereRadius;
  }
  g->reserved = 0;
  return 0;
}

// ---------------------------------------------------------------------------------------------
// Philox4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw, "Parallel random numbers:
// as easy as 1, 2, 3", SC'11): 10 rounds of two 32x32->64 multiplies with the published
// multipliers and Weyl key increments.
// ---------------------------------------------------------------------------------------------
ST_HD uint32_t st_mulhi32(uint32_t a, uint32_t b) {
#ifdef __CUDA_ARCH__
  return __umulhi(a, b);
#else
  return (uint32_t)(((uint64_t)a * (uint64_t)b) >> 32);
#endif
}

ST_HD void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r > 0) { k0 += W0; k1 += W1; }
    const uint32_t hi0 = st_mulhi32(M0, c[0]), lo0 = M0 * c[0];
    const uint32_t hi1 = st_mulhi32(M1, c[2]), lo1 = M1 * c[2];
    const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
  }
}

// Stream constant placed in the fourth counter word of every shift draw ("SHFT").
constexpr uint32_t kShiftStream = 0x53484654u;

// A uniform float in (0, 1]: 24 random bits, +1, times 2^-24 (every value exactly representable).
ST_HD float u01_from_bits(uint32_t r) { return (float)((r >> 8) + 1u) * 5.9604644775390625e-08f; }

// The two uniforms of oversample `os` of track (seed, track_id). The reference draws 2*N_os
// uniforms in (0,1] per task and uses the pair (2*os, 2*os+1)
// (VoxelConstrainedSphereMethod.cu:61-83, :176-177); here the pair is a pure function of
// (seed, track_id, os), so any oversample can be regenerated or exported on its own.
ST_HD void shift_uniforms(uint64_t seed, uint64_t track_id, uint32_t os, int shift_track,
                          float* ux, float* uy) {
  if (!shift_track) {  // ShiftTrack=false fills the uniforms with 0.5 (SetRandomValsToHalf)
    *ux = 0.5f; *uy = 0.5f;
    return;
  }
  uint32_t c[4] = {os, (uint32_t)track_id, (uint32_t)(track_id >> 32), kShiftStream};
  philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  *ux = u01_from_bits(c[0]);
  *uy = u01_from_bits(c[1]);
}

// sx = u*L - HL' in double, each operation rounded on its own (VoxelConstrainedSphereMethod.cu:176-177).
ST_HD double shift_from_uniform(float u, double L, double HL) {
  return st_dsub(st_dmul((double)u, L), HL);
}

// ---------------------------------------------------------------------------------------------
// Exact per-sphere energy accumulation.
//
// Each lineal-energy contribution v = edep/((2/3)d) is a double m*2^e (m < 2^53). A job fixes
// one grid exponent E0 (the smallest e among its nonzero contributions, raised only if the
// job's dynamic range would not fit) and every contribution becomes the integer m*2^(e-E0),
// held as a 128-bit two's-complement value (lo, hi). Integer sums are associative, so the
// per-sphere total does not depend on the order or grouping in which hits are combined; the
// sphere's lineal energy is that exact total rounded once to double.
// ---------------------------------------------------------------------------------------------

// Exponent of the unit in the last place of a finite nonzero double.
ST_HD int ulp_exponent(double v) {
#ifdef __CUDA_ARCH__
  const uint64_t bits = (uint64_t)__double_as_longlong(v);
#else
  union { double d; uint64_t u; } cv; cv.d = v; const uint64_t bits = cv.u;
#endif
  const int biased = (int)((bits >> 52) & 0x7FF);
  return biased ? biased - 1075 : -1074;
}

ST_HD int bit_length_u64(uint64_t x) {
  int n = 0;
  while (x) { ++n; x >>= 1; }
  return n;
}

// e_min/e_max: min and max ulp exponents over the job's nonzero contributions; n: the number
// of contributions that can meet in one sphere (bounded by the job's deposit count).
// The bound keeps |sum| < 2^127, the signed range of the accumulator.
ST_HD int choose_grid_exponent(int e_min, int e_max, int64_t n, int any_nonzero) {
  if (!any_nonzero) return 0;
  const int need = e_max + 53 + bit_length_u64((uint64_t)(n > 0 ? n : 1)) - 127;
  return e_min > need ? e_min : need;
}

// Converts v to the fixed-point grid 2^E0 (round-to-nearest-even when v is finer than the grid,
// which only happens for jobs whose dynamic range exceeded the accumulator).
ST_HD void to_fixed(double v, int E0, uint64_t* lo_out, uint64_t* hi_out) {
#ifdef __CUDA_ARCH__
  const uint64_t bits = (uint64_t)__double_as_longlong(v);
#else
  union { double d; uint64_t u; } cv; cv.d = v; const uint64_t bits = cv.u;
#endif
  const int biased = (int)((bits >> 52) & 0x7FF);
  uint64_t m = bits & 0x000FFFFFFFFFFFFFull;
  int e;
  if (biased) { m |= 0x0010000000000000ull; e = biased - 1075; } else { e = -1074; }
  uint64_t lo = 0, hi = 0;
  if (m != 0) {
    const int s = e - E0;
    if (s >= 0) {
      if (s == 0) { lo = m; }
      else if (s < 64) { lo = m << s; hi = m >> (64 - s); }
      else if (s < 128) { hi = m << (s - 64); }
    } else {
      const int rs = -s;
      if (rs <= 53) {
        const uint64_t q = m >> rs;
        const uint64_t rem = m & ((1ull << rs) - 1);
        const uint64_t half = 1ull << (rs - 1);
        lo = q + ((rem > half || (rem == half && (q & 1))) ? 1 : 0);
      }
    }
    if (bits >> 63) {  // negate the 128-bit value
      lo = ~lo + 1;
      hi = ~hi + (lo == 0 ? 1 : 0);
    }
  }
  *lo_out = lo;
  *hi_out = hi;
}

ST_HD int clz64(uint64_t x) {
#ifdef __CUDA_ARCH__
  return __clzll((long long)x);
#else
  return x ? __builtin_clzll(x) : 64;
#endif
}

ST_HD double u64_to_double_rn(uint64_t x) {
#ifdef __CUDA_ARCH__
  return __ull2double_rn(x);
#else
  return (double)x;  // x86-64 conversion honours the (default) round-to-nearest mode
#endif
}

// x * 2^e for a power-of-two scale, exact unless the result leaves the normal range.
ST_HD double scale_pow2(double x, int e) {
  while (e > 1000) { x = st_dmul(x, 0x1p1000); e -= 1000; }
  while (e < -1000) { x = st_dmul(x, 0x1p-1000); e += 1000; }
#ifdef __CUDA_ARCH__
  const double p = __longlong_as_double((long long)(uint64_t)(e + 1023) << 52);
#else
  union { uint64_t u; double d; } cv; cv.u = (uint64_t)(e + 1023) << 52; const double p = cv.d;
#endif
  return st_dmul(x, p);
}

// The 128-bit grid value (lo, hi) times 2^E0, rounded once to the nearest double (ties to even).
ST_HD double from_fixed(uint64_t lo, uint64_t hi, int E0) {
  const bool neg = (int64_t)hi < 0;
  if (neg) { lo = ~lo + 1; hi = ~hi + (lo == 0 ? 1 : 0); }
  double mag;
  if (hi == 0) {
    mag = u64_to_double_rn(lo);
  } else {
    const int sh = 64 - clz64(hi);                 // 1..64 bits live in hi
    uint64_t top = (sh == 64) ? hi : ((hi << (64 - sh)) | (lo >> sh));
    const uint64_t dropped = (sh == 64) ? lo : (lo & ((1ull << sh) - 1));
    if (dropped) top |= 1;                         // sticky bit below the rounding position
    mag = scale_pow2(u64_to_double_rn(top), sh);
  }
  mag = scale_pow2(mag, E0);
  return neg ? -mag : mag;
}

// ---------------------------------------------------------------------------------------------
// Histogram binning with the HistogramRange rule used by the reference
// (Histogram.cu:158): bin b iff edges[b] <= y < edges[b+1]; out of range and NaN are dropped.
// ---------------------------------------------------------------------------------------------
ST_HD int find_bin(const double* edges, int nbins, double y) {
  if (!(y >= edges[0]) || !(y < edges[nbins])) return -1;
  int lo = 0, hi = nbins;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (edges[mid] <= y) lo = mid; else hi = mid;
  }
  return lo;
}

}  // namespace st
