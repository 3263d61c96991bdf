// Device-side data layout shared by the kernels (vcs_kernels.cu) and the host runtime (capi.cu).
//
// HBM layout of one batch:
//   * input tracks: SoA float64 x, y, z, edep per job (caller memory or the context's arena);
//   * prepared arena (written once per job, read once per oversample): for every job its kept
//     deposits (those that can lie inside the voxel for some shift; in source order, or grouped
//     by cell inside each prepare block) as a padded run of warp tiles of kWarpTile deposits.
//     Lane l of a warp tile owns the kDepPerLane consecutive deposits 4l..4l+3 of the tile,
//     stored "pair-blocked" (prep_slot in vcs_kernels.cu): the pair 4l, 4l+1 at tile slots
//     2l, 2l+1 and the pair 4l+2, 4l+3 at 64+2l, 64+2l+1, so a warp reads one pair per lane with
//     one 16-byte load per lane (512 contiguous bytes):
//       PXY     : {x, y} as loaded, one 16-byte record per slot (padding slots hold NaN so the
//                 box test rejects them); a lane's pair of slots is one 32-byte load
//       PDZ2    : (k_z*d - a_z)^2, +inf when the deposit is outside the box in z
//       PV      : v = edep / ((2/3) d) on the job's fixed-point grid, a 128-bit integer stored
//                 as one 16-byte {low, high} record (one vector load per hit)
//       PKEY    : k_z * N*N (the z part of the sphere key); bit 63 flags boundary deposits
//   * spill tables: one open-addressing table per resident CTA for spheres that do not fit
//     the CTA's shared-memory table (keys, 128-bit accumulators, used-slot list);
//   * histograms: int64 counts and float64 y*f(y) sums per bin, one set per histogram.
#pragma once
#include <stdint.h>
#include "st_core.cuh"

namespace st {

constexpr int kDepPerLane = 4;                  // deposits owned by one lane inside a warp tile
constexpr int kWarpTile = 32 * kDepPerLane;     // deposits per warp tile
constexpr uint64_t kEmptyKey = ~0ull;           // never a valid sphere key (keys < 2^63)

struct JobDev {
  const double* x;
  const double* y;
  const double* z;
  const double* edep;
  int64_t n;          // deposits in the track
  int64_t n_pad;      // n rounded up to a whole number of warp tiles
  int64_t prep_off;   // first slot of this job in the prepared arena
  double HL;          // scoringRegionHalfLength (after lattice fitting)
  double L;           // scoringRegionLength
  double gSO;         // greatestSphereOffset
  double d;           // sphere diameter
  double inv_d;       // RN(1/d), used by the fast lattice-index path
  double r2;          // RN(r*r)
  double denom;       // RN(RN(2/3)*d): lineal-energy denominator
  double zsh;         // z-origin shift added to every z
  double xy_keep;     // |x|, |y| at or beyond this can never be inside the voxel after a shift
  uint64_t N2;        // N*N
  uint64_t seed;
  uint64_t track_id;
  uint32_t N;
  int32_t n_os;
  int32_t shift_track;
  int32_t hist;       // histogram index
  // boundary flags (see k_prep_flag): computed when `flagged`; the cell hash of the job lives in
  // the cell arena at [cell_off, cell_off + cell_cap); its cells have a side slightly above d (27
  // neighbour cells probed per deposit) or, with cell_nbr8, slightly above 2d (eight probed)
  int32_t flagged;
  uint32_t cell_cap;
  int64_t cell_off;
  double cell_size;
  double inv_cell;    // RN(1 / cell_size)
  // FP32 geometry variant: HL', gSO, d, RN(1/d) and r^2 rounded to float (1/d in float)
  float f_HL;
  float f_gSO;
  float f_d;
  float f_inv_d;
  float f_r2;
  int32_t cell_nbr8;
};

// Deposits of a windowed job are processed in windows of consecutive kept deposits: kWindow (two
// warp tiles per warp of the fused kernel's CTA), or twice that for jobs with coarse windows. A
// kept deposit is a boundary deposit when a kept deposit of another window lies within distance d
// of it; the flag travels in bit 63 of its PKEY word (keys are below 2^63).
constexpr unsigned long long kBoundaryBit = 1ull << 63;

// Per-job values produced on the device.
struct JobAux {
  int32_t e_min;          // min ulp exponent over nonzero contributions
  int32_t e_max;          // max ulp exponent over nonzero contributions
  int32_t flags;          // kAuxNonzero | kAuxNonfinite
  int32_t windowed;       // set by k_prep_scan: the job runs with window flags (JobDev::flagged
                          // and more than PrepareParams::flag_min_kept kept deposits)
  long long kept;              // deposits that can be inside the voxel for some shift
  unsigned long long hits;     // in-sphere deposits summed over all oversamples
  unsigned long long spheres;  // (oversample, sphere) pairs with at least one hit
  unsigned long long binned;   // of those, the ones that landed inside the histogram range
  unsigned long long inbox;    // deposit*oversamples inside the voxel after the shift
  unsigned long long cells;    // occupied cells of the boundary-flag hash (windowed jobs)
};
constexpr int kAuxNonzero = 1;
constexpr int kAuxNonfinite = 2;

struct HistDev {
  const double* edges;            // nbins + 1 edges
  unsigned long long* counts;     // nbins
  double* yfy;                    // nbins
  int32_t nbins;
  int32_t mode;                   // bin guess: 0 linear in y, 1 linear in log2(y)
  double ca, cb;                  // guess = (y - ca) * cb  or  (log2(y) - ca) * cb
};

// One unit of work for the persistent kernel: a contiguous block of oversamples of one job.
struct WorkItem {
  int32_t job;
  int32_t os_begin;
  int32_t os_count;
  int32_t unit;       // -1: the CTA does every window of os_begin..+os_count; else a helper of
                      // shared unit `unit` (one oversample of a large job, split into chunks)
};

// One exported sphere: (oversample, key, lineal energy, hit deposits).
struct SphereRecord {
  uint64_t key;
  double y;
  int32_t os;
  int32_t job;
};

struct FusedParams {
  const JobDev* jobs;
  JobAux* aux;
  const HistDev* hists;
  const WorkItem* items;
  const int* n_items;         // written by the planner
  int32_t flush_threshold;    // smem table occupancy that triggers a flush to the spill table
  unsigned int* work_counter; // next item to claim
  const double2* PXY;         // {x, y} per slot (FP32 variant: float2 {x, y} at the slot's index)
  const double* PDZ2;
  const ulonglong2* PV;            // contribution on the job's grid: {low, high} 64-bit words
  const unsigned long long* PKEY;  // k_z * N*N, bit 63 = boundary deposit
  // spill tables: gridDim.x tables of gcap slots each
  uint64_t* gkeys;
  unsigned long long* glo;
  unsigned long long* ghi;
  uint32_t* gused;
  unsigned int* gcount;       // gridDim.x counters
  uint32_t gcap;              // power of two
  int32_t smem_hist_bins;     // histograms with more bins accumulate straight into HBM
  // optional export of every sphere (os, key, y); null when not requested
  SphereRecord* export_buf;
  unsigned long long* export_count;
  unsigned long long export_cap;
  int* error_flags;           // bit 0: spill table full, bit 1: export buffer full,
                              // bit 2: spill-table pool exhausted, bit 3: unit wait gave up
  // shared units (one oversample of a large job, processed in chunks by several CTAs)
  unsigned int* unit_next;    // next chunk to claim
  unsigned int* unit_done;    // chunks finished
  int* unit_table;            // spill table of the unit (-1 none yet, -2 being acquired)
  unsigned int* pool_bits;    // spill tables in use (one bit per table, gridDim.x tables)
  int32_t chunk_windows;      // windows per chunk
  int32_t fp32;               // 1: FP32 geometry variant (float records, float x/y geometry)
};

// One slot of the cell hash used for boundary flags: the cell key (EMPTY when free), the
// smallest window with a deposit in the cell and the bitwise complement of the largest one, so
// that an all-ones fill is the empty state and both bounds are kept with atomicMin. One 16-byte
// load reads a whole slot.
struct __align__(16) CellSlot {
  unsigned long long key;
  unsigned int wmin;
  unsigned int nwmax;
};

struct PrepareParams {
  const JobDev* jobs;
  JobAux* aux;
  int32_t n_jobs;
  int64_t blk_base;           // prepare block of blockIdx.x 0 (jobs and blk_prefix may start
                              // at a later job of the batch; block indices stay batch-wide)
  const int64_t* blk_prefix;  // n_jobs+1 prefix sums of prepare blocks per job
  const int32_t* blk_job;     // batch-wide job index of each prepare block (null: searched in
                              // blk_prefix)
  int32_t job_base;           // batch-wide index of jobs[0]
  int32_t* blk_count;         // kept deposits per prepare block
  int64_t* blk_offset;        // first kept index of each prepare block inside its job
  CellSlot* cells;            // cell arena (flagged jobs)
  double* PZ;                 // z after the z-origin shift (flagged jobs only)
  double2* PXY;               // {x, y} per slot; FP32 variant: float2 {x, y} at the slot's index
  double* PDZ2;               // FP32 variant: float dz^2 at the slot's float index
  ulonglong2* PV;
  unsigned long long* PKEY;
  int32_t fp32;               // 1: records for the FP32 geometry variant
  int64_t flag_min_kept;      // a flagged job runs with window flags only above this many kept
                              // deposits (fewer spheres than that fit the table without them)
  int32_t sort;               // prepare blocks that write their kept deposits grouped by cell
                              // (see k_prep_write): 0 none, 1 those of window-flagged jobs,
                              // 2 all; the others write them in source order
};

// Device-side planning of the fused kernel's work items from the kept deposit counts.
constexpr int kPlanBuckets = 64;
struct JobPlan {
  int32_t items;
  int32_t bucket;
  int32_t unit_base;   // -1: private items
  int32_t blk_os;      // oversamples per private item, or helpers per unit
};
struct PlanParams {
  const JobDev* jobs;
  const JobAux* aux;
  int32_t n_jobs;
  int32_t chunk_windows;
  int32_t max_helpers;
  int32_t grid;
  long long item_cost;
  int32_t share_divisor;             // a job is shared when kept > total / (share_divisor * grid)
  int32_t min_chunks;                // ... and kept > min_chunks chunks; share_divisor 0: never
  unsigned long long* total_units;   // sum of kept * n_os
  unsigned int* bucket_count;        // kPlanBuckets
  unsigned int* bucket_start;        // kPlanBuckets
  unsigned int* bucket_cursor;       // kPlanBuckets
  unsigned int* unit_counter;
  JobPlan* plan;
  WorkItem* items;
  int* n_items;
  long long item_cap;
};

constexpr int kPrepThreads = 256;
constexpr int kPrepSlotsPerBlock = 1024;                // source deposits per prepare block
constexpr int kFusedWarps = 32;                       // warps of the fused kernel's CTA
constexpr int kCtaTile = kFusedWarps * kWarpTile;    // kept deposits of one warp tile per warp
constexpr int kWinTiles = 2;                          // warp tiles per warp in a window
constexpr int kCoarseTiles = 4;                       // ... in a coarse window (dense spheres)
constexpr int kWindow = kWinTiles * kCtaTile;         // kept deposits per window (8192)
// A flagged job uses flag cells of side 2d (eight probes per deposit instead of 27, but more
// deposits flagged, whose spheres then pass through the spill log at every oversample) when its
// deposits per sphere diameter of track length, n * d / (2 HL), times its oversamples are at most
// this (context parameter flag_cells_limit).
constexpr int64_t kFlagCellsLimit = 25000;
constexpr int kCellBits = 21;                         // bits per axis of a cell key

}  // namespace st
