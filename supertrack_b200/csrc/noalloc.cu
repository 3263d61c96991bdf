// st_superimpose_noalloc: one track's superimposition with no device allocation.
//
// Who needs it: callers that must not call cudaMalloc/cudaFree on their path. cudaFree
// synchronises the whole device and stalls every other stream, which a serving thread sharing the
// GPU cannot afford; and frameworks that own all device memory through their own pool leave no
// room for, or forbid, allocations of their plug-ins. The regular entry points grow their arenas
// with cudaMalloc on first use; this one works entirely inside a fixed scratch array that is part
// of the library image.
//
// The scratch below is a file-scope __device__ array: every GPU that loads the library holds it
// (kScratchBytes, about 6.2 MB) until the process exits. Host code cannot pass the symbol
// itself to a kernel (on the host it names a host-side stand-in), so the first call on each
// device, with that device current, resolves its device address with cudaGetSymbolAddress and
// sets the fused kernel's shared-memory attribute; that first call should therefore come before
// any stream capture. Every call shares the one array and re-initialises the parts that must start
// empty (hash tables, counters, flags) itself, so two calls whose work overlapped on the GPU would
// race. Sharing a stream does not prevent that: the host-to-device copies of one call could be
// enqueued between the copies and the kernels of another. Calls are therefore serialised on the
// host: each holds a per-device lock from its first enqueue until its final stream
// synchronisation, and returns only after its work on the GPU has finished.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <mutex>

#include "../../include/supertrack_b200.h"
#include "host_model.h"
#include "st_device.cuh"

namespace st {
cudaError_t launch_prepare(const PrepareParams& p, int64_t n_blocks, bool any_flagged,
                           cudaStream_t s);
cudaError_t configure_fused();
cudaError_t launch_fused(FusedParams p, int max_nbins, int grid, int table_slots, cudaStream_t s);
cudaError_t launch_plan(const PlanParams& q, cudaStream_t s);
}  // namespace st

namespace {

constexpr int64_t kNaMaxDeposits = 16384;       // deposits per track
constexpr int32_t kNaMaxBins = 4096;            // histogram bins
constexpr int64_t kNaMaxOversamples = 65536;    // oversamples per call
constexpr int kNaGrid = 4;                      // resident CTAs (and spill tables)
constexpr uint32_t kNaTableCap = 2 * kNaMaxDeposits;   // spill-table slots (power of two)
constexpr uint32_t kNaCellCap = 2 * kNaMaxDeposits;    // cell-hash slots (power of two)
constexpr int64_t kNaBlocks = kNaMaxDeposits / st::kPrepSlotsPerBlock;
// planning parameters: the regular context's defaults
constexpr int64_t kNaFlagMinKept = 16384;       // window flags only above this many kept deposits
constexpr int64_t kNaItemCost = 1 << 18;        // deposit*oversamples per private work item
constexpr int kNaChunkWindows = 4;              // windows per chunk (shared units; none here)

constexpr size_t al(size_t v) { return (v + 255) / 256 * 256; }

// Byte offsets of every region inside the scratch array.
struct Layout {
  size_t jobs, aux, hists, blk_prefix, blk_count, blk_off;
  size_t pxy, pdz2, pv, pkey, pz;
  size_t cells;
  size_t gkeys, glo, ghi, gused, gcount, pool;
  size_t items, plan, plan_misc, counter, err, edges, units;
  size_t total;
};

constexpr Layout make_layout() {
  Layout L{};
  size_t o = 0;
  L.jobs = o;       o += al(sizeof(st::JobDev));
  L.aux = o;        o += al(sizeof(st::JobAux));
  L.hists = o;      o += al(sizeof(st::HistDev));
  L.blk_prefix = o; o += al(2 * 8);
  L.blk_count = o;  o += al(kNaBlocks * 4);
  L.blk_off = o;    o += al(kNaBlocks * 8);
  L.pxy = o;        o += al(kNaMaxDeposits * 16);

  L.pdz2 = o;       o += al(kNaMaxDeposits * 8);
  L.pv = o;         o += al(kNaMaxDeposits * 16);
  L.pkey = o;       o += al(kNaMaxDeposits * 8);
  L.pz = o;         o += al(kNaMaxDeposits * 8);
  L.cells = o;      o += al((size_t)kNaCellCap * sizeof(st::CellSlot));
  L.gkeys = o;      o += al((size_t)kNaGrid * kNaTableCap * 8);
  L.glo = o;        o += al((size_t)kNaGrid * kNaTableCap * 8);
  L.ghi = o;        o += al((size_t)kNaGrid * kNaTableCap * 8);
  L.gused = o;      o += al((size_t)kNaGrid * kNaTableCap * 4);
  L.gcount = o;     o += al((size_t)kNaGrid * 4);
  L.pool = o;       o += al(4);
  L.items = o;      o += al((size_t)kNaMaxOversamples * sizeof(st::WorkItem));
  L.plan = o;       o += al(sizeof(st::JobPlan));
  L.plan_misc = o;  o += al(16 + 3 * 4 * st::kPlanBuckets);
  L.counter = o;    o += al(16);
  L.err = o;        o += al(16);
  L.edges = o;      o += al((size_t)(kNaMaxBins + 1) * 8);
  L.units = o;      o += al(3 * 4);
  L.total = o;
  return L;
}

constexpr Layout kLayout = make_layout();
constexpr size_t kScratchBytes = kLayout.total;

std::mutex g_setup_mu;
constexpr int kMaxDevices = 64;
unsigned char* g_scratch_addr[kMaxDevices] = {};
// held by a call from its first enqueue to its final synchronisation (one scratch per device)
std::mutex g_call_mu[kMaxDevices];

}  // namespace

// The scratch memory of st_superimpose_noalloc (see the file comment).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

namespace {

// Per-device set-up, once: the device address of the scratch array and the fused kernel's
// shared-memory attribute. Must run with `device` current.
st_status noalloc_setup(int device, unsigned char** base) {
  if (device < 0 || device >= kMaxDevices) return ST_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (!g_scratch_addr[device]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
      cudaGetLastError();
      return ST_ERR_CUDA;
    }
    if (st::configure_fused() != cudaSuccess) {
      cudaGetLastError();
      return ST_ERR_CUDA;
    }
    g_scratch_addr[device] = (unsigned char*)p;
  }
  *base = g_scratch_addr[device];
  return ST_OK;
}

}  // namespace

extern "C" st_status st_superimpose_noalloc(const st_track_view* track, const st_job_desc* desc,
                                            int32_t hist_type, int32_t nbins, float lower,
                                            float upper, int64_t* d_counts, double* d_yfy,
                                            void* stream, st_job_stats* stats_out) {
  // ---- argument checks (sizes beyond the scratch limits are rejected here)
  if (!track || !desc || !d_counts || !d_yfy) return ST_ERR_INVALID_ARGUMENT;
  if (!track->on_device) return ST_ERR_INVALID_ARGUMENT;
  if (track->n > 0 &&
      (((uintptr_t)track->x | (uintptr_t)track->y | (uintptr_t)track->z | (uintptr_t)track->edep) & 7))
    return ST_ERR_INVALID_ARGUMENT;  // read in place as doubles: a misaligned array would fault
  if (track->n < 0 || (track->n > 0 && (!track->x || !track->y || !track->z || !track->edep)))
    return ST_ERR_INVALID_ARGUMENT;
  if (track->n > kNaMaxDeposits) return ST_ERR_CAPACITY;
  if (nbins < 1 || nbins > kNaMaxBins) return ST_ERR_CAPACITY;
  if ((int64_t)desc->n_oversamples > kNaMaxOversamples) return ST_ERR_CAPACITY;
  if (desc->zshift < ST_ZSHIFT_PLUS || desc->zshift > ST_ZSHIFT_NONE) return ST_ERR_INVALID_ARGUMENT;
  st::Geometry g;
  if (st::make_geometry(desc->half_length, desc->sphere_diameter, &g) != 0) return ST_ERR_BAD_GEOMETRY;
  double edges[kNaMaxBins + 1];
  if (hist_type == ST_HIST_LIN) st::LinSpace(lower, upper, nbins, edges);
  else if (hist_type == ST_HIST_LOG) st::LogSpace(lower, upper, nbins, edges);
  else return ST_ERR_BAD_HISTOGRAM;
  for (int i = 0; i <= nbins; ++i)
    if (!std::isfinite(edges[i]) || (i > 0 && !(edges[i] > edges[i - 1]))) return ST_ERR_BAD_HISTOGRAM;

  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) return ST_ERR_NO_DEVICE;
  unsigned char* base = nullptr;
  st_status s = noalloc_setup(device, &base);
  if (s != ST_OK) return s;
  std::lock_guard<std::mutex> call_lock(g_call_mu[device]);
  const cudaStream_t st_ = (cudaStream_t)stream;
  const Layout& L = kLayout;

  // ---- job, histogram and launch descriptors (host stack), copied into the scratch
  const int64_t n = track->n;
  const int64_t n_pad = std::max<int64_t>(256, (n + 255) / 256 * 256);
  st::JobDev D;
  std::memset(&D, 0, sizeof(D));
  D.x = track->x; D.y = track->y; D.z = track->z; D.edep = track->edep;
  D.n = n;
  D.n_pad = n_pad;
  D.prep_off = 0;
  D.HL = g.scoringRegionHalfLength;
  D.L = g.scoringRegionLength;
  D.gSO = g.greatestSphereOffset;
  D.d = g.sphereDiameter;
  D.inv_d = 1.0 / g.sphereDiameter;
  D.r2 = g.sphereRadius * g.sphereRadius;
  D.denom = (2. / 3.) * g.sphereDiameter;
  D.zsh = desc->zshift == ST_ZSHIFT_PLUS ? g.scoringRegionHalfLength
        : desc->zshift == ST_ZSHIFT_MINUS ? -g.scoringRegionHalfLength : 0.0;
  D.xy_keep = desc->shift_track ? 2.0 * g.scoringRegionHalfLength * (1.0 + 0x1p-30)
                                : g.scoringRegionHalfLength;
  D.N = (uint32_t)g.numSpheresLinear;
  D.N2 = (uint64_t)D.N * (uint64_t)D.N;
  D.seed = desc->seed;
  D.track_id = desc->track_id;
  D.n_os = (int32_t)desc->n_oversamples;
  D.shift_track = desc->shift_track ? 1 : 0;
  D.hist = 0;
  D.flagged = (n > 2 * st::kCtaTile && desc->n_oversamples >= 4 && D.N >= 128 &&
               D.N < (1u << (st::kCellBits - 2))) ? 1 : 0;
  D.cell_cap = kNaCellCap;
  D.cell_off = 0;
  const double per_d = (double)n * g.sphereDiameter / (2.0 * g.scoringRegionHalfLength);
  D.cell_nbr8 = (D.flagged && per_d * desc->n_oversamples <= (double)st::kFlagCellsLimit) ? 1 : 0;
  D.cell_size = (D.cell_nbr8 ? 2.0 : 1.0) * g.sphereDiameter * (1.0 + 0x1p-10);
  D.inv_cell = 1.0 / D.cell_size;

  st::JobAux A;
  std::memset(&A, 0, sizeof(A));
  A.e_min = INT_MAX;
  A.e_max = INT_MIN;

  st::HistDev H;
  std::memset(&H, 0, sizeof(H));
  H.edges = (const double*)(base + L.edges);
  H.counts = (unsigned long long*)d_counts;
  H.yfy = d_yfy;
  H.nbins = nbins;
  if (hist_type == ST_HIST_LOG && edges[0] > 0) {
    H.mode = 1;
    H.ca = std::log2(edges[0]);
    H.cb = nbins / (std::log2(edges[nbins]) - std::log2(edges[0]));
  } else {
    H.mode = 0;
    H.ca = edges[0];
    H.cb = nbins / (edges[nbins] - edges[0]);
  }
  const int64_t n_blocks = (n_pad + st::kPrepSlotsPerBlock - 1) / st::kPrepSlotsPerBlock;
  const int64_t blk[2] = {0, n_blocks};

#define NA_CUDA(call)                                        \
  do {                                                       \
    if ((call) != cudaSuccess) { cudaGetLastError(); return ST_ERR_CUDA; } \
  } while (0)

  NA_CUDA(cudaMemcpyAsync(base + L.jobs, &D, sizeof(D), cudaMemcpyHostToDevice, st_));
  NA_CUDA(cudaMemcpyAsync(base + L.aux, &A, sizeof(A), cudaMemcpyHostToDevice, st_));
  NA_CUDA(cudaMemcpyAsync(base + L.hists, &H, sizeof(H), cudaMemcpyHostToDevice, st_));
  NA_CUDA(cudaMemcpyAsync(base + L.blk_prefix, blk, sizeof(blk), cudaMemcpyHostToDevice, st_));
  NA_CUDA(cudaMemcpyAsync(base + L.edges, edges, (size_t)(nbins + 1) * 8, cudaMemcpyHostToDevice, st_));
  // everything that must start empty: hash tables, counters, flags
  NA_CUDA(cudaMemsetAsync(base + L.gkeys, 0xFF, (size_t)kNaGrid * kNaTableCap * 8, st_));
  NA_CUDA(cudaMemsetAsync(base + L.glo, 0, (size_t)kNaGrid * kNaTableCap * 8, st_));
  NA_CUDA(cudaMemsetAsync(base + L.ghi, 0, (size_t)kNaGrid * kNaTableCap * 8, st_));
  NA_CUDA(cudaMemsetAsync(base + L.gcount, 0, (size_t)kNaGrid * 4, st_));
  NA_CUDA(cudaMemsetAsync(base + L.pool, 0, 4, st_));
  NA_CUDA(cudaMemsetAsync(base + L.plan_misc, 0, 16 + 3 * 4 * st::kPlanBuckets, st_));
  NA_CUDA(cudaMemsetAsync(base + L.counter, 0, 16, st_));
  NA_CUDA(cudaMemsetAsync(base + L.err, 0, 16, st_));
  NA_CUDA(cudaMemsetAsync(base + L.units, 0, 8, st_));
  NA_CUDA(cudaMemsetAsync(base + L.units + 8, 0xFF, 4, st_));
  if (D.flagged) {
    NA_CUDA(cudaMemsetAsync(base + L.cells, 0xFF, (size_t)kNaCellCap * sizeof(st::CellSlot), st_));
  }

  st::PrepareParams pp;
  std::memset(&pp, 0, sizeof(pp));
  pp.jobs = (const st::JobDev*)(base + L.jobs);
  pp.aux = (st::JobAux*)(base + L.aux);
  pp.n_jobs = 1;
  pp.blk_prefix = (const int64_t*)(base + L.blk_prefix);
  pp.blk_count = (int32_t*)(base + L.blk_count);
  pp.blk_offset = (int64_t*)(base + L.blk_off);
  pp.cells = (st::CellSlot*)(base + L.cells);
  pp.blk_base = 0;
  pp.PZ = (double*)(base + L.pz);
  pp.PXY = (double2*)(base + L.pxy);

  pp.PDZ2 = (double*)(base + L.pdz2);
  pp.PV = (ulonglong2*)(base + L.pv);
  pp.PKEY = (unsigned long long*)(base + L.pkey);
  // the regular path's default: window flags only above this many kept deposits (a track here
  // keeps at most kNaMaxDeposits, so the scratch path never runs windowed, as the regular path
  // would not for the same track)
  pp.flag_min_kept = kNaFlagMinKept;

  st::PlanParams q;
  std::memset(&q, 0, sizeof(q));
  unsigned char* m = base + L.plan_misc;
  q.jobs = pp.jobs;
  q.aux = pp.aux;
  q.n_jobs = 1;
  q.chunk_windows = kNaChunkWindows;
  q.max_helpers = 1;
  q.grid = kNaGrid;
  q.item_cost = kNaItemCost;
  // deliberate difference from the regular path: share_divisor 0 (left zero) rules out shared
  // units, whose helpers would need a spill table each from a pool sized for kNaGrid CTAs;
  // min_chunks only matters for shared units
  q.total_units = (unsigned long long*)m;
  q.n_items = (int*)(m + 8);
  q.unit_counter = (unsigned int*)(m + 12);
  q.bucket_count = (unsigned int*)(m + 16);
  q.bucket_start = q.bucket_count + st::kPlanBuckets;
  q.bucket_cursor = q.bucket_start + st::kPlanBuckets;
  q.plan = (st::JobPlan*)(base + L.plan);
  q.items = (st::WorkItem*)(base + L.items);
  q.item_cap = kNaMaxOversamples;

  st::FusedParams fp;
  std::memset(&fp, 0, sizeof(fp));
  fp.jobs = pp.jobs;
  fp.aux = pp.aux;
  fp.hists = (const st::HistDev*)(base + L.hists);
  fp.items = q.items;
  fp.n_items = q.n_items;
  fp.work_counter = (unsigned int*)(base + L.counter);
  fp.PXY = pp.PXY; fp.PDZ2 = pp.PDZ2;
  fp.PV = pp.PV; fp.PKEY = pp.PKEY;
  fp.gkeys = (uint64_t*)(base + L.gkeys);
  fp.glo = (unsigned long long*)(base + L.glo);
  fp.ghi = (unsigned long long*)(base + L.ghi);
  fp.gused = (uint32_t*)(base + L.gused);
  fp.gcount = (unsigned int*)(base + L.gcount);
  fp.gcap = kNaTableCap;
  fp.error_flags = (int*)(base + L.err);
  fp.unit_next = (unsigned int*)(base + L.units);
  fp.unit_done = (unsigned int*)(base + L.units + 4);
  fp.unit_table = (int*)(base + L.units + 8);
  fp.pool_bits = (unsigned int*)(base + L.pool);
  fp.chunk_windows = kNaChunkWindows;

  NA_CUDA(st::launch_prepare(pp, n_blocks, D.flagged != 0, st_));
  NA_CUDA(st::launch_plan(q, st_));
  NA_CUDA(st::launch_fused(fp, nbins, kNaGrid, 0, st_));

  // ---- status: job counters and device error flags (host stack destinations)
  st::JobAux out;
  int errflags[4] = {0, 0, 0, 0};
  NA_CUDA(cudaMemcpyAsync(&out, base + L.aux, sizeof(out), cudaMemcpyDeviceToHost, st_));
  NA_CUDA(cudaMemcpyAsync(errflags, base + L.err, sizeof(errflags), cudaMemcpyDeviceToHost, st_));
  NA_CUDA(cudaStreamSynchronize(st_));
#undef NA_CUDA
  if (stats_out) {
    stats_out->hits = out.hits;
    stats_out->spheres = out.spheres;
    stats_out->binned = out.binned;
    stats_out->inbox = out.inbox;
    stats_out->grid_exponent =
        st::choose_grid_exponent(out.e_min, out.e_max, n, out.flags & st::kAuxNonzero);
    stats_out->status = (out.flags & st::kAuxNonfinite) ? ST_ERR_NONFINITE_EDEP : ST_OK;
  }
  // after an error the caller's d_counts / d_yfy may hold part of this call's sums
  if (out.flags & st::kAuxNonfinite) return ST_ERR_NONFINITE_EDEP;
  if (errflags[0] & 1) return ST_ERR_DEVICE_OVERFLOW;       // spill table full
  if (errflags[0] & (4 | 8)) return ST_ERR_DEVICE_WAIT;     // pool exhausted / unit wait expired
  if (errflags[0]) return ST_ERR_DEVICE_OVERFLOW;
  return ST_OK;
}

extern "C" int64_t st_noalloc_scratch_bytes(void) { return (int64_t)kScratchBytes; }
