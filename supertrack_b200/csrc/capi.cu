// Host runtime behind the C ABI (include/supertrack_b200.h): contexts, device arenas,
// histograms, job queues and the launches of the prepare and fused kernels.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/supertrack_b200.h"
#include "host_model.h"
#include "st_device.cuh"

namespace st {
cudaError_t launch_prepare(const PrepareParams& p, int64_t n_blocks, bool any_flagged,
                           cudaStream_t s);
cudaError_t configure_fused();
cudaError_t launch_fused(FusedParams p, int max_nbins, int grid, int table_slots, cudaStream_t s);
cudaError_t launch_fp64_probe(double* out, int blocks, int iters, cudaStream_t s);
cudaError_t launch_unit_wait_probe(int* table, int* error_flags, int* out, long long max_polls,
                                   cudaStream_t s);
cudaError_t launch_smem_atomic_probe(unsigned long long* out, int blocks, int iters, cudaStream_t s);
cudaError_t launch_plan(const PlanParams& q, cudaStream_t s);
cudaError_t launch_reset_aux(JobAux* aux, int n, cudaStream_t s);
}  // namespace st

namespace {

using st::HistDev;
using st::JobAux;
using st::JobDev;
using st::WorkItem;

// Host time spent allocating (and freeing) device and pinned memory in the calling thread,
// reported per run through st_ctx_get_param.
thread_local double g_alloc_us = 0;
thread_local int64_t g_allocs = 0;

double now_us() {
  return std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

// Grow-only device buffer. A buffer that has to grow again takes at least half as much more, so
// that contexts running batches of changing size (serving) reallocate rarely: cudaFree waits
// for the whole device.
cudaError_t ensure(DevBuf& b, size_t bytes) {
  if (bytes == 0) bytes = 16;
  if (b.bytes >= bytes) return cudaSuccess;
  if (b.bytes > 0) bytes = std::max(bytes, b.bytes + b.bytes / 2);
  const double t0 = now_us();
  struct Tally {
    double t0;
    ~Tally() { g_alloc_us += now_us() - t0; ++g_allocs; }
  } tally{t0};
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.bytes = 0;
  cudaError_t e = cudaMalloc(&b.p, bytes);
  if (e != cudaSuccess) { b.p = nullptr; return e; }
  b.bytes = bytes;
  return cudaSuccess;
}

// Page-locked host staging for the per-run tables: copies from pageable memory would make the
// host wait until the stream reaches them, i.e. behind whatever the GPU runs before this stream's
// work gets SMs. Grow-only (by half again), freed with the context.
struct PinnedBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

cudaError_t ensure_pinned(PinnedBuf& b, size_t bytes) {
  if (b.bytes >= bytes) return cudaSuccess;
  const size_t cap = std::max(bytes, b.bytes + b.bytes / 2);
  struct Tally {
    double t0;
    ~Tally() { g_alloc_us += now_us() - t0; ++g_allocs; }
  } tally{now_us()};
  if (b.p) cudaFreeHost(b.p);
  b.p = nullptr;
  b.bytes = 0;
  cudaError_t e = cudaMallocHost(&b.p, cap);
  if (e != cudaSuccess) { b.p = nullptr; return e; }
  b.bytes = cap;
  return cudaSuccess;
}

size_t align256(size_t v) { return (v + 255) / 256 * 256; }

void release(DevBuf& b) {
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.bytes = 0;
}

struct HistHost {
  int32_t type = 0, nbins = 0;
  float lower = 0, upper = 0;
  std::vector<double> edges;
  int64_t off = 0;        // first bin in the context's count/yfy arenas
  int64_t eoff = 0;       // first edge in the context's edge arena
};

struct JobHost {
  st_track_view track{};
  st_job_desc desc{};
  st::Geometry g{};
  int64_t n_pad = 0;
  int64_t prep_off = 0;
  int64_t arena_off = -1;  // host tracks: offset of the device copy inside the track arena
  bool ran = false;
  st_job_stats stats{};
};

int64_t round_up(int64_t v, int64_t m) { return (v + m - 1) / m * m; }

uint32_t next_pow2(uint64_t v) {
  uint64_t p = 1;
  while (p < v) p <<= 1;
  return (uint32_t)std::min<uint64_t>(p, 1ull << 31);
}

}  // namespace

struct st_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int sm_count = 0;
  std::string err;
  std::vector<HistHost> hists;
  std::vector<JobHost> jobs;

  DevBuf track_arena;
  DevBuf pxy, pdz2, pv, pkey;
  DevBuf d_jobs, d_aux, d_hists, d_items, d_blk, d_counter, d_err, d_blk_count, d_blk_off, d_blk_job;
  DevBuf c_cells, pz;               // cell arena and shifted z of flagged jobs
  DevBuf u_next, u_done, u_table, pool;  // shared units and the spill-table pool
  DevBuf d_plan, d_plan_misc;             // planner: per-job plans and scratch counters
  DevBuf g_keys, g_lo, g_hi, g_used, g_count;
  uint32_t gcap = 0;
  int ggrid = 0;
  bool g_dirty = false;
  DevBuf ex_buf, ex_count;
  // all histograms live in three arenas so that every spectrum can be read in two copies
  DevBuf h_counts, h_yfy, h_edges;
  int64_t h_bins = 0, h_edge_total = 0;

  bool timing = false;
  // run events: 0 start, 1 prepare and plan done, 4 fused start (after any cross-context wait),
  // 2 fused done, 3 results copied to the host
  cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  cudaEvent_t order_after = nullptr;  // the next run's fused kernel waits for this event
  // CUDA graph of a whole run, captured at the first rerun of the same tables
  bool use_graphs = true;
  cudaGraphExec_t gexec = nullptr;
  int64_t build_id = 0, gexec_build = -1;
  const void* gexec_aux = nullptr;
  const void* gexec_stage = nullptr;
  int64_t graph_launches = 0;
  int table_slots = 0;        // shared-memory sphere table: 0 automatic, 4096 or 8192
  // pipelined runs of host tracks: jobs in groups of about pipeline_bytes of track data; the
  // copy stream uploads group g+1 while the context's stream runs group g
  int64_t pipeline_bytes = (int64_t)1 << 28;
  // ... only when the host tracks average at most this many oversamples per deposit: past it a
  // batch computes longer than it uploads, and each group's fused-kernel tail costs more than the
  // overlap saves
  int64_t pipeline_max_os = 50;
  cudaStream_t copy_stream = nullptr;
  std::vector<cudaEvent_t> up_ev;
  std::vector<int64_t> cache_blk;    // prepare-block prefix of the batch (host copy)
  std::vector<char> cache_flagged;   // jobs with boundary flags
  float t_prep = 0, t_fused = 0;
  int32_t launches = 0;

  int64_t item_cost = 1 << 18;
  int grid_override = 0;
  int smem_hist_bins = 4096;
  bool fused_configured = false;

  // launch set-up of the last batched range, reused when the same jobs run again
  bool cache_valid = false;
  size_t cache_first = 0, cache_last = 0;
  st::PrepareParams cache_pp{};
  st::FusedParams cache_fp{};
  int64_t cache_blocks = 0;
  int cache_grid = 0;
  int64_t cache_arena_total = 0;
  int cache_max_nbins = 0;
  int64_t cache_cells = 0;
  bool cache_any_flagged = false;
  int64_t cache_units = 0;
  int64_t cache_item_cap = 0;
  st::PlanParams cache_plan{};
  int chunk_windows = 4;      // windows (8192 deposits each) per chunk of a shared unit
  int max_helpers = 32;       // helper items per shared unit
  int64_t spill_budget = 0;   // bytes for the spill tables; 0: 30% of free memory (or the full
                              // grid's tables if they leave 16 GB free), at most 48 GB
  int share_divisor = 8;      // shared units: kept > batch units / (share_divisor * grid) ...
  int min_chunks = 4;         // ... and kept > min_chunks chunks
  int precision = 64;         // 32: FP32 geometry variant (x/y geometry in float)
  int64_t flag_min_kept = 16384;  // window flags only for jobs with more kept deposits
  int64_t flag_cells_limit = st::kFlagCellsLimit;  // flag cells of side 2d up to this density*OS
  int sort_deposits = 1;          // prepare blocks that group kept deposits by cell: 0 none,
                                  // 1 those of window-flagged jobs, 2 all

  // results of an enqueued run are copied into pinned buffers and picked up at finish
  JobAux* h_aux = nullptr;
  size_t h_aux_cap = 0;
  PinnedBuf stage;                // job, histogram and prepare-block tables of the run
  // host time of the last launch (microseconds): whole launch, table building, allocations
  // inside it (and their number), the free-memory query
  double host_launch_us = 0, host_tables_us = 0, host_alloc_us = 0, host_meminfo_us = 0;
  int64_t host_allocs = 0;
  int* h_err = nullptr;           // 4 ints + export count (8 bytes)
  bool pending = false;
  size_t pend_first = 0, pend_last = 0;
  bool pend_export = false;
};

namespace {

st_status cuda_fail(st_ctx* c, cudaError_t e, const char* what) {
  c->err = std::string(what) + ": " + cudaGetErrorString(e);
  return e == cudaErrorMemoryAllocation ? ST_ERR_OUT_OF_MEMORY : ST_ERR_CUDA;
}

#define ST_CUDA(call, what)                              \
  do {                                                   \
    cudaError_t e__ = (call);                            \
    if (e__ != cudaSuccess) return cuda_fail(c, e__, what); \
  } while (0)

st_status init_spill_tables(st_ctx* c, uint32_t gcap, int grid) {
  const size_t slots = (size_t)gcap * (size_t)grid;
  ST_CUDA(ensure(c->g_keys, slots * 8), "spill table keys");
  ST_CUDA(ensure(c->g_lo, slots * 8), "spill table lo");
  ST_CUDA(ensure(c->g_hi, slots * 8), "spill table hi");
  ST_CUDA(ensure(c->g_used, slots * 4), "spill table used list");
  ST_CUDA(ensure(c->g_count, (size_t)grid * 4), "spill table counters");
  ST_CUDA(cudaMemsetAsync(c->g_keys.p, 0xFF, slots * 8, c->stream), "spill init");
  ST_CUDA(cudaMemsetAsync(c->g_lo.p, 0, slots * 8, c->stream), "spill init");
  ST_CUDA(cudaMemsetAsync(c->g_hi.p, 0, slots * 8, c->stream), "spill init");
  ST_CUDA(cudaMemsetAsync(c->g_count.p, 0, (size_t)grid * 4, c->stream), "spill init");
  c->gcap = gcap;
  c->ggrid = grid;
  c->g_dirty = false;
  return ST_OK;
}

// Copies the host-resident tracks of jobs [first, last) into the track arena; adjacent host
// ranges are merged into one copy per coordinate array.
st_status upload_host_tracks(st_ctx* c, size_t first, size_t last, int64_t arena_total,
                             cudaStream_t stream) {
  double* arena = (double*)c->track_arena.p;
  size_t j = first;
  while (j < last) {
    JobHost& J = c->jobs[j];
    if (J.track.on_device || J.track.n == 0) { ++j; continue; }
    size_t k = j + 1;
    int64_t n = J.track.n;
    while (k < last) {
      const JobHost& K = c->jobs[k];
      if (K.track.on_device || K.track.n == 0 || K.arena_off != J.arena_off + n ||
          K.track.x != J.track.x + n || K.track.y != J.track.y + n ||
          K.track.z != J.track.z + n || K.track.edep != J.track.edep + n)
        break;
      n += K.track.n;
      ++k;
    }
    const double* src[4] = {J.track.x, J.track.y, J.track.z, J.track.edep};
    for (int a = 0; a < 4; ++a)
      ST_CUDA(cudaMemcpyAsync(arena + (size_t)arena_total * a + J.arena_off, src[a],
                              (size_t)n * 8, cudaMemcpyHostToDevice, stream),
              "track upload");
    j = k;
  }
  return ST_OK;
}

// Builds the device tables (jobs, aux, histograms, work items, prepare blocks) of jobs
// [first, last) and the launch parameters; stores them in the context cache.
st_status build_tables(st_ctx* c, size_t first, size_t last, bool want_export) {
  const size_t nj = last - first;
  // a job whose histogram was forgotten (st_hists_clear) has nothing to add into
  for (size_t j = first; j < last; ++j) {
    const int32_t h = c->jobs[j].desc.hist_id;
    if (h < 0 || h >= (int32_t)c->hists.size()) return ST_ERR_STATE;
  }
  ++c->build_id;
  int64_t prep_total = 0, arena_total = 0, max_pad = 0;
  for (size_t j = first; j < last; ++j) {
    JobHost& J = c->jobs[j];
    J.n_pad = round_up(std::max<int64_t>(J.track.n, 1), st::kWarpTile);
    J.prep_off = prep_total;
    prep_total += J.n_pad;
    max_pad = std::max(max_pad, J.n_pad);
    J.arena_off = -1;
    if (!J.track.on_device && J.track.n > 0) {
      J.arena_off = arena_total;
      arena_total += J.track.n;
    }
  }
  ST_CUDA(ensure(c->pxy, prep_total * 16), "prepared arena");

  ST_CUDA(ensure(c->pdz2, prep_total * 8), "prepared arena");
  ST_CUDA(ensure(c->pv, prep_total * 16), "prepared arena");
  ST_CUDA(ensure(c->pkey, prep_total * 8), "prepared arena");
  ST_CUDA(ensure(c->track_arena, (size_t)arena_total * 32), "track arena");
  double* arena = (double*)c->track_arena.p;

  std::vector<JobDev> jd(nj);
  std::vector<int64_t> blk(nj + 1, 0);
  int64_t cells_total = 0;
  bool any_flagged = false;
  for (size_t i = 0; i < nj; ++i) {
    JobHost& J = c->jobs[first + i];
    JobDev& D = jd[i];
    if (J.track.on_device) {
      D.x = J.track.x; D.y = J.track.y; D.z = J.track.z; D.edep = J.track.edep;
    } else {
      D.x = arena + J.arena_off;
      D.y = arena + (size_t)arena_total + J.arena_off;
      D.z = arena + (size_t)arena_total * 2 + J.arena_off;
      D.edep = arena + (size_t)arena_total * 3 + J.arena_off;
    }
    D.n = J.track.n;
    D.n_pad = J.n_pad;
    D.prep_off = J.prep_off;
    D.HL = J.g.scoringRegionHalfLength;
    D.L = J.g.scoringRegionLength;
    D.gSO = J.g.greatestSphereOffset;
    D.d = J.g.sphereDiameter;
    D.inv_d = 1.0 / J.g.sphereDiameter;
    D.r2 = J.g.sphereRadius * J.g.sphereRadius;
    D.denom = (2. / 3.) * J.g.sphereDiameter;
    D.zsh = J.desc.zshift == ST_ZSHIFT_PLUS ? J.g.scoringRegionHalfLength
          : J.desc.zshift == ST_ZSHIFT_MINUS ? -J.g.scoringRegionHalfLength : 0.0;
    // with shifts in (-HL', HL'] a deposit at |x| >= 2HL'(1+2^-30) stays outside the voxel
    // (2HL'(1+2^-20) when x, the shift and their sum are rounded to float); without shifts
    // (x + 0 = x) the box test itself decides, and rounding x to float keeps |x| >= HL' outside
    const bool f32 = c->precision == 32;
    D.xy_keep = J.desc.shift_track
                    ? 2.0 * J.g.scoringRegionHalfLength * (1.0 + (f32 ? 0x1p-20 : 0x1p-30))
                    : J.g.scoringRegionHalfLength;
    D.N = (uint32_t)J.g.numSpheresLinear;
    D.N2 = (uint64_t)D.N * (uint64_t)D.N;
    D.seed = J.desc.seed;
    D.track_id = J.desc.track_id;
    D.n_os = (int32_t)J.desc.n_oversamples;
    D.shift_track = J.desc.shift_track ? 1 : 0;
    D.hist = J.desc.hist_id;
    // boundary flags pay off for multi-window jobs on fine lattices with several oversamples
    D.flagged = (J.track.n > 2 * st::kCtaTile && J.desc.n_oversamples >= 4 &&
                 D.N >= 128 && D.N < (1u << (st::kCellBits - 2))) ? 1 : 0;
    D.cell_cap = 0;
    D.cell_off = 0;
    // flag cells: two hits of one sphere are within d of each other; in the FP32 form within d
    // plus a few float roundings of coordinates below 4HL' (HL' 2^-16 covers them). Side twice
    // that for tracks with few deposits per d of track length times oversamples.
    const double per_d = (double)J.track.n * J.g.sphereDiameter /
                         (2.0 * J.g.scoringRegionHalfLength);
    D.cell_nbr8 = (D.flagged && per_d * J.desc.n_oversamples <= (double)c->flag_cells_limit) ? 1 : 0;
    D.cell_size = (D.cell_nbr8 ? 2.0 : 1.0) *
                  (J.g.sphereDiameter * (1.0 + 0x1p-10) +
                   (f32 ? J.g.scoringRegionHalfLength * 0x1p-16 : 0.0));
    D.inv_cell = 1.0 / D.cell_size;
    D.f_HL = (float)J.g.scoringRegionHalfLength;
    D.f_gSO = (float)J.g.greatestSphereOffset;
    D.f_d = (float)J.g.sphereDiameter;
    D.f_inv_d = 1.0f / D.f_d;
    D.f_r2 = (float)D.r2;
    if (D.flagged) {
      D.cell_cap = next_pow2((uint64_t)2 * (uint64_t)J.track.n);
      D.cell_off = cells_total;
      cells_total += D.cell_cap;
      any_flagged = true;
    }
    blk[i + 1] = blk[i] + (J.n_pad + st::kPrepSlotsPerBlock - 1) / st::kPrepSlotsPerBlock;
  }
  std::vector<HistDev> hd(c->hists.size());
  for (size_t h = 0; h < c->hists.size(); ++h) {
    hd[h].edges = (const double*)c->h_edges.p + c->hists[h].eoff;
    hd[h].counts = (unsigned long long*)c->h_counts.p + c->hists[h].off;
    hd[h].yfy = (double*)c->h_yfy.p + c->hists[h].off;
    hd[h].nbins = c->hists[h].nbins;
    const std::vector<double>& e = c->hists[h].edges;
    const double lo = e.front(), hi = e.back();
    if (c->hists[h].type == ST_HIST_LOG && lo > 0) {
      hd[h].mode = 1;
      hd[h].ca = std::log2(lo);
      hd[h].cb = c->hists[h].nbins / (std::log2(hi) - std::log2(lo));
    } else {
      hd[h].mode = 0;
      hd[h].ca = lo;
      hd[h].cb = c->hists[h].nbins / (hi - lo);
    }
  }
  int max_nbins = 0;
  for (size_t i = 0; i < nj; ++i)
    max_nbins = std::max(max_nbins, c->hists[c->jobs[first + i].desc.hist_id].nbins);
  c->cache_max_nbins = max_nbins;

  // work items are planned on the device from the kept counts (k_plan_*); here only their
  // capacity: every job as shared units with the most helpers is the upper bound
  int64_t total_os = 0, work_jobs = 0;
  for (size_t i = 0; i < nj; ++i) {
    const JobHost& J = c->jobs[first + i];
    if (J.desc.n_oversamples == 0 || J.track.n == 0) continue;
    total_os += J.desc.n_oversamples;
    ++work_jobs;
  }
  const int64_t item_cap = std::max<int64_t>(1, total_os * std::max(1, c->max_helpers));
  const int64_t units = std::max<int64_t>(1, total_os);
  ST_CUDA(ensure(c->u_next, (size_t)units * 4), "units");
  ST_CUDA(ensure(c->u_done, (size_t)units * 4), "units");
  ST_CUDA(ensure(c->u_table, (size_t)units * 4), "units");
  ST_CUDA(ensure(c->d_items, (size_t)item_cap * sizeof(WorkItem)), "items");
  ST_CUDA(ensure(c->d_plan, nj * sizeof(st::JobPlan)), "plan");
  ST_CUDA(ensure(c->d_plan_misc, 4096), "plan scratch");

  ST_CUDA(ensure(c->d_jobs, nj * sizeof(JobDev)), "job table");
  ST_CUDA(ensure(c->d_aux, nj * sizeof(JobAux)), "job aux");
  ST_CUDA(ensure(c->d_hists, std::max<size_t>(1, hd.size()) * sizeof(HistDev)), "hist table");
  ST_CUDA(ensure(c->d_blk, (nj + 1) * 8), "prepare blocks");
  ST_CUDA(ensure(c->d_blk_count, (size_t)blk[nj] * 4), "prepare block counts");
  ST_CUDA(ensure(c->d_blk_job, (size_t)std::max<int64_t>(1, blk[nj]) * 4), "prepare block jobs");
  ST_CUDA(ensure(c->c_cells, (size_t)cells_total * sizeof(st::CellSlot)), "cell arena");
  ST_CUDA(ensure(c->pz, any_flagged ? (size_t)prep_total * 8 : 16), "shifted z");
  ST_CUDA(ensure(c->d_blk_off, (size_t)blk[nj] * 8), "prepare block offsets");
  ST_CUDA(ensure(c->d_counter, 16), "work counter");
  ST_CUDA(ensure(c->d_err, 16), "error flags");
  {
    // tables through pinned staging (the previous run's copies from it have completed)
    const size_t o_hists = align256(nj * sizeof(JobDev));
    const size_t o_blk = o_hists + align256(hd.size() * sizeof(HistDev));
    const size_t o_bj = o_blk + align256((nj + 1) * 8);
    ST_CUDA(ensure_pinned(c->stage, o_bj + align256((size_t)blk[nj] * 4)), "pinned staging");
    char* st_base = (char*)c->stage.p;
    std::memcpy(st_base, jd.data(), nj * sizeof(JobDev));
    if (!hd.empty()) std::memcpy(st_base + o_hists, hd.data(), hd.size() * sizeof(HistDev));
    std::memcpy(st_base + o_blk, blk.data(), (nj + 1) * 8);
    int32_t* bj = (int32_t*)(st_base + o_bj);  // job of each prepare block
    for (size_t i = 0; i < nj; ++i)
      for (int64_t b = blk[i]; b < blk[i + 1]; ++b) bj[b] = (int32_t)i;
    ST_CUDA(cudaMemcpyAsync(c->d_jobs.p, st_base, nj * sizeof(JobDev), cudaMemcpyHostToDevice, c->stream), "upload jobs");
    if (!hd.empty())
      ST_CUDA(cudaMemcpyAsync(c->d_hists.p, st_base + o_hists, hd.size() * sizeof(HistDev), cudaMemcpyHostToDevice, c->stream), "upload hists");
    ST_CUDA(cudaMemcpyAsync(c->d_blk.p, st_base + o_blk, (nj + 1) * 8, cudaMemcpyHostToDevice, c->stream), "upload blocks");
    if (blk[nj] > 0)
      ST_CUDA(cudaMemcpyAsync(c->d_blk_job.p, st_base + o_bj, (size_t)blk[nj] * 4, cudaMemcpyHostToDevice, c->stream), "upload block jobs");
  }

  // spill tables: one per resident CTA, able to hold every distinct sphere of the largest job;
  // the number of resident CTAs shrinks if the tables would exceed the spill budget (by default
  // 30% of free memory, at most 48 GB)
  int grid = c->grid_override > 0 ? c->grid_override : c->sm_count;
  // never more CTAs than work items can exist (every oversample as a shared unit with the
  // most helpers)
  grid = (int)std::max<int64_t>(1, std::min<int64_t>(grid, item_cap));
  const uint32_t gcap = std::max(c->gcap, next_pow2((uint64_t)std::max<int64_t>(2 * max_pad, 1024)));
  if (gcap > c->gcap || grid > c->ggrid) {
    // the free-memory query waits for other streams' work, so it is made only when the
    // tables have to grow
    size_t free_b = 0, total_b = 0;
    const double tm = now_us();
    if (c->spill_budget <= 0) cudaMemGetInfo(&free_b, &total_b);
    c->host_meminfo_us = now_us() - tm;
    const size_t have = (size_t)c->gcap * (size_t)c->ggrid * 28;
    // default: 30% of free memory, or the whole grid's tables when they still leave 16 GB free
    // (a batch of huge tracks, whose tables are large, would otherwise run on a fraction of the
    // SMs); at most 48 GB
    const double avail = (double)(free_b + have);
    const double full = (double)gcap * 28.0 * (double)grid;
    const double budget = c->spill_budget > 0
                              ? (double)c->spill_budget
                              : std::min(std::max(0.3 * avail, full <= avail - 16e9 ? full : 0.0),
                                         48e9);
    const int fit = (int)std::max(1.0, std::floor(budget / ((double)gcap * 28.0)));
    grid = std::min(grid, fit);
  }
  if (gcap > c->gcap || grid > c->ggrid || c->g_dirty) {
    st_status s = init_spill_tables(c, gcap, grid);
    if (s != ST_OK) return s;
  }
  ST_CUDA(ensure(c->pool, (size_t)((grid + 31) / 32) * 4), "spill-table pool");
  if (!c->fused_configured) {
    ST_CUDA(st::configure_fused(), "configure fused kernel");
    c->fused_configured = true;
  }

  st::PrepareParams& pp = c->cache_pp;
  pp.jobs = (const JobDev*)c->d_jobs.p;
  pp.aux = (JobAux*)c->d_aux.p;
  pp.n_jobs = (int32_t)nj;
  pp.blk_base = 0;
  pp.blk_prefix = (const int64_t*)c->d_blk.p;
  pp.blk_job = (const int32_t*)c->d_blk_job.p;
  pp.job_base = 0;
  pp.blk_count = (int32_t*)c->d_blk_count.p;
  pp.blk_offset = (int64_t*)c->d_blk_off.p;
  pp.cells = (st::CellSlot*)c->c_cells.p;
  pp.PZ = (double*)c->pz.p;
  pp.PXY = (double2*)c->pxy.p;

  pp.PDZ2 = (double*)c->pdz2.p;
  pp.PV = (ulonglong2*)c->pv.p;
  pp.PKEY = (unsigned long long*)c->pkey.p;
  pp.fp32 = c->precision == 32 ? 1 : 0;
  pp.flag_min_kept = c->flag_min_kept;
  pp.sort = c->sort_deposits;

  st::FusedParams& fp = c->cache_fp;
  fp.jobs = pp.jobs;
  fp.aux = pp.aux;
  fp.hists = (const HistDev*)c->d_hists.p;
  fp.items = (const WorkItem*)c->d_items.p;
  fp.n_items = (const int*)((char*)c->d_plan_misc.p + 8);
  fp.flush_threshold = 1024;
  fp.work_counter = (unsigned int*)c->d_counter.p;
  fp.PXY = pp.PXY; fp.PDZ2 = pp.PDZ2;
  fp.PV = pp.PV; fp.PKEY = pp.PKEY;
  fp.gkeys = (uint64_t*)c->g_keys.p;
  fp.glo = (unsigned long long*)c->g_lo.p;
  fp.ghi = (unsigned long long*)c->g_hi.p;
  fp.gused = (uint32_t*)c->g_used.p;
  fp.gcount = (unsigned int*)c->g_count.p;
  fp.gcap = c->gcap;
  fp.smem_hist_bins = c->smem_hist_bins;
  fp.export_buf = nullptr;
  fp.export_count = nullptr;
  fp.export_cap = 0;
  fp.error_flags = (int*)c->d_err.p;
  fp.unit_next = (unsigned int*)c->u_next.p;
  fp.unit_done = (unsigned int*)c->u_done.p;
  fp.unit_table = (int*)c->u_table.p;
  fp.pool_bits = (unsigned int*)c->pool.p;
  fp.chunk_windows = c->chunk_windows;
  fp.fp32 = pp.fp32;

  c->cache_blk = blk;
  c->cache_flagged.resize(nj);
  for (size_t i = 0; i < nj; ++i) c->cache_flagged[i] = (char)jd[i].flagged;
  c->cache_blocks = blk[nj];
  c->cache_grid = work_jobs == 0 ? 0 : grid;
  c->cache_item_cap = item_cap;
  c->cache_arena_total = arena_total;
  c->cache_cells = cells_total;
  c->cache_any_flagged = any_flagged;
  c->cache_units = units;
  // planner parameters; the scratch block holds total_units (8 B), n_items (4 B), the unit
  // counter (4 B) and the three bucket arrays
  st::PlanParams& q = c->cache_plan;
  char* m = (char*)c->d_plan_misc.p;
  q.jobs = (const JobDev*)c->d_jobs.p;
  q.aux = (const JobAux*)c->d_aux.p;
  q.n_jobs = (int32_t)nj;
  q.chunk_windows = c->chunk_windows;
  q.max_helpers = c->max_helpers;
  q.grid = std::max(1, grid);
  q.item_cost = c->item_cost;
  q.share_divisor = c->share_divisor;
  q.min_chunks = c->min_chunks;
  q.total_units = (unsigned long long*)m;
  q.n_items = (int*)(m + 8);
  q.unit_counter = (unsigned int*)(m + 12);
  q.bucket_count = (unsigned int*)(m + 16);
  q.bucket_start = q.bucket_count + st::kPlanBuckets;
  q.bucket_cursor = q.bucket_start + st::kPlanBuckets;
  q.plan = (st::JobPlan*)c->d_plan.p;
  q.items = (WorkItem*)c->d_items.p;
  q.item_cap = item_cap;
  c->cache_first = first;
  c->cache_last = last;
  c->cache_valid = !want_export;
  return ST_OK;
}

// Enqueues the device side of a run on the context's stream: the resets, the prepare, plan and
// fused kernels, and the copies of the job counters and error flags into pinned host memory,
// with the run's events. Nothing waits; finish_range picks the results up. While the stream is
// being captured into a CUDA graph the events become event-record nodes.
st_status enqueue_run(st_ctx* c, const st::FusedParams& fp, size_t nj, bool want_export,
                      bool capturing) {
  const unsigned evf = capturing ? cudaEventRecordExternal : cudaEventRecordDefault;
  ST_CUDA(st::launch_reset_aux((JobAux*)c->d_aux.p, (int)nj, c->stream), "reset aux");
  ST_CUDA(cudaMemsetAsync(c->d_counter.p, 0, 16, c->stream), "reset counter");
  if (c->cache_grid > 0)
    ST_CUDA(cudaMemsetAsync(c->pool.p, 0, (size_t)((c->cache_grid + 31) / 32) * 4, c->stream), "pool reset");
  ST_CUDA(cudaMemsetAsync(c->d_plan_misc.p, 0, 16 + 3 * 4 * st::kPlanBuckets, c->stream), "plan reset");
  if (c->cache_units > 0) {
    ST_CUDA(cudaMemsetAsync(c->u_next.p, 0, (size_t)c->cache_units * 4, c->stream), "unit reset");
    ST_CUDA(cudaMemsetAsync(c->u_done.p, 0, (size_t)c->cache_units * 4, c->stream), "unit reset");
    ST_CUDA(cudaMemsetAsync(c->u_table.p, 0xFF, (size_t)c->cache_units * 4, c->stream), "unit reset");
  }
  if (c->cache_cells > 0) {
    ST_CUDA(cudaMemsetAsync(c->c_cells.p, 0xFF, (size_t)c->cache_cells * sizeof(st::CellSlot), c->stream), "cell reset");
  }
  ST_CUDA(cudaMemsetAsync(c->d_err.p, 0, 16, c->stream), "reset errors");
  if (want_export) ST_CUDA(cudaMemsetAsync(c->ex_count.p, 0, 16, c->stream), "export counter");

  ST_CUDA(cudaEventRecordWithFlags(c->ev[0], c->stream, evf), "event");
  ST_CUDA(st::launch_prepare(c->cache_pp, c->cache_blocks, c->cache_any_flagged, c->stream), "prepare launch");
  ST_CUDA(st::launch_plan(c->cache_plan, c->stream), "plan launch");
  ST_CUDA(cudaEventRecordWithFlags(c->ev[1], c->stream, evf), "event");
  if (c->order_after && !capturing) {
    ST_CUDA(cudaStreamWaitEvent(c->stream, c->order_after, 0), "order after");
    c->order_after = nullptr;
  }
  ST_CUDA(cudaEventRecordWithFlags(c->ev[4], c->stream, evf), "event");
  ST_CUDA(st::launch_fused(fp, c->cache_max_nbins, c->cache_grid, c->table_slots, c->stream), "fused launch");
  ST_CUDA(cudaEventRecordWithFlags(c->ev[2], c->stream, evf), "event");
  ST_CUDA(cudaMemcpyAsync(c->h_aux, c->d_aux.p, nj * sizeof(JobAux), cudaMemcpyDeviceToHost, c->stream), "read aux");
  ST_CUDA(cudaMemcpyAsync(c->h_err, c->d_err.p, 16, cudaMemcpyDeviceToHost, c->stream), "read errors");
  if (want_export) ST_CUDA(cudaMemcpyAsync(c->h_err + 4, c->ex_count.p, 8, cudaMemcpyDeviceToHost, c->stream), "read export count");
  ST_CUDA(cudaEventRecordWithFlags(c->ev[3], c->stream, evf), "event");
  return ST_OK;
}

// Pipelined form of enqueue_run: after the batch-wide uploads and resets, each group of jobs
// [groups[g], groups[g+1]) waits for its track upload, then runs its own prepare, plan and fused
// launches on the jobs, aux and plan tables offset to its first job (the tables are batch-wide,
// so every job keeps its slot). Events: 0 start, 1 and 4 before the first fused kernel, 2 after
// the last one, 3 results copied.
st_status enqueue_groups(st_ctx* c, const st::FusedParams& fp, size_t first,
                         const std::vector<size_t>& groups) {
  const size_t nj = groups.back() - first;
  ST_CUDA(st::launch_reset_aux((JobAux*)c->d_aux.p, (int)nj, c->stream), "reset aux");
  if (c->cache_cells > 0) {
    ST_CUDA(cudaMemsetAsync(c->c_cells.p, 0xFF, (size_t)c->cache_cells * sizeof(st::CellSlot), c->stream), "cell reset");
  }
  ST_CUDA(cudaMemsetAsync(c->d_err.p, 0, 16, c->stream), "reset errors");
  ST_CUDA(cudaEventRecord(c->ev[0], c->stream), "event");
  for (size_t g = 0; g + 1 < groups.size(); ++g) {
    const size_t j0 = groups[g] - first, j1 = groups[g + 1] - first;
    ST_CUDA(cudaStreamWaitEvent(c->stream, c->up_ev[g], 0), "upload wait");
    ST_CUDA(cudaMemsetAsync(c->d_counter.p, 0, 16, c->stream), "reset counter");
    if (c->cache_grid > 0)
      ST_CUDA(cudaMemsetAsync(c->pool.p, 0, (size_t)((c->cache_grid + 31) / 32) * 4, c->stream), "pool reset");
    ST_CUDA(cudaMemsetAsync(c->d_plan_misc.p, 0, 16 + 3 * 4 * st::kPlanBuckets, c->stream), "plan reset");
    if (c->cache_units > 0) {
      ST_CUDA(cudaMemsetAsync(c->u_next.p, 0, (size_t)c->cache_units * 4, c->stream), "unit reset");
      ST_CUDA(cudaMemsetAsync(c->u_done.p, 0, (size_t)c->cache_units * 4, c->stream), "unit reset");
      ST_CUDA(cudaMemsetAsync(c->u_table.p, 0xFF, (size_t)c->cache_units * 4, c->stream), "unit reset");
    }
    st::PrepareParams pp = c->cache_pp;
    pp.jobs += j0;
    pp.aux += j0;
    pp.n_jobs = (int32_t)(j1 - j0);
    pp.blk_prefix += j0;
    pp.job_base = (int32_t)j0;
    pp.blk_base = c->cache_blk[j0];
    bool flagged = false;
    for (size_t j = j0; j < j1; ++j) flagged |= c->cache_flagged[j] != 0;
    ST_CUDA(st::launch_prepare(pp, c->cache_blk[j1] - c->cache_blk[j0], flagged, c->stream), "prepare launch");
    st::PlanParams q = c->cache_plan;
    q.jobs += j0;
    q.aux += j0;
    q.plan += j0;
    q.n_jobs = (int32_t)(j1 - j0);
    ST_CUDA(st::launch_plan(q, c->stream), "plan launch");
    if (g == 0) {
      ST_CUDA(cudaEventRecord(c->ev[1], c->stream), "event");
      ST_CUDA(cudaEventRecord(c->ev[4], c->stream), "event");
    }
    st::FusedParams f = fp;
    f.jobs += j0;
    f.aux += j0;
    ST_CUDA(st::launch_fused(f, c->cache_max_nbins, c->cache_grid, c->table_slots, c->stream), "fused launch");
  }
  ST_CUDA(cudaEventRecord(c->ev[2], c->stream), "event");
  ST_CUDA(cudaMemcpyAsync(c->h_aux, c->d_aux.p, nj * sizeof(JobAux), cudaMemcpyDeviceToHost, c->stream), "read aux");
  ST_CUDA(cudaMemcpyAsync(c->h_err, c->d_err.p, 16, cudaMemcpyDeviceToHost, c->stream), "read errors");
  ST_CUDA(cudaEventRecord(c->ev[3], c->stream), "event");
  return ST_OK;
}

void drop_graph(st_ctx* c) {
  if (c->gexec) cudaGraphExecDestroy(c->gexec);
  c->gexec = nullptr;
}

// Captures enqueue_run into a CUDA graph (once per set of tables); false if capture is not
// possible here, in which case the caller enqueues directly and graphs stay off.
bool capture_run(st_ctx* c, const st::FusedParams& fp, size_t nj) {
  drop_graph(c);
  if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    c->use_graphs = false;
    return false;
  }
  const st_status s = enqueue_run(c, fp, nj, false, true);
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
  cudaGraphExec_t x = nullptr;
  const bool ok = s == ST_OK && e == cudaSuccess && g &&
                  cudaGraphInstantiate(&x, g, 0) == cudaSuccess;
  if (g) cudaGraphDestroy(g);
  if (!ok) {
    cudaGetLastError();
    if (x) cudaGraphExecDestroy(x);
    c->use_graphs = false;
    return false;
  }
  c->gexec = x;
  c->gexec_build = c->build_id;
  c->gexec_aux = c->h_aux;
  c->gexec_stage = c->stage.p;
  return true;
}

// Enqueues jobs [first, last) of the context: tables (unless the same jobs ran last), uploads,
// the prepare and plan launches, the fused launch, and the copy of the job counters and error
// flags into pinned host buffers. A rerun of the same jobs replays a captured CUDA graph of all
// of it. Nothing waits; finish_range picks the results up.
st_status launch_range(st_ctx* c, size_t first, size_t last, bool want_export, int64_t ex_cap) {
  const double t_begin = now_us();
  g_alloc_us = 0;
  g_allocs = 0;
  c->host_meminfo_us = 0;
  struct Stamp {
    st_ctx* c;
    double t0;
    ~Stamp() {
      c->host_launch_us = now_us() - t0;
      c->host_alloc_us = g_alloc_us;
      c->host_allocs = g_allocs;
    }
  } stamp{c, t_begin};
  const size_t nj = last - first;
  const bool reuse = !want_export && c->cache_valid && c->cache_first == first && c->cache_last == last;
  c->host_tables_us = 0;
  if (!reuse) {
    st_status s = build_tables(c, first, last, want_export);
    c->host_tables_us = now_us() - t_begin;
    if (s != ST_OK) { c->cache_valid = false; return s; }
  }
  // groups of host track data (one group when every track is on the device): their uploads
  // run on the copy stream, ahead of the groups' kernels. The first and the last group hold
  // about a quarter of pipeline_bytes (the upload before the first kernels and the kernels after
  // the last upload are not overlapped), the others about pipeline_bytes. A batch averaging more
  // than pipeline_max_os oversamples per uploaded deposit is uploaded whole, then run at once.
  std::vector<size_t> groups(1, first);
  {
    int64_t total = 0;
    double host_units = 0.0;
    for (size_t j = first; j < last; ++j)
      if (!c->jobs[j].track.on_device) {
        total += 32 * c->jobs[j].track.n;
        host_units += (double)c->jobs[j].track.n * (double)c->jobs[j].desc.n_oversamples;
      }
    const bool upload_bound = host_units <= (double)c->pipeline_max_os * (double)(total / 32);
    const int64_t P = c->pipeline_bytes, q = std::max<int64_t>(P / 4, 1);
    std::vector<int64_t> cuts;
    if (total > 2 * q && upload_bound) {
      for (int64_t t = q; t < total - q && cuts.size() < 62; t += P) cuts.push_back(t);
      cuts.push_back(total - q);
    }
    int64_t acc = 0;
    size_t k = 0;
    for (size_t j = first; j < last && k < cuts.size(); ++j) {
      if (!c->jobs[j].track.on_device) acc += 32 * c->jobs[j].track.n;
      if (acc >= cuts[k] && j + 1 < last) {
        groups.push_back(j + 1);
        while (k < cuts.size() && acc >= cuts[k]) ++k;
      }
    }
    groups.push_back(last);
  }
  const bool pipelined = groups.size() > 2 && !want_export;
  if (!pipelined) {
    groups.assign({first, last});
    st_status s = upload_host_tracks(c, first, last, c->cache_arena_total, c->stream);
    if (s != ST_OK) return s;
  } else {
    if (!c->copy_stream)
      ST_CUDA(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking), "copy stream");
    while (c->up_ev.size() < groups.size()) {
      cudaEvent_t e;
      ST_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "upload event");
      c->up_ev.push_back(e);
    }
    // the copies start after everything already queued on the context's stream
    ST_CUDA(cudaEventRecord(c->up_ev.back(), c->stream), "event");
    ST_CUDA(cudaStreamWaitEvent(c->copy_stream, c->up_ev.back(), 0), "copy stream wait");
    for (size_t g = 0; g + 1 < groups.size(); ++g) {
      st_status s = upload_host_tracks(c, groups[g], groups[g + 1], c->cache_arena_total, c->copy_stream);
      if (s != ST_OK) return s;
      ST_CUDA(cudaEventRecord(c->up_ev[g], c->copy_stream), "event");
    }
  }

  st::FusedParams fp = c->cache_fp;
  if (want_export) {
    ST_CUDA(ensure(c->ex_buf, (size_t)std::max<int64_t>(ex_cap, 1) * sizeof(st::SphereRecord)), "export buffer");
    ST_CUDA(ensure(c->ex_count, 16), "export counter");
    fp.export_buf = (st::SphereRecord*)c->ex_buf.p;
    fp.export_count = (unsigned long long*)c->ex_count.p;
    fp.export_cap = (unsigned long long)ex_cap;
  }
  if (c->h_aux_cap < nj) {
    const size_t cap = std::max<size_t>(std::max<size_t>(nj, 1024), c->h_aux_cap + c->h_aux_cap / 2);
    if (c->h_aux) cudaFreeHost(c->h_aux);
    c->h_aux = nullptr;
    c->h_aux_cap = 0;
    ST_CUDA(cudaMallocHost(&c->h_aux, cap * sizeof(JobAux)), "pinned aux");
    c->h_aux_cap = cap;
  }
  if (!c->h_err) ST_CUDA(cudaMallocHost(&c->h_err, 32), "pinned flags");

  const bool graph = reuse && c->use_graphs && !c->order_after && !pipelined;
  bool launched = false;
  if (pipelined) {
    st_status s = enqueue_groups(c, fp, first, groups);
    if (s != ST_OK) return s;
    launched = true;
  }
  if (graph) {
    if (!c->gexec || c->gexec_build != c->build_id || c->gexec_aux != c->h_aux ||
        c->gexec_stage != c->stage.p)
      capture_run(c, fp, nj);
    if (c->gexec) {
      ST_CUDA(cudaGraphLaunch(c->gexec, c->stream), "graph launch");
      launched = true;
      ++c->graph_launches;
    }
  }
  if (!launched) {
    st_status s = enqueue_run(c, fp, nj, want_export, false);
    if (s != ST_OK) return s;
  }
  const size_t n_groups = groups.size() - 1;
  c->launches += (nj > 0 ? 1 : 0) +
                 (int32_t)n_groups * ((c->cache_blocks > 0 ? (c->cache_any_flagged ? 5 : 4) : 0) +
                                      (nj > 0 ? 4 : 0) + (c->cache_grid > 0 ? 1 : 0));
  c->pending = true;
  c->pend_first = first;
  c->pend_last = last;
  c->pend_export = want_export;
  return ST_OK;
}

// Waits for the enqueued run and turns its counters and flags into job statistics and a status.
st_status finish_range(st_ctx* c, st_sphere* ex_out, int64_t ex_cap, int64_t* ex_n) {
  if (!c->pending) return ST_OK;
  c->pending = false;
  const size_t first = c->pend_first, last = c->pend_last, nj = last - first;
  ST_CUDA(cudaEventSynchronize(c->ev[3]), "run");
  const JobAux* aux = c->h_aux;
  int errflags[4] = {c->h_err[0], c->h_err[1], c->h_err[2], c->h_err[3]};
  unsigned long long exn = 0;
  if (c->pend_export) std::memcpy(&exn, c->h_err + 4, 8);
  {
    float a = 0, b = 0;
    cudaEventElapsedTime(&a, c->ev[0], c->ev[1]);
    cudaEventElapsedTime(&b, c->ev[4], c->ev[2]);
    c->t_prep += a;
    c->t_fused += b;
  }
  st_status result = ST_OK;
  for (size_t i = 0; i < nj; ++i) {
    JobHost& J = c->jobs[first + i];
    J.ran = true;
    J.stats.hits = aux[i].hits;
    J.stats.spheres = aux[i].spheres;
    J.stats.binned = aux[i].binned;
    J.stats.inbox = aux[i].inbox;
    J.stats.grid_exponent = st::choose_grid_exponent(aux[i].e_min, aux[i].e_max, J.track.n,
                                                     aux[i].flags & st::kAuxNonzero);
    J.stats.status = (aux[i].flags & st::kAuxNonfinite) ? ST_ERR_NONFINITE_EDEP : ST_OK;
    if (J.stats.status != ST_OK && result == ST_OK) {
      result = ST_ERR_NONFINITE_EDEP;
      c->err = "job " + std::to_string(first + i) + " has a non-finite edep/((2/3)d); it was skipped";
    }
  }
  if (errflags[0] & 1) {
    c->g_dirty = true;
    c->cache_valid = false;
    c->err = "spill table overflow";
    return ST_ERR_DEVICE_OVERFLOW;
  }
  if (errflags[0] & (4 | 8)) {
    // a work item gave up (no free spill table, or a shared unit's table was never published)
    c->g_dirty = true;
    c->cache_valid = false;
    c->err = (errflags[0] & 4) ? "spill-table pool exhausted" : "shared-unit table wait expired";
    return ST_ERR_DEVICE_WAIT;
  }
  if (ex_out) {
    if ((errflags[0] & 2) || exn > (unsigned long long)ex_cap) {
      if (ex_n) *ex_n = (int64_t)exn;
      c->err = "export buffer too small";
      return ST_ERR_CAPACITY;
    }
    std::vector<st::SphereRecord> rec((size_t)exn);
    if (exn) {
      ST_CUDA(cudaMemcpy(rec.data(), c->ex_buf.p, (size_t)exn * sizeof(st::SphereRecord), cudaMemcpyDeviceToHost), "read export");
    }
    for (size_t i = 0; i < rec.size(); ++i) {
      ex_out[i].key = rec[i].key;
      ex_out[i].y = rec[i].y;
      ex_out[i].os = rec[i].os;
      ex_out[i].job = rec[i].job + (int32_t)first;
    }
    if (ex_n) *ex_n = (int64_t)exn;
  }
  return result;
}

// Runs jobs [first, last) of the context in one batched launch sequence and waits for it.
st_status run_range(st_ctx* c, size_t first, size_t last, st_sphere* ex_out, int64_t ex_cap,
                    int64_t* ex_n) {
  if (first >= last) {
    if (ex_n) *ex_n = 0;
    return ST_OK;
  }
  if (c->pending) {
    st_status s = finish_range(c, nullptr, 0, nullptr);
    if (s != ST_OK) return s;
  }
  st_status s = launch_range(c, first, last, ex_out != nullptr, ex_cap);
  if (s != ST_OK) return s;
  return finish_range(c, ex_out, ex_cap, ex_n);
}

}  // namespace

// =============================================================================================
// C ABI
// =============================================================================================
extern "C" {

const char* st_status_string(st_status s) {
  switch (s) {
    case ST_OK: return "ok";
    case ST_ERR_INVALID_ARGUMENT: return "invalid argument";
    case ST_ERR_BAD_GEOMETRY: return "bad geometry";
    case ST_ERR_BAD_HISTOGRAM: return "bad histogram specification";
    case ST_ERR_CUDA: return "CUDA error";
    case ST_ERR_OUT_OF_MEMORY: return "out of device memory";
    case ST_ERR_CAPACITY: return "capacity exceeded";
    case ST_ERR_NONFINITE_EDEP: return "non-finite energy deposit";
    case ST_ERR_DEVICE_OVERFLOW: return "device table overflow";
    case ST_ERR_NOT_FOUND: return "not found";
    case ST_ERR_STATE: return "invalid state";
    case ST_ERR_IO: return "I/O error";
    case ST_ERR_CONFIG: return "configuration error";
    case ST_ERR_NO_DEVICE: return "no CUDA device";
    case ST_ERR_DEVICE_WAIT: return "device-side wait expired";
  }
  return "unknown status";
}

const char* st_version(void) { return "supertrack_b200 0.1.0 (sm_100a)"; }

st_status st_geometry_make(double half_length, double sphere_diameter, st_geometry* out) {
  if (!out) return ST_ERR_INVALID_ARGUMENT;
  st::Geometry g;
  if (st::make_geometry(half_length, sphere_diameter, &g) != 0) return ST_ERR_BAD_GEOMETRY;
  out->scoring_region_length = g.scoringRegionLength;
  out->scoring_region_half_length = g.scoringRegionHalfLength;
  out->greatest_sphere_offset = g.greatestSphereOffset;
  out->num_spheres_linear = g.numSpheresLinear;
  out->reserved = 0;
  out->sphere_diameter = g.sphereDiameter;
  out->sphere_radius = g.sphereRadius;
  return ST_OK;
}

st_status st_hist_edges(int32_t type, int32_t nbins, float lower, float upper, double* edges_out) {
  if (!edges_out) return ST_ERR_INVALID_ARGUMENT;
  std::vector<double> e;
  if (!st::MakeEdges(type, nbins, lower, upper, &e)) return ST_ERR_BAD_HISTOGRAM;
  std::memcpy(edges_out, e.data(), e.size() * sizeof(double));
  return ST_OK;
}

st_status st_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  if (!ctr || !key || !out) return ST_ERR_INVALID_ARGUMENT;
  uint32_t c[4] = {ctr[0], ctr[1], ctr[2], ctr[3]};
  st::philox4x32_10(c, key[0], key[1]);
  for (int i = 0; i < 4; ++i) out[i] = c[i];
  return ST_OK;
}

st_status st_oversample_shifts(const st_geometry* g, int32_t shift_track, uint64_t seed,
                               uint64_t track_id, uint32_t os_begin, uint32_t n_os,
                               double* sxsy) {
  if (!g || (!sxsy && n_os)) return ST_ERR_INVALID_ARGUMENT;
  for (uint32_t i = 0; i < n_os; ++i) {
    float ux, uy;
    st::shift_uniforms(seed, track_id, os_begin + i, shift_track, &ux, &uy);
    sxsy[2 * i] = st::shift_from_uniform(ux, g->scoring_region_length, g->scoring_region_half_length);
    sxsy[2 * i + 1] = st::shift_from_uniform(uy, g->scoring_region_length, g->scoring_region_half_length);
  }
  return ST_OK;
}

int32_t st_grid_exponent(int32_t e_min, int32_t e_max, int64_t n, int32_t any_nonzero) {
  return st::choose_grid_exponent(e_min, e_max, n, any_nonzero);
}

void st_to_fixed(double v, int32_t e0, uint64_t* lo, uint64_t* hi) {
  uint64_t a = 0, b = 0;
  st::to_fixed(v, e0, &a, &b);
  if (lo) *lo = a;
  if (hi) *hi = b;
}

double st_from_fixed(uint64_t lo, uint64_t hi, int32_t e0) { return st::from_fixed(lo, hi, e0); }

st_status st_ctx_create(int32_t device, void* stream, st_ctx** out) {
  if (!out) return ST_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return ST_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= ndev) return ST_ERR_INVALID_ARGUMENT;
  if (cudaSetDevice(device) != cudaSuccess) return ST_ERR_CUDA;
  st_ctx* c = new st_ctx();
  c->device = device;
  cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device);
  if (stream) {
    c->stream = (cudaStream_t)stream;
  } else {
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete c;
      return ST_ERR_CUDA;
    }
    c->own_stream = true;
  }
  for (auto& e : c->ev) cudaEventCreate(&e);
  *out = c;
  return ST_OK;
}

st_status st_ctx_destroy(st_ctx* c) {
  if (!c) return ST_ERR_INVALID_ARGUMENT;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  DevBuf* bufs[] = {&c->track_arena, &c->pxy, &c->pdz2, &c->pv, &c->pkey,
                    &c->d_jobs, &c->d_aux, &c->d_hists, &c->d_items, &c->d_blk,
                    &c->d_counter, &c->d_err, &c->d_blk_count, &c->d_blk_off, &c->d_blk_job, &c->c_cells,
                    &c->pz, &c->u_next, &c->u_done, &c->u_table,
                    &c->pool, &c->d_plan, &c->d_plan_misc, &c->g_keys, &c->g_lo, &c->g_hi,
                    &c->g_used, &c->g_count, &c->ex_buf, &c->ex_count, &c->h_counts,
                    &c->h_yfy, &c->h_edges};
  drop_graph(c);
  if (c->copy_stream) {
    cudaStreamSynchronize(c->copy_stream);
    cudaStreamDestroy(c->copy_stream);
  }
  for (cudaEvent_t e : c->up_ev) cudaEventDestroy(e);
  for (DevBuf* b : bufs) release(*b);
  for (auto& e : c->ev) if (e) cudaEventDestroy(e);
  if (c->h_aux) cudaFreeHost(c->h_aux);
  if (c->h_err) cudaFreeHost(c->h_err);
  if (c->stage.p) cudaFreeHost(c->stage.p);
  if (c->own_stream) cudaStreamDestroy(c->stream);
  delete c;
  return ST_OK;
}

st_status st_ctx_set_stream(st_ctx* c, void* stream) {
  if (!c) return ST_ERR_INVALID_ARGUMENT;
  cudaStreamSynchronize(c->stream);
  if (c->own_stream) cudaStreamDestroy(c->stream);
  c->own_stream = false;
  if (stream) {
    c->stream = (cudaStream_t)stream;
  } else {
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) return ST_ERR_CUDA;
    c->own_stream = true;
  }
  return ST_OK;
}

st_status st_ctx_last_error(const st_ctx* c, char* buf, size_t len) {
  if (!c || !buf || !len) return ST_ERR_INVALID_ARGUMENT;
  std::snprintf(buf, len, "%s", c->err.c_str());
  return ST_OK;
}

int32_t st_ctx_sm_count(const st_ctx* c) { return c ? c->sm_count : 0; }

st_status st_ctx_order_after(st_ctx* c, const st_ctx* other) {
  if (!c || !other || c == other) return ST_ERR_INVALID_ARGUMENT;
  c->order_after = other->ev[2];
  return ST_OK;
}

st_status st_ctx_enable_timing(st_ctx* c, int32_t on) {
  if (!c) return ST_ERR_INVALID_ARGUMENT;
  c->timing = on != 0;
  return ST_OK;
}

st_status st_ctx_last_timing(const st_ctx* c, float* prepare_ms, float* fused_ms, int32_t* launches) {
  if (!c) return ST_ERR_INVALID_ARGUMENT;
  if (prepare_ms) *prepare_ms = c->t_prep;
  if (fused_ms) *fused_ms = c->t_fused;
  if (launches) *launches = c->launches;
  return ST_OK;
}

st_status st_ctx_set_tuning(st_ctx* c, int64_t item_cost, int32_t grid) {
  if (!c || item_cost < 0 || grid < 0) return ST_ERR_INVALID_ARGUMENT;
  if (item_cost > 0) c->item_cost = item_cost;
  c->grid_override = grid;
  return ST_OK;
}

st_status st_ctx_set_param(st_ctx* c, const char* name, int64_t v) {
  if (!c || !name) return ST_ERR_INVALID_ARGUMENT;
  const std::string n(name);
  if (n == "item_cost" && v >= 256 && v <= ((int64_t)1 << 40)) c->item_cost = v;
  else if (n == "grid" && v >= 0 && v <= 1 << 20) c->grid_override = (int)v;
  else if (n == "chunk_windows" && v >= 1 && v <= 1024) c->chunk_windows = (int)v;
  else if (n == "max_helpers" && v >= 1 && v <= 4096) c->max_helpers = (int)v;
  else if (n == "share_divisor" && v >= 0 && v <= 1 << 20) c->share_divisor = (int)v;
  else if (n == "shared_min_chunks" && v >= 1 && v <= 1 << 20) c->min_chunks = (int)v;
  else if (n == "precision" && (v == 64 || v == 32)) { c->precision = (int)v; drop_graph(c); }
  else if (n == "flag_min_kept" && v >= 0) c->flag_min_kept = v;
  else if (n == "flag_cells_limit" && v >= 0) c->flag_cells_limit = v;
  else if (n == "sort_deposits" && v >= 0 && v <= 2) c->sort_deposits = (int)v;
  else if (n == "spill_budget_bytes" && v >= 0) c->spill_budget = v;
  else if (n == "table_slots" && (v == 0 || v == 4096 || v == 8192)) c->table_slots = (int)v;
  else if (n == "pipeline_bytes" && v >= 0) c->pipeline_bytes = v > 0 ? v : ((int64_t)1 << 62);
  else if (n == "pipeline_max_os" && v >= 0) c->pipeline_max_os = v;
  else if (n == "graphs" && (v == 0 || v == 1)) { c->use_graphs = v != 0; drop_graph(c); }
  else return ST_ERR_INVALID_ARGUMENT;
  c->cache_valid = false;
  return ST_OK;
}

st_status st_ctx_get_param(const st_ctx* c, const char* name, int64_t* v) {
  if (!c || !name || !v) return ST_ERR_INVALID_ARGUMENT;
  const std::string n(name);
  if (n == "item_cost") *v = c->item_cost;
  else if (n == "grid") *v = c->grid_override;
  else if (n == "chunk_windows") *v = c->chunk_windows;
  else if (n == "max_helpers") *v = c->max_helpers;
  else if (n == "share_divisor") *v = c->share_divisor;
  else if (n == "shared_min_chunks") *v = c->min_chunks;
  else if (n == "precision") *v = c->precision;
  else if (n == "flag_min_kept") *v = c->flag_min_kept;
  else if (n == "flag_cells_limit") *v = c->flag_cells_limit;
  else if (n == "sort_deposits") *v = c->sort_deposits;
  else if (n == "spill_budget_bytes") *v = c->spill_budget;
  else if (n == "table_slots") *v = c->table_slots;
  else if (n == "pipeline_bytes") *v = c->pipeline_bytes;
  else if (n == "pipeline_max_os") *v = c->pipeline_max_os;
  else if (n == "graphs") *v = c->use_graphs ? 1 : 0;
  else if (n == "graph_launches") *v = c->graph_launches;  // read-only: runs replayed from a graph
  else if (n == "last_grid") *v = c->cache_grid;       // read-only: CTAs of the last fused launch
  else if (n == "last_host_launch_us") *v = (int64_t)c->host_launch_us;
  else if (n == "last_host_tables_us") *v = (int64_t)c->host_tables_us;
  else if (n == "last_host_alloc_us") *v = (int64_t)c->host_alloc_us;
  else if (n == "last_host_allocs") *v = c->host_allocs;
  else if (n == "last_host_meminfo_us") *v = (int64_t)c->host_meminfo_us;
  else if (n == "spill_slots") *v = (int64_t)c->gcap;  // read-only: slots per spill table
  else return ST_ERR_INVALID_ARGUMENT;
  return ST_OK;
}

// Work-planning autotuner: coordinate descent over the planning parameters on the context's
// queued jobs, each candidate timed (prepare + fused device time, best of two runs). Results are
// exact and order-free, so parameters change only the time. The histograms are saved before the
// trials and restored after them.
st_status st_ctx_autotune(st_ctx* c, int32_t max_trials, st_tune_result* out) {
  if (!c || !out || max_trials < 1) return ST_ERR_INVALID_ARGUMENT;
  if (c->jobs.empty()) return ST_ERR_STATE;
  cudaSetDevice(c->device);
  if (c->pending) {
    const st_status s = finish_range(c, nullptr, 0, nullptr);
    if (s != ST_OK && s != ST_ERR_NONFINITE_EDEP) return s;
  }
  DevBuf save_c, save_y;
  const size_t hb = (size_t)c->h_bins * 8;
  if (hb) {
    ST_CUDA(ensure(save_c, hb), "autotune save");
    ST_CUDA(ensure(save_y, hb), "autotune save");
    ST_CUDA(cudaMemcpyAsync(save_c.p, c->h_counts.p, hb, cudaMemcpyDeviceToDevice, c->stream), "autotune save");
    ST_CUDA(cudaMemcpyAsync(save_y.p, c->h_yfy.p, hb, cudaMemcpyDeviceToDevice, c->stream), "autotune save");
  }
  std::vector<char> ran(c->jobs.size());
  for (size_t j = 0; j < c->jobs.size(); ++j) ran[j] = c->jobs[j].ran;
  st_status fail = ST_OK;
  auto trial = [&]() -> double {
    double best = 1e300;
    for (int rep = 0; rep < 2 && fail == ST_OK; ++rep) {
      for (auto& j : c->jobs) j.ran = false;
      c->t_prep = c->t_fused = 0;
      const st_status s = run_range(c, 0, c->jobs.size(), nullptr, 0, nullptr);
      if (s != ST_OK && s != ST_ERR_NONFINITE_EDEP) { fail = s; break; }
      best = std::min(best, (double)c->t_prep + (double)c->t_fused);
    }
    return best;
  };
  struct Knob {
    const char* name;
    std::vector<int64_t> values;
  };
  const Knob knobs[] = {
      {"item_cost", {1 << 16, 1 << 17, 1 << 18, 1 << 19, 1 << 20, 1 << 21}},
      {"sort_deposits", {0, 1, 2}},
      {"chunk_windows", {1, 2, 4, 8, 16}},
      {"max_helpers", {8, 16, 32, 64, 148}},
      {"share_divisor", {2, 4, 8, 16, 0}},
      {"table_slots", {0, 4096}},
      {"flag_cells_limit", {0, st::kFlagCellsLimit, (int64_t)1 << 50}},
  };
  out->default_ms = trial();
  double best = out->default_ms;
  int trials = 1;
  for (const Knob& k : knobs) {
    int64_t cur = 0;
    st_ctx_get_param(c, k.name, &cur);
    for (int64_t v : k.values) {
      if (v == cur || trials >= max_trials || fail != ST_OK) continue;
      st_ctx_set_param(c, k.name, v);
      const double t = trial();
      ++trials;
      if (fail == ST_OK && t < best * 0.99) {
        best = t;
        cur = v;
      } else {
        st_ctx_set_param(c, k.name, cur);
      }
    }
  }
  if (hb) {
    ST_CUDA(cudaMemcpyAsync(c->h_counts.p, save_c.p, hb, cudaMemcpyDeviceToDevice, c->stream), "autotune restore");
    ST_CUDA(cudaMemcpyAsync(c->h_yfy.p, save_y.p, hb, cudaMemcpyDeviceToDevice, c->stream), "autotune restore");
    ST_CUDA(cudaStreamSynchronize(c->stream), "autotune restore");
  }
  release(save_c);
  release(save_y);
  for (size_t j = 0; j < c->jobs.size(); ++j) c->jobs[j].ran = ran[j] != 0;
  if (fail != ST_OK) return fail;
  out->best_ms = best;
  out->item_cost = c->item_cost;
  out->chunk_windows = c->chunk_windows;
  out->max_helpers = c->max_helpers;
  out->share_divisor = c->share_divisor;
  out->table_slots = c->table_slots;
  out->trials = trials;
  out->sort_deposits = c->sort_deposits;
  out->flag_cells_limit = c->flag_cells_limit;
  return ST_OK;
}

// Grows a histogram arena to `bytes`, keeping its contents.
static st_status grow_arena(st_ctx* c, DevBuf& b, size_t used, size_t bytes) {
  if (b.bytes >= bytes) return ST_OK;
  size_t cap = std::max<size_t>(bytes, b.bytes * 2);
  void* p = nullptr;
  ST_CUDA(cudaMalloc(&p, cap), "histogram arena");
  if (used) ST_CUDA(cudaMemcpyAsync(p, b.p, used, cudaMemcpyDeviceToDevice, c->stream), "histogram arena");
  ST_CUDA(cudaStreamSynchronize(c->stream), "histogram arena");
  if (b.p) cudaFree(b.p);
  b.p = p;
  b.bytes = cap;
  return ST_OK;
}

st_status st_hist_create(st_ctx* c, int32_t type, int32_t nbins, float lower, float upper,
                         int32_t* hist_id) {
  if (!c || !hist_id) return ST_ERR_INVALID_ARGUMENT;
  HistHost h;
  if (!st::MakeEdges(type, nbins, lower, upper, &h.edges)) return ST_ERR_BAD_HISTOGRAM;
  h.type = type; h.nbins = nbins; h.lower = lower; h.upper = upper;
  cudaSetDevice(c->device);
  h.off = c->h_bins;
  h.eoff = c->h_edge_total;
  st_status s;
  if ((s = grow_arena(c, c->h_counts, (size_t)c->h_bins * 8, (size_t)(c->h_bins + nbins) * 8)) != ST_OK) return s;
  if ((s = grow_arena(c, c->h_yfy, (size_t)c->h_bins * 8, (size_t)(c->h_bins + nbins) * 8)) != ST_OK) return s;
  if ((s = grow_arena(c, c->h_edges, (size_t)c->h_edge_total * 8, (size_t)(c->h_edge_total + nbins + 1) * 8)) != ST_OK) return s;
  ST_CUDA(cudaMemcpyAsync((double*)c->h_edges.p + h.eoff, h.edges.data(), h.edges.size() * 8, cudaMemcpyHostToDevice, c->stream), "histogram edges");
  ST_CUDA(cudaMemsetAsync((unsigned long long*)c->h_counts.p + h.off, 0, (size_t)nbins * 8, c->stream), "histogram counts");
  ST_CUDA(cudaMemsetAsync((double*)c->h_yfy.p + h.off, 0, (size_t)nbins * 8, c->stream), "histogram yfy");
  c->h_bins += nbins;
  c->h_edge_total += nbins + 1;
  c->hists.push_back(std::move(h));
  *hist_id = (int32_t)c->hists.size() - 1;
  c->cache_valid = false;
  return ST_OK;
}

st_status st_hist_read(st_ctx* c, int32_t hist_id, int64_t* counts, double* yfy) {
  if (!c || hist_id < 0 || hist_id >= (int32_t)c->hists.size()) return ST_ERR_INVALID_ARGUMENT;
  const HistHost& h = c->hists[hist_id];
  if (counts) ST_CUDA(cudaMemcpyAsync(counts, (unsigned long long*)c->h_counts.p + h.off, (size_t)h.nbins * 8, cudaMemcpyDeviceToHost, c->stream), "histogram read");
  if (yfy) ST_CUDA(cudaMemcpyAsync(yfy, (double*)c->h_yfy.p + h.off, (size_t)h.nbins * 8, cudaMemcpyDeviceToHost, c->stream), "histogram read");
  ST_CUDA(cudaStreamSynchronize(c->stream), "histogram read");
  return ST_OK;
}

st_status st_hist_read_all(st_ctx* c, int64_t* counts, double* yfy, int64_t cap, int64_t* n_bins) {
  if (!c) return ST_ERR_INVALID_ARGUMENT;
  if (n_bins) *n_bins = c->h_bins;
  if (!counts && !yfy) return ST_OK;
  if (cap < c->h_bins) return ST_ERR_CAPACITY;
  if (c->h_bins == 0) return ST_OK;
  // cudaMemcpyDefault: the destination may be host memory or device memory (a multi-GPU
  // caller gathers the spectra in a device buffer for its all-reduce)
  if (counts) ST_CUDA(cudaMemcpyAsync(counts, c->h_counts.p, (size_t)c->h_bins * 8, cudaMemcpyDefault, c->stream), "histogram read");
  if (yfy) ST_CUDA(cudaMemcpyAsync(yfy, c->h_yfy.p, (size_t)c->h_bins * 8, cudaMemcpyDefault, c->stream), "histogram read");
  ST_CUDA(cudaStreamSynchronize(c->stream), "histogram read");
  return ST_OK;
}

st_status st_hist_offset(const st_ctx* c, int32_t hist_id, int64_t* first_bin) {
  if (!c || !first_bin || hist_id < 0 || hist_id >= (int32_t)c->hists.size()) return ST_ERR_INVALID_ARGUMENT;
  *first_bin = c->hists[hist_id].off;
  return ST_OK;
}

st_status st_hist_read_bins_async(st_ctx* c, int64_t first_bin, int64_t n_bins, int64_t* counts,
                                  double* yfy) {
  if (!c || first_bin < 0 || n_bins < 0 || first_bin + n_bins > c->h_bins) return ST_ERR_INVALID_ARGUMENT;
  if (n_bins == 0) return ST_OK;
  cudaSetDevice(c->device);
  if (counts) ST_CUDA(cudaMemcpyAsync(counts, (unsigned long long*)c->h_counts.p + first_bin, (size_t)n_bins * 8, cudaMemcpyDeviceToHost, c->stream), "histogram read");
  if (yfy) ST_CUDA(cudaMemcpyAsync(yfy, (double*)c->h_yfy.p + first_bin, (size_t)n_bins * 8, cudaMemcpyDeviceToHost, c->stream), "histogram read");
  // an enqueued run now completes only once the copies have landed
  if (c->pending) ST_CUDA(cudaEventRecord(c->ev[3], c->stream), "event");
  return ST_OK;
}

st_status st_hist_reset(st_ctx* c, int32_t hist_id) {
  if (!c || hist_id < -1 || hist_id >= (int32_t)c->hists.size()) return ST_ERR_INVALID_ARGUMENT;
  const int64_t off = hist_id < 0 ? 0 : c->hists[hist_id].off;
  const int64_t nb = hist_id < 0 ? c->h_bins : c->hists[hist_id].nbins;
  if (nb == 0) return ST_OK;
  ST_CUDA(cudaMemsetAsync((unsigned long long*)c->h_counts.p + off, 0, (size_t)nb * 8, c->stream), "histogram reset");
  ST_CUDA(cudaMemsetAsync((double*)c->h_yfy.p + off, 0, (size_t)nb * 8, c->stream), "histogram reset");
  return ST_OK;
}

st_status st_hist_nbins(const st_ctx* c, int32_t hist_id, int32_t* nbins) {
  if (!c || !nbins || hist_id < 0 || hist_id >= (int32_t)c->hists.size()) return ST_ERR_INVALID_ARGUMENT;
  *nbins = c->hists[hist_id].nbins;
  return ST_OK;
}

st_status st_hist_edges_of(const st_ctx* c, int32_t hist_id, double* edges) {
  if (!c || !edges || hist_id < 0 || hist_id >= (int32_t)c->hists.size()) return ST_ERR_INVALID_ARGUMENT;
  const auto& e = c->hists[hist_id].edges;
  std::memcpy(edges, e.data(), e.size() * 8);
  return ST_OK;
}

st_status st_job_submit(st_ctx* c, const st_track_view* track, const st_job_desc* desc,
                        int32_t* job_id) {
  if (!c || !track || !desc) return ST_ERR_INVALID_ARGUMENT;
  if (track->n < 0 || (track->n > 0 && (!track->x || !track->y || !track->z || !track->edep)))
    return ST_ERR_INVALID_ARGUMENT;
  // device arrays are read in place as doubles: a misaligned one would fault the prepare kernels
  if (track->on_device && track->n > 0 &&
      (((uintptr_t)track->x | (uintptr_t)track->y | (uintptr_t)track->z | (uintptr_t)track->edep) & 7))
    return ST_ERR_INVALID_ARGUMENT;
  if (track->n > (int64_t)1 << 40) return ST_ERR_CAPACITY;
  if (desc->hist_id < 0 || desc->hist_id >= (int32_t)c->hists.size()) return ST_ERR_INVALID_ARGUMENT;
  if (desc->zshift < ST_ZSHIFT_PLUS || desc->zshift > ST_ZSHIFT_NONE) return ST_ERR_INVALID_ARGUMENT;
  if (desc->n_oversamples > 0x7fffffffu) return ST_ERR_INVALID_ARGUMENT;
  JobHost J;
  if (st::make_geometry(desc->half_length, desc->sphere_diameter, &J.g) != 0) return ST_ERR_BAD_GEOMETRY;
  J.track = *track;
  J.desc = *desc;
  c->jobs.push_back(J);
  c->cache_valid = false;
  if (job_id) *job_id = (int32_t)c->jobs.size() - 1;
  return ST_OK;
}

static size_t first_unrun(const st_ctx* c) {
  size_t f = c->jobs.size();
  while (f > 0 && !c->jobs[f - 1].ran) --f;
  return f;
}

st_status st_run(st_ctx* c, int32_t mode) {
  if (!c) return ST_ERR_INVALID_ARGUMENT;
  cudaSetDevice(c->device);
  c->t_prep = c->t_fused = 0;
  c->launches = 0;
  const size_t first = first_unrun(c), last = c->jobs.size();
  if (mode == ST_RUN_BATCHED) return run_range(c, first, last, nullptr, 0, nullptr);
  if (mode != ST_RUN_PLAIN) return ST_ERR_INVALID_ARGUMENT;
  st_status worst = ST_OK;
  for (size_t j = first; j < last; ++j) {
    const st_status s = run_range(c, j, j + 1, nullptr, 0, nullptr);
    if (s != ST_OK && s != ST_ERR_NONFINITE_EDEP) return s;
    if (s != ST_OK) worst = s;
  }
  return worst;
}

st_status st_run_export(st_ctx* c, st_sphere* spheres_out, int64_t cap, int64_t* n_out) {
  if (!c || !spheres_out || cap < 0) return ST_ERR_INVALID_ARGUMENT;
  cudaSetDevice(c->device);
  c->t_prep = c->t_fused = 0;
  c->launches = 0;
  return run_range(c, first_unrun(c), c->jobs.size(), spheres_out, cap, n_out);
}

st_status st_run_async(st_ctx* c) {
  if (!c) return ST_ERR_INVALID_ARGUMENT;
  cudaSetDevice(c->device);
  if (c->pending) return ST_ERR_STATE;
  c->t_prep = c->t_fused = 0;
  c->launches = 0;
  const size_t first = first_unrun(c), last = c->jobs.size();
  if (first >= last) return ST_OK;
  return launch_range(c, first, last, false, 0);
}

st_status st_run_query(st_ctx* c, int32_t* done) {
  if (!c || !done) return ST_ERR_INVALID_ARGUMENT;
  if (!c->pending) { *done = 1; return ST_OK; }
  const cudaError_t e = cudaEventQuery(c->ev[3]);
  if (e == cudaErrorNotReady) { *done = 0; return ST_OK; }
  *done = 1;
  return finish_range(c, nullptr, 0, nullptr);
}

st_status st_run_finish(st_ctx* c) {
  if (!c) return ST_ERR_INVALID_ARGUMENT;
  cudaSetDevice(c->device);
  return finish_range(c, nullptr, 0, nullptr);
}

st_status st_hists_clear(st_ctx* c) {
  if (!c) return ST_ERR_INVALID_ARGUMENT;
  if (c->pending) return ST_ERR_STATE;
  c->hists.clear();
  c->h_bins = 0;
  c->h_edge_total = 0;
  c->cache_valid = false;
  return ST_OK;
}

st_status st_job_stats_get(st_ctx* c, int32_t job_id, st_job_stats* out) {
  if (!c || !out || job_id < 0 || job_id >= (int32_t)c->jobs.size()) return ST_ERR_INVALID_ARGUMENT;
  if (!c->jobs[job_id].ran) return ST_ERR_STATE;
  *out = c->jobs[job_id].stats;
  return ST_OK;
}

st_status st_jobs_clear(st_ctx* c) {
  if (!c) return ST_ERR_INVALID_ARGUMENT;
  c->jobs.clear();
  c->cache_valid = false;
  return ST_OK;
}

st_status st_jobs_reset(st_ctx* c) {
  if (!c) return ST_ERR_INVALID_ARGUMENT;
  for (auto& j : c->jobs) j.ran = false;
  return ST_OK;
}

st_status st_job_submit_many(st_ctx* c, int32_t n, const st_track_view* tracks,
                             const st_job_desc* descs, int32_t* job_ids) {
  if (!c || n < 0 || (n && (!tracks || !descs))) return ST_ERR_INVALID_ARGUMENT;
  for (int32_t i = 0; i < n; ++i) {
    int32_t id = -1;
    const st_status s = st_job_submit(c, &tracks[i], &descs[i], &id);
    if (s != ST_OK) return s;
    if (job_ids) job_ids[i] = id;
  }
  return ST_OK;
}

st_status st_measure_fp64_peak(st_ctx* c, double* ops_per_second) {
  if (!c || !ops_per_second) return ST_ERR_INVALID_ARGUMENT;
  cudaSetDevice(c->device);
  DevBuf out;
  ST_CUDA(ensure(out, 4096 * 8), "fp64 probe buffer");
  const int blocks = c->sm_count * 8, iters = 4096;
  float best = 1e30f;
  for (int rep = 0; rep < 4; ++rep) {
    ST_CUDA(cudaEventRecord(c->ev[0], c->stream), "event");
    ST_CUDA(st::launch_fp64_probe((double*)out.p, blocks, iters, c->stream), "fp64 probe");
    ST_CUDA(cudaEventRecord(c->ev[1], c->stream), "event");
    ST_CUDA(cudaEventSynchronize(c->ev[1]), "fp64 probe");
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
    if (rep > 0) best = std::min(best, ms);
  }
  release(out);
  // two FP64 operations (one multiply, one add) per chain step
  *ops_per_second = 2.0 * 8.0 * iters * (double)blocks * 256.0 / (best * 1e-3);
  return ST_OK;
}

st_status st_probe_unit_wait(st_ctx* c, int32_t published, int64_t max_polls, int32_t* table,
                             int32_t* error_flags) {
  if (!c || !table || !error_flags || max_polls < 0 || max_polls > ((int64_t)1 << 24))
    return ST_ERR_INVALID_ARGUMENT;
  cudaSetDevice(c->device);
  DevBuf buf;
  ST_CUDA(ensure(buf, 16), "wait probe buffer");
  // the unit's table slot: published, or "being acquired" (-2) by a first helper that never
  // publishes it; then the error flags and the probe's result
  const int init[3] = {published >= 0 ? published : -2, 0, 0};
  int out[3] = {0, 0, 0};
  int* d = (int*)buf.p;
  st_status s = ST_OK;
  if (cudaMemcpyAsync(d, init, sizeof(init), cudaMemcpyHostToDevice, c->stream) != cudaSuccess ||
      st::launch_unit_wait_probe(d, d + 1, d + 2, (long long)max_polls, c->stream) != cudaSuccess ||
      cudaMemcpyAsync(out, d, sizeof(out), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
      cudaStreamSynchronize(c->stream) != cudaSuccess) {
    c->err = std::string("wait probe: ") + cudaGetErrorString(cudaGetLastError());
    s = ST_ERR_CUDA;
  }
  release(buf);
  *table = out[2];
  *error_flags = out[1];
  return s;
}

st_status st_measure_smem_atomic_peak(st_ctx* c, double* atomics_per_second) {
  if (!c || !atomics_per_second) return ST_ERR_INVALID_ARGUMENT;
  cudaSetDevice(c->device);
  DevBuf out;
  ST_CUDA(ensure(out, (size_t)c->sm_count * 8), "smem probe buffer");
  const int blocks = c->sm_count, iters = 8192;
  float best = 1e30f;
  for (int rep = 0; rep < 4; ++rep) {
    ST_CUDA(cudaEventRecord(c->ev[0], c->stream), "event");
    ST_CUDA(st::launch_smem_atomic_probe((unsigned long long*)out.p, blocks, iters, c->stream),
            "smem probe");
    ST_CUDA(cudaEventRecord(c->ev[1], c->stream), "event");
    ST_CUDA(cudaEventSynchronize(c->ev[1]), "smem probe");
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
    if (rep > 0) best = std::min(best, ms);
  }
  release(out);
  *atomics_per_second = (double)iters * 1024.0 * (double)blocks / (best * 1e-3);
  return ST_OK;
}

st_status st_jobs_count(const st_ctx* c, int32_t* n) {
  if (!c || !n) return ST_ERR_INVALID_ARGUMENT;
  *n = (int32_t)c->jobs.size();
  return ST_OK;
}

}  // extern "C"
