/*
 * supertrack_b200 — C ABI of the B200-native VoxelConstrainedSphere superimposition path.
 *
 * The reference (JDecunha/SuperTrack) has no C ABI: its C++ run loop calls CUDA directly. Every
 * entry point below states which reference interface it replaces (file:line in the reference
 * tree). Conventions:
 *   - every function returns st_status (ST_OK == 0) and never aborts or throws;
 *   - plain pointers and sizes only; "device" pointers are CUDA device addresses on the
 *     context's device, everything else is host memory;
 *   - a context is used by one host thread at a time.
 */
#ifndef SUPERTRACK_B200_H
#define SUPERTRACK_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ST_API __attribute__((visibility("default")))

typedef enum {
  ST_OK = 0,
  ST_ERR_INVALID_ARGUMENT = 1,
  ST_ERR_BAD_GEOMETRY = 2,     /* sphere diameter <= 0, non-finite input, lattice too large */
  ST_ERR_BAD_HISTOGRAM = 3,    /* unknown type, nbins < 1, edges not finite/increasing      */
  ST_ERR_CUDA = 4,             /* a CUDA call failed; st_ctx_last_error has the text         */
  ST_ERR_OUT_OF_MEMORY = 5,
  ST_ERR_CAPACITY = 6,         /* a caller buffer or a fixed capacity is too small           */
  ST_ERR_NONFINITE_EDEP = 7,   /* a job's edep/((2/3)d) is NaN or infinite                   */
  ST_ERR_DEVICE_OVERFLOW = 8,  /* a device-side table or export buffer overflowed            */
  ST_ERR_NOT_FOUND = 9,
  ST_ERR_STATE = 10,           /* call out of order (e.g. reading stats before st_run)       */
  ST_ERR_IO = 11,
  ST_ERR_CONFIG = 12,          /* unusable .ini macro                                        */
  ST_ERR_NO_DEVICE = 13,
  ST_ERR_DEVICE_WAIT = 14      /* a bounded device-side wait expired; the run is incomplete */
} st_status;

typedef enum { ST_ZSHIFT_PLUS = 0, ST_ZSHIFT_MINUS = 1, ST_ZSHIFT_NONE = 2 } st_zshift_mode;
typedef enum { ST_HIST_LIN = 0, ST_HIST_LOG = 1 } st_hist_type;
typedef enum { ST_RUN_BATCHED = 0, ST_RUN_PLAIN = 1 } st_run_mode;

/* Fitted lattice; same fields as SphericalGeometry (SphericalGeometry.cuh:8-23). */
typedef struct {
  double scoring_region_length;
  double scoring_region_half_length;
  double greatest_sphere_offset;
  int32_t num_spheres_linear;
  int32_t reserved;
  double sphere_diameter;
  double sphere_radius;
} st_geometry;

/* One track: float64 SoA deposits (x, y, z in nm; edep in eV). on_device != 0 means the four
 * pointers are 8-byte-aligned device addresses (submit rejects others) that stay valid and
 * unchanged until st_jobs_clear; otherwise they are host memory (pinned memory makes the copy
 * asynchronous) read during st_run. The track is never modified. */
typedef struct {
  const double* x;
  const double* y;
  const double* z;
  const double* edep;
  int64_t n;
  int32_t on_device;
  int32_t reserved;
} st_track_view;

/* One superimposition job: a track, its geometry, its oversamples and the histogram it feeds. */
typedef struct {
  double half_length;        /* [VoxelConstrainedSphere] ScoringRegionHalfLength (nm)      */
  double sphere_diameter;    /* [VoxelConstrainedSphere] ScoringSphereDiameter (nm)        */
  int32_t zshift;            /* st_zshift_mode: z-origin shift +HL', -HL' or none          */
  int32_t shift_track;       /* [VoxelConstrainedSphere] ShiftTrack                        */
  uint32_t n_oversamples;    /* [Run] Oversamples                                          */
  int32_t hist_id;           /* from st_hist_create                                        */
  uint64_t seed;             /* task seed (ThreadAllocation.cc:28-31)                      */
  uint64_t track_id;         /* second Philox key word; 0 for tasks seeded per track       */
} st_job_desc;

typedef struct {
  uint64_t hits;             /* in-sphere deposits over all oversamples                    */
  uint64_t spheres;          /* (oversample, sphere) pairs with at least one hit           */
  uint64_t binned;           /* of those, the ones inside the histogram range              */
  uint64_t inbox;            /* deposit*oversamples inside the voxel after the shift       */
  int32_t grid_exponent;     /* exponent E0 of the job's exact accumulation grid           */
  int32_t status;            /* st_status of this job                                      */
} st_job_stats;

/* One exported sphere of one oversample (the reference's reduced VolumeEdepPair entry,
 * Histogram.cu:153): key = ix + iy*N + iz*N*N and its lineal energy y in keV/um. */
typedef struct {
  uint64_t key;
  double y;
  int32_t os;
  int32_t job;
} st_sphere;

typedef struct st_ctx st_ctx;

ST_API const char* st_status_string(st_status s);
ST_API const char* st_version(void);

/* --- host-only helpers (no GPU needed) ------------------------------------------------------ */

/* SphericalGeometry(half_length, sphere_diameter) — SphericalGeometry.cu:7-32. */
ST_API st_status st_geometry_make(double half_length, double sphere_diameter, st_geometry* out);

/* utils::LinSpace / utils::LogSpace as used by Histogram::ConstructBins —
 * utils.cc:8-31, Histogram.cu:53-72. edges_out holds nbins+1 doubles. */
ST_API st_status st_hist_edges(int32_t type, int32_t nbins, float lower, float upper,
                               double* edges_out);

/* The Philox4x32-10 block function used for the oversample shifts. */
ST_API st_status st_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* (sx, sy) of oversamples os_begin .. os_begin+n_os-1, interleaved in sxsy[2*n_os]: the shift
 * the fused kernel applies (replaces the cuRAND draw of GenerateRandomXYShift,
 * VoxelConstrainedSphereMethod.cu:61-83, and the shift formula at :176-177). */
ST_API st_status st_oversample_shifts(const st_geometry* g, int32_t shift_track, uint64_t seed,
                                      uint64_t track_id, uint32_t os_begin, uint32_t n_os,
                                      double* sxsy);

/* Fixed-point helpers of the exact per-sphere accumulation (exposed for verification). */
ST_API int32_t st_grid_exponent(int32_t e_min, int32_t e_max, int64_t n, int32_t any_nonzero);
ST_API void st_to_fixed(double v, int32_t e0, uint64_t* lo, uint64_t* hi);
ST_API double st_from_fixed(uint64_t lo, uint64_t hi, int32_t e0);

/* --- context ---------------------------------------------------------------------------- */

/* Creates a context on `device`; stream NULL creates a private non-blocking stream, otherwise
 * all work is enqueued on the given cudaStream_t. Replaces the per-worker CUDA state of
 * SuperTrackManager::Run's forked processes (SuperTrackManager.cu:53-56). */
ST_API st_status st_ctx_create(int32_t device, void* stream, st_ctx** out);
ST_API st_status st_ctx_destroy(st_ctx* ctx);
ST_API st_status st_ctx_set_stream(st_ctx* ctx, void* stream);
ST_API st_status st_ctx_last_error(const st_ctx* ctx, char* buf, size_t len);
ST_API int32_t st_ctx_sm_count(const st_ctx* ctx);
/* Kept for callers that switch timing on: every run is timed with CUDA events. */
ST_API st_status st_ctx_enable_timing(st_ctx* ctx, int32_t on);
/* Milliseconds of the last st_run / st_run_async (summed over its launches): prepare and plan
 * kernels, fused kernel (from its start, after any st_ctx_order_after wait), and the number of
 * kernel launches. */
ST_API st_status st_ctx_last_timing(const st_ctx* ctx, float* prepare_ms, float* fused_ms,
                                    int32_t* launches);
/* Measured FP64 add/multiply issue rate of the device (operations per second). */
ST_API st_status st_measure_fp64_peak(st_ctx* ctx, double* ops_per_second);
/* Runs, on the context's stream, the fused kernel's one cross-CTA wait (a helper of a shared
 * unit waiting for the unit's spill table to be published) against a unit table set to
 * `published` (>= 0), or never published (< 0), with at most max_polls sleeps (at most 2^24,
 * the fused kernel's own limit). *table receives what the wait got (-1 when it ran out) and
 * *error_flags the device error flags it set (8: a wait ran out, which st_run reports as
 * ST_ERR_DEVICE_WAIT). No counterpart in the reference: it checks on the device, without a
 * fault or a hang, that the wait gives up and reports instead of waiting forever. */
ST_API st_status st_probe_unit_wait(st_ctx* ctx, int32_t published, int64_t max_polls,
                                    int32_t* table, int32_t* error_flags);
/* Measured rate of conflict-free 64-bit shared-memory atomic additions of the device (one CTA
 * of 1024 threads per SM, the fused kernel's shape), in atomics per second. No counterpart in the
 * reference: the peak that the shared-memory roofline term of the fused kernel is set against. */
ST_API st_status st_measure_smem_atomic_peak(st_ctx* ctx, double* atomics_per_second);
/* Tuning knobs: target deposit*oversamples per work item, resident CTAs (0 = one per SM). */
ST_API st_status st_ctx_set_tuning(st_ctx* ctx, int64_t item_cost, int32_t grid);
/* Named work-planning parameters (all take effect at the next run):
 *   item_cost          deposit*oversamples per private work item            (default 262144)
 *   grid               resident CTAs of the fused kernel, 0 = one per SM     (default 0)
 *   chunk_windows      windows of 8192 kept deposits per chunk of a shared unit   (default 4)
 *   max_helpers        helper items per shared unit                          (default 32)
 *   share_divisor      a job runs as shared units (one per oversample) when its kept deposits
 *                      exceed batch units / (share_divisor * grid); 0 = never (default 8)
 *   shared_min_chunks  ... and exceed this many chunks                       (default 4)
 *   flag_min_kept      a multi-window job on a fine lattice (more than 8192 deposits, at least 4
 *                      oversamples, 128 or more spheres along an axis) gets window boundary flags
 *                      when more than this many of its deposits are kept; with fewer, its
 *                      spheres fit the shared-memory table without them      (default 16384)
 *   flag_cells_limit   boundary flags of such a job are found in a hash of cells of side d (27
 *                      cells probed per kept deposit) or of side 2d (8 probed; more deposits come
 *                      out flagged, whose spheres are then summed through the spill log at every
 *                      oversample): side 2d when its deposits per sphere diameter of track
 *                      length, n * d / (2 HL), times its oversamples are at most this; 0 = side
 *                      d for every job. Results do not depend on it          (default 25000)
 *   sort_deposits      prepare blocks (1024 source deposits) that write their kept deposits
 *                      grouped by d-cell, the groups in the order of their first deposit, so
 *                      that deposits of one sphere arrive together in the fused kernel: 0 none
 *                      (source order), 1 the blocks of jobs with window boundary flags (dense
 *                      multi-window tracks), 2 all. Results do not depend on it (sums are
 *                      exact)                                                (default 1)
 *   precision          64 = the reference's FP64 arithmetic; 32 = FP32 geometry variant: x, y,
 *                      shifts, the x/y box test, x/y lattice index and sphere distance in float
 *                      (z, keys and energies as in FP64). No reference counterpart: the
 *                      reference's readme asks for a float form (readme.md:29). Results are
 *                      not bound to the reference's                           (default 64)
 *   table_slots        shared-memory sphere table: 0 = 8192 slots when every histogram has at
 *                      most 600 bins, else 4096; 4096 = always 4096          (default 0)
 *   pipeline_bytes     runs with host-resident tracks upload them in groups on a second stream
 *                      while earlier groups compute; groups hold about this many bytes of
 *                      track data (the first and last about a quarter); 0 = one upload, then
 *                      one launch                                            (default 256 MiB)
 *   pipeline_max_os    ... only when the host tracks average at most this many oversamples
 *                      per deposit; a batch above it computes longer than it uploads and is
 *                      uploaded whole, then run at once (each group's launch tail would cost
 *                      more than the overlap saves)                          (default 50)
 *   graphs             1 = a rerun of the same jobs replays a CUDA graph of the whole run
 *                      (captured at the first rerun); 0 = enqueue every call (default 1)
 *   spill_budget_bytes device bytes for the spill tables (one per resident CTA, each able to
 *                      hold every sphere of the batch's largest job); the grid shrinks to fit;
 *                      0 = 30% of free device memory, or the full grid's tables when they
 *                      leave 16 GB free; at most 48 GB                       (default 0)
 * st_ctx_get_param also reads "last_grid" (CTAs of the last fused launch), "spill_slots"
 * (slots of each CTA's spill table), "graph_launches" (runs replayed from a CUDA graph) and
 * the host cost of the last launch in microseconds:
 * "last_host_launch_us", "last_host_tables_us", "last_host_alloc_us" (with "last_host_allocs"
 * allocations) and "last_host_meminfo_us". */
ST_API st_status st_ctx_set_param(st_ctx* ctx, const char* name, int64_t value);
ST_API st_status st_ctx_get_param(const st_ctx* ctx, const char* name, int64_t* value);

/* Autotuner: picks item_cost, sort_deposits, chunk_windows, max_helpers, share_divisor,
 * table_slots and flag_cells_limit for the context's queued jobs by timing them (coordinate descent, at most max_trials batched runs of
 * all jobs, best of two each). Replaces the reference's SuggestedCudaBlocks/SuggestedCudaThreads
 * keys (VoxelConstrainedSphereMethod.cu:27-28, Histogram.cu:37-38). Histograms and job states are
 * as before the call;
 * the chosen parameters stay set. */
typedef struct {
  double default_ms;           /* prepare + fused device time with the parameters on entry */
  double best_ms;              /* ... with the chosen parameters                           */
  int64_t item_cost;
  int32_t chunk_windows, max_helpers, share_divisor, table_slots;
  int32_t trials, sort_deposits;
  int64_t flag_cells_limit;
} st_tune_result;
ST_API st_status st_ctx_autotune(st_ctx* ctx, int32_t max_trials, st_tune_result* out);

/* --- histograms (device accumulators) ------------------------------------------------------ */

/* Histogram(nbins, binLower, binUpper, type) — Histogram.cu:16-28 / :30-43. */
ST_API st_status st_hist_create(st_ctx* ctx, int32_t type, int32_t nbins, float lower,
                                float upper, int32_t* hist_id);
/* Copies the accumulated f(y) counts (int64) and y*f(y) sums (float64) to host arrays of nbins
 * (either may be NULL). Replaces Histogram::AccumulateCPUHistogram/GetCPUHistogram
 * (Histogram.cu:177-186, Histogram.cuh:47). */
ST_API st_status st_hist_read(st_ctx* ctx, int32_t hist_id, int64_t* counts, double* yfy);
/* Zeroes one histogram, or all of them with hist_id = -1. */
ST_API st_status st_hist_reset(st_ctx* ctx, int32_t hist_id);
/* Copies every histogram of the context in two transfers: counts/yfy (host or device memory)
 * receive all bins in histogram creation order (st_hist_offset gives each histogram's first
 * bin); cap is the room in each array; n_bins receives the total. */
ST_API st_status st_hist_read_all(st_ctx* ctx, int64_t* counts, double* yfy, int64_t cap,
                                  int64_t* n_bins);
ST_API st_status st_hist_offset(const st_ctx* ctx, int32_t hist_id, int64_t* first_bin);
/* Copies bins [first_bin, first_bin + n_bins) of the context's histograms (in creation order,
 * see st_hist_offset) to counts/yfy, enqueued on the context's stream only (host arrays should
 * be pinned); a run in flight (st_run_async) reports completion only after these copies. */
ST_API st_status st_hist_read_bins_async(st_ctx* ctx, int64_t first_bin, int64_t n_bins,
                                         int64_t* counts, double* yfy);
ST_API st_status st_hist_nbins(const st_ctx* ctx, int32_t hist_id, int32_t* nbins);
ST_API st_status st_hist_edges_of(const st_ctx* ctx, int32_t hist_id, double* edges);

/* --- jobs ---------------------------------------------------------------------------------- */

/* Queues one track for superimposition. Replaces, per task, Track::AllocateAndLoadTrack +
 * VoxelConstrainedSphereMethod::AllocateTrackProcess + the N_os calls of ProcessTrack and
 * Histogram::SortReduceAndAddToHistogram (SuperTrackManager.cu:61-75). */
ST_API st_status st_job_submit(st_ctx* ctx, const st_track_view* track, const st_job_desc* desc,
                               int32_t* job_id);
/* Runs every queued job that has not run yet. ST_RUN_BATCHED: one prepare launch and one
 * persistent work-stealing launch for all of them; ST_RUN_PLAIN: one track at a time, each
 * with its own launches and a host synchronisation (the reference's per-task loop shape). */
ST_API st_status st_run(st_ctx* ctx, int32_t mode);
ST_API st_status st_job_stats_get(st_ctx* ctx, int32_t job_id, st_job_stats* out);
/* Asynchronous form of st_run(ST_RUN_BATCHED): enqueues the run on the context's stream and
 * returns; st_run_query reports whether it finished (and then collects its statistics and
 * status), st_run_finish waits for it. One run per context may be in flight. */
ST_API st_status st_run_async(st_ctx* ctx);
ST_API st_status st_run_query(st_ctx* ctx, int32_t* done);
ST_API st_status st_run_finish(st_ctx* ctx);
/* The fused kernel of ctx's next run starts only after the fused kernel last enqueued by other
 * (a context on another stream of the same device) has finished; its prepare stage may overlap. */
ST_API st_status st_ctx_order_after(st_ctx* ctx, const st_ctx* other);
/* Forgets every histogram of the context (device memory is kept for reuse); ids restart at 0.
 * Queued jobs that refer to a forgotten histogram make the next run return ST_ERR_STATE (clear
 * or resubmit them); st_hist_reset(ctx, -1) zeroes every histogram instead. */
ST_API st_status st_hists_clear(st_ctx* ctx);
/* Queues n jobs at once (tracks[i] with descs[i]); job_ids may be NULL. */
ST_API st_status st_job_submit_many(st_ctx* ctx, int32_t n, const st_track_view* tracks,
                                    const st_job_desc* descs, int32_t* job_ids);
/* Marks every queued job as not yet run, so the next st_run runs the same jobs again (host
 * tracks are copied again; the launch set-up of an unchanged batch is reused). */
ST_API st_status st_jobs_reset(st_ctx* ctx);
/* Forgets all jobs (their device copies are released for reuse). */
ST_API st_status st_jobs_clear(st_ctx* ctx);
ST_API st_status st_jobs_count(const st_ctx* ctx, int32_t* n);

/* Like st_run(ST_RUN_BATCHED) but also returns every (oversample, sphere) with its lineal
 * energy, in no particular order; spheres_out has room for cap records. The exported list is
 * the reference's per-oversample reduced VolumeEdepPair (Histogram.cu:150-153). */
ST_API st_status st_run_export(st_ctx* ctx, st_sphere* spheres_out, int64_t cap, int64_t* n_out);

/* --- serving: continuous batching of arriving jobs ------------------------------------------
 * Replaces the reference's static, fork-per-thread task loop (SuperTrackManager.cu:49-102) for
 * jobs that arrive over time. A worker thread admits queued jobs while their device footprint
 * (prepared records, boundary cells, histogram) fits the budget, batches them into one launch
 * sequence on one of two contexts (two streams: the next batch is enqueued while the previous one
 * is still on the GPU), and on completion copies each job's spectrum to the caller's host arrays
 * and records its latency. Tracks must be device-resident and stay valid until completion. */
typedef struct st_server st_server;
typedef struct {
  uint64_t tag;              /* the caller's tag from st_server_submit                      */
  int32_t status;            /* st_status of the job                                        */
  int32_t batch;             /* index of the batch that ran it                              */
  int64_t submit_ns;         /* steady-clock times: submitted, its batch launched, done     */
  int64_t start_ns;
  int64_t done_ns;
} st_completion;

typedef struct {
  int32_t batch, slot, n_jobs, status;
  double units;              /* deposit x oversamples of the batch                           */
  int64_t launch_ns;         /* steady clock: launch began, launch calls returned,           */
  int64_t launched_ns;       /* predicted end of the fused kernel, completion handled        */
  int64_t end_est_ns;
  int64_t done_ns;
  float prepare_ms, fused_ms;  /* device time of the prepare stage and of the fused kernel   */
  float host_jobs_ms;          /* host time to queue the jobs and histograms of the batch    */
  float host_run_ms;           /* host time of st_run_async (tables, uploads, launches)      */
  int32_t grid;                /* CTAs of the fused launch                                   */
  int32_t host_allocs;         /* device/pinned allocations made by the launch               */
  float host_tables_ms;        /* ... of which building the tables                           */
  float host_alloc_ms;         /* ... of which allocating                                    */
} st_batch_record;

ST_API st_status st_server_create(int32_t device, int64_t budget_bytes, int64_t max_track_deposits,
                                  int32_t max_batch_jobs, st_server** out);
ST_API st_status st_server_destroy(st_server* server);
/* Device bytes a job is charged against the budget while its batch is in flight. */
ST_API st_status st_server_job_footprint(const st_track_view* track, const st_job_desc* desc,
                                         int32_t nbins, int64_t* bytes);
/* Bytes of the budget set aside for the two contexts' spill tables (per-sphere scratch). */
ST_API st_status st_server_reserve_bytes(const st_server* server, int64_t* bytes);
/* Queues one job. counts_out (int64[nbins]) and yfy_out (float64[nbins]) receive its spectrum. */
ST_API st_status st_server_submit(st_server* server, const st_track_view* track,
                                  const st_job_desc* desc, int32_t hist_type, int32_t nbins,
                                  float lower, float upper, int64_t* counts_out, double* yfy_out,
                                  uint64_t tag);
/* Submits n jobs from a server-side thread at start + arrival_ns[i] (steady clock), returning at
 * once; outputs are counts_out/yfy_out + i*nbins. All jobs share one histogram specification. */
ST_API st_status st_server_replay(st_server* server, int32_t n, const st_track_view* tracks,
                                  const st_job_desc* descs, const int64_t* arrival_ns,
                                  int32_t hist_type, int32_t nbins, float lower, float upper,
                                  int64_t* counts_out, double* yfy_out);
/* Moves up to cap finished-job records into out; n_out receives the number moved. */
ST_API st_status st_server_poll(st_server* server, st_completion* out, int32_t cap, int32_t* n_out);
/* Moves up to cap records of finished batches into out; n_out receives the number moved. */
ST_API st_status st_server_batches(st_server* server, st_batch_record* out, int32_t cap,
                                   int32_t* n_out);
/* Waits until every submitted (and replayed) job has completed, or timeout_ms elapses. */
ST_API st_status st_server_drain(st_server* server, int64_t timeout_ms);

/* --- superimposition without device allocation ------------------------------------------------
 * No counterpart in the reference. For callers that must not allocate device memory on their
 * path: cudaFree synchronises the whole device and stalls every other stream (a serving thread
 * sharing the GPU cannot afford that), and frameworks that own all device memory through their
 * own pool leave no room for, or forbid, allocations by their plug-ins. The call allocates
 * nothing: it works in a fixed scratch array compiled into the library
 * (st_noalloc_scratch_bytes() bytes, about 6.2 MB, held by every GPU that loads the library
 * until the process exits). Limits: one device-resident track (track->on_device != 0) of at
 * most 16384 deposits, at most 65536 oversamples, a histogram of at most 4096 bins; larger
 * requests return ST_ERR_CAPACITY. d_counts (int64) and d_yfy (float64) are device arrays of
 * nbins that the call adds into; after an error status they may hold part of the call's sums.
 * desc->hist_id is ignored. Work is enqueued on `stream` (NULL: the legacy default stream) on the
 * current device, and the call synchronises that stream before it returns.
 * The first call on each device resolves the scratch array's device address (and sets a kernel
 * attribute), so that first call should come before any stream capture. All calls share the one
 * scratch array, and two calls whose GPU work overlapped would race; a shared stream does not
 * prevent that, since one call's copies could be enqueued between another's copies and kernels.
 * The library therefore serialises the calls of a process per device: each call holds a lock
 * from its first enqueue to its final synchronisation. */
ST_API st_status st_superimpose_noalloc(const st_track_view* track, const st_job_desc* desc,
                                        int32_t hist_type, int32_t nbins, float lower,
                                        float upper, int64_t* d_counts, double* d_yfy,
                                        void* stream, st_job_stats* stats_out);
ST_API int64_t st_noalloc_scratch_bytes(void);

/* --- macro-level run (SuperTrackManager) ----------------------------------------------------- */

typedef struct {
  int64_t n_tracks;          /* "Number of Tracks"                                        */
  int64_t n_oversamples;     /* "Number of Oversamples"                                   */
  int64_t n_effective;       /* "Effective Number of Tracks"                              */
  int64_t random_seed;       /* [Run] RandomSeed after the time(NULL) default             */
  int64_t deposits;          /* deposits over all tracks                                  */
  int32_t nbins;
  int32_t reserved;
} st_run_info;

/* SuperTrackManager::Initialize(new INIReader(path)) + Run() (SuperTrackManager.cu:28-102):
 * reads the macro, enumerates the track folder, derives the task seeds, runs every task on
 * the GPU and writes <[Output] Path><NamePrefix><seed>.csv/.json unless write_output == 0.
 * counts/yfy receive the summed spectrum (nbins_cap entries available). A macro or track folder
 * that cannot be used returns ST_ERR_CONFIG; a failed library call returns its own status (for
 * example ST_ERR_NO_DEVICE without a GPU, or a job's rejection); err receives the reason. */
ST_API st_status st_run_macro(const char* ini_path, int32_t device, int32_t write_output,
                              int64_t* counts, double* yfy, int32_t nbins_cap,
                              st_run_info* info, char* err, size_t err_len);

/* Writes a track file (the format SuperTrackManager's folder loop reads). */
ST_API st_status st_track_file_write(const char* path, uint64_t n_tracks, const uint64_t* index,
                                     uint64_t n_deposits, const double* x, const double* y,
                                     const double* z, const double* edep);

/* --- .ini access (INIReader, extern/inih/INIReader.h) --------------------------------------- */
typedef struct st_ini st_ini;
ST_API st_status st_ini_open(const char* path, st_ini** out, int32_t* parse_error);
ST_API st_status st_ini_from_string(const char* text, st_ini** out, int32_t* parse_error);
ST_API void st_ini_close(st_ini* ini);
ST_API st_status st_ini_get(const st_ini* ini, const char* section, const char* name,
                            const char* default_value, char* buf, size_t len);
ST_API long st_ini_get_integer(const st_ini* ini, const char* section, const char* name, long dflt);
ST_API double st_ini_get_real(const st_ini* ini, const char* section, const char* name, double dflt);
ST_API float st_ini_get_float(const st_ini* ini, const char* section, const char* name, float dflt);
ST_API int32_t st_ini_get_boolean(const st_ini* ini, const char* section, const char* name,
                                  int32_t dflt);

/* --- spectrum post-processing (host; CPUHistogramUtils, utils.cc:37-117) --------------------
 * `contents` uses ROOT's TH1 layout: nbins + 2 values, [0] underflow, [1..nbins] the bins
 * (st_hist_read's bin b is contents[b + 1]), [nbins + 1] overflow; `edges` has nbins + 1 values.
 * The reference's loops cover indices 0..nbins-1 (the underflow bin, with ROOT's equidistant low
 * edge below the axis, and every bin but the last) and sum the normalisation in float; these
 * functions do the same, so they return the reference's numbers. */
/* BinLogX (utils.cc:37-57): edges 10^(from + i*(to - from)/nbins), i = 0..nbins. */
ST_API st_status st_spectrum_bin_log_x(int32_t nbins, double from_log10, double to_log10,
                                       double* edges);
/* PMF_to_PDF (utils.cc:81-102): divide by bin width, then by the sum of the original contents. */
ST_API st_status st_spectrum_pmf_to_pdf(int32_t nbins, const double* edges, double* contents);
/* Prepare_for_Semilog (utils.cc:104-117): multiply by the bin midpoint (f(y) -> y*f(y)). */
ST_API st_status st_spectrum_prepare_for_semilog(int32_t nbins, const double* edges,
                                                 double* contents);

/* Task list of a macro: ThreadAllocator::ReturnThreadAllocations (ThreadAllocator.cc:51-109)
 * flattened; per task: thread id, entry/exit points, task seed, file ordinal (1-based). */
typedef struct {
  int64_t entry;
  int64_t exit;
  int64_t seed;
  int32_t thread_id;
  int32_t file_ordinal;
  int32_t n_oversamples;
  int32_t track_in_file;
} st_task;
ST_API st_status st_macro_tasks(const char* ini_path, st_task* tasks, int64_t cap, int64_t* n_out,
                                char* err, size_t err_len);

#ifdef __cplusplus
}
#endif
#endif /* SUPERTRACK_B200_H */
