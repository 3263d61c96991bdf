// Serving: continuous batching of superimposition jobs that arrive over time.
//
// The reference runs a fixed list of tasks, one forked process per thread, each looping over its
// tracks (SuperTrackManager.cu:49-102). A server instead takes (track, geometry, oversamples,
// histogram) jobs while earlier ones are on the GPU:
//   - a worker thread owns two contexts, each with its own stream and device arenas;
//   - when a context is idle and jobs are queued, the worker admits queued jobs in arrival
//     order while their device footprint fits the budget, and launches them as one batch
//     (prepare, plan, fused kernel, histogram read-back) without waiting. While the other
//     context's batch runs, the launch waits until that batch is expected to end within the
//     time a launch takes on the host (its duration is predicted from the measured device
//     throughput of earlier batches), so that the batch collects every job that arrives
//     meanwhile and the GPU still does not idle between batches. The new batch's prepare
//     kernels may overlap the running batch, its fused kernel is ordered after the running
//     one's (st_ctx_order_after): a persistent kernel that has not yet placed all its CTAs is
//     never starved by the next batch;
//   - a finished batch (polled with an event query) hands every job its own spectrum, copied
//     from pinned staging into the caller's arrays, and a completion record with its times.
// Every job's spectrum depends only on its own track, geometry, seed and track id (the fused
// kernel sums per-sphere energies exactly), so it is the same whichever batch it lands in.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <tuple>
#include <vector>

#include "../../include/supertrack_b200.h"
#include "st_core.cuh"

namespace {

int64_t now_ns() {
  return std::chrono::duration_cast<std::chrono::nanoseconds>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

struct HistSpec {
  int32_t type, nbins;
  float lower, upper;
  bool operator<(const HistSpec& o) const {
    return std::tie(type, nbins, lower, upper) < std::tie(o.type, o.nbins, o.lower, o.upper);
  }
};

struct ServedJob {
  st_track_view track{};
  st_job_desc desc{};
  HistSpec spec{};
  int64_t* counts = nullptr;
  double* yfy = nullptr;
  uint64_t tag = 0;
  int64_t submit_ns = 0;
  int64_t footprint = 0;
};

int64_t pad256(int64_t n) { return (std::max<int64_t>(n, 1) + 255) / 256 * 256; }

uint64_t pow2_at_least(uint64_t v) {
  uint64_t p = 1;
  while (p < v) p <<= 1;
  return p;
}

// Device bytes one job holds while its batch is in flight: its track (x, y, z, edep), the
// prepared records (x, y, dz^2, two fixed-point words, key), the boundary-cell hash and shifted z
// of window-flagged jobs, its histogram (counts, y*f(y), edges), its job tables and work items.
int64_t job_footprint(const st_track_view& t, const st_job_desc& d, int32_t nbins, uint32_t n_lin) {
  const int64_t n = t.n, np = pad256(n);
  int64_t b = 32 * n + 48 * np;
  const bool flagged = n > 2 * 4096 && d.n_oversamples >= 4 && n_lin >= 128 && n_lin < (1u << 19);
  if (flagged) b += 16 * (int64_t)pow2_at_least(2 * (uint64_t)n) + 8 * np;
  b += 24 * (int64_t)nbins + 8;
  b += 512 + 16 * 32 * (int64_t)d.n_oversamples + 12 * (int64_t)d.n_oversamples;
  return b;
}

struct Slot {
  st_ctx* ctx = nullptr;
  std::vector<ServedJob> jobs;
  std::vector<int32_t> hist_of_job;
  std::map<HistSpec, std::vector<int32_t>> hist_pool;  // histogram ids kept for reuse, by spec
  bool busy = false;
  int32_t batch = -1;
  int64_t start_ns = 0;
  int64_t footprint = 0;
  double units = 0;          // deposit x oversamples of the batch
  int64_t launched_ns = 0;   // host time when the launch calls returned
  int64_t host_phase_ns[2] = {0, 0};  // run launch began, run launch returned
  int64_t end_est_ns = 0;    // predicted end of its fused kernel
  int64_t read_bins = 0;     // histogram bins read back (the used prefix of the arena)
  int64_t* pin_counts = nullptr;
  double* pin_yfy = nullptr;
  int64_t pin_cap = 0;
};

}  // namespace

struct st_server {
  int device = 0;
  int64_t budget = 0;          // bytes for jobs in flight, after the per-context reserve
  int64_t reserve = 0;         // spill tables of both contexts
  int64_t max_deposits = 0;
  int32_t max_batch = 0;
  Slot slots[2];

  std::mutex mu;
  std::condition_variable cv_work;  // queue grew, or stop
  std::condition_variable cv_done;  // jobs completed
  std::deque<ServedJob> queue;
  std::vector<st_completion> done;
  std::vector<st_batch_record> batch_log;
  int64_t in_flight_bytes = 0;
  int64_t outstanding = 0;  // submitted or scheduled, not yet completed
  int32_t next_batch = 0;
  int next_slot = 0;
  // predictions for the launch policy: fused-kernel throughput (deposit x oversamples per ms),
  // the prepare stage of a batch that starts on an idle GPU, and the host time of a launch
  double rate_per_ms = 5e7;
  double batch_fixed_ms = 0.5;
  double launch_ms = 0.5;
  std::atomic<bool> stop{false};
  std::thread worker;
  std::vector<std::thread> replayers;

  st_status check_job(const st_track_view* t, const st_job_desc* d, int32_t type, int32_t nbins,
                      float lower, float upper, const void* counts, const void* yfy,
                      int64_t* footprint) const;
  void run_worker();
  void launch(Slot& s, Slot& other, std::vector<ServedJob>&& batch);
  void complete(Slot& s, st_status run_status);
};

st_status st_server::check_job(const st_track_view* t, const st_job_desc* d, int32_t type,
                               int32_t nbins, float lower, float upper, const void* counts,
                               const void* yfy, int64_t* footprint) const {
  if (!t || !d || !counts || !yfy) return ST_ERR_INVALID_ARGUMENT;
  if (!t->on_device) return ST_ERR_INVALID_ARGUMENT;  // served tracks stay resident on the device
  if (t->n < 0 || (t->n > 0 && (!t->x || !t->y || !t->z || !t->edep))) return ST_ERR_INVALID_ARGUMENT;
  if (t->n > max_deposits) return ST_ERR_CAPACITY;
  if (d->zshift < ST_ZSHIFT_PLUS || d->zshift > ST_ZSHIFT_NONE) return ST_ERR_INVALID_ARGUMENT;
  if (d->n_oversamples > 0x7fffffffu) return ST_ERR_INVALID_ARGUMENT;
  if ((type != ST_HIST_LIN && type != ST_HIST_LOG) || nbins <= 0 || !(upper > lower) ||
      (type == ST_HIST_LOG && !(lower > 0)))
    return ST_ERR_BAD_HISTOGRAM;
  st::Geometry g;
  if (st::make_geometry(d->half_length, d->sphere_diameter, &g) != 0) return ST_ERR_BAD_GEOMETRY;
  const int64_t f = job_footprint(*t, *d, nbins, (uint32_t)g.numSpheresLinear);
  if (f > budget) return ST_ERR_CAPACITY;
  *footprint = f;
  return ST_OK;
}

// Enqueues one batch on an idle context: jobs, one histogram each (reused from earlier batches
// when the spec matches, all zeroed first), the asynchronous run and the read-back of every bin
// into pinned staging behind it.
void st_server::launch(Slot& s, Slot& other, std::vector<ServedJob>&& batch) {
  s.jobs = std::move(batch);
  s.busy = true;
  s.start_ns = now_ns();
  s.units = 0;
  for (const ServedJob& J : s.jobs) s.units += (double)J.track.n * (double)J.desc.n_oversamples;
  {
    std::lock_guard<std::mutex> lk(mu);
    s.batch = next_batch++;
  }
  s.launched_ns = 0;
  st_status st = st_jobs_clear(s.ctx);
  if (st == ST_OK) {
    int64_t total = 0;
    st = st_hist_read_all(s.ctx, nullptr, nullptr, 0, &total);
    if (st == ST_OK && total > 0) st = st_hist_reset(s.ctx, -1);
  }
  std::map<HistSpec, size_t> used;
  s.hist_of_job.assign(s.jobs.size(), -1);
  for (size_t i = 0; st == ST_OK && i < s.jobs.size(); ++i) {
    ServedJob& J = s.jobs[i];
    std::vector<int32_t>& pool = s.hist_pool[J.spec];
    size_t& k = used[J.spec];
    if (k == pool.size()) {
      int32_t id = -1;
      st = st_hist_create(s.ctx, J.spec.type, J.spec.nbins, J.spec.lower, J.spec.upper, &id);
      if (st != ST_OK) break;
      pool.push_back(id);
    }
    s.hist_of_job[i] = pool[k++];
    st_job_desc d = J.desc;
    d.hist_id = s.hist_of_job[i];
    st = st_job_submit(s.ctx, &J.track, &d, nullptr);
  }
  if (st == ST_OK) {
    int64_t bins = 0;
    for (int32_t id : s.hist_of_job) {
      int64_t off = 0;
      int32_t nb = 0;
      st_hist_offset(s.ctx, id, &off);
      st_hist_nbins(s.ctx, id, &nb);
      bins = std::max<int64_t>(bins, off + nb);
    }
    s.read_bins = bins;
    if (bins > s.pin_cap) {
      if (s.pin_counts) cudaFreeHost(s.pin_counts);
      if (s.pin_yfy) cudaFreeHost(s.pin_yfy);
      s.pin_counts = nullptr;
      s.pin_yfy = nullptr;
      s.pin_cap = 0;
      const int64_t cap = std::max<int64_t>(bins + bins / 2, 4096);
      if (cudaMallocHost(&s.pin_counts, (size_t)cap * 8) != cudaSuccess ||
          cudaMallocHost(&s.pin_yfy, (size_t)cap * 8) != cudaSuccess)
        st = ST_ERR_OUT_OF_MEMORY;
      else
        s.pin_cap = cap;
    }
    if (st == ST_OK && other.busy) st = st_ctx_order_after(s.ctx, other.ctx);
    s.host_phase_ns[0] = now_ns();
    if (st == ST_OK) st = st_run_async(s.ctx);
    s.host_phase_ns[1] = now_ns();
    if (st == ST_OK) st = st_hist_read_bins_async(s.ctx, 0, bins, s.pin_counts, s.pin_yfy);
  }
  const int64_t t1 = now_ns();
  s.launched_ns = t1;
  launch_ms = 0.8 * launch_ms + 0.2 * (t1 - s.start_ns) * 1e-6;
  const int64_t fused_start = other.busy ? std::max<int64_t>(t1, other.end_est_ns)
                                         : t1 + (int64_t)(batch_fixed_ms * 1e6);
  s.end_est_ns = fused_start + (int64_t)(s.units / rate_per_ms * 1e6);
  if (st != ST_OK) {
    st_run_finish(s.ctx);
    complete(s, st);
  }
}

// Hands every job of a finished batch its spectrum and completion record.
void st_server::complete(Slot& s, st_status run_status) {
  st_batch_record rec{};
  rec.batch = s.batch;
  rec.slot = (int32_t)(&s - slots);
  rec.n_jobs = (int32_t)s.jobs.size();
  rec.status = run_status;
  rec.units = s.units;
  rec.launch_ns = s.start_ns;
  rec.launched_ns = s.launched_ns;
  rec.end_est_ns = s.end_est_ns;
  rec.host_jobs_ms = (float)((s.host_phase_ns[0] - s.start_ns) * 1e-6);
  rec.host_run_ms = (float)((s.host_phase_ns[1] - s.host_phase_ns[0]) * 1e-6);
  {
    int64_t g = 0;
    st_ctx_get_param(s.ctx, "last_grid", &g);
    rec.grid = (int32_t)g;
    st_ctx_get_param(s.ctx, "last_host_allocs", &g);
    rec.host_allocs = (int32_t)g;
    st_ctx_get_param(s.ctx, "last_host_tables_us", &g);
    rec.host_tables_ms = (float)(g * 1e-3);
    st_ctx_get_param(s.ctx, "last_host_alloc_us", &g);
    rec.host_alloc_ms = (float)(g * 1e-3);
  }
  st_ctx_last_timing(s.ctx, &rec.prepare_ms, &rec.fused_ms, nullptr);
  if (run_status == ST_OK || run_status == ST_ERR_NONFINITE_EDEP) {
    // the fused kernel's own time (its prepare stage may have shared the GPU with the batch
    // before it, so only the fused time measures this batch)
    float fused = 0;
    st_ctx_last_timing(s.ctx, nullptr, &fused, nullptr);
    const double dev_ms = (double)fused;
    if (s.units > 0 && dev_ms > 0.05) {
      const double r = s.units / dev_ms;
      rate_per_ms = 0.7 * rate_per_ms + 0.3 * r;
    }
  }
  std::vector<st_completion> out(s.jobs.size());
  for (size_t i = 0; i < s.jobs.size(); ++i) {
    ServedJob& J = s.jobs[i];
    st_status js = run_status;
    if (run_status == ST_OK || run_status == ST_ERR_NONFINITE_EDEP) {
      st_job_stats stats;
      js = st_job_stats_get(s.ctx, (int32_t)i, &stats) == ST_OK ? (st_status)stats.status : run_status;
      int64_t off = 0;
      int32_t nb = 0;
      if (s.hist_of_job[i] >= 0 && st_hist_offset(s.ctx, s.hist_of_job[i], &off) == ST_OK &&
          st_hist_nbins(s.ctx, s.hist_of_job[i], &nb) == ST_OK) {
        std::memcpy(J.counts, s.pin_counts + off, (size_t)nb * 8);
        std::memcpy(J.yfy, s.pin_yfy + off, (size_t)nb * 8);
      }
    }
    out[i].tag = J.tag;
    out[i].status = js;
    out[i].batch = s.batch;
    out[i].submit_ns = J.submit_ns;
    out[i].start_ns = s.start_ns;
  }
  const int64_t t = now_ns();
  for (auto& c : out) c.done_ns = t;
  rec.done_ns = t;
  {
    std::lock_guard<std::mutex> lk(mu);
    batch_log.push_back(rec);
    in_flight_bytes -= s.footprint;
    outstanding -= (int64_t)s.jobs.size();
    done.insert(done.end(), out.begin(), out.end());
  }
  cv_done.notify_all();
  s.jobs.clear();
  s.footprint = 0;
  s.busy = false;
}

void st_server::run_worker() {
  cudaSetDevice(device);
  for (;;) {
    for (Slot& s : slots) {
      if (!s.busy) continue;
      int32_t fin = 0;
      const st_status q = st_run_query(s.ctx, &fin);
      if (fin || q != ST_OK) complete(s, q);
    }
    bool any_busy = slots[0].busy || slots[1].busy;
    {
      // batches alternate between the two contexts
      const int k = next_slot;
      Slot& s = slots[k];
      Slot& other = slots[1 - k];
      if (s.busy) goto wait;
      // while the other batch runs, launch only once it is about to end
      if (other.busy && now_ns() < other.end_est_ns - (int64_t)((launch_ms + 0.3) * 1e6)) goto wait;
      std::vector<ServedJob> batch;
      {
        std::lock_guard<std::mutex> lk(mu);
        int64_t taken = 0;
        while (!queue.empty() && (int32_t)batch.size() < max_batch &&
               in_flight_bytes + taken + queue.front().footprint <= budget) {
          taken += queue.front().footprint;
          batch.push_back(std::move(queue.front()));
          queue.pop_front();
        }
        in_flight_bytes += taken;
        s.footprint = taken;
      }
      if (batch.empty()) goto wait;
      launch(s, other, std::move(batch));
      next_slot = 1 - k;
      any_busy = true;
    }
  wait:
    std::unique_lock<std::mutex> lk(mu);
    if (stop && queue.empty() && !any_busy) break;
    if (any_busy) {
      // a batch is on the GPU: poll its event every few tens of microseconds, or sooner when
      // a job arrives
      cv_work.wait_for(lk, std::chrono::microseconds(20));
    } else {
      cv_work.wait(lk, [&] { return stop || !queue.empty(); });
    }
  }
}

extern "C" {

st_status st_server_create(int32_t device, int64_t budget_bytes, int64_t max_track_deposits,
                           int32_t max_batch_jobs, st_server** out) {
  if (!out || budget_bytes <= 0 || max_track_deposits <= 0 || max_batch_jobs <= 0)
    return ST_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  st_server* s = new st_server();
  s->device = device;
  s->max_deposits = max_track_deposits;
  s->max_batch = max_batch_jobs;
  for (Slot& sl : s->slots) {
    const st_status st = st_ctx_create(device, nullptr, &sl.ctx);
    if (st != ST_OK) {
      for (Slot& o : s->slots)
        if (o.ctx) st_ctx_destroy(o.ctx);
      delete s;
      return st;
    }
  }
  // per-sphere scratch: each context keeps one spill table per resident CTA, able to hold every
  // sphere of the largest admissible job (2 * padded deposits slots of 28 bytes)
  const int64_t slots_per_table =
      (int64_t)pow2_at_least((uint64_t)std::max<int64_t>(2 * pad256(max_track_deposits), 1024));
  const int32_t sms = st_ctx_sm_count(s->slots[0].ctx);
  s->reserve = 2 * slots_per_table * 28 * (int64_t)std::max(sms, 1);
  for (Slot& sl : s->slots) st_ctx_set_param(sl.ctx, "spill_budget_bytes", s->reserve / 2);
  s->budget = budget_bytes - s->reserve;
  if (s->budget <= 0) {
    for (Slot& o : s->slots) st_ctx_destroy(o.ctx);
    delete s;
    return ST_ERR_CAPACITY;
  }
  s->worker = std::thread([s] { s->run_worker(); });
  *out = s;
  return ST_OK;
}

st_status st_server_job_footprint(const st_track_view* track, const st_job_desc* desc,
                                  int32_t nbins, int64_t* bytes) {
  if (!track || !desc || !bytes || nbins <= 0 || track->n < 0) return ST_ERR_INVALID_ARGUMENT;
  st::Geometry g;
  if (st::make_geometry(desc->half_length, desc->sphere_diameter, &g) != 0) return ST_ERR_BAD_GEOMETRY;
  *bytes = job_footprint(*track, *desc, nbins, (uint32_t)g.numSpheresLinear);
  return ST_OK;
}

st_status st_server_reserve_bytes(const st_server* s, int64_t* bytes) {
  if (!s || !bytes) return ST_ERR_INVALID_ARGUMENT;
  *bytes = s->reserve;
  return ST_OK;
}

st_status st_server_submit(st_server* s, const st_track_view* track, const st_job_desc* desc,
                           int32_t hist_type, int32_t nbins, float lower, float upper,
                           int64_t* counts_out, double* yfy_out, uint64_t tag) {
  if (!s) return ST_ERR_INVALID_ARGUMENT;
  int64_t f = 0;
  const st_status st = s->check_job(track, desc, hist_type, nbins, lower, upper, counts_out, yfy_out, &f);
  if (st != ST_OK) return st;
  ServedJob J;
  J.track = *track;
  J.desc = *desc;
  J.spec = {hist_type, nbins, lower, upper};
  J.counts = counts_out;
  J.yfy = yfy_out;
  J.tag = tag;
  J.footprint = f;
  J.submit_ns = now_ns();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return ST_ERR_STATE;
    ++s->outstanding;
    s->queue.push_back(J);
  }
  s->cv_work.notify_one();
  return ST_OK;
}

st_status st_server_replay(st_server* s, int32_t n, const st_track_view* tracks,
                           const st_job_desc* descs, const int64_t* arrival_ns, int32_t hist_type,
                           int32_t nbins, float lower, float upper, int64_t* counts_out,
                           double* yfy_out) {
  if (!s || n < 0 || (n > 0 && (!tracks || !descs || !arrival_ns))) return ST_ERR_INVALID_ARGUMENT;
  std::vector<ServedJob> jobs((size_t)n);
  for (int32_t i = 0; i < n; ++i) {
    if (i > 0 && arrival_ns[i] < arrival_ns[i - 1]) return ST_ERR_INVALID_ARGUMENT;
    int64_t f = 0;
    const st_status st = s->check_job(&tracks[i], &descs[i], hist_type, nbins, lower, upper,
                                      counts_out, yfy_out, &f);
    if (st != ST_OK) return st;
    ServedJob& J = jobs[(size_t)i];
    J.track = tracks[i];
    J.desc = descs[i];
    J.spec = {hist_type, nbins, lower, upper};
    J.counts = counts_out + (size_t)i * nbins;
    J.yfy = yfy_out + (size_t)i * nbins;
    J.tag = (uint64_t)i;
    J.footprint = f;
  }
  std::vector<int64_t> at(arrival_ns, arrival_ns + n);
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return ST_ERR_STATE;
    s->outstanding += n;
  }
  // jobs are released at their arrival times; the recorded submit time is the scheduled arrival,
  // so a late release counts against latency
  s->replayers.emplace_back([s, jobs = std::move(jobs), at = std::move(at)]() mutable {
    const int64_t t0 = now_ns();
    size_t i = 0;
    while (i < jobs.size()) {
      const int64_t due = t0 + at[i];
      int64_t t = now_ns();
      if (s->stop) {
        // the server is shutting down: the jobs not yet released are dropped
        std::lock_guard<std::mutex> lk(s->mu);
        s->outstanding -= (int64_t)(jobs.size() - i);
        break;
      }
      if (due - t > 200000) {  // sleep in slices of at most 10 ms so that a shutdown is seen
        std::this_thread::sleep_for(std::chrono::nanoseconds(std::min<int64_t>(due - t - 100000, 10000000)));
        continue;
      }
      while ((t = now_ns()) < due) std::this_thread::yield();
      std::lock_guard<std::mutex> lk(s->mu);
      while (i < jobs.size() && t0 + at[i] <= t) {
        jobs[i].submit_ns = t0 + at[i];
        s->queue.push_back(std::move(jobs[i]));
        ++i;
      }
      s->cv_work.notify_one();
    }
    s->cv_done.notify_all();
  });
  return ST_OK;
}

st_status st_server_poll(st_server* s, st_completion* out, int32_t cap, int32_t* n_out) {
  if (!s || !n_out || cap < 0 || (cap > 0 && !out)) return ST_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(s->mu);
  const size_t k = std::min<size_t>((size_t)cap, s->done.size());
  std::copy(s->done.begin(), s->done.begin() + k, out);
  s->done.erase(s->done.begin(), s->done.begin() + k);
  *n_out = (int32_t)k;
  return ST_OK;
}

st_status st_server_batches(st_server* s, st_batch_record* out, int32_t cap, int32_t* n_out) {
  if (!s || !n_out || cap < 0 || (cap > 0 && !out)) return ST_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(s->mu);
  const size_t k = std::min<size_t>((size_t)cap, s->batch_log.size());
  std::copy(s->batch_log.begin(), s->batch_log.begin() + k, out);
  s->batch_log.erase(s->batch_log.begin(), s->batch_log.begin() + k);
  *n_out = (int32_t)k;
  return ST_OK;
}

st_status st_server_drain(st_server* s, int64_t timeout_ms) {
  if (!s) return ST_ERR_INVALID_ARGUMENT;
  std::unique_lock<std::mutex> lk(s->mu);
  const bool ok = s->cv_done.wait_for(lk, std::chrono::milliseconds(std::max<int64_t>(timeout_ms, 0)),
                                      [&] { return s->outstanding == 0; });
  return ok ? ST_OK : ST_ERR_STATE;
}

st_status st_server_destroy(st_server* s) {
  if (!s) return ST_ERR_INVALID_ARGUMENT;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  for (std::thread& t : s->replayers) t.join();
  s->cv_work.notify_all();
  if (s->worker.joinable()) s->worker.join();
  for (Slot& sl : s->slots) {
    if (sl.ctx) st_ctx_destroy(sl.ctx);
    if (sl.pin_counts) cudaFreeHost(sl.pin_counts);
    if (sl.pin_yfy) cudaFreeHost(sl.pin_yfy);
  }
  delete s;
  return ST_OK;
}

}  // extern "C"
