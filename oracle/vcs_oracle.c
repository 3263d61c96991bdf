/*
 * CPU oracle of the VoxelConstrainedSphere superimposition path — TEST INFRASTRUCTURE ONLY.
 *
 * This file restates the reference algorithm in plain C so that the GPU path can be checked
 * against it. It is the checker, never the product: only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline / reference arm load it. It shares no code with supertrack_b200/.
 *
 * The reference itself cannot be compiled here (it needs CERN ROOT, and its histogram stage
 * calls cudaDeviceSynchronize() from device code, which CUDA 12 rejects), so this restatement
 * is pinned against the reference's own known-answer tests (tst/tests/SuperTrackVoxelConstrainedTests.cu and
 * tst/tests/HistogramTests.cu, regenerated
 * fixtures in tests/golden/).
 *
 * Reference lines restated:
 *   geometry            src/Simulation_method/VoxelConstrainedSphereMethod/SphericalGeometry.cu:7-32
 *   bin edges           src/utils.cc:8-31 (float-typed bounds, Histogram.cu:34-35, :53-72)
 *   z-origin shift      VoxelConstrainedSphereMethod.cu:138-154 (called at :45)
 *   xy shift            VoxelConstrainedSphereMethod.cu:176-177, :183-184
 *   box filter          VoxelConstrainedSphereMethod.cu:198 (strict, |z| included)
 *   sphere filter       VoxelConstrainedSphereMethod.cu:249-271 (IEEE '/', llrint, inclusive <=)
 *   key and value       VoxelConstrainedSphereMethod.cu:302-322
 *   reduce + binning    Histogram.cu:150-158 (sort by key, sum per key, HistogramRange [lo,hi))
 *   accumulation        Histogram.cu:161-171, SuperTrackManager.cu:71-75 (per oversample, summed)
 *   FP32 variant        or_job_f32: the readme's float wish (readme.md:29), no reference code
 *
 * Per-sphere sums: the reference's CUB sort + ReduceByKey order is not deterministic, so the
 * oracle fixes two definitions:
 *   OR_SUM_EXACT : the exact real sum of the contributions (integer accumulation on a per-job
 *                  power-of-two grid, __int128), rounded once to double — the definition the GPU
 *                  path reproduces bit for bit;
 *   OR_SUM_SEQ   : left-to-right double sum in ascending deposit order — the literal FP64
 *                  reduction, used to check energies within 1e-12 relative.
 * Build with -ffp-contract=off: no a*b+c may be fused.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include <time.h>

#define OR_SUM_EXACT 0
#define OR_SUM_SEQ 1

typedef struct {
  double L, HL, gSO, d, r;
  int N;
} or_geom;

typedef struct {
  int64_t hits, spheres, binned;
  int32_t grid_exponent;
  int32_t status;
} or_stats;

typedef struct {
  uint64_t key;
  double y;       /* OR_SUM_EXACT value                                */
  double y_seq;   /* OR_SUM_SEQ value                                  */
  int64_t nhits;  /* deposits of this oversample inside this sphere    */
  int32_t os;
  int32_t bin;    /* histogram bin of y, -1 when outside               */
} or_sphere;

/* SphericalGeometry.cu:7-32 */
int or_geometry(double hl, double d, or_geom* g) {
  if (!(d > 0) || !isfinite(d) || !isfinite(hl)) return 1;
  g->d = d;
  g->r = d / 2;
  double nd = floor((hl * 2) / d);
  if (nd > 2097151.0) return 2;
  if (nd < -2147483648.0) nd = -2147483648.0;
  g->N = (int)nd;
  g->L = g->N * d;
  g->HL = g->L / 2;
  g->gSO = -g->HL + g->r;
  if (g->r > g->HL) {
    g->HL = g->r;
    g->N = 1;
    g->L = g->HL * 2;
    g->gSO = -g->HL + g->r;
  }
  return 0;
}

/* utils.cc:8-31 */
int or_edges(int type, int nbins, float lo, float hi, double* e) {
  if (nbins < 1) return 1;
  if (type == 0) {
    double width = (hi - lo) / (nbins);
    for (int i = 0; i <= nbins; i++) e[i] = lo + (i * width);
  } else if (type == 1) {
    float blo = (float)log10((double)lo), bhi = (float)log10((double)hi);
    double width = (bhi - blo) / (nbins);
    for (int i = 0; i <= nbins; i++) e[i] = pow(10.0, blo + (i * width));
  } else {
    return 1;
  }
  for (int i = 0; i <= nbins; i++) {
    if (!isfinite(e[i])) return 2;
    if (i > 0 && !(e[i] > e[i - 1])) return 2;
  }
  return 0;
}

/* Philox4x32-10 (Salmon et al., SC'11), written from the paper's round definition. */
void or_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; r++) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
    uint32_t n1 = (uint32_t)p1;
    uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
    uint32_t n3 = (uint32_t)p0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* The shift contract of the GPU path: uniforms u in (0,1] from 24 Philox bits (+1, /2^24) with
 * counter (os, track_id lo, track_id hi, "SHFT") and key (seed lo, seed hi); u = 0.5 when
 * shifting is off (SetRandomValsToHalf, VoxelConstrainedSphereMethod.cu:125-136). */
void or_shifts(const or_geom* g, int shift_track, uint64_t seed, uint64_t track_id,
               uint32_t os_begin, uint32_t n_os, double* sxsy) {
  for (uint32_t i = 0; i < n_os; i++) {
    float u[2] = {0.5f, 0.5f};
    if (shift_track) {
      uint32_t ctr[4] = {os_begin + i, (uint32_t)track_id, (uint32_t)(track_id >> 32), 0x53484654u};
      uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
      uint32_t out[4];
      or_philox(ctr, key, out);
      for (int a = 0; a < 2; a++) u[a] = (float)((out[a] >> 8) + 1u) / 16777216.0f;
    }
    for (int a = 0; a < 2; a++) sxsy[2 * i + a] = ((u[a] * g->L) - g->HL);
  }
}

/* ---------------------------------------------------------------------------------------- */
/* exact accumulation grid                                                                    */

static int ulp_exp(double v) {
  int ex;
  double a = fabs(v);
  if (a < DBL_MIN) return -1074;
  frexp(a, &ex);
  return ex - 53;
}

static int bitlen(uint64_t v) {
  int n = 0;
  while (v) { n++; v >>= 1; }
  return n;
}

int or_grid_exponent(int e_min, int e_max, int64_t n, int any) {
  if (!any) return 0;
  int need = e_max + 53 + bitlen((uint64_t)(n > 0 ? n : 1)) - 127;
  return e_min > need ? e_min : need;
}

static __int128 fixed_of(double v, int E0) {
  if (v == 0) return 0;
  int ex;
  double f = frexp(fabs(v), &ex);            /* |v| = f * 2^ex, f in [0.5, 1)           */
  int64_t m = (int64_t)ldexp(f, 53);          /* exact integer                           */
  int e = ex - 53;
  int s = e - E0;
  __int128 r;
  if (s >= 0) {
    r = (__int128)m << s;
  } else {
    int rs = -s;
    if (rs > 60) {
      r = 0;
    } else {
      int64_t q = m >> rs, rem = m & (((int64_t)1 << rs) - 1), half = (int64_t)1 << (rs - 1);
      if (rem > half || (rem == half && (q & 1))) q++;
      r = q;
    }
  }
  return v < 0 ? -r : r;
}

/* Rounds the integer a*2^E0 to the nearest double (ties to even) by taking the top 53 bits. */
static double double_of(__int128 a, int E0) {
  if (a == 0) return 0.0;
  int neg = a < 0;
  unsigned __int128 m = neg ? (unsigned __int128)(-a) : (unsigned __int128)a;
  int L = 0;
  for (unsigned __int128 t = m; t; t >>= 1) L++;
  double r;
  if (L <= 53) {
    r = ldexp((double)(uint64_t)m, E0);
  } else {
    int sh = L - 53;
    unsigned __int128 q = m >> sh;
    unsigned __int128 rem = m - (q << sh);
    unsigned __int128 half = (unsigned __int128)1 << (sh - 1);
    if (rem > half || (rem == half && (q & 1))) q++;
    r = ldexp((double)(uint64_t)q, sh + E0);
  }
  return neg ? -r : r;
}

/* ---------------------------------------------------------------------------------------- */

typedef struct {
  uint64_t key;
  int64_t idx;
  double v;
} hit_t;

static int cmp_hit(const void* a, const void* b) {
  const hit_t* x = (const hit_t*)a;
  const hit_t* y = (const hit_t*)b;
  if (x->key != y->key) return x->key < y->key ? -1 : 1;
  return (x->idx > y->idx) - (x->idx < y->idx);
}

/* CUB HistogramRange (Histogram.cu:158): bin = (first i with y < e[i]) - 1, valid in [0,nbins). */
static int bin_of(const double* e, int nbins, double y) {
  int lo = 0, hi = nbins + 1; /* search in e[0..nbins] for the first e[i] > y */
  while (lo < hi) {
    int mid = (lo + hi) / 2;
    if (y < e[mid]) hi = mid; else lo = mid + 1;
  }
  int b = lo - 1;
  return (b >= 0 && b < nbins) ? b : -1;
}

/*
 * One job: n deposits, n_os oversamples with the given shifts (sxsy[2*os], sxsy[2*os+1]),
 * z-origin shift mode 0 (+HL'), 1 (-HL'), 2 (none). counts/yfy (nbins) are accumulated into.
 * Optionally writes every (os, sphere) record to spheres_out (cap entries; *n_spheres gets
 * the number produced even when it exceeds cap). Returns 0, or 1 bad geometry, 2 non-finite
 * contribution, 3 out of memory.
 */
static int job_impl(const double* x, const double* y, const double* z, const double* edep,
                    int64_t n, double half_length, double d, int zshift_mode, uint32_t n_os,
                    const double* sxsy, const double* edges, int nbins, int sum_mode,
                    int64_t* counts, double* yfy, or_stats* st, or_sphere* spheres_out,
                    int64_t cap, int64_t* n_spheres, int fp32) {
  or_geom g;
  if (or_geometry(half_length, d, &g)) return 1;
  const double zsh = zshift_mode == 0 ? g.HL : (zshift_mode == 1 ? -g.HL : 0.0);
  const double lineal = (2. / 3.) * g.d;
  const double r2 = g.r * g.r;
  const uint64_t N = (uint64_t)g.N;

  /* the job's accumulation grid */
  int e_min = 0, e_max = 0, any = 0;
  for (int64_t i = 0; i < n; i++) {
    double v = edep[i] / lineal;
    if (!isfinite(v)) return 2;
    if (v != 0) {
      int e = ulp_exp(v);
      if (!any || e < e_min) e_min = e;
      if (!any || e > e_max) e_max = e;
      any = 1;
    }
  }
  const int E0 = or_grid_exponent(e_min, e_max, n, any);
  if (st) { memset(st, 0, sizeof(*st)); st->grid_exponent = E0; }

  double* zs = (double*)malloc(sizeof(double) * (n > 0 ? n : 1));
  double *bx = (double*)malloc(sizeof(double) * (n > 0 ? n : 1));
  double *by = (double*)malloc(sizeof(double) * (n > 0 ? n : 1));
  int64_t* bi = (int64_t*)malloc(sizeof(int64_t) * (n > 0 ? n : 1));
  hit_t* hits = (hit_t*)malloc(sizeof(hit_t) * (n > 0 ? n : 1));
  if (!zs || !bx || !by || !bi || !hits) {
    free(zs); free(bx); free(by); free(bi); free(hits);
    return 3;
  }
  for (int64_t i = 0; i < n; i++) zs[i] = z[i] + zsh; /* ShiftTrackZOrigin, not in place */
  int64_t nsph_total = 0;

  for (uint32_t os = 0; os < n_os; os++) {
    const double sx = sxsy[2 * os], sy = sxsy[2 * os + 1];
    /* FilterInScoringBox (FP32 form: x, y and the shift rounded to float, the sum in float;
       the float results are held exactly in bx/by) */
    const float f_sx = (float)sx, f_sy = (float)sy, f_HL = (float)g.HL;
    int64_t nbox = 0;
    for (int64_t i = 0; i < n; i++) {
      double xs, ys;
      int in;
      if (fp32) {
        const float fx = (float)x[i] + f_sx, fy = (float)y[i] + f_sy;
        xs = fx; ys = fy;
        in = fabsf(fx) < f_HL && fabsf(fy) < f_HL;
      } else {
        xs = x[i] + sx; ys = y[i] + sy;
        in = fabs(xs) < g.HL && fabs(ys) < g.HL;
      }
      if (in && fabs(zs[i]) < g.HL) {
        bx[nbox] = xs; by[nbox] = ys; bi[nbox] = i; nbox++;
      }
    }
    /* FilterTrackInSphere + ScoreTrackInSphere (FP32 form: a = x' - gSO, k = rint(a * (1/d)),
       dx = k*d - a and dist = (dx^2 + dy^2) + RN32(dz^2) in float; z as in the FP64 form) */
    const float f_gSO = (float)g.gSO, f_d = (float)g.d, f_inv_d = 1.0f / f_d;
    const float f_r2 = (float)r2;
    int64_t nh = 0;
    for (int64_t k = 0; k < nbox; k++) {
      const int64_t i = bi[k];
      long long kx, ky, kz;
      int hit;
      if (fp32) {
        const float ax = (float)bx[k] - f_gSO, ay = (float)by[k] - f_gSO;
        const float fkx = rintf(ax * f_inv_d), fky = rintf(ay * f_inv_d);
        const float dx = (fkx * f_d) - ax, dy = (fky * f_d) - ay;
        const double az = zs[i] - g.gSO;
        kz = llrint(az / g.d);
        const double dz = (kz * g.d) - az;
        const float dist = ((dx * dx) + (dy * dy)) + (float)(dz * dz);
        kx = (long long)fkx;
        ky = (long long)fky;
        hit = dist <= f_r2;
      } else {
        double ax = bx[k] - g.gSO, ay = by[k] - g.gSO, az = zs[i] - g.gSO;
        kx = llrint(ax / g.d); ky = llrint(ay / g.d); kz = llrint(az / g.d);
        double dx = (kx * g.d) - ax, dy = (ky * g.d) - ay, dz = (kz * g.d) - az;
        double dist = (dx * dx) + (dy * dy) + (dz * dz);
        hit = dist <= r2;
      }
      if (hit) {
        hits[nh].key = (uint64_t)kx + (uint64_t)ky * N + (uint64_t)kz * N * N;
        hits[nh].idx = i;
        hits[nh].v = edep[i] / lineal;
        nh++;
      }
    }
    if (st) st->hits += nh;
    /* sort by (key, deposit index); reduce per key; bin */
    qsort(hits, (size_t)nh, sizeof(hit_t), cmp_hit);
    for (int64_t a = 0; a < nh;) {
      int64_t b = a;
      __int128 acc = 0;
      double seq = 0.0;
      while (b < nh && hits[b].key == hits[a].key) {
        acc += fixed_of(hits[b].v, E0);
        seq = (b == a) ? hits[b].v : seq + hits[b].v;
        b++;
      }
      const double yx = double_of(acc, E0);
      const double yv = sum_mode == OR_SUM_SEQ ? seq : yx;
      const int bin = bin_of(edges, nbins, yv);
      if (st) st->spheres++;
      if (bin >= 0) {
        counts[bin] += 1;
        yfy[bin] += yv;
        if (st) st->binned++;
      }
      if (spheres_out && nsph_total < cap) {
        or_sphere* s = &spheres_out[nsph_total];
        s->key = hits[a].key;
        s->y = yx;
        s->y_seq = seq;
        s->nhits = b - a;
        s->os = (int32_t)os;
        s->bin = bin;
      }
      nsph_total++;
      a = b;
    }
  }
  if (n_spheres) *n_spheres = nsph_total;
  free(zs); free(bx); free(by); free(bi); free(hits);
  return 0;
}

int or_job(const double* x, const double* y, const double* z, const double* edep, int64_t n,
           double half_length, double d, int zshift_mode, uint32_t n_os, const double* sxsy,
           const double* edges, int nbins, int sum_mode, int64_t* counts, double* yfy,
           or_stats* st, or_sphere* spheres_out, int64_t cap, int64_t* n_spheres) {
  return job_impl(x, y, z, edep, n, half_length, d, zshift_mode, n_os, sxsy, edges, nbins,
                  sum_mode, counts, yfy, st, spheres_out, cap, n_spheres, 0);
}

/*
 * The FP32 geometry variant of or_job (not a reference algorithm: the reference computes in
 * FP64 throughout and only wishes for a float form, readme.md:29). x, y, the shifts, the box
 * test in x and y, the x/y lattice index and the sphere distance are computed in float, every
 * operation rounded on its own; z (box test, lattice index, dz), keys and energies are as in
 * or_job.
 */
int or_job_f32(const double* x, const double* y, const double* z, const double* edep, int64_t n,
               double half_length, double d, int zshift_mode, uint32_t n_os,
               const double* sxsy, const double* edges, int nbins, int sum_mode,
               int64_t* counts, double* yfy, or_stats* st, or_sphere* spheres_out, int64_t cap,
               int64_t* n_spheres) {
  return job_impl(x, y, z, edep, n, half_length, d, zshift_mode, n_os, sxsy, edges, nbins,
                  sum_mode, counts, yfy, st, spheres_out, cap, n_spheres, 1);
}

/*
 * Many jobs, threads over jobs (the CPU baseline). Job j reads deposits [off[j], off[j]+n[j])
 * of the SoA arrays, geometry (hl[j], d[j]), its own shifts from the Philox contract, and adds
 * into histogram hist[j] (counts/yfy laid out hist-major, nbins[h] bins at hoff[h], edges at
 * eoff[h]). Threads claim jobs from a shared counter in the given order (callers pass the
 * largest first). job_stats (may be NULL) receives each job's hits, spheres and binned spheres;
 * job_seconds (may be NULL) the thread time each job took (CLOCK_MONOTONIC around it, measured
 * while the other threads work on their own jobs). Returns the number of failed jobs.
 */
typedef struct {
  int64_t n_jobs;
  const double *x, *y, *z, *edep;
  const int64_t *off, *n;
  const double *hl, *d;
  const int32_t *zshift, *shift_track;
  const uint32_t* n_os;
  const uint64_t *seed, *track_id;
  const int32_t* hist;
  const double* edges;
  const int64_t* eoff;
  const int32_t* nbins;
  const int64_t* hoff;
  int64_t* counts;
  double* yfy;
  or_stats* job_stats;
  double* job_seconds;
  int64_t next;
  int failed;
  pthread_mutex_t lock;
} batch_t;

static void* batch_worker(void* arg) {
  batch_t* B = (batch_t*)arg;
  for (;;) {
    int64_t j = __atomic_fetch_add(&B->next, 1, __ATOMIC_RELAXED);
    if (j >= B->n_jobs) break;
    struct timespec t0, t1;
    clock_gettime(CLOCK_MONOTONIC, &t0);
    or_geom g;
    int rc = or_geometry(B->hl[j], B->d[j], &g);
    if (!rc) {
      const int h = B->hist[j];
      double* sxsy = (double*)malloc(sizeof(double) * 2 * (B->n_os[j] ? B->n_os[j] : 1));
      int64_t* c = (int64_t*)calloc((size_t)B->nbins[h], sizeof(int64_t));
      double* w = (double*)calloc((size_t)B->nbins[h], sizeof(double));
      or_stats js;
      memset(&js, 0, sizeof(js));
      or_shifts(&g, B->shift_track[j], B->seed[j], B->track_id[j], 0, B->n_os[j], sxsy);
      rc = or_job(B->x + B->off[j], B->y + B->off[j], B->z + B->off[j], B->edep + B->off[j],
                  B->n[j], B->hl[j], B->d[j], B->zshift[j], B->n_os[j], sxsy,
                  B->edges + B->eoff[h], B->nbins[h], OR_SUM_EXACT, c, w, &js, NULL, 0, NULL);
      if (B->job_stats) B->job_stats[j] = js;
      pthread_mutex_lock(&B->lock);
      for (int b = 0; b < B->nbins[h]; b++) {
        B->counts[B->hoff[h] + b] += c[b];
        B->yfy[B->hoff[h] + b] += w[b];
      }
      pthread_mutex_unlock(&B->lock);
      free(c); free(w); free(sxsy);
    }
    clock_gettime(CLOCK_MONOTONIC, &t1);
    if (B->job_seconds)
      B->job_seconds[j] = (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec);
    if (rc) __atomic_fetch_add(&B->failed, 1, __ATOMIC_RELAXED);
  }
  return NULL;
}

int or_run_batch(int64_t n_jobs, const double* x, const double* y, const double* z,
                 const double* edep, const int64_t* off, const int64_t* n, const double* hl,
                 const double* d, const int32_t* zshift, const int32_t* shift_track,
                 const uint32_t* n_os, const uint64_t* seed, const uint64_t* track_id,
                 const int32_t* hist, const double* edges, const int64_t* eoff,
                 const int32_t* nbins, const int64_t* hoff, int64_t* counts, double* yfy,
                 or_stats* job_stats, double* job_seconds, int32_t threads) {
  batch_t B = {n_jobs, x, y, z, edep, off, n, hl, d, zshift, shift_track, n_os, seed, track_id,
               hist, edges, eoff, nbins, hoff, counts, yfy, job_stats, job_seconds, 0, 0,
               PTHREAD_MUTEX_INITIALIZER};
  if (threads < 1) threads = 1;
  pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)threads);
  int started = 0;
  for (int t = 0; t < threads; t++)
    if (pthread_create(&th[t], NULL, batch_worker, &B) == 0) started++; else break;
  if (started == 0) batch_worker(&B);
  for (int t = 0; t < started; t++) pthread_join(th[t], NULL);
  free(th);
  return B.failed;
}
