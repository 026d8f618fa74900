/*
 * oracle.c -- CPU restatement of the reference star join (TEST INFRASTRUCTURE;
 * see oracle.h).  Plain C11 + pthreads.
 */
#define _GNU_SOURCE
#include "oracle.h"

#include <pthread.h>
#include <sched.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

int or_available_cores(void) {
  cpu_set_t set;
  if (sched_getaffinity(0, sizeof(set), &set) == 0) {
    int n = CPU_COUNT(&set);
    if (n > 0) return n;
  }
  long n = sysconf(_SC_NPROCESSORS_ONLN);
  return n > 0 ? (int)n : 1;
}

/* Dimension predicate, as the build kernels evaluate it
 * (src/ssb-jo/q33/0-lip.cu:130-135: BlockPredEQ then BlockPredOrEQ over the
 * IN codes; :187-190: the GTE/LTE range form). */
static int or_pred(const or_dim* d, int64_t i) {
  if (d->pred_kind == 0) return 1;
  int32_t a = d->filter_attr[i];
  if (d->pred_kind == 2) return a >= d->pred_lo && a <= d->pred_hi;
  for (int32_t c = 0; c < d->in_count; ++c)
    if (a == d->in_codes[c]) return 1;
  return 0;
}

/* HASH(X, len, min) = (X - min) % len (crystal/join.cuh:27), with the
 * difference taken as an unsigned 32-bit offset. */
static inline uint32_t or_slot(int32_t k, int32_t kmin, int32_t len) {
  return ((uint32_t)k - (uint32_t)kmin) % (uint32_t)len;
}

/* BlockBuildSelectivePHT_2 (crystal/join.cuh:260-335): atomicCAS(ht[2h], 0, key)
 * then ht[2h+1] = val, for every qualifying row.  Sequential order: the first
 * qualifying key claims the slot, the last qualifying value stays. */
int or_build_pht(const or_dim* d, int32_t* ht) {
  if (d->ht_len <= 0) return OR_ERR_INVALID;
  memset(ht, 0, sizeof(int32_t) * 2 * (size_t)d->ht_len);
  for (int64_t i = 0; i < d->rows; ++i) {
    if (!or_pred(d, i)) continue;
    uint32_t h = or_slot(d->key[i], d->key_min, d->ht_len);
    if (ht[2 * h] == 0) ht[2 * h] = d->key[i];
    ht[2 * h + 1] = d->payload ? d->payload[i] : 0;
  }
  return OR_OK;
}

typedef struct or_job {
  const or_plan* plan;
  int32_t* ht[OR_MAX_DIMS];
  int64_t stride[OR_MAX_DIMS];
  uint64_t* sum;
  uint64_t* cnt;
  int64_t begin, end;
  int bad_payload;
} or_job;

/* Probe loop of src/ssb-jo/q33/0-naive.cu:28-91 (PHT probes in join order,
 * early exit on the first miss) with the uint64 aggregate of
 * src/ssb-jo/q31/0-lip.cu:98-113. */
static void* or_worker(void* arg) {
  or_job* j = (or_job*)arg;
  const or_plan* p = j->plan;
  const int nd = p->n_dims;
  for (int64_t r = j->begin; r < j->end; ++r) {
    int64_t g = 0;
    int ok = 1;
    for (int s = 0; s < nd; ++s) {
      int d = p->order[s];
      const or_dim* dim = &p->dims[d];
      uint32_t h = or_slot(dim->fact_fk[r], dim->key_min, dim->ht_len);
      const int32_t* slot = j->ht[d] + 2 * (size_t)h;
      if (slot[0] == 0) { ok = 0; break; }
      if (dim->group) {
        int32_t v = slot[1];
        if (v < dim->payload_min || v > dim->payload_max) { j->bad_payload = 1; ok = 0; break; }
        g += (int64_t)(v - dim->payload_min) * j->stride[d];
      }
    }
    if (!ok) continue;
    int64_t m = (int64_t)p->measure[r];
    if (p->measure_sub) m -= (int64_t)p->measure_sub[r];
    __atomic_fetch_add(&j->sum[g], (uint64_t)m, __ATOMIC_RELAXED);
    __atomic_fetch_add(&j->cnt[g], (uint64_t)1, __ATOMIC_RELAXED);
  }
  return NULL;
}

int or_starjoin(const or_plan* p, int threads, or_group_row* out, int64_t cap, int64_t* n_out) {
  if (!p || p->n_dims < 1 || p->n_dims > OR_MAX_DIMS || !p->measure) return OR_ERR_INVALID;
  if (p->row_begin < 0 || p->row_end < p->row_begin) return OR_ERR_INVALID;
  int used[OR_MAX_DIMS] = {0};
  for (int s = 0; s < p->n_dims; ++s) {
    int d = p->order[s];
    if (d < 0 || d >= p->n_dims || used[d]) return OR_ERR_INVALID;
    used[d] = 1;
  }
  /* group strides: dimension 0 most significant */
  int64_t stride[OR_MAX_DIMS] = {0};
  int64_t groups = 1;
  for (int d = p->n_dims - 1; d >= 0; --d) {
    const or_dim* dim = &p->dims[d];
    if (dim->ht_len <= 0) return OR_ERR_INVALID;
    if (!dim->group) continue;
    if (!dim->payload || dim->payload_max < dim->payload_min) return OR_ERR_INVALID;
    stride[d] = groups;
    groups *= (int64_t)dim->payload_max - dim->payload_min + 1;
    if (groups > ((int64_t)1 << 28)) return OR_ERR_INVALID;
  }
  or_job base;
  memset(&base, 0, sizeof(base));
  base.plan = p;
  int rc = OR_OK;
  for (int d = 0; d < p->n_dims; ++d) {
    base.ht[d] = (int32_t*)malloc(sizeof(int32_t) * 2 * (size_t)p->dims[d].ht_len);
    base.stride[d] = stride[d];
    if (!base.ht[d]) { rc = OR_ERR_INVALID; goto done; }
    or_build_pht(&p->dims[d], base.ht[d]);
  }
  base.sum = (uint64_t*)calloc((size_t)groups, sizeof(uint64_t));
  base.cnt = (uint64_t*)calloc((size_t)groups, sizeof(uint64_t));
  if (!base.sum || !base.cnt) { rc = OR_ERR_INVALID; goto done; }

  {
    int64_t rows = p->row_end - p->row_begin;
    if (threads <= 0) threads = or_available_cores();
    if (threads > 256) threads = 256;
    if (rows < (int64_t)threads * 65536) threads = (int)(rows / 65536) + 1;
    or_job jobs[256];
    pthread_t tids[256];
    for (int t = 0; t < threads; ++t) {
      jobs[t] = base;
      jobs[t].begin = p->row_begin + rows * t / threads;
      jobs[t].end = p->row_begin + rows * (t + 1) / threads;
    }
    for (int t = 1; t < threads; ++t) pthread_create(&tids[t], NULL, or_worker, &jobs[t]);
    or_worker(&jobs[0]);
    for (int t = 1; t < threads; ++t) pthread_join(tids[t], NULL);
    int bad = 0;
    for (int t = 0; t < threads; ++t) bad |= jobs[t].bad_payload;
    if (bad) { rc = OR_ERR_PAYLOAD_DOMAIN; goto done; }
  }

  {
    int64_t n = 0;
    for (int64_t g = 0; g < groups; ++g) {
      if (!base.cnt[g]) continue;
      if (n < cap && out) {
        or_group_row* row = &out[n];
        memset(row, 0, sizeof(*row));
        for (int d = 0; d < p->n_dims; ++d) {
          if (!p->dims[d].group) continue;
          const int64_t span = (int64_t)p->dims[d].payload_max - p->dims[d].payload_min + 1;
          row->attr[d] = (int32_t)((g / stride[d]) % span + p->dims[d].payload_min);
        }
        row->count = base.cnt[g];
        row->sum = base.sum[g];
      }
      ++n;
    }
    *n_out = n;
    if (n > cap) rc = OR_ERR_CAPACITY;
  }

done:
  for (int d = 0; d < OR_MAX_DIMS; ++d) free(base.ht[d]);
  free(base.sum);
  free(base.cnt);
  return rc;
}

/* ---- seeded synthetic columns (the generator header is plain C) ---------- */
#include "../crystal-opt_b200/csrc/sj_datagen.h"

typedef struct or_gen_job {
  int32_t* dst;
  int64_t begin, end, row0;
  uint64_t key;
  int32_t kind, lo, hi;
} or_gen_job;

static void* or_gen_worker(void* arg) {
  const or_gen_job* j = (const or_gen_job*)arg;
  for (int64_t i = j->begin; i < j->end; ++i)
    j->dst[i] = sj_gen_value(j->key, j->kind, j->lo, j->hi, (uint64_t)(j->row0 + i));
  return NULL;
}

void or_gen_column(int32_t* dst, int64_t n, uint64_t seed, int32_t col, int32_t kind, int32_t lo, int32_t hi,
                   int threads) {
  or_gen_rows(dst, 0, n, seed, col, kind, lo, hi, threads);
}

void or_gen_rows(int32_t* dst, int64_t row0, int64_t n, uint64_t seed, int32_t col, int32_t kind, int32_t lo,
                 int32_t hi, int threads) {
  if (n <= 0 || row0 < 0) return;
  if (threads <= 0) threads = or_available_cores();
  if (threads > 256) threads = 256;
  if (n < (int64_t)threads * 65536) threads = (int)(n / 65536) + 1;
  or_gen_job jobs[256];
  pthread_t tids[256];
  const uint64_t key = sj_stream_key(seed, (uint32_t)col);
  for (int t = 0; t < threads; ++t) {
    jobs[t].dst = dst;
    jobs[t].begin = n * t / threads;
    jobs[t].end = n * (t + 1) / threads;
    jobs[t].row0 = row0;
    jobs[t].key = key;
    jobs[t].kind = kind;
    jobs[t].lo = lo;
    jobs[t].hi = hi;
  }
  for (int t = 1; t < threads; ++t) pthread_create(&tids[t], NULL, or_gen_worker, &jobs[t]);
  or_gen_worker(&jobs[0]);
  for (int t = 1; t < threads; ++t) pthread_join(tids[t], NULL);
}
