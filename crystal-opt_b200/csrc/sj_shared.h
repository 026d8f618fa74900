// sj_shared.h -- internals of the shared-scan forms (batch and serving).
//
// One probe kernel serves both forms.  It reads a step descriptor (SjbStep)
// that names, for up to 64 query slots, the fact rows each slot needs in this
// step, how its group key is formed and where its accumulators live.  The
// batch form writes the descriptor on the device (sjb_layout_kernel) so the
// whole batch replays as a CUDA graph; the serving loop writes it on the host
// between scan steps.  Both use the same layout functions below.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "sj_l2.h"

#include "../../include/starjoin_batch.h"

namespace sj {

constexpr int kBq = SJB_MAX_QUERIES;
constexpr int kBMaxJobs = SJB_MAX_QUERIES * SJ_MAX_DIMS;
constexpr int kBInWords = SJ_MAX_IN_CODES / 32;
constexpr int kBMaxIn = 128;  // IN-list predicates per batch
constexpr uint32_t kBErrGroupCapacity = 1u;
constexpr uint32_t kBErrSmem = 2u;
constexpr uint32_t kBErrCollision = 4u;

struct SjbDimRt {
  const int32_t* fact_fk;
  const int32_t* key;
  const int32_t* attr[SJB_MAX_ATTRS];
  const int32_t* slot_attr[SJB_MAX_ATTRS];  // attribute of the row held by each PHT slot
  uint64_t* mask;                           // per slot: bit q = slot q's predicate accepts the row
  int64_t rows;
  uint64_t fastmod_m;
  int32_t key_min;
  uint32_t len;
  uint32_t n_attrs;
};

struct SjbSchemaRt {
  SjbDimRt dim[SJ_MAX_DIMS];
  const int32_t* measure;
  const int32_t* measure_sub;
  int64_t fact_rows;
  uint32_t n_dims;
};

// Filter statistics of one cached (dimension, predicate) bitmap.  min/max of
// each attribute over the qualifying rows are kept as order-preserving
// unsigned codes so that a zeroed record is the identity of both reductions.
struct SjbEntryStats {
  uint32_t count;
  uint32_t umax[SJB_MAX_ATTRS];  // max of (v ^ 0x80000000)
  uint32_t nmin[SJB_MAX_ATTRS];  // max of ~(v ^ 0x80000000)
  uint32_t pad[3];
};
static_assert(sizeof(SjbEntryStats) == 48, "stats record");

__host__ __device__ inline int32_t stats_max(const SjbEntryStats& s, int a) {
  return (int32_t)(s.umax[a] ^ 0x80000000u);
}
__host__ __device__ inline int32_t stats_min(const SjbEntryStats& s, int a) {
  return (int32_t)((~s.nmin[a]) ^ 0x80000000u);
}

// A filter-bitmap build: predicate of one query dimension over the dimension rows.
struct SjbJob {
  uint32_t dim;
  int32_t attr;
  int32_t kind;
  int32_t lo, hi;
  uint32_t words;        // bitmap words (ceil(len / 32))
  int32_t in_index;      // row of the IN-code bitmaps, -1 if none
  uint32_t stats_mask;   // bit a: reduce min/max of attribute a; kJobStatsOnly: see below
  uint32_t* bitmap;
  SjbEntryStats* stats;
};

// A job that only adds attributes' min/max to the statistics of a filter that is
// already built (and may be in use): it neither zeroes nor writes the bitmap and
// leaves the count alone.
constexpr uint32_t kJobStatsOnly = 1u << 31;
constexpr uint32_t kJobAllStats = (1u << SJB_MAX_ATTRS) - 1u;

struct SjbAcc {
  unsigned long long cnt;
  unsigned long long sum;
};

struct SjbSlot {                 // 128 bytes
  int64_t b, e;                  // fact rows of this step; b >= e: nothing to do
  uint64_t group_base;           // first accumulator entry (global array)
  const int32_t* gtab[SJ_MAX_DIMS];  // slot-attribute table of each grouped dimension
  int32_t pmin[SJ_MAX_DIMS];
  uint32_t stride[SJ_MAX_DIMS];
  uint32_t width[SJ_MAX_DIMS];
  int32_t smem_off;              // first entry of the CTA's shared partials, -1: global atomics
  uint32_t span;                 // accumulator entries (0: the query cannot match)
  uint8_t n_g;                   // grouped dimensions
  uint8_t gpos[SJ_MAX_DIMS];     // lookup position of each grouped dimension in this step
  uint8_t gk[SJ_MAX_DIMS];       // predicate index in the query (output column)
  uint8_t gd[SJ_MAX_DIMS];       // schema dimension
  uint8_t pad_[3];
};
static_assert(sizeof(SjbSlot) == 128, "slot record");

struct SjbStep {
  int64_t seg_b, seg_e;          // fact rows of this step
  uint64_t active;               // slots with rows in this step
  uint64_t use[SJ_MAX_DIMS];     // slots that use each dimension
  uint32_t order[SJ_MAX_DIMS];   // dimension lookup order
  uint32_t n_dims;
  uint32_t smem_entries;         // shared partial entries in use
  uint32_t error;
  uint32_t pad_[3];
  SjbSlot slot[kBq];
  const uint32_t* bm[kBq][SJ_MAX_DIMS];  // filter bitmap of slot q on dimension d (NULL: unused)
  float sel[kBq][SJ_MAX_DIMS];           // qualifying fraction of the dimension's rows
};

// What the batch pipeline receives from the host (copied in one transfer).
struct SjbBatchQuery {
  int64_t b, e;
  uint32_t n_preds;
  uint32_t dim[SJ_MAX_DIMS];
  int32_t group_attr[SJ_MAX_DIMS];
  const SjbEntryStats* stats[SJ_MAX_DIMS];
  const uint32_t* bitmap[SJ_MAX_DIMS];
};

struct SjbBatchDesc {
  uint32_t n_jobs;
  uint32_t n_queries;
  uint64_t group_capacity;
  uint32_t smem_capacity;
  uint32_t pad_;
  SjbJob jobs[kBMaxJobs];
  SjbBatchQuery q[kBq];
  uint32_t in_bits[kBMaxIn][kBInWords];
};

struct SjbCounters {
  unsigned long long rows_scanned;
  unsigned long long out_rows;
  unsigned int error;
  unsigned int pad_;
};

// ------------------------------------------------------------ layout ----
// Group layout of one query slot from its filters' statistics: the group key is
// a mixed-radix number over the grouped attributes, each offset by the minimum
// over the rows its predicate accepts (the last grouped predicate varies
// fastest).  span = 0 when some predicate accepts no row.  Returns
// kBErrGroupCapacity (and span 0) when the key space exceeds span_limit.
__host__ __device__ inline uint32_t sjb_group_layout(const SjbSchemaRt& S, const SjbBatchQuery& q,
                                                     const SjbEntryStats* const* st, SjbSlot& out,
                                                     float* sel, uint64_t span_limit) {
  out.n_g = 0;
  out.span = 1;
  out.smem_off = -1;
  bool empty = false;
  for (uint32_t k = 0; k < q.n_preds; ++k) {
    const SjbEntryStats& s = *st[k];
    const uint32_t d = q.dim[k];
    if (s.count == 0) empty = true;
    sel[d] = S.dim[d].rows > 0 ? (float)s.count / (float)S.dim[d].rows : 0.f;
    const int32_t a = q.group_attr[k];
    if (a < 0 || s.count == 0) continue;
    const uint32_t g = out.n_g++;
    out.gd[g] = (uint8_t)d;
    out.gk[g] = (uint8_t)k;
    out.gtab[g] = S.dim[d].slot_attr[a];
    out.pmin[g] = stats_min(s, a);
    out.width[g] = (uint32_t)((int64_t)stats_max(s, a) - (int64_t)out.pmin[g] + 1);
  }
  uint64_t span = 1;
  uint32_t err = 0;
  for (int g = (int)out.n_g - 1; g >= 0; --g) {
    out.stride[g] = (uint32_t)span;
    span *= out.width[g];
    if (span > span_limit) {
      err = kBErrGroupCapacity;
      break;
    }
  }
  out.span = (empty || err) ? 0u : (uint32_t)span;
  return err;
}

// Dimension order number `idx` (0 <= idx < n!) by its factorial-base digits.
__host__ __device__ inline void sjb_perm_of(uint32_t idx, uint32_t n, uint32_t* out) {
  uint32_t pool[SJ_MAX_DIMS] = {0, 1, 2, 3};
  uint32_t fact = 1;
  for (uint32_t i = 2; i < n; ++i) fact *= i;
  for (uint32_t k = 0; k < n; ++k) {
    const uint32_t left = n - 1 - k;
    const uint32_t r = left ? idx / fact : 0u;
    if (left) idx %= fact;
    out[k] = pool[r];
    for (uint32_t j = r; j + 1 < n - k; ++j) pool[j] = pool[j + 1];
    if (left > 1) fact /= left;
  }
}

// Expected mask-word lookups per scanned row for a dimension order: position k
// is looked up when some query still alive uses its dimension, and query q is
// alive there with probability cover[q] (its share of the scanned rows) times
// its selectivities on the dimensions before k.  Queries are taken as
// independent of one another.
__host__ __device__ inline float sjb_order_lookups(const SjbStep& st, const float* cover, const uint32_t* perm,
                                                   uint32_t nd) {
  float alive[kBq];
  for (int q = 0; q < kBq; ++q) alive[q] = ((st.active >> q) & 1ull) ? cover[q] : 0.f;
  float cost = 0.f;
  for (uint32_t k = 0; k < nd; ++k) {
    const uint32_t d = perm[k];
    float none = 1.f;
    for (int q = 0; q < kBq; ++q) {
      if (!((st.use[d] >> q) & 1ull)) continue;
      none *= 1.f - alive[q];
      alive[q] *= st.sel[q][d];
    }
    cost += 1.f - none;
  }
  return cost;
}

// Share of the step's segment that each active slot's row range covers.
__host__ __device__ inline void sjb_cover(const SjbStep& st, float* cover) {
  const double seg = st.seg_e > st.seg_b ? (double)(st.seg_e - st.seg_b) : 1.0;
  for (int q = 0; q < kBq; ++q) {
    const SjbSlot& s = st.slot[q];
    cover[q] = ((st.active >> q) & 1ull) ? (float)((double)(s.e - s.b) / seg) : 0.f;
  }
}

// Per-step fields: dimension use masks, lookup order (fewest expected mask-word
// lookups per row over every order), grouped-dimension positions and
// shared-memory partials (smallest spans first, while they fit).
__host__ __device__ inline void sjb_step_layout(SjbStep& st, uint32_t n_dims, uint32_t smem_capacity) {
  st.n_dims = n_dims;
  for (uint32_t d = 0; d < SJ_MAX_DIMS; ++d) st.use[d] = 0;
  for (int q = 0; q < kBq; ++q) {
    if (!((st.active >> q) & 1ull)) continue;
    for (uint32_t d = 0; d < n_dims; ++d)
      if (st.bm[q][d]) st.use[d] |= 1ull << q;
  }
  float cover[kBq];
  sjb_cover(st, cover);
  uint32_t n_perm = 1;
  for (uint32_t i = 2; i <= n_dims; ++i) n_perm *= i;
  float best = 3.4e38f;
  for (uint32_t d = 0; d < SJ_MAX_DIMS; ++d) st.order[d] = d;
  for (uint32_t i = 0; i < n_perm; ++i) {
    uint32_t perm[SJ_MAX_DIMS];
    sjb_perm_of(i, n_dims, perm);
    const float c = sjb_order_lookups(st, cover, perm, n_dims);
    if (c < best) {
      best = c;
      for (uint32_t k = 0; k < n_dims; ++k) st.order[k] = perm[k];
    }
  }
  uint8_t pos[SJ_MAX_DIMS] = {0, 0, 0, 0};
  for (uint32_t k = 0; k < n_dims; ++k) pos[st.order[k]] = (uint8_t)k;
  uint32_t used = 0;
  int cand[kBq];
  int nc = 0;
  for (int q = 0; q < kBq; ++q) {
    st.slot[q].smem_off = -1;
    for (int g = 0; g < st.slot[q].n_g; ++g) st.slot[q].gpos[g] = pos[st.slot[q].gd[g]];
    if (((st.active >> q) & 1ull) && st.slot[q].span > 0 && st.slot[q].span <= 2048u) cand[nc++] = q;
  }
  for (int i = 1; i < nc; ++i)  // smallest span first (insertion sort, stable)
    for (int j = i; j > 0 && st.slot[cand[j]].span < st.slot[cand[j - 1]].span; --j) {
      int t = cand[j];
      cand[j] = cand[j - 1];
      cand[j - 1] = t;
    }
  for (int i = 0; i < nc; ++i) {
    SjbSlot& s = st.slot[cand[i]];
    if (used + s.span > smem_capacity) break;
    s.smem_off = (int32_t)used;
    used += s.span;
  }
  st.smem_entries = used;
}

// ---------------------------------------------------------- launchers ----
cudaError_t sjb_launch_register(const SjbSchemaRt& S, uint32_t* slot_rows, SjbCounters* ctr, cudaStream_t st);
cudaError_t sjb_launch_build(const SjbSchemaRt& S, const SjbBatchDesc* desc, uint32_t max_jobs,
                             uint32_t jobs_hint, int sm_count, cudaStream_t st);
cudaError_t sjb_launch_layout(const SjbSchemaRt& S, const SjbBatchDesc* desc, SjbStep* step, SjbCounters* ctr,
                              cudaStream_t st);
cudaError_t sjb_launch_zero_groups(const SjbStep* step, uint64_t zero_mask, SjbAcc* acc, int sm_count,
                                   cudaStream_t st);
cudaError_t sjb_launch_compose(const SjbSchemaRt& S, const SjbStep* step, int sm_count, cudaStream_t st);
cudaError_t sjb_launch_probe(const SjbSchemaRt& S, const SjbStep* step, SjbAcc* acc, SjbCounters* ctr,
                             uint32_t threads, uint32_t smem_entries, int sm_count, cudaStream_t st,
                             const L2Window& masks_window);
cudaError_t sjb_launch_finalize(const SjbStep* step, uint64_t mask, const SjbAcc* acc, sjb_row* out,
                                uint64_t cap, SjbCounters* ctr, const int32_t* slot_query, int sm_count,
                                cudaStream_t st);
uint32_t sjb_probe_smem_bytes(uint32_t smem_entries);

}  // namespace sj
