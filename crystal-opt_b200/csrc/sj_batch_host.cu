// sj_batch_host.cu -- host side of the batch form (include/starjoin_batch.h):
// schema registration, filter resolution against the cache, and the batch
// pipeline, recorded once as a CUDA graph and replayed for every batch.
//
// Everything a batch needs on the device is decided on the device (filter
// statistics -> group layout -> accumulator ranges), so the host only writes
// the batch description into pinned memory and launches the graph; its first
// node copies the description in and its last nodes copy the counters and the
// first rows back.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "sj_cache.h"
#include "sj_internal.h"
#include "sj_shared.h"

namespace sj {

sj_status fail_fmt(sj_status s, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  return set_error(s, buf);
}

sj_status cuda_fail(cudaError_t e, const char* what) {
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    return fail_fmt(SJ_ERR_OUT_OF_MEMORY, "%s: %s", what, cudaGetErrorString(e));
  }
  return fail_fmt(SJ_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define SJB_CUDA(call)                                      \
  do {                                                      \
    cudaError_t _e = (call);                                \
    if (_e != cudaSuccess) return cuda_fail(_e, #call);     \
  } while (0)

static bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// ------------------------------------------------------------------ schema ----
void schema_release(SchemaState& st) {
  if (st.masks) cudaFree(st.masks);
  if (st.slot_attr) cudaFree(st.slot_attr);
  st.masks = nullptr;
  st.slot_attr = nullptr;
}

sj_status schema_register(sj_engine* eng, const sjb_schema* sc, SchemaState& st) {
  SjNvtxRange nvtx_range("sjb.schema_register");
  if (!sc) return fail_fmt(SJ_ERR_INVALID_ARGUMENT, "schema is NULL");
  if (sc->n_dims < 1 || sc->n_dims > SJ_MAX_DIMS) return fail_fmt(SJ_ERR_INVALID_ARGUMENT, "n_dims=%d", sc->n_dims);
  if (!sc->measure || !aligned16(sc->measure) || (sc->measure_sub && !aligned16(sc->measure_sub)))
    return fail_fmt(SJ_ERR_INVALID_ARGUMENT, "measure column NULL or not 16-byte aligned");
  if (sc->fact_rows < 0 || sc->fact_rows > 0xFFFFFFF0ll)
    return fail_fmt(SJ_ERR_UNSUPPORTED, "fact_rows=%lld (max 2^32-16)", (long long)sc->fact_rows);
  uint64_t total_len = 0, total_attr = 0;
  for (int d = 0; d < sc->n_dims; ++d) {
    const sjb_dim& D = sc->dims[d];
    if (!D.fact_fk || !aligned16(D.fact_fk) || !D.key)
      return fail_fmt(SJ_ERR_INVALID_ARGUMENT, "dim %d: NULL or misaligned column", d);
    if (D.rows < 0 || D.rows > 0x7FFFFFFFll || D.ht_len < 1)
      return fail_fmt(SJ_ERR_INVALID_ARGUMENT, "dim %d: rows=%lld ht_len=%d", d, (long long)D.rows, D.ht_len);
    if (D.n_attrs < 0 || D.n_attrs > SJB_MAX_ATTRS) return fail_fmt(SJ_ERR_INVALID_ARGUMENT, "dim %d: n_attrs", d);
    for (int a = 0; a < D.n_attrs; ++a)
      if (!D.attr[a]) return fail_fmt(SJ_ERR_INVALID_ARGUMENT, "dim %d: attr %d is NULL", d, a);
    total_len += (uint64_t)D.ht_len;
    total_attr += (uint64_t)D.ht_len * (uint64_t)D.n_attrs;
  }
  st.schema = *sc;
  SjbSchemaRt& R = st.rt;
  memset(&R, 0, sizeof(R));
  R.n_dims = (uint32_t)sc->n_dims;
  R.measure = sc->measure;
  R.measure_sub = sc->measure_sub;
  R.fact_rows = sc->fact_rows;
  SJB_CUDA(cudaSetDevice(eng->device));
  SJB_CUDA(cudaMalloc(&st.masks, std::max<uint64_t>(total_len, 1) * sizeof(uint64_t)));
  st.masks_bytes = std::max<uint64_t>(total_len, 1) * sizeof(uint64_t);
  SJB_CUDA(cudaMalloc(&st.slot_attr, std::max<uint64_t>(total_attr, 1) * sizeof(int32_t)));
  SJB_CUDA(cudaMemset(st.masks, 0, std::max<uint64_t>(total_len, 1) * sizeof(uint64_t)));
  SJB_CUDA(cudaMemset(st.slot_attr, 0, std::max<uint64_t>(total_attr, 1) * sizeof(int32_t)));
  uint64_t lo = 0, ao = 0;
  for (int d = 0; d < sc->n_dims; ++d) {
    const sjb_dim& D = sc->dims[d];
    SjbDimRt& T = R.dim[d];
    T.fact_fk = D.fact_fk;
    T.key = D.key;
    T.rows = D.rows;
    T.key_min = D.key_min;
    T.len = (uint32_t)D.ht_len;
    T.fastmod_m = ~0ull / (uint64_t)(uint32_t)D.ht_len + 1ull;
    T.n_attrs = (uint32_t)D.n_attrs;
    T.mask = st.masks + lo;
    for (int a = 0; a < D.n_attrs; ++a) {
      T.attr[a] = D.attr[a];
      T.slot_attr[a] = st.slot_attr + ao;
      ao += (uint64_t)D.ht_len;
    }
    lo += (uint64_t)D.ht_len;
    st.words[d] = (uint32_t)(((uint64_t)D.ht_len + 31) / 32);
  }

  // one row per slot, and each attribute's range over the rows (an ALL filter per dimension)
  uint32_t* slot_rows = nullptr;
  SjbCounters* ctr = nullptr;
  SjbBatchDesc* desc_d = nullptr;
  uint32_t* bm = nullptr;
  SjbEntryStats* stats = nullptr;
  SjbBatchDesc* desc_h = new SjbBatchDesc();
  sj_status rc = SJ_OK;
  cudaError_t e = cudaSuccess;
  auto step = [&](cudaError_t x) {
    if (e == cudaSuccess) e = x;
  };
  step(cudaMalloc(&slot_rows, std::max<uint64_t>(total_len, 1) * sizeof(uint32_t)));
  step(cudaMalloc(&ctr, sizeof(SjbCounters)));
  step(cudaMalloc(&desc_d, sizeof(SjbBatchDesc)));
  uint64_t bm_words = 0;
  for (int d = 0; d < sc->n_dims; ++d) bm_words += st.words[d];
  step(cudaMalloc(&bm, std::max<uint64_t>(bm_words, 1) * 4));
  step(cudaMalloc(&stats, sizeof(SjbEntryStats) * SJ_MAX_DIMS));
  if (e == cudaSuccess) {
    step(cudaMemset(slot_rows, 0, std::max<uint64_t>(total_len, 1) * sizeof(uint32_t)));
    step(cudaMemset(ctr, 0, sizeof(SjbCounters)));
    memset(desc_h, 0, sizeof(*desc_h));
    desc_h->n_jobs = (uint32_t)sc->n_dims;
    uint64_t wo = 0;
    for (int d = 0; d < sc->n_dims; ++d) {
      SjbJob& J = desc_h->jobs[d];
      J.dim = (uint32_t)d;
      J.attr = -1;
      J.kind = SJ_PRED_ALL;
      J.words = st.words[d];
      J.in_index = -1;
      J.stats_mask = kJobAllStats;  // the schema's attribute ranges
      J.bitmap = bm + wo;
      J.stats = stats + d;
      wo += st.words[d];
    }
    step(cudaMemcpy(desc_d, desc_h, sizeof(SjbBatchDesc), cudaMemcpyHostToDevice));
    if (e == cudaSuccess) step(sjb_launch_register(R, slot_rows, ctr, 0));
    if (e == cudaSuccess) step(sjb_launch_build(R, desc_d, (uint32_t)sc->n_dims, 1, eng->sm_count, 0));
    step(cudaDeviceSynchronize());
  }
  SjbCounters hc{};
  SjbEntryStats hs[SJ_MAX_DIMS];
  if (e == cudaSuccess) step(cudaMemcpy(&hc, ctr, sizeof(hc), cudaMemcpyDeviceToHost));
  if (e == cudaSuccess) step(cudaMemcpy(hs, stats, sizeof(hs), cudaMemcpyDeviceToHost));
  if (e != cudaSuccess) {
    rc = cuda_fail(e, "schema registration");
  } else if (hc.error & kBErrCollision) {
    rc = fail_fmt(SJ_ERR_UNSUPPORTED,
                  "two dimension rows share a PHT slot; the shared-scan forms need one row per slot");
  } else {
    for (int d = 0; d < sc->n_dims; ++d)
      for (int a = 0; a < sc->dims[d].n_attrs; ++a) {
        st.attr_min[d][a] = hs[d].count ? stats_min(hs[d], a) : 0;
        st.attr_max[d][a] = hs[d].count ? stats_max(hs[d], a) : 0;
      }
  }
  cudaFree(slot_rows);
  cudaFree(ctr);
  cudaFree(desc_d);
  cudaFree(bm);
  cudaFree(stats);
  delete desc_h;
  if (rc != SJ_OK) schema_release(st);
  return rc;
}

sj_status validate_query(const SchemaState& S, const sjb_query& q, uint64_t* worst) {
  const sjb_schema& sc = S.schema;
  if (q.n_preds < 1 || q.n_preds > sc.n_dims) return fail_fmt(SJ_ERR_INVALID_ARGUMENT, "n_preds=%d", q.n_preds);
  if (q.row_begin < 0 || q.row_end < q.row_begin || q.row_end > sc.fact_rows)
    return fail_fmt(SJ_ERR_INVALID_ARGUMENT, "row range [%lld, %lld) outside [0, %lld)", (long long)q.row_begin,
                    (long long)q.row_end, (long long)sc.fact_rows);
  int seen = 0;
  uint64_t span = 1;
  for (int k = 0; k < q.n_preds; ++k) {
    const sjb_pred& p = q.preds[k];
    if (p.dim < 0 || p.dim >= sc.n_dims || ((seen >> p.dim) & 1))
      return fail_fmt(SJ_ERR_INVALID_ARGUMENT, "pred %d: dim %d missing or repeated", k, p.dim);
    seen |= 1 << p.dim;
    const int na = sc.dims[p.dim].n_attrs;
    if (p.kind < SJ_PRED_ALL || p.kind > SJ_PRED_RANGE)
      return fail_fmt(SJ_ERR_INVALID_ARGUMENT, "pred %d: kind %d", k, p.kind);
    if (p.kind != SJ_PRED_ALL && (p.attr < 0 || p.attr >= na))
      return fail_fmt(SJ_ERR_INVALID_ARGUMENT, "pred %d: attr %d (dim has %d)", k, p.attr, na);
    if (p.kind == SJ_PRED_IN) {
      if (p.in_count < 0 || (p.in_count > 0 && !p.in_codes))
        return fail_fmt(SJ_ERR_INVALID_ARGUMENT, "pred %d: IN list", k);
      for (int i = 0; i < p.in_count; ++i)
        if (p.in_codes[i] < 0 || p.in_codes[i] >= SJ_MAX_IN_CODES)
          return fail_fmt(SJ_ERR_UNSUPPORTED, "pred %d: IN code %d outside [0, %d)", k, p.in_codes[i],
                          SJ_MAX_IN_CODES);
    }
    if (p.group_attr >= na || p.group_attr < -1)
      return fail_fmt(SJ_ERR_INVALID_ARGUMENT, "pred %d: group_attr %d", k, p.group_attr);
    if (p.group_attr >= 0) {
      span *= (uint64_t)(S.attr_max[p.dim][p.group_attr] - S.attr_min[p.dim][p.group_attr] + 1);
      if (span > 0xFFFFFFFFull) return fail_fmt(SJ_ERR_UNSUPPORTED, "group key space exceeds 2^32");
    }
  }
  *worst = span;
  return SJ_OK;
}

}  // namespace sj

using namespace sj;

// ------------------------------------------------------------------- batch ----
struct sjb_batch {
  sj_engine* eng = nullptr;
  SchemaState S;
  sjb_limits lim{};
  uint32_t threads = 512;
  uint32_t smem_entries = 6144;
  uint64_t prefix_rows = 8192;  // rows copied back inside the graph
  // device
  SjbAcc* acc = nullptr;
  sjb_row* rows_d = nullptr;
  SjbCounters* ctr_d = nullptr;
  SjbStep* step_d = nullptr;
  SjbBatchDesc* desc_d = nullptr;
  uint8_t* arena = nullptr;
  SjbEntryStats* stats_d = nullptr;
  // pinned host
  SjbBatchDesc* desc_h = nullptr;
  SjbCounters* ctr_h = nullptr;
  sjb_row* rows_h = nullptr;
  FilterCache cache;
  cudaStream_t cap_stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  sjb_stats last{};
};

static void batch_free(sjb_batch* b) {
  if (!b) return;
  cudaSetDevice(b->eng->device);
  cudaDeviceSynchronize();
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
  for (auto& e : b->ev)
    if (e) cudaEventDestroy(e);
  cudaFree(b->acc);
  cudaFree(b->rows_d);
  cudaFree(b->ctr_d);
  cudaFree(b->step_d);
  cudaFree(b->desc_d);
  cudaFree(b->arena);
  cudaFree(b->stats_d);
  cudaFreeHost(b->desc_h);
  cudaFreeHost(b->ctr_h);
  cudaFreeHost(b->rows_h);
  schema_release(b->S);
  delete b;
}

extern "C" sj_status sjb_batch_create(sj_engine* eng, const sjb_schema* schema, const sjb_limits* limits,
                                      sjb_batch** out) {
  if (!eng || !out) return fail_fmt(SJ_ERR_INVALID_ARGUMENT, "engine or out is NULL");
  *out = nullptr;
  sjb_batch* b = new sjb_batch();
  b->eng = eng;
  if (limits) b->lim = *limits;
  sjb_limits& L = b->lim;
  if (L.group_entries <= 0) L.group_entries = 1ll << 24;
  if (L.result_rows <= 0) L.result_rows = 1ll << 20;
  if (L.filter_cache_bytes <= 0) L.filter_cache_bytes = 1ll << 30;
  b->threads = L.threads ? (uint32_t)L.threads : 1024u;
  if (b->threads != 256 && b->threads != 512 && b->threads != 1024) {
    const int threads = L.threads;
    delete b;
    return fail_fmt(SJ_ERR_INVALID_ARGUMENT, "threads=%d (256, 512 or 1024)", threads);
  }
  b->smem_entries = L.smem_group_entries > 0 ? (uint32_t)L.smem_group_entries : 6144u;
  if (sjb_probe_smem_bytes(b->smem_entries) + 1024 > eng->smem_optin) {
    const int entries = L.smem_group_entries;
    delete b;
    return fail_fmt(SJ_ERR_INVALID_ARGUMENT, "smem_group_entries=%d does not fit shared memory", entries);
  }
  b->prefix_rows = std::min<uint64_t>(b->prefix_rows, (uint64_t)L.result_rows);
  sj_status rc = schema_register(eng, schema, b->S);
  if (rc != SJ_OK) {
    delete b;
    return rc;
  }
  cudaError_t e = cudaSuccess;
  auto step = [&](cudaError_t x) {
    if (e == cudaSuccess) e = x;
  };
  step(cudaMalloc(&b->acc, sizeof(SjbAcc) * (size_t)L.group_entries));
  step(cudaMalloc(&b->rows_d, sizeof(sjb_row) * (size_t)L.result_rows));
  step(cudaMalloc(&b->ctr_d, sizeof(SjbCounters)));
  step(cudaMalloc(&b->step_d, sizeof(SjbStep)));
  step(cudaMalloc(&b->desc_d, sizeof(SjbBatchDesc)));
  step(cudaMalloc(&b->arena, (size_t)L.filter_cache_bytes));
  const uint32_t max_entries = 4096;
  step(cudaMalloc(&b->stats_d, sizeof(SjbEntryStats) * max_entries));
  step(cudaMallocHost(&b->desc_h, sizeof(SjbBatchDesc)));
  step(cudaMallocHost(&b->ctr_h, sizeof(SjbCounters)));
  step(cudaMallocHost(&b->rows_h, sizeof(sjb_row) * std::max<uint64_t>(b->prefix_rows, 1)));
  step(cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking));
  for (auto& ev : b->ev) step(cudaEventCreate(&ev));
  if (e != cudaSuccess) {
    rc = cuda_fail(e, "sjb_batch_create");
    batch_free(b);
    return rc;
  }
  b->cache.init(b->arena, (uint64_t)L.filter_cache_bytes, b->stats_d, max_entries);
  memset(b->desc_h, 0, sizeof(SjbBatchDesc));
  *out = b;
  return SJ_OK;
}

extern "C" void sjb_batch_destroy(sjb_batch* b) { batch_free(b); }

// The whole device pipeline of one batch, in stream order.
static cudaError_t batch_enqueue(sjb_batch* b, cudaStream_t st) {
  const int sm = b->eng->sm_count;
  cudaError_t e;
#define SJB_Q(x)                         \
  do {                                   \
    e = (x);                             \
    if (e != cudaSuccess) return e;      \
  } while (0)
  SJB_Q(cudaMemcpyAsync(b->desc_d, b->desc_h, sizeof(SjbBatchDesc), cudaMemcpyHostToDevice, st));
  SJB_Q(cudaMemsetAsync(b->ctr_d, 0, sizeof(SjbCounters), st));
  SJB_Q(sjb_launch_build(b->S.rt, b->desc_d, kBMaxJobs, 96, sm, st));
  SJB_Q(sjb_launch_layout(b->S.rt, b->desc_d, b->step_d, b->ctr_d, st));
  SJB_Q(sjb_launch_zero_groups(b->step_d, ~0ull, b->acc, sm, st));
  SJB_Q(sjb_launch_compose(b->S.rt, b->step_d, sm, st));
  SJB_Q(cudaEventRecordWithFlags(b->ev[1], st, b->lim.use_graph ? cudaEventRecordExternal : cudaEventRecordDefault));
  SJB_Q(sjb_launch_probe(b->S.rt, b->step_d, b->acc, b->ctr_d, b->threads, b->smem_entries, sm, st,
                         l2_window(b->S.masks, b->S.masks_bytes, b->eng->l2_persist_bytes, b->eng->l2_window_max)));
  SJB_Q(cudaEventRecordWithFlags(b->ev[2], st, b->lim.use_graph ? cudaEventRecordExternal : cudaEventRecordDefault));
  SJB_Q(sjb_launch_finalize(b->step_d, ~0ull, b->acc, b->rows_d, (uint64_t)b->lim.result_rows, b->ctr_d, nullptr,
                            sm, st));
  SJB_Q(cudaMemcpyAsync(b->ctr_h, b->ctr_d, sizeof(SjbCounters), cudaMemcpyDeviceToHost, st));
  if (b->prefix_rows)
    SJB_Q(cudaMemcpyAsync(b->rows_h, b->rows_d, sizeof(sjb_row) * b->prefix_rows, cudaMemcpyDeviceToHost, st));
#undef SJB_Q
  return cudaSuccess;
}

// The whole-batch events are recorded on the caller's stream around the graph
// launch (or the direct launches); the probe's events are nodes of the graph.
static cudaError_t batch_launch(sjb_batch* b, cudaStream_t st) {
  cudaError_t e = cudaEventRecord(b->ev[0], st);
  if (e != cudaSuccess) return e;
  if (!b->lim.use_graph) {
    e = batch_enqueue(b, st);
    return e != cudaSuccess ? e : cudaEventRecord(b->ev[3], st);
  }
  if (!b->exec) {
    e = cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeRelaxed);
    if (e != cudaSuccess) return e;
    cudaError_t eq = batch_enqueue(b, b->cap_stream);
    e = cudaStreamEndCapture(b->cap_stream, &b->graph);
    if (eq != cudaSuccess) return eq;
    if (e != cudaSuccess) return e;
    e = cudaGraphInstantiate(&b->exec, b->graph, 0);
    if (e != cudaSuccess) return e;
  }
  e = cudaGraphLaunch(b->exec, st);
  return e != cudaSuccess ? e : cudaEventRecord(b->ev[3], st);
}

extern "C" sj_status sjb_batch_run(sjb_batch* b, const sjb_query* queries, int32_t n, sjb_row* out, int64_t cap,
                                   int64_t* n_out, void* stream) {
  SjNvtxRange nvtx_range("sjb.batch_run");
  if (!b || !queries || !n_out) return fail_fmt(SJ_ERR_INVALID_ARGUMENT, "NULL argument");
  if (n < 1 || n > SJB_MAX_QUERIES) return fail_fmt(SJ_ERR_INVALID_ARGUMENT, "n=%d (1..%d)", n, SJB_MAX_QUERIES);
  *n_out = 0;
  uint64_t worst_total = 0;
  for (int i = 0; i < n; ++i) {
    uint64_t w = 0;
    sj_status rc = validate_query(b->S, queries[i], &w);
    if (rc != SJ_OK) return fail_fmt(rc, "query %d: %s", i, sj_last_error());
    worst_total += w;
  }
  if (worst_total > (uint64_t)b->lim.group_entries)
    return fail_fmt(SJ_ERR_CAPACITY, "batch may need %llu group entries (limit %lld); split it",
                    (unsigned long long)worst_total, (long long)b->lim.group_entries);
  cudaSetDevice(b->eng->device);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);

  // resolve filters
  SjbBatchDesc& D = *b->desc_h;
  D.n_jobs = 0;
  D.n_queries = (uint32_t)n;
  D.group_capacity = (uint64_t)b->lim.group_entries;
  D.smem_capacity = b->smem_entries;
  std::vector<int> held;
  std::unordered_map<std::string, int> local;  // dedupe within the batch when the cache is off
  uint32_t n_in = 0;
  uint64_t built = 0, cached = 0;
  // a filter this batch created but did not build leaves the cache
  auto release_all = [&]() {
    for (int id : held)
      if (b->cache.at(id).built) b->cache.release(id);
      else b->cache.discard_new(id);
  };
  // Jobs this batch: a full build for each new filter, and a statistics-only job
  // for a cached filter that lacks the min/max of an attribute some query here
  // groups by.  job_of maps an entry to its job of this batch.
  std::unordered_map<int, uint32_t> job_of;
  std::vector<int> job_entry;
  auto add_job = [&](int id, uint32_t mask) -> bool {
    const FilterEntry& fe = b->cache.at(id);
    if (fe.kind == SJ_PRED_IN && n_in >= (uint32_t)kBMaxIn) return false;
    SjbJob& J = D.jobs[D.n_jobs];
    memset(&J, 0, sizeof(J));
    J.dim = fe.dim;
    J.attr = fe.kind == SJ_PRED_ALL ? -1 : fe.attr;
    J.kind = fe.kind;
    J.lo = fe.lo;
    J.hi = fe.hi;
    J.words = b->S.words[fe.dim];
    J.in_index = -1;
    J.stats_mask = mask;
    if (fe.kind == SJ_PRED_IN) {
      J.in_index = (int32_t)n_in;
      uint32_t* bits = D.in_bits[n_in++];
      memset(bits, 0, sizeof(uint32_t) * kBInWords);
      for (int32_t c : fe.codes) bits[c >> 5] |= 1u << (c & 31);
    }
    J.bitmap = b->cache.bitmap(id);
    J.stats = b->cache.stats(id);
    job_of[id] = D.n_jobs++;
    job_entry.push_back(id);
    return true;
  };
  for (int i = 0; i < n; ++i) {
    const sjb_query& q = queries[i];
    SjbBatchQuery& Q = D.q[i];
    memset(&Q, 0, sizeof(Q));
    Q.b = q.row_begin;
    Q.e = q.row_end;
    Q.n_preds = (uint32_t)q.n_preds;
    for (int k = 0; k < q.n_preds; ++k) {
      const sjb_pred& p = q.preds[k];
      const uint32_t gbit = p.group_attr >= 0 ? 1u << p.group_attr : 0u;
      int id = -1;
      bool is_new = false;
      const std::string key = FilterCache::make_key(p, nullptr);
      auto it = local.find(key);
      if (it != local.end()) {
        id = it->second;
      } else {
        id = b->cache.acquire(p, b->S.words[p.dim], b->lim.cache_filters != 0, &is_new);
        if (id < 0) {
          release_all();
          return fail_fmt(SJ_ERR_OUT_OF_MEMORY, "filter cache (%lld bytes) cannot hold this batch's filters",
                          (long long)b->lim.filter_cache_bytes);
        }
        held.push_back(id);
        local[key] = id;
        if (is_new) ++built;
        else ++cached;
      }
      auto jt = job_of.find(id);
      bool ok = true;
      if (jt != job_of.end()) {
        D.jobs[jt->second].stats_mask |= gbit;  // built or completed in this batch
      } else if (is_new) {
        ok = add_job(id, gbit);
      } else if (gbit & ~b->cache.at(id).stats_have) {
        ok = add_job(id, kJobStatsOnly | (gbit & ~b->cache.at(id).stats_have));
      }
      if (!ok) {
        release_all();
        return fail_fmt(SJ_ERR_UNSUPPORTED, "more than %d IN-list filters to build in one batch", kBMaxIn);
      }
      Q.dim[k] = (uint32_t)p.dim;
      Q.group_attr[k] = p.group_attr;
      Q.stats[k] = b->cache.stats(id);
      Q.bitmap[k] = b->cache.bitmap(id);
    }
  }
  cudaError_t e = batch_launch(b, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    release_all();
    return cuda_fail(e, "batch pipeline");
  }
  for (int id : held) b->cache.at(id).built = true;
  for (uint32_t j = 0; j < D.n_jobs; ++j) b->cache.at(job_entry[j]).stats_have |= D.jobs[j].stats_mask & kJobAllStats;
  e = cudaGetLastError();  // an error no call above reported
  if (e != cudaSuccess) {
    release_all();
    return cuda_fail(e, "batch pipeline (deferred error)");
  }
  const SjbCounters c = *b->ctr_h;
  float ms = 0.f, msp = 0.f;
  if (cudaEventElapsedTime(&ms, b->ev[0], b->ev[3]) != cudaSuccess) ms = -1.f;
  if (cudaEventElapsedTime(&msp, b->ev[1], b->ev[2]) != cudaSuccess) msp = -1.f;
  cudaGetLastError();  // a timing that could not be read leaves no error behind
  b->last.ms_total = ms;
  b->last.ms_probe = msp;
  b->last.rows_scanned = c.rows_scanned;
  b->last.filters_built = built;
  b->last.filters_cached = cached;
  b->last.error_flags = c.error;
  release_all();
  if (c.error & kBErrGroupCapacity)
    return fail_fmt(SJ_ERR_CAPACITY, "group accumulators exceeded %lld entries", (long long)b->lim.group_entries);
  const uint64_t rows = c.out_rows;
  *n_out = (int64_t)rows;
  if (rows > (uint64_t)b->lim.result_rows)
    return fail_fmt(SJ_ERR_CAPACITY, "batch produced %llu rows (result_rows limit %lld)", (unsigned long long)rows,
                    (long long)b->lim.result_rows);
  if ((int64_t)rows > cap || (rows && !out))
    return fail_fmt(SJ_ERR_CAPACITY, "batch produced %llu rows, buffer holds %lld", (unsigned long long)rows,
                    (long long)cap);
  const uint64_t head = std::min<uint64_t>(rows, b->prefix_rows);
  if (head) memcpy(out, b->rows_h, sizeof(sjb_row) * head);
  if (rows > head) {
    e = cudaMemcpy(out + head, b->rows_d + head, sizeof(sjb_row) * (rows - head), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "result read-back");
  }
  return SJ_OK;
}

extern "C" sj_status sjb_batch_get_stats(sjb_batch* b, sjb_stats* out) {
  if (!b || !out) return fail_fmt(SJ_ERR_INVALID_ARGUMENT, "NULL argument");
  *out = b->last;
  return SJ_OK;
}

// ------------------------------------------------------------------ tuner ----
// Probe shape of the batched form, chosen by timing: every candidate CTA size x
// shared-memory group-partial budget runs the caller's sample batch on a batch
// of its own (same schema, same other limits), `reps` times after one warm-up;
// the median probe time (CUDA events around the probe) decides.  Every
// candidate's groups must equal the first candidate's.
namespace {
bool row_less_b(const sjb_row& a, const sjb_row& b) {
  if (a.query != b.query) return a.query < b.query;
  for (int d = 0; d < SJ_MAX_DIMS; ++d)
    if (a.attr[d] != b.attr[d]) return a.attr[d] < b.attr[d];
  return false;
}
bool rows_same_b(std::vector<sjb_row> a, std::vector<sjb_row> b) {
  if (a.size() != b.size()) return false;
  std::sort(a.begin(), a.end(), row_less_b);
  std::sort(b.begin(), b.end(), row_less_b);
  for (size_t i = 0; i < a.size(); ++i)
    if (a[i].query != b[i].query || a[i].count != b[i].count || a[i].sum != b[i].sum ||
        memcmp(a[i].attr, b[i].attr, sizeof(a[i].attr)) != 0)
      return false;
  return true;
}
}  // namespace

extern "C" sj_status sjb_batch_tune(sj_engine* eng, const sjb_schema* schema, const sjb_limits* base,
                                    const sjb_query* sample, int32_t n, int32_t reps, sjb_limits* chosen,
                                    sjb_tune_report* report) {
  if (!eng || !schema || !sample || !chosen || n < 1 || n > SJB_MAX_QUERIES)
    return fail_fmt(SJ_ERR_INVALID_ARGUMENT, "sjb_batch_tune: bad arguments");
  if (reps < 1) reps = 3;
  sjb_limits lim0;
  memset(&lim0, 0, sizeof(lim0));
  if (base) lim0 = *base;
  sjb_tune_report rep;
  memset(&rep, 0, sizeof(rep));
  const int threads[] = {1024, 512, 256};
  const int entries[] = {6144, 2048, 12288};
  std::vector<sjb_row> first, rows;
  float best = 3.4e38f;
  sjb_limits best_lim = lim0;
  for (int t : threads)
    for (int e : entries) {
      sjb_limits L = lim0;
      L.threads = t;
      L.smem_group_entries = e;
      sjb_batch* b = nullptr;
      if (sjb_batch_create(eng, schema, &L, &b) != SJ_OK) continue;  // a shape that does not fit
      std::vector<float> ms;
      sj_status st = SJ_OK;
      for (int r = 0; r <= reps && st == SJ_OK; ++r) {
        int64_t got = 0;
        rows.resize(std::max<size_t>(rows.size(), 4096));
        st = sjb_batch_run(b, sample, n, rows.data(), (int64_t)rows.size(), &got, nullptr);
        if (st == SJ_ERR_CAPACITY && got > (int64_t)rows.size()) {  // more result rows than the buffer
          rows.resize((size_t)got);
          st = sjb_batch_run(b, sample, n, rows.data(), (int64_t)rows.size(), &got, nullptr);
        }
        if (st != SJ_OK) break;
        if (r == 0) {  // warm-up run: the groups to compare
          std::vector<sjb_row> mine(rows.begin(), rows.begin() + got);
          if (first.empty() && rep.candidates == 0) first = mine;
          else if (!rows_same_b(first, mine)) ++rep.mismatches;
          continue;
        }
        sjb_stats s;
        sjb_batch_get_stats(b, &s);
        ms.push_back(s.ms_probe);
      }
      sjb_batch_destroy(b);
      if (st != SJ_OK || ms.empty()) continue;
      std::sort(ms.begin(), ms.end());
      const float med = ms[ms.size() / 2];
      if (rep.candidates == 0) rep.default_probe_ms = med;
      ++rep.candidates;
      if (med < best) {
        best = med;
        best_lim = L;
      }
    }
  if (!rep.candidates) return fail_fmt(SJ_ERR_UNSUPPORTED, "sjb_batch_tune: no candidate shape ran");
  rep.threads = best_lim.threads;
  rep.smem_group_entries = best_lim.smem_group_entries;
  rep.best_probe_ms = best;
  *chosen = best_lim;
  if (report) *report = rep;
  if (rep.mismatches) return fail_fmt(SJ_ERR_CUDA, "sjb_batch_tune: %d candidate shapes changed the groups", rep.mismatches);
  return SJ_OK;
}
