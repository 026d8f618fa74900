// sj_serve.cu -- the serving loop (include/starjoin_batch.h, sjs_*).
//
// A request loop over a resident fact table.  Queries are admitted while query
// slots (64) and device memory (filter cache + group accumulators, sized from
// the free HBM at start) allow; each admitted query attaches to a circular
// shared scan at its current position and leaves once the scan has covered its
// fact row range, so a query that arrives while others run shares their scan
// (continuous batching in the sense of shared-scan engines: CJOIN's continuous
// pipeline, Crescando's ClockScan).  Between scan steps the loop admits new
// queries, builds the filters the cache lacks, recomposes the 64-bit slot
// words when the set of queries changed, and returns finished queries' groups.
//
// `plain = 1` serves the same requests one at a time through the plain engine
// (sj_run_plain), the baseline the shared form is measured against.
// `solo_plain = 1` sends a query that finds the scan idle and no other query
// waiting through the plain engine too, when its row range fits in one scan
// step: alone, the plain probe reads only the fact columns its survivors need
// (the shared scan reads every column over the query's range), so a short
// query's latency is the plain engine's.  A longer query still starts the
// shared scan, which later arrivals join at the next step instead of queueing
// behind it.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "sj_cache.h"
#include "sj_internal.h"
#include "sj_shared.h"

using namespace sj;

namespace {

double now_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

struct Ticket {
  sjb_query q{};
  std::vector<int32_t> codes[SJ_MAX_DIMS];
  uint64_t worst = 0;
  double submit_s = 0, admit_s = 0, finish_s = 0;
  int status = SJ_OK;
  bool done = false;
  bool cancel = false;  // asked to leave the scan (sjs_cancel)
  std::vector<sjb_row> rows;
};

struct Slot {
  bool used = false;
  uint64_t ticket = 0;
  int entry[SJ_MAX_DIMS] = {-1, -1, -1, -1};
  int n_entries = 0;
  uint64_t group_off = 0, group_span = 0;
  SjbSlot lay{};
  float sel[SJ_MAX_DIMS] = {1.f, 1.f, 1.f, 1.f};
  const uint32_t* bm[SJ_MAX_DIMS] = {nullptr, nullptr, nullptr, nullptr};
  std::vector<Interval> remaining;  // fact rows still to scan (at most two pieces)
  bool cancelled = false;           // leaves at the next step boundary; groups discarded
};

}  // namespace

struct sjs_server {
  sj_engine* eng = nullptr;
  SchemaState S;
  sjs_config cfg{};
  int64_t step_rows = 0;
  int max_active = kBq;
  uint64_t result_rows = 1ull << 20;
  // device
  SjbAcc* acc = nullptr;
  sjb_row* rows_d = nullptr;
  SjbCounters* ctr_d = nullptr;
  SjbStep* step_d = nullptr;
  SjbBatchDesc* desc_d = nullptr;
  uint8_t* arena = nullptr;
  SjbEntryStats* stats_d = nullptr;
  int32_t* slot_query_d = nullptr;
  // pinned (double-buffered per step: [buffer][0 = composition, 1 = probe])
  SjbStep* step_h[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
  SjbBatchDesc* desc_h = nullptr;
  SjbCounters* ctr_h = nullptr;
  SjbEntryStats* stats_h = nullptr;
  int32_t* slot_query_h = nullptr;
  sjb_row* rows_h[2] = {nullptr, nullptr};
  cudaStream_t st = nullptr;   // scan steps
  cudaStream_t stb = nullptr;  // admission: filter builds, accumulator clears
  cudaEvent_t ev_probe[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
  cudaEvent_t ev_done[2] = {nullptr, nullptr};
  cudaEvent_t ev_admitted = nullptr;
  struct StepRec {
    bool valid = false;
    bool probed = false;
    uint64_t fin = 0;          // slots whose groups this step reads back
    uint64_t bound = 0;        // result rows copied back (sum of their spans)
  } rec[2];
  int next_buf = 0;            // buffer of the next step launch
  uint64_t fin_queued = 0;     // finished slots whose read-back is enqueued
  int64_t next_pos = 0;        // scan position after the last launched step
  FilterCache cache;
  RangeAlloc groups;
  // loop state
  std::thread th;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<uint64_t> pending;
  std::unordered_map<uint64_t, Ticket> tickets;
  uint64_t next_ticket = 1;
  bool stop = false;
  int waiters = 0;             // threads inside sjs_wait
  uint64_t admissions = 0;     // admission attempts (fault injection counts these)
  Slot slots[kBq];
  bool masks_dirty = true;
  sjs_stats stats{};
  std::string loop_error;
};

namespace {

void finish_ticket(sjs_server* s, uint64_t id, int status, std::vector<sjb_row>&& rows) {
  std::lock_guard<std::mutex> g(s->mu);
  auto it = s->tickets.find(id);
  if (it == s->tickets.end()) return;
  Ticket& t = it->second;
  t.status = status;
  t.rows = std::move(rows);
  t.finish_s = now_s();
  t.done = true;
  ++s->stats.finished;
  s->cv_done.notify_all();
}

// Next row at or after `pos` (cyclically over [0, n)) that an admitted query still needs.
int64_t next_needed(sjs_server* s, int64_t pos, int64_t n) {
  int64_t best = -1, best_dist = INT64_MAX;
  for (const Slot& sl : s->slots) {
    if (!sl.used) continue;
    int64_t dist = 0;
    const int64_t cand = first_needed(sl.remaining, pos, n, &dist);
    if (cand >= 0 && dist < best_dist) {
      best_dist = dist;
      best = cand;
    }
  }
  return best;
}

void release_slot(sjs_server* s, int q) {
  Slot& sl = s->slots[q];
  for (int k = 0; k < sl.n_entries; ++k) s->cache.release(sl.entry[k]);
  if (sl.group_span) s->groups.release(sl.group_off, sl.group_span);
  sl = Slot();
  s->masks_dirty = true;
}

// A pending ticket's query, copied under s->mu (the ticket itself may be
// cancelled and released while the copy is in use).
struct QueryCopy {
  sjb_query q{};
  std::vector<int32_t> codes[SJ_MAX_DIMS];
};

bool pending_query(sjs_server* s, uint64_t id, QueryCopy& out) {
  auto it = s->tickets.find(id);
  if (it == s->tickets.end() || it->second.done) return false;
  out.q = it->second.q;
  for (int k = 0; k < SJ_MAX_DIMS; ++k) {
    out.codes[k] = it->second.codes[k];
    if (k < out.q.n_preds && out.q.preds[k].in_count > 0) out.q.preds[k].in_codes = out.codes[k].data();
  }
  return true;
}

// Remove id from the queue (under s->mu); false if it left meanwhile (cancelled).
bool take_pending(sjs_server* s, uint64_t id) {
  auto p = std::find(s->pending.begin(), s->pending.end(), id);
  if (p == s->pending.end()) return false;
  s->pending.erase(p);
  return true;
}

// Admit pending tickets into free slots while memory allows.  Returns false on a CUDA error.
bool admit(sjs_server* s) {
  SjNvtxRange nvtx_range("sjs.admit");
  std::vector<uint64_t> cand;
  bool idle = true;
  for (const Slot& sl : s->slots) idle &= !sl.used;
  {
    std::lock_guard<std::mutex> g(s->mu);
    int free_slots = 0, used = 0;
    for (const Slot& sl : s->slots) (sl.used ? used : free_slots) += 1;
    const int room = std::min(free_slots, s->max_active - used);
    for (size_t i = 0; i < s->pending.size() && (int)cand.size() < room; ++i) cand.push_back(s->pending[i]);
  }
  if (cand.empty()) return true;
  struct Adm {
    uint64_t id;
    int entry[SJ_MAX_DIMS];
    int n;
    QueryCopy qc;
  };
  std::vector<Adm> adm;
  SjbBatchDesc& D = *s->desc_h;
  D.n_jobs = 0;
  uint32_t n_in = 0;
  uint64_t hits = 0;
  std::vector<int> new_ids;  // entries built or completed this round (statistics read back)
  // A full build for each new filter; a statistics-only job for a built filter
  // that lacks the min/max of an attribute an admitted query groups by.
  std::unordered_map<int, uint32_t> job_of;
  std::vector<int> job_entry;
  auto add_job = [&](int eid, uint32_t mask) -> bool {
    const FilterEntry& fe = s->cache.at(eid);
    if (D.n_jobs >= (uint32_t)kBMaxJobs || (fe.kind == SJ_PRED_IN && n_in >= (uint32_t)kBMaxIn)) return false;
    SjbJob& J = D.jobs[D.n_jobs];
    memset(&J, 0, sizeof(J));
    J.dim = fe.dim;
    J.attr = fe.kind == SJ_PRED_ALL ? -1 : fe.attr;
    J.kind = fe.kind;
    J.lo = fe.lo;
    J.hi = fe.hi;
    J.words = s->S.words[fe.dim];
    J.in_index = -1;
    J.stats_mask = mask;
    if (fe.kind == SJ_PRED_IN) {
      J.in_index = (int32_t)n_in;
      uint32_t* bits = D.in_bits[n_in++];
      memset(bits, 0, sizeof(uint32_t) * kBInWords);
      for (int32_t c : fe.codes) bits[c >> 5] |= 1u << (c & 31);
    }
    J.bitmap = s->cache.bitmap(eid);
    J.stats = s->cache.stats(eid);
    job_of[eid] = D.n_jobs++;
    job_entry.push_back(eid);
    new_ids.push_back(eid);
    return true;
  };
  for (uint64_t id : cand) {
    Adm a{id, {-1, -1, -1, -1}, 0, {}};
    {
      std::lock_guard<std::mutex> g(s->mu);
      if (!pending_query(s, id, a.qc)) continue;  // cancelled since the queue was read
    }
    if (s->cfg.fault_admit_every > 0 && ++s->admissions % (uint64_t)s->cfg.fault_admit_every == 0) {
      // injected fault: this admission fails as a device allocation would
      bool was;
      {
        std::lock_guard<std::mutex> g(s->mu);
        was = take_pending(s, id);
      }
      if (was) finish_ticket(s, id, SJ_ERR_OUT_OF_MEMORY, {});
      continue;
    }
    const sjb_query& tq = a.qc.q;
    bool ok = true;
    for (int k = 0; k < tq.n_preds && ok; ++k) {
      const sjb_pred& p = tq.preds[k];
      const uint32_t gbit = p.group_attr >= 0 ? 1u << p.group_attr : 0u;
      bool is_new = false;
      const int eid = s->cache.acquire(p, s->S.words[p.dim], s->cfg.limits.cache_filters != 0, &is_new);
      if (eid < 0) {
        ok = false;
        break;
      }
      auto jt = job_of.find(eid);
      bool fits = true;
      if (jt != job_of.end()) {
        D.jobs[jt->second].stats_mask |= gbit;  // built or completed this round
      } else if (is_new) {
        fits = add_job(eid, gbit);
      } else if (gbit & ~s->cache.at(eid).stats_have) {
        fits = add_job(eid, kJobStatsOnly | (gbit & ~s->cache.at(eid).stats_have));
      }
      if (!fits) {
        if (is_new) s->cache.discard_new(eid);
        else s->cache.release(eid);
        ok = false;
        break;
      }
      a.entry[a.n++] = eid;
      if (!is_new) ++hits;
    }
    if (!ok) {
      for (int k = 0; k < a.n; ++k) s->cache.release(a.entry[k]);
      if (idle && adm.empty()) {  // cannot fit even alone: refuse it
        bool was;
        {
          std::lock_guard<std::mutex> g(s->mu);
          was = take_pending(s, id);
          if (was) ++s->stats.rejected;
        }
        if (was) finish_ticket(s, id, SJ_ERR_REJECTED, {});
      }
      break;  // memory is full: keep FIFO order, retry after queries leave
    }
    adm.push_back(std::move(a));
  }
  // build the new filters and read back every admitted predicate's statistics
  if (D.n_jobs) {
    // upload the header and the jobs in use, then the IN-code bitmaps in use
    const size_t head = offsetof(SjbBatchDesc, jobs) + sizeof(SjbJob) * D.n_jobs;
    if (cudaMemcpyAsync(s->desc_d, s->desc_h, head, cudaMemcpyHostToDevice, s->stb) != cudaSuccess) return false;
    if (n_in && cudaMemcpyAsync(s->desc_d->in_bits, s->desc_h->in_bits, sizeof(uint32_t) * kBInWords * n_in,
                                cudaMemcpyHostToDevice, s->stb) != cudaSuccess)
      return false;
    if (sjb_launch_build(s->S.rt, s->desc_d, D.n_jobs, D.n_jobs, s->eng->sm_count, s->stb) != cudaSuccess)
      return false;
    // one read-back of the statistics records (indexed by entry id)
    uint32_t hi = 0;
    for (int id : new_ids) hi = std::max(hi, s->cache.at(id).stats_idx + 1);
    if (cudaMemcpyAsync(s->stats_h, s->stats_d, sizeof(SjbEntryStats) * hi, cudaMemcpyDeviceToHost, s->stb) !=
        cudaSuccess)
      return false;
    if (cudaStreamSynchronize(s->stb) != cudaSuccess) return false;
    for (size_t i = 0; i < new_ids.size(); ++i) {
      FilterEntry& e = s->cache.at(new_ids[i]);
      e.host = s->stats_h[e.stats_idx];
      e.host_valid = true;
      e.built = true;
    }
    uint64_t full_builds = 0;
    for (uint32_t j = 0; j < D.n_jobs; ++j) {
      s->cache.at(job_entry[j]).stats_have |= D.jobs[j].stats_mask & kJobAllStats;
      full_builds += (D.jobs[j].stats_mask & kJobStatsOnly) ? 0u : 1u;
    }
    std::lock_guard<std::mutex> g(s->mu);
    s->stats.filters_built += full_builds;
  }
  // group layout and accumulator ranges
  const double t_adm = now_s();
  for (const Adm& a : adm) {
    const sjb_query& tq = a.qc.q;
    SjbBatchQuery bq{};
    bq.b = tq.row_begin;
    bq.e = tq.row_end;
    bq.n_preds = (uint32_t)tq.n_preds;
    const SjbEntryStats* stp[SJ_MAX_DIMS];
    for (int k = 0; k < a.n; ++k) {
      bq.dim[k] = (uint32_t)tq.preds[k].dim;
      bq.group_attr[k] = tq.preds[k].group_attr;
      stp[k] = &s->cache.at(a.entry[k]).host;
    }
    SjbSlot lay{};
    float sel[SJ_MAX_DIMS] = {1.f, 1.f, 1.f, 1.f};
    const uint32_t err = sjb_group_layout(s->S.rt, bq, stp, lay, sel, 1ull << 32);
    const uint64_t span = lay.span;
    uint64_t off = 0;
    if (span && !err) {
      off = s->groups.alloc(span);
      if (off == ~0ull) {  // accumulators full: this and later tickets wait
        for (const Adm& rest : adm)
          if (&rest >= &a)
            for (int k = 0; k < rest.n; ++k) s->cache.release(rest.entry[k]);
        bool any = false;
        for (const Slot& sl : s->slots) any |= sl.used;
        if (!any) {  // cannot fit even alone: refuse it
          bool was;
          {
            std::lock_guard<std::mutex> g(s->mu);
            was = take_pending(s, a.id);
            if (was) ++s->stats.rejected;
          }
          if (was) finish_ticket(s, a.id, SJ_ERR_REJECTED, {});
        }
        break;
      }
    }
    bool still;
    {
      std::lock_guard<std::mutex> g(s->mu);
      still = take_pending(s, a.id);
      if (still) {
        s->tickets[a.id].admit_s = t_adm;
        ++s->stats.admitted;
      }
    }
    if (!still) {  // cancelled while its filters were built
      if (span && !err) s->groups.release(off, span);
      for (int k = 0; k < a.n; ++k) s->cache.release(a.entry[k]);
      continue;
    }
    if (err || span == 0 || bq.e <= bq.b) {  // no row can match (or key space too large)
      for (int k = 0; k < a.n; ++k) s->cache.release(a.entry[k]);
      finish_ticket(s, a.id, err ? SJ_ERR_CAPACITY : SJ_OK, {});
      continue;
    }
    int q = 0;
    while (s->slots[q].used) ++q;
    Slot& sl = s->slots[q];
    sl.used = true;
    sl.ticket = a.id;
    sl.n_entries = a.n;
    for (int k = 0; k < a.n; ++k) {
      sl.entry[k] = a.entry[k];
      sl.bm[bq.dim[k]] = s->cache.bitmap(a.entry[k]);
      sl.sel[bq.dim[k]] = sel[bq.dim[k]];
    }
    sl.group_off = off;
    sl.group_span = span;
    sl.lay = lay;
    sl.lay.group_base = off;
    // the next step starts at next_pos: rows [next_pos, e) come first, then [b, next_pos) after the wrap
    const int64_t b = bq.b, e = bq.e, p = s->next_pos;
    sl.remaining = attach(b, e, p);
    if (cudaMemsetAsync(s->acc + off, 0, sizeof(SjbAcc) * span, s->stb) != cudaSuccess) return false;
    s->masks_dirty = true;
  }
  // the next scan step waits for the accumulator clears
  if (cudaEventRecord(s->ev_admitted, s->stb) != cudaSuccess) return false;
  if (cudaStreamWaitEvent(s->st, s->ev_admitted, 0) != cudaSuccess) return false;
  uint64_t act = 0;
  for (const Slot& sl : s->slots) act += sl.used;
  std::lock_guard<std::mutex> g(s->mu);
  s->stats.filters_cached += hits;
  s->stats.peak_active = std::max<uint64_t>(s->stats.peak_active, act);
  return true;
}

// Fill a step descriptor from the admitted slots; `step` selects which slots
// are active (rows in this step) -- all admitted slots for mask composition.
void fill_step(sjs_server* s, SjbStep& st, bool all, int64_t seg_b, int64_t seg_e) {
  memset(&st, 0, sizeof(SjbStep));
  st.seg_b = seg_b;
  st.seg_e = seg_e;
  uint64_t active = 0;
  for (int q = 0; q < kBq; ++q) {
    Slot& sl = s->slots[q];
    st.slot[q] = sl.lay;
    st.slot[q].b = st.slot[q].e = 0;
    for (int d = 0; d < SJ_MAX_DIMS; ++d) {
      st.bm[q][d] = sl.used ? sl.bm[d] : nullptr;
      st.sel[q][d] = sl.sel[d];
    }
    if (!sl.used) continue;
    if (all) {  // slot words for the slots still scanning
      if (!sl.remaining.empty()) active |= 1ull << q;
      else for (int d = 0; d < SJ_MAX_DIMS; ++d) st.bm[q][d] = nullptr;
      continue;
    }
    const Interval iv = take(sl.remaining, seg_b, seg_e);
    if (iv.e > iv.b) {
      st.slot[q].b = iv.b;
      st.slot[q].e = iv.e;
      active |= 1ull << q;
    }
  }
  st.active = active;
  sjb_step_layout(st, s->S.rt.n_dims, 6144u);
}

// Launch the next scan step into buffer set `b` (asynchronous): recompose the
// slot words if the set of queries changed, probe the next segment some query
// still needs, and queue the read-back of every query that step finishes.
// Which queries a step finishes is known when it is planned, so their group
// compaction and copies go into the stream right behind the probe; the host
// collects them (complete_step) while the next step already runs.
bool launch_step(sjs_server* s, bool* launched) {
  SjNvtxRange nvtx_range("sjs.launch_step");
  *launched = false;
  const int b = s->next_buf;
  const int64_t n = s->S.rt.fact_rows;
  if (s->masks_dirty) {
    fill_step(s, *s->step_h[b][0], true, 0, 0);
    if (cudaMemcpyAsync(s->step_d, s->step_h[b][0], sizeof(SjbStep), cudaMemcpyHostToDevice, s->st) != cudaSuccess)
      return false;
    if (sjb_launch_compose(s->S.rt, s->step_d, s->eng->sm_count, s->st) != cudaSuccess) return false;
    s->masks_dirty = false;
  }
  SjbCounters* ctr = s->ctr_d + 2 * b;
  const int64_t p = next_needed(s, s->next_pos, n);
  bool probed = false;
  if (p >= 0) {
    const int64_t seg_b = p, seg_e = std::min<int64_t>(n, p + s->step_rows);
    SjbStep& st = *s->step_h[b][1];
    fill_step(s, st, false, seg_b, seg_e);
    if (cudaMemcpyAsync(s->step_d, s->step_h[b][1], sizeof(SjbStep), cudaMemcpyHostToDevice, s->st) != cudaSuccess)
      return false;
    if (cudaMemsetAsync(ctr, 0, 2 * sizeof(SjbCounters), s->st) != cudaSuccess) return false;
    const uint32_t threads = s->cfg.limits.threads ? (uint32_t)s->cfg.limits.threads : 1024u;
    if (cudaEventRecord(s->ev_probe[b][0], s->st) != cudaSuccess) return false;
    const L2Window w = l2_window(s->S.masks, s->S.masks_bytes, s->eng->l2_persist_bytes, s->eng->l2_window_max);
    if (sjb_launch_probe(s->S.rt, s->step_d, s->acc, ctr, threads, st.smem_entries, s->eng->sm_count, s->st, w) !=
        cudaSuccess)
      return false;
    if (cudaEventRecord(s->ev_probe[b][1], s->st) != cudaSuccess) return false;
    for (int q = 0; q < kBq; ++q)
      if ((st.active >> q) & 1ull) cover(s->slots[q].remaining, {st.slot[q].b, st.slot[q].e});
    s->next_pos = seg_e >= n ? 0 : seg_e;
    probed = true;
  }
  // read back the finished slots (as many as the result buffer holds; the rest next time)
  uint64_t fin = 0, bound = 0;
  for (int q = 0; q < kBq; ++q) {
    const Slot& sl = s->slots[q];
    if (!sl.used || !sl.remaining.empty() || ((s->fin_queued >> q) & 1ull)) continue;
    if (fin && bound + sl.group_span > s->result_rows) continue;
    fin |= 1ull << q;
    bound += sl.group_span;
  }
  if (!probed && !fin) return true;
  if (fin) {
    // step_d holds every used slot's layout (each upload copies them all)
    if (!probed && cudaMemsetAsync(ctr + 1, 0, sizeof(SjbCounters), s->st) != cudaSuccess) return false;
    if (sjb_launch_finalize(s->step_d, fin, s->acc, s->rows_d, s->result_rows, ctr + 1, s->slot_query_d,
                            s->eng->sm_count, s->st) != cudaSuccess)
      return false;
    if (cudaMemcpyAsync(s->rows_h[b], s->rows_d, sizeof(sjb_row) * bound, cudaMemcpyDeviceToHost, s->st) !=
        cudaSuccess)
      return false;
  }
  if (cudaMemcpyAsync(s->ctr_h + 2 * b, ctr, 2 * sizeof(SjbCounters), cudaMemcpyDeviceToHost, s->st) != cudaSuccess)
    return false;
  if (cudaEventRecord(s->ev_done[b], s->st) != cudaSuccess) return false;
  s->rec[b].valid = true;
  s->rec[b].probed = probed;
  s->rec[b].fin = fin;
  s->rec[b].bound = bound;
  s->fin_queued |= fin;
  s->next_buf = b ^ 1;
  *launched = true;
  return true;
}

// Wait for the step in buffer set `b` and hand out the groups it read back.
bool complete_step(sjs_server* s, int b) {
  SjNvtxRange nvtx_range("sjs.complete_step");
  auto& r = s->rec[b];
  if (!r.valid) return true;
  if (cudaEventSynchronize(s->ev_done[b]) != cudaSuccess) return false;
  r.valid = false;
  const SjbCounters* c = s->ctr_h + 2 * b;
  if (r.fin) {
    const uint64_t nrows = std::min<uint64_t>(c[1].out_rows, r.bound);
    std::vector<std::vector<sjb_row>> per(kBq);
    for (uint64_t i = 0; i < nrows; ++i) per[s->rows_h[b][i].query].push_back(s->rows_h[b][i]);
    for (int q = 0; q < kBq; ++q) {
      if (!((r.fin >> q) & 1ull)) continue;
      for (sjb_row& x : per[q]) x.query = 0;
      const uint64_t id = s->slots[q].ticket;
      const bool cancelled = s->slots[q].cancelled;
      release_slot(s, q);
      s->fin_queued &= ~(1ull << q);
      if (cancelled) per[q].clear();
      finish_ticket(s, id, cancelled ? SJ_ERR_CANCELLED : SJ_OK, std::move(per[q]));
    }
  }
  if (r.probed) {
    float pms = 0.f;
    if (cudaEventElapsedTime(&pms, s->ev_probe[b][0], s->ev_probe[b][1]) != cudaSuccess) pms = 0.f;
    std::lock_guard<std::mutex> g(s->mu);
    s->stats.rows_scanned += c[0].rows_scanned;
    s->stats.probe_device_s += pms * 1e-3;
    ++s->stats.steps;
  }
  return true;
}

// Run ticket `id` (the queue's head) through the plain engine; false if it was
// cancelled before it started.
bool plain_one(sjs_server* s, uint64_t id) {
  SjNvtxRange nvtx_range("sjs.plain_query");
  QueryCopy qc;
  {
    std::lock_guard<std::mutex> g(s->mu);
    if (s->pending.empty() || s->pending.front() != id) return false;  // cancelled meanwhile
    s->pending.pop_front();
    if (!pending_query(s, id, qc)) return false;
    s->tickets[id].admit_s = now_s();
    ++s->stats.admitted;
  }
  const sjb_query& q = qc.q;
  sj_plan plan;
  memset(&plan, 0, sizeof(plan));
  plan.n_dims = q.n_preds;
  for (int k = 0; k < q.n_preds; ++k) {
    const sjb_pred& p = q.preds[k];
    const sjb_dim& D = s->S.schema.dims[p.dim];
    sj_dim& d = plan.dims[k];
    d.fact_fk = D.fact_fk;
    d.key = D.key;
    d.filter_attr = p.kind == SJ_PRED_ALL ? nullptr : D.attr[p.attr];
    d.payload = p.group_attr >= 0 ? D.attr[p.group_attr] : nullptr;
    d.rows = D.rows;
    d.key_min = D.key_min;
    d.ht_len = D.ht_len;
    d.pred_kind = p.kind;
    d.pred_lo = p.lo;
    d.pred_hi = p.hi;
    d.in_count = p.in_count;
    d.in_codes = p.in_codes;
    d.group = p.group_attr >= 0;
    if (d.group) {
      d.payload_min = (int32_t)s->S.attr_min[p.dim][p.group_attr];
      d.payload_max = (int32_t)s->S.attr_max[p.dim][p.group_attr];
    }
    plan.order[k] = k;
  }
  plan.measure = s->S.schema.measure;
  plan.measure_sub = s->S.schema.measure_sub;
  plan.fact_rows = s->S.schema.fact_rows;
  plan.row_begin = q.row_begin;
  plan.row_end = q.row_end;
  plan.lip = 1;
  plan.bf_bits_per_key = 0;
  plan.bf_hashes = 2;
  std::vector<sj_group_row> rows(4096);
  int64_t n = 0;
  float ms = 0.f;
  sj_status rc = sj_run_plain(s->eng, &plan, 0, rows.data(), (int64_t)rows.size(), &n, &ms, s->st);
  if (rc == SJ_ERR_CAPACITY && n > (int64_t)rows.size()) {
    rows.resize((size_t)n);
    rc = sj_run_plain(s->eng, &plan, 0, rows.data(), (int64_t)rows.size(), &n, &ms, s->st);
  }
  std::vector<sjb_row> out;
  {
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->tickets.find(id);
    if (rc == SJ_OK && it != s->tickets.end() && it->second.cancel) rc = SJ_ERR_CANCELLED;
  }
  if (rc == SJ_OK) {
    out.resize((size_t)n);
    for (int64_t i = 0; i < n; ++i) {
      sjb_row& r = out[(size_t)i];
      memset(&r, 0, sizeof(r));
      for (int k = 0; k < q.n_preds; ++k) r.attr[k] = q.preds[k].group_attr >= 0 ? rows[(size_t)i].attr[k] : 0;
      r.count = rows[(size_t)i].count;
      r.sum = rows[(size_t)i].sum;
    }
    std::lock_guard<std::mutex> g(s->mu);
    s->stats.rows_scanned += (uint64_t)(q.row_end - q.row_begin);
    ++s->stats.steps;
  }
  finish_ticket(s, id, rc, std::move(out));
  return true;
}

// Whether the plain engine can answer q: its group space (full ranges of the
// grouped attributes, as plain_one lays it out) within the plain engine's limits.
bool plain_fits(const sjs_server* s, const sjb_query& q) {
  uint64_t groups = 1;
  for (int k = 0; k < q.n_preds; ++k) {
    const sjb_pred& p = q.preds[k];
    if (p.group_attr < 0) continue;
    const int64_t span = s->S.attr_max[p.dim][p.group_attr] - s->S.attr_min[p.dim][p.group_attr] + 1;
    if (span < 1 || span > SJ_MAX_PAYLOAD_SPAN) return false;
    groups *= (uint64_t)span;
    if (groups > (1ull << 26)) return false;
  }
  return true;
}

// The one waiting query when the scan is idle, nothing else waits and its row
// range fits in one scan step (0 otherwise).
uint64_t solo_candidate(sjs_server* s) {
  if (!s->cfg.solo_plain || s->rec[0].valid || s->rec[1].valid) return 0;
  for (const Slot& sl : s->slots)
    if (sl.used) return 0;
  std::lock_guard<std::mutex> g(s->mu);
  if (s->pending.size() != 1) return 0;
  const uint64_t id = s->pending.front();
  auto it = s->tickets.find(id);
  if (it == s->tickets.end() || it->second.done) return 0;
  const sjb_query& q = it->second.q;
  if (q.row_end - q.row_begin > s->step_rows || !plain_fits(s, q)) return 0;
  return id;
}

void loop(sjs_server* s) {
  cudaSetDevice(s->eng->device);
  for (;;) {
    bool any_active = false;
    for (const Slot& sl : s->slots) any_active |= sl.used;
    {
      std::unique_lock<std::mutex> g(s->mu);
      if (!any_active && !s->rec[0].valid && !s->rec[1].valid)
        s->cv_work.wait(g, [&] { return s->stop || !s->pending.empty(); });
      if (s->stop) break;
    }
    const double t0 = now_s();
    bool ok = true;
    uint64_t solo = 0;
    if (s->cfg.plain) {
      uint64_t id = 0;
      {
        std::lock_guard<std::mutex> g(s->mu);
        if (!s->pending.empty()) id = s->pending.front();
      }
      if (id) plain_one(s, id);
    } else if ((solo = solo_candidate(s)) != 0) {
      if (plain_one(s, solo)) {
        std::lock_guard<std::mutex> g(s->mu);
        ++s->stats.solo;
      }
    } else {
      // admission (filter builds on the second stream) overlaps the steps in flight;
      // step k+1 is launched before step k's results are collected
      ok = admit(s);
      const double t1 = now_s();
      bool active = false;
      for (const Slot& sl : s->slots) active |= sl.used;
      {  // running queries asked to stop leave the scan: nothing left to read
        std::lock_guard<std::mutex> g(s->mu);
        for (Slot& sl : s->slots) {
          if (!sl.used || sl.cancelled) continue;
          auto it = s->tickets.find(sl.ticket);
          if (it != s->tickets.end() && it->second.cancel) {
            sl.cancelled = true;
            sl.remaining.clear();
            s->masks_dirty = true;
          }
        }
      }
      bool launched = false;
      if (ok && active) ok = launch_step(s, &launched);
      if (ok && launched) ok = complete_step(s, s->next_buf);  // the older of the two buffer sets
      else if (ok) ok = complete_step(s, 0) && complete_step(s, 1);  // nothing new: drain
      std::lock_guard<std::mutex> g(s->mu);
      s->stats.admit_s += t1 - t0;
      s->stats.scan_s += now_s() - t1;
    }
    {
      std::lock_guard<std::mutex> g(s->mu);
      s->stats.busy_s += now_s() - t0;
    }
    if (!ok) {  // a CUDA error ends the loop; every waiting ticket fails
      std::lock_guard<std::mutex> g(s->mu);
      s->loop_error = cudaGetErrorString(cudaGetLastError());
      for (auto& kv : s->tickets)
        if (!kv.second.done) {
          kv.second.done = true;
          kv.second.status = SJ_ERR_CUDA;
          kv.second.finish_s = now_s();
        }
      s->pending.clear();
      s->cv_done.notify_all();
      break;
    }
  }
}

void server_free(sjs_server* s) {
  if (!s) return;
  cudaSetDevice(s->eng->device);
  if (s->st) cudaStreamSynchronize(s->st);
  if (s->stb) cudaStreamSynchronize(s->stb);
  cudaFree(s->acc);
  cudaFree(s->rows_d);
  cudaFree(s->ctr_d);
  cudaFree(s->step_d);
  cudaFree(s->desc_d);
  cudaFree(s->arena);
  cudaFree(s->stats_d);
  cudaFree(s->slot_query_d);
  for (auto& pair : s->step_h)
    for (auto& h : pair) cudaFreeHost(h);
  cudaFreeHost(s->desc_h);
  cudaFreeHost(s->ctr_h);
  cudaFreeHost(s->stats_h);
  cudaFreeHost(s->slot_query_h);
  for (auto& h : s->rows_h) cudaFreeHost(h);
  if (s->st) cudaStreamDestroy(s->st);
  if (s->stb) cudaStreamDestroy(s->stb);
  if (s->ev_admitted) cudaEventDestroy(s->ev_admitted);
  for (auto& pair : s->ev_probe)
    for (auto& e : pair)
      if (e) cudaEventDestroy(e);
  for (auto& e : s->ev_done)
    if (e) cudaEventDestroy(e);
  schema_release(s->S);
  delete s;
}

}  // namespace

extern "C" double sjs_now(void) { return now_s(); }

extern "C" sj_status sjs_server_create(sj_engine* eng, const sjb_schema* schema, const sjs_config* cfg,
                                       sjs_server** out) {
  if (!eng || !out) return fail_fmt(SJ_ERR_INVALID_ARGUMENT, "engine or out is NULL");
  *out = nullptr;
  sjs_server* s = new sjs_server();
  s->eng = eng;
  if (cfg) s->cfg = *cfg;
  sj_status rc = schema_register(eng, schema, s->S);
  if (rc != SJ_OK) {
    delete s;
    return rc;
  }
  const int64_t n = s->S.rt.fact_rows;
  s->step_rows = s->cfg.step_rows > 0 ? s->cfg.step_rows : std::max<int64_t>(1 << 20, n / 8);
  s->step_rows = (s->step_rows + 127) / 128 * 128;
  s->max_active = s->cfg.max_active > 0 ? std::min(s->cfg.max_active, kBq) : kBq;
  const uint32_t threads = s->cfg.limits.threads ? (uint32_t)s->cfg.limits.threads : 1024u;
  if (threads != 256 && threads != 512 && threads != 1024) {
    server_free(s);
    return fail_fmt(SJ_ERR_INVALID_ARGUMENT, "threads=%d (256, 512 or 1024)", s->cfg.limits.threads);
  }
  // admission budget: device memory that is free now, minus the reserve
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  const int64_t reserve = s->cfg.hbm_reserve_bytes > 0 ? s->cfg.hbm_reserve_bytes : (2ll << 30);
  const int64_t budget = std::max<int64_t>(64ll << 20, (int64_t)free_b - reserve);
  int64_t groups = s->cfg.limits.group_entries > 0 ? s->cfg.limits.group_entries : (1ll << 24);
  int64_t fcache = s->cfg.limits.filter_cache_bytes > 0 ? s->cfg.limits.filter_cache_bytes : (1ll << 30);
  groups = std::min<int64_t>(groups, budget / 2 / (int64_t)sizeof(SjbAcc));
  fcache = std::min<int64_t>(fcache, budget / 2);
  s->cfg.limits.group_entries = groups;
  s->cfg.limits.filter_cache_bytes = fcache;
  cudaError_t e = cudaSuccess;
  auto step = [&](cudaError_t x) {
    if (e == cudaSuccess) e = x;
  };
  const uint32_t max_entries = 8192;
  step(cudaMalloc(&s->acc, sizeof(SjbAcc) * (size_t)groups));
  step(cudaMalloc(&s->rows_d, sizeof(sjb_row) * s->result_rows));
  step(cudaMalloc(&s->ctr_d, 4 * sizeof(SjbCounters)));
  step(cudaMalloc(&s->step_d, sizeof(SjbStep)));
  step(cudaMalloc(&s->desc_d, sizeof(SjbBatchDesc)));
  step(cudaMalloc(&s->arena, (size_t)fcache));
  step(cudaMalloc(&s->stats_d, sizeof(SjbEntryStats) * max_entries));
  step(cudaMalloc(&s->slot_query_d, sizeof(int32_t) * kBq));
  for (auto& pair : s->step_h)
    for (auto& h : pair) step(cudaMallocHost(&h, sizeof(SjbStep)));
  step(cudaMallocHost(&s->desc_h, sizeof(SjbBatchDesc)));
  step(cudaMallocHost(&s->ctr_h, 4 * sizeof(SjbCounters)));
  step(cudaMallocHost(&s->stats_h, sizeof(SjbEntryStats) * max_entries));
  step(cudaMallocHost(&s->slot_query_h, sizeof(int32_t) * kBq));
  step(cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking));
  step(cudaStreamCreateWithFlags(&s->stb, cudaStreamNonBlocking));
  step(cudaEventCreateWithFlags(&s->ev_admitted, cudaEventDisableTiming));
  for (auto& h : s->rows_h) step(cudaMallocHost(&h, sizeof(sjb_row) * s->result_rows));
  for (auto& pair : s->ev_probe)
    for (auto& ev : pair) step(cudaEventCreate(&ev));
  for (auto& ev : s->ev_done) step(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  if (e != cudaSuccess) {
    rc = cuda_fail(e, "sjs_server_create");
    server_free(s);
    return rc;
  }
  memset(s->desc_h, 0, sizeof(SjbBatchDesc));
  for (int q = 0; q < kBq; ++q) s->slot_query_h[q] = q;
  e = cudaMemcpy(s->slot_query_d, s->slot_query_h, sizeof(int32_t) * kBq, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    rc = cuda_fail(e, "sjs_server_create");
    server_free(s);
    return rc;
  }
  s->cache.init(s->arena, (uint64_t)fcache, s->stats_d, max_entries);
  s->groups.reset((uint64_t)groups, 1);
  s->th = std::thread(loop, s);
  *out = s;
  return SJ_OK;
}

extern "C" sj_status sjs_submit(sjs_server* s, const sjb_query* q, uint64_t* ticket) {
  if (!s || !q || !ticket) return fail_fmt(SJ_ERR_INVALID_ARGUMENT, "NULL argument");
  uint64_t worst = 0;
  sj_status rc = validate_query(s->S, *q, &worst);
  if (rc != SJ_OK) return rc;
  if (worst > (uint64_t)s->cfg.limits.group_entries || worst > s->result_rows) {
    std::lock_guard<std::mutex> g(s->mu);
    ++s->stats.rejected;
    return fail_fmt(SJ_ERR_REJECTED, "query may need %llu group entries (server holds %lld)",
                    (unsigned long long)worst, (long long)s->cfg.limits.group_entries);
  }
  std::lock_guard<std::mutex> g(s->mu);
  if (!s->loop_error.empty()) return fail_fmt(SJ_ERR_CUDA, "server stopped: %s", s->loop_error.c_str());
  const uint64_t id = s->next_ticket++;
  Ticket& t = s->tickets[id];
  t.q = *q;
  for (int k = 0; k < q->n_preds; ++k) {
    if (q->preds[k].kind == SJ_PRED_IN && q->preds[k].in_count > 0) {
      t.codes[k].assign(q->preds[k].in_codes, q->preds[k].in_codes + q->preds[k].in_count);
      t.q.preds[k].in_codes = t.codes[k].data();
    } else {
      t.q.preds[k].in_codes = nullptr;
      t.q.preds[k].in_count = 0;
    }
  }
  t.worst = worst;
  t.submit_s = now_s();
  s->pending.push_back(id);
  ++s->stats.submitted;
  *ticket = id;
  s->cv_work.notify_one();
  return SJ_OK;
}

static sj_status take_result(sjs_server* s, Ticket& t, uint64_t ticket, sjs_ticket_info* info, sjb_row* out,
                             int64_t cap) {
  if (info) {
    info->done = t.done;
    info->status = t.status;
    info->n_rows = (int64_t)t.rows.size();
    info->submit_s = t.submit_s;
    info->admit_s = t.admit_s;
    info->finish_s = t.finish_s;
  }
  if (!t.done || !out) return SJ_OK;
  if ((int64_t)t.rows.size() > cap)
    return fail_fmt(SJ_ERR_CAPACITY, "ticket has %zu rows, buffer holds %lld", t.rows.size(), (long long)cap);
  if (!t.rows.empty()) memcpy(out, t.rows.data(), sizeof(sjb_row) * t.rows.size());
  const int status = t.status;
  s->tickets.erase(ticket);
  return status == SJ_OK ? SJ_OK : fail_fmt((sj_status)status, "query failed: %s", sj_status_string((sj_status)status));
}

extern "C" sj_status sjs_poll(sjs_server* s, uint64_t ticket, sjs_ticket_info* info, sjb_row* out, int64_t cap) {
  if (!s) return fail_fmt(SJ_ERR_INVALID_ARGUMENT, "NULL server");
  std::lock_guard<std::mutex> g(s->mu);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) return fail_fmt(SJ_ERR_INVALID_ARGUMENT, "unknown ticket %llu", (unsigned long long)ticket);
  return take_result(s, it->second, ticket, info, out, cap);
}

extern "C" sj_status sjs_wait(sjs_server* s, uint64_t ticket, double timeout_s, sjs_ticket_info* info, sjb_row* out,
                              int64_t cap) {
  if (!s) return fail_fmt(SJ_ERR_INVALID_ARGUMENT, "NULL server");
  std::unique_lock<std::mutex> g(s->mu);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) return fail_fmt(SJ_ERR_INVALID_ARGUMENT, "unknown ticket %llu", (unsigned long long)ticket);
  Ticket& t = it->second;  // references survive a rehash by concurrent submits; iterators do not
  auto ready = [&] { return t.done; };
  ++s->waiters;
  sj_status rc;
  if (timeout_s > 0 && !s->cv_done.wait_for(g, std::chrono::duration<double>(timeout_s), ready)) {
    take_result(s, t, ticket, info, nullptr, 0);
    rc = fail_fmt(SJ_ERR_TIMEOUT, "ticket %llu not finished after %.3f s", (unsigned long long)ticket, timeout_s);
  } else {
    if (timeout_s <= 0) s->cv_done.wait(g, ready);
    rc = take_result(s, t, ticket, info, out, cap);
  }
  --s->waiters;
  s->cv_done.notify_all();
  return rc;
}

extern "C" sj_status sjs_cancel(sjs_server* s, uint64_t ticket) {
  if (!s) return fail_fmt(SJ_ERR_INVALID_ARGUMENT, "NULL server");
  std::lock_guard<std::mutex> g(s->mu);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) return fail_fmt(SJ_ERR_INVALID_ARGUMENT, "unknown ticket %llu", (unsigned long long)ticket);
  Ticket& t = it->second;
  if (t.done) return SJ_OK;
  auto p = std::find(s->pending.begin(), s->pending.end(), ticket);
  if (p != s->pending.end()) {  // not admitted yet: drop it here
    s->pending.erase(p);
    t.done = true;
    t.status = SJ_ERR_CANCELLED;
    t.finish_s = now_s();
    ++s->stats.finished;
    s->cv_done.notify_all();
    return SJ_OK;
  }
  t.cancel = true;  // running: the loop takes it out of the scan
  return SJ_OK;
}

extern "C" sj_status sjs_get_stats(sjs_server* s, sjs_stats* out) {
  if (!s || !out) return fail_fmt(SJ_ERR_INVALID_ARGUMENT, "NULL argument");
  std::lock_guard<std::mutex> g(s->mu);
  *out = s->stats;
  return SJ_OK;
}

extern "C" void sjs_server_destroy(sjs_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> g(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  if (s->th.joinable()) s->th.join();
  {
    std::unique_lock<std::mutex> g(s->mu);
    for (auto& kv : s->tickets)
      if (!kv.second.done) {
        kv.second.done = true;
        kv.second.status = SJ_ERR_CANCELLED;
        kv.second.finish_s = now_s();
      }
    s->pending.clear();
    s->cv_done.notify_all();
    s->cv_done.wait(g, [&] { return s->waiters == 0; });
  }
  for (int q = 0; q < kBq; ++q)
    if (s->slots[q].used) release_slot(s, q);
  server_free(s);
}
