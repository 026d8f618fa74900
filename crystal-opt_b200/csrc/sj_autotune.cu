// sj_autotune.cu -- the plain engine's autotuner (sj_autotune in include/starjoin.h).
//
// Candidates are timed on the plan's own device columns with CUDA events around
// sj_query_probe (the build is re-run before every timed probe, as a query
// would).  Search order, each step keeping the best so far:
//   1. filter kind   direct bitmap, per-dimension auto layout, 8 or 16 bits per
//                    key -- with every join order when the order is searched too
//   2. geometry      threads x rows per lane, then rows per stage x stages
//   3. join order    (when not searched in 1) most selective first, or every
//                    permutation; then bits set per key 1..4 and 4 / 8 / 16
//                    bits per key for the chosen order and geometry
// The groups of every candidate are compared with the first candidate's.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "sj_cache.h"
#include "sj_internal.h"

using namespace sj;

namespace {

std::mutex g_cache_mu;

bool rows_equal(const std::vector<sj_group_row>& a, const std::vector<sj_group_row>& b) {
  if (a.size() != b.size()) return false;
  for (size_t i = 0; i < a.size(); ++i)
    if (memcmp(&a[i], &b[i], sizeof(sj_group_row)) != 0) return false;
  return true;
}

struct Timed {
  sj_status st = SJ_OK;
  float ms = 0.f;
  std::vector<sj_group_row> rows;
  sj_query_stats stats{};
};

Timed time_plan(sj_engine* eng, const sj_plan& plan, int reps, cudaStream_t stream, bool want_rows) {
  Timed t;
  sj_query* q = nullptr;
  t.st = sj_query_prepare(eng, &plan, &q);
  if (t.st != SJ_OK) return t;
  cudaEvent_t a = nullptr, b = nullptr;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  std::vector<float> ms;
  for (int i = 0; i < 2 + reps && t.st == SJ_OK; ++i) {
    t.st = sj_query_build(q, stream);
    if (t.st != SJ_OK) break;
    cudaEventRecord(a, stream);
    t.st = sj_query_probe(q, stream);
    cudaEventRecord(b, stream);
    if (t.st != SJ_OK) break;
    if (i >= 2) {
      cudaEventSynchronize(b);
      float v = 0.f;
      if (cudaEventElapsedTime(&v, a, b) == cudaSuccess) ms.push_back(v);
    }
  }
  if (t.st == SJ_OK) {
    int64_t n = 0;
    std::vector<sj_group_row> rows(1 << 12);
    sj_status f = sj_query_fetch(q, rows.data(), (int64_t)rows.size(), &n, stream);
    if (f == SJ_ERR_CAPACITY) {
      rows.resize((size_t)n);
      f = sj_query_fetch(q, rows.data(), (int64_t)rows.size(), &n, stream);
    }
    if (f != SJ_OK) {
      t.st = f;
    } else if (want_rows) {
      rows.resize((size_t)n);
      t.rows.swap(rows);
    }
    sj_query_get_stats(q, &t.stats);
  }
  std::sort(ms.begin(), ms.end());
  t.ms = ms.empty() ? 0.f : ms[ms.size() / 2];
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  sj_query_release(q);
  return t;
}

std::string signature(const sj_plan& p, const double* sel, const sj_autotune_opts& o) {
  std::ostringstream s;
  s << "v1|n" << p.n_dims << "|r" << (int)std::lround(std::log2((double)std::max<int64_t>(1, p.row_end - p.row_begin)))
    << "|lip" << p.lip << "|ad" << p.adaptive << "|sub" << (p.measure_sub ? 1 : 0);
  if (!o.tune_filter) s << "|bf" << p.bf_bits_per_key << "x" << p.bf_hashes;
  if (!o.tune_order) {
    s << "|o";
    for (int i = 0; i < p.n_dims; ++i) s << p.order[i];
  }
  for (int d = 0; d < p.n_dims; ++d) {
    const sj_dim& D = p.dims[d];
    const int sb = sel[d] > 0 ? std::max(-24, (int)std::lround(std::log2(sel[d]))) : -99;
    s << "|d" << D.ht_len << "," << D.rows << "," << D.group << "," << (D.group ? D.payload_max - D.payload_min + 1 : 0)
      << ",s" << sb;
  }
  return s.str();
}

bool cache_get(const char* path, const std::string& sig, sj_plan& p) {
  if (!path) return false;
  std::lock_guard<std::mutex> g(g_cache_mu);
  std::ifstream f(path);
  std::string line;
  bool found = false;
  sj_plan best = p;
  while (std::getline(f, line)) {  // the last entry for a signature wins
    const size_t tab = line.find('\t');
    if (tab == std::string::npos || line.compare(0, tab, sig) != 0 || tab != sig.size()) continue;
    std::istringstream v(line.substr(tab + 1));
    sj_plan c = p;
    sj_tuning& t = c.tune;
    if (!(v >> t.threads >> t.chunk_rows >> t.stages >> t.ctas_per_sm >> t.compact_threshold >> t.bf_smem_bytes >>
          c.bf_bits_per_key >> c.bf_hashes))
      continue;
    bool ok = true;
    for (int i = 0; i < SJ_MAX_DIMS; ++i) ok = ok && (bool)(v >> c.order[i]);
    if (!ok) continue;
    best = c;
    found = true;
  }
  if (found) p = best;
  return found;
}

void cache_put(const char* path, const std::string& sig, const sj_plan& p) {
  if (!path) return;
  std::lock_guard<std::mutex> g(g_cache_mu);
  std::ofstream f(path, std::ios::app);
  const sj_tuning& t = p.tune;
  f << sig << '\t' << t.threads << ' ' << t.chunk_rows << ' ' << t.stages << ' ' << t.ctas_per_sm << ' '
    << t.compact_threshold << ' ' << t.bf_smem_bytes << ' ' << p.bf_bits_per_key << ' ' << p.bf_hashes;
  for (int i = 0; i < SJ_MAX_DIMS; ++i) f << ' ' << p.order[i];
  f << '\n';
}

}  // namespace

extern "C" sj_status sj_autotune(sj_engine* eng, sj_plan* plan, const sj_autotune_opts* opts,
                                 sj_autotune_report* report, void* stream) {
  SjNvtxRange nvtx_range("sj.autotune");
  if (!eng || !plan) return fail_fmt(SJ_ERR_INVALID_ARGUMENT, "engine or plan is NULL");
  sj_autotune_opts o{};
  if (opts) o = *opts;
  const int reps = o.reps > 0 ? o.reps : 5;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  sj_autotune_report rep{};
  sj_plan cur = *plan;

  // the plan as given: reference time, reference groups, selectivities
  Timed base = time_plan(eng, cur, reps, st, true);
  if (base.st != SJ_OK) return base.st;
  rep.candidates = 1;
  rep.default_ms = base.ms;
  for (int d = 0; d < cur.n_dims; ++d)
    rep.selectivity[d] = cur.dims[d].rows > 0 ? (double)base.stats.bf_inserted[d] / (double)cur.dims[d].rows : 0.0;
  if (o.tune_order == 1) {  // most selective dimension first
    int ord[SJ_MAX_DIMS];
    for (int i = 0; i < cur.n_dims; ++i) ord[i] = i;
    std::stable_sort(ord, ord + cur.n_dims, [&](int x, int y) { return rep.selectivity[x] < rep.selectivity[y]; });
    for (int i = 0; i < cur.n_dims; ++i) cur.order[i] = ord[i];
  }
  const std::string sig = signature(cur, rep.selectivity, o);
  if (cache_get(o.cache_path, sig, cur)) {
    Timed t = time_plan(eng, cur, reps, st, o.verify != 0);
    if (t.st == SJ_OK) {
      if (o.verify && !rows_equal(t.rows, base.rows)) ++rep.mismatches;
      rep.cache_hit = 1;
      rep.best_ms = t.ms;
      rep.candidates = 2;
      *plan = cur;
      if (report) *report = rep;
      return rep.mismatches ? fail_fmt(SJ_ERR_CUDA, "cached plan changed the groups") : SJ_OK;
    }
    cur = *plan;  // unusable cache entry: search
  }

  sj_plan best = cur;
  float best_ms = 0.f;
  {
    Timed t = time_plan(eng, cur, reps, st, o.verify != 0);
    if (t.st != SJ_OK) return t.st;
    ++rep.candidates;
    if (o.verify && !rows_equal(t.rows, base.rows)) ++rep.mismatches;
    best_ms = t.ms;
  }
  auto consider = [&](const sj_plan& c) {
    Timed t = time_plan(eng, c, reps, st, o.verify != 0);
    if (t.st != SJ_OK) return;  // geometry the engine does not build, or too large
    ++rep.candidates;
    if (o.verify && !rows_equal(t.rows, base.rows)) {
      ++rep.mismatches;
      return;
    }
    if (t.ms < best_ms) {
      best_ms = t.ms;
      best = c;
    }
  };
  // 1. filter kind, jointly with the join order when both are searched: a
  //    large, selective dimension pays off first in the order only with a
  //    filter that fits shared memory, so neither choice is right alone
  auto for_orders = [&](const sj_plan& base, bool all_orders) {
    if (!all_orders || cur.n_dims < 2) {
      consider(base);
      return;
    }
    int perm[SJ_MAX_DIMS];
    for (int i = 0; i < cur.n_dims; ++i) perm[i] = i;
    do {
      sj_plan c = base;
      for (int i = 0; i < cur.n_dims; ++i) c.order[i] = perm[i];
      consider(c);
    } while (std::next_permutation(perm, perm + cur.n_dims));
  };
  const bool joint = o.tune_filter && o.tune_order == 2;
  if (o.tune_filter) {
    const sj_plan start = best;
    const int kinds[][2] = {{0, 2}, {SJ_BF_AUTO, 2}, {SJ_BF_AUTO, 3}, {8, 2}, {16, 2}};
    for (auto& kd : kinds) {
      sj_plan c = start;
      c.bf_bits_per_key = kd[0];
      c.bf_hashes = kd[1];
      for_orders(c, joint);
    }
  }
  // 2. geometry: CTA size x rows per lane, then rows per stage x stages
  {
    const sj_plan start = best;
    const int shapes[][2] = {{256, 0}, {256, 16}, {512, 0}, {512, 16}, {768, 0}};
    for (auto& sh : shapes) {
      sj_plan c = start;
      c.tune.threads = sh[0];
      c.tune.compact_threshold = sh[1];
      c.tune.chunk_rows = 0;
      c.tune.stages = 0;
      if (c.tune.threads == start.tune.threads && c.tune.compact_threshold == start.tune.compact_threshold &&
          start.tune.chunk_rows == 0 && start.tune.stages == 0)
        continue;
      consider(c);
    }
    const sj_plan mid = best;
    const int threads = mid.tune.threads ? mid.tune.threads : 512;
    const int rpl = (mid.tune.compact_threshold == 16 && threads <= 512) ? 16 : 8;
    const int pass = (threads / 32 - 1) * 32 * rpl;
    const int passes[] = {2, 4, 8};
    const int stages[] = {2, 3, 4};
    for (int np : passes)
      for (int sg : stages) {
        sj_plan c = mid;
        c.tune.chunk_rows = np * pass;
        c.tune.stages = sg;
        if ((int64_t)c.tune.chunk_rows * 4 > (1 << 19)) continue;
        consider(c);
      }
  }
  // 3. join order (when not searched with the filter), then bits set per key
  //    and the other filter sizes for the chosen order and geometry
  if (o.tune_order == 2 && !joint && cur.n_dims > 1) for_orders(best, true);
  if (o.tune_filter) {
    const sj_plan start = best;
    const int bpks[] = {SJ_BF_AUTO, 4, 8, 16};
    for (int bpk : bpks)
      for (int k = 1; k <= (bpk > 0 ? 4 : 3); ++k) {
        if (bpk < 0 && k == 1) continue;
        if (bpk == start.bf_bits_per_key && k == start.bf_hashes) continue;
        sj_plan c = start;
        c.bf_bits_per_key = bpk;
        c.bf_hashes = k;
        consider(c);
      }
  }
  rep.best_ms = best_ms;
  *plan = best;
  cache_put(o.cache_path, sig, best);
  if (report) *report = rep;
  if (rep.mismatches) return fail_fmt(SJ_ERR_CUDA, "%d candidate plans changed the groups", rep.mismatches);
  return SJ_OK;
}
