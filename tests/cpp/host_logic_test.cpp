// Host-side logic of the shared-scan forms, checked without a GPU: the range
// allocator, the filter cache, the circular-scan coverage bookkeeping, and the
// group / step layout functions the batch kernel and the serving loop share.
#include <cassert>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "sj_cache.h"
#include "sj_internal.h"

using namespace sj;

#define CHECK(c)                                                      \
  do {                                                                \
    if (!(c)) {                                                       \
      std::fprintf(stderr, "FAIL %s:%d: %s\n", __FILE__, __LINE__, #c); \
      std::exit(1);                                                   \
    }                                                                 \
  } while (0)

static void test_range_alloc() {
  std::mt19937_64 rng(1);
  for (int trial = 0; trial < 50; ++trial) {
    const uint64_t cap = 1 + rng() % 5000, align = 1u << (rng() % 4);
    RangeAlloc a(cap, align);
    std::vector<char> used(cap, 0);
    std::vector<std::pair<uint64_t, uint64_t>> live;
    for (int op = 0; op < 400; ++op) {
      if (live.empty() || rng() % 3) {
        const uint64_t sz = 1 + rng() % 300;
        const uint64_t off = a.alloc(sz);
        if (off == ~0ull) continue;
        const uint64_t r = a.round(sz);
        CHECK(off % align == 0 && off + r <= a.capacity());
        for (uint64_t i = off; i < off + r; ++i) {
          CHECK(!used[i]);
          used[i] = 1;
        }
        live.push_back({off, sz});
      } else {
        const size_t k = rng() % live.size();
        const auto blk = live[k];
        live.erase(live.begin() + k);
        a.release(blk.first, blk.second);
        for (uint64_t i = blk.first; i < blk.first + a.round(blk.second); ++i) used[i] = 0;
      }
      uint64_t u = 0;
      for (char c : used) u += c;
      CHECK(u == a.used());
    }
    for (auto& blk : live) a.release(blk.first, blk.second);
    CHECK(a.used() == 0 && a.largest_free() == a.capacity());  // frees coalesce back to one block
  }
}

static sjb_pred range_pred(int dim, int lo, int hi) {
  sjb_pred p{};
  p.dim = dim;
  p.kind = SJ_PRED_RANGE;
  p.attr = 1;
  p.lo = lo;
  p.hi = hi;
  p.group_attr = -1;
  return p;
}

static void test_filter_cache() {
  std::vector<uint8_t> arena(256 * 8);
  std::vector<SjbEntryStats> stats(4);
  FilterCache c;
  c.init(arena.data(), arena.size(), stats.data(), 4);
  bool is_new = false;
  const int a = c.acquire(range_pred(0, 1, 5), 64, true, &is_new);  // 256 B
  CHECK(a >= 0 && is_new);
  const int a2 = c.acquire(range_pred(0, 1, 5), 64, true, &is_new);
  CHECK(a2 == a && !is_new);  // same predicate: served from the cache
  sjb_pred in{};
  in.dim = 0;
  in.kind = SJ_PRED_IN;
  in.attr = 0;
  int32_t codes1[] = {5, 3, 3, 9}, codes2[] = {9, 5, 3};
  in.in_codes = codes1;
  in.in_count = 4;
  const int b = c.acquire(in, 64, true, &is_new);
  CHECK(is_new);
  in.in_codes = codes2;
  in.in_count = 3;
  CHECK(c.acquire(in, 64, true, &is_new) == b && !is_new);  // IN lists compare as sets
  const int d = c.acquire(range_pred(1, 1, 5), 64, true, &is_new);
  CHECK(is_new && d != a && d != b);  // another dimension is another filter
  const int e = c.acquire(range_pred(2, 0, 0), 64, true, &is_new);
  CHECK(e >= 0);
  // arena (8 x 256 B) and the 4-entry table are now in use: with every entry
  // referenced, nothing can be evicted
  CHECK(c.acquire(range_pred(3, 0, 0), 64, true, &is_new) == -1);
  c.release(b);
  c.release(b);
  const int f = c.acquire(range_pred(3, 0, 0), 64, true, &is_new);
  CHECK(f >= 0 && is_new);  // the unreferenced IN filter was evicted for it
  in.in_codes = codes1;
  in.in_count = 4;
  c.release(f);
  const int g = c.acquire(in, 64, true, &is_new);
  CHECK(g >= 0 && is_new);  // evicted before, so it is built again
  // entries outside the index (cache off) are freed when unreferenced
  c.release(g);
  c.release(a);
  c.release(a);
  c.release(d);
  c.release(e);
  c.clear_unreferenced();
  CHECK(c.bytes_used() == 0);
  const int h = c.acquire(range_pred(0, 7, 7), 64, false, &is_new);
  CHECK(is_new && c.bytes_used() == 256);
  c.release(h);
  CHECK(c.bytes_used() == 0);
}

// A circular scan with random step sizes and queries attaching between steps:
// every query's rows are covered exactly once, and it finishes within one wrap.
static void test_coverage() {
  std::mt19937_64 rng(2);
  for (int trial = 0; trial < 200; ++trial) {
    const int64_t n = 1 + (int64_t)(rng() % 2000);
    struct Q {
      std::vector<Interval> rem;
      std::vector<int> hits;
      int64_t b, e;
      int64_t scanned;
    };
    std::vector<Q> qs;
    int64_t pos = 0;
    for (int step = 0; step < 400; ++step) {
      if (rng() % 3 == 0 && qs.size() < 20) {
        Q q;
        q.b = (int64_t)(rng() % (uint64_t)(n + 1));
        q.e = q.b + (int64_t)(rng() % (uint64_t)(n - q.b + 1));
        q.rem = attach(q.b, q.e, pos);
        q.hits.assign((size_t)n, 0);
        q.scanned = 0;
        qs.push_back(q);
      }
      int64_t best = -1, best_dist = INT64_MAX;
      for (auto& q : qs) {
        int64_t dist = 0;
        const int64_t c = first_needed(q.rem, pos, n, &dist);
        if (c >= 0 && dist < best_dist) {
          best_dist = dist;
          best = c;
        }
      }
      if (best < 0) continue;
      const int64_t seg_b = best, seg_e = std::min<int64_t>(n, best + 1 + (int64_t)(rng() % 300));
      for (auto& q : qs) {
        const Interval iv = take(q.rem, seg_b, seg_e);
        if (iv.e <= iv.b) continue;
        CHECK(iv.b >= q.b && iv.e <= q.e);
        for (int64_t r = iv.b; r < iv.e; ++r) ++q.hits[(size_t)r];
        q.scanned += iv.e - iv.b;
        cover(q.rem, iv);
        CHECK(q.rem.size() <= 2);
      }
      pos = seg_e >= n ? 0 : seg_e;
    }
    for (auto& q : qs) {
      for (int64_t r = 0; r < n; ++r) CHECK(q.hits[(size_t)r] <= 1);
      if (q.rem.empty())
        for (int64_t r = q.b; r < q.e; ++r) CHECK(q.hits[(size_t)r] == 1);
    }
  }
}

static void test_layouts() {
  SjbSchemaRt S{};
  S.n_dims = 3;
  for (int d = 0; d < 3; ++d) S.dim[d].rows = 1000;
  std::mt19937_64 rng(3);
  for (int trial = 0; trial < 100; ++trial) {
    SjbStep st{};
    std::vector<SjbEntryStats> es(kBq * 3);
    for (int q = 0; q < kBq; ++q) {
      SjbBatchQuery bq{};
      bq.n_preds = 1 + rng() % 3;
      const SjbEntryStats* stp[SJ_MAX_DIMS];
      for (uint32_t k = 0; k < bq.n_preds; ++k) {
        bq.dim[k] = k;
        bq.group_attr[k] = (rng() % 2) ? 0 : -1;
        SjbEntryStats& e = es[q * 3 + k];
        e.count = (rng() % 8) ? 1 + rng() % 1000 : 0;
        const int32_t lo = (int32_t)(rng() % 50) - 10, hi = lo + (int32_t)(rng() % 30);
        e.umax[0] = (uint32_t)hi ^ 0x80000000u;
        e.nmin[0] = ~((uint32_t)lo ^ 0x80000000u);
        stp[k] = &e;
        st.bm[q][k] = reinterpret_cast<const uint32_t*>(&e);  // any non-null marks the dimension as used
      }
      SjbSlot& sl = st.slot[q];
      const uint32_t err = sjb_group_layout(S, bq, stp, sl, st.sel[q], 1ull << 32);
      CHECK(err == 0);
      bool empty = false;
      uint64_t span = 1;
      for (uint32_t k = 0; k < bq.n_preds; ++k) {
        empty |= es[q * 3 + k].count == 0;
        if (bq.group_attr[k] >= 0 && es[q * 3 + k].count)
          span *= (uint64_t)(stats_max(es[q * 3 + k], 0) - stats_min(es[q * 3 + k], 0) + 1);
      }
      CHECK(sl.span == (empty ? 0u : span));
      if (sl.span) {  // mixed radix: the last grouped predicate varies fastest
        uint64_t stride = 1;
        for (int g = (int)sl.n_g - 1; g >= 0; --g) {
          CHECK(sl.stride[g] == stride);
          stride *= sl.width[g];
        }
      }
      if (sl.span && rng() % 4) st.active |= 1ull << q;
    }
    const uint32_t cap = 1 + rng() % 4000;
    sjb_step_layout(st, 3, cap);
    CHECK(st.smem_entries <= cap);
    // shared partials: disjoint, smallest spans first
    uint32_t max_assigned = 0, min_unassigned = ~0u;
    std::vector<char> seen(cap + 1, 0);
    for (int q = 0; q < kBq; ++q) {
      const SjbSlot& sl = st.slot[q];
      if (!((st.active >> q) & 1ull) || sl.span == 0 || sl.span > 2048) continue;
      if (sl.smem_off >= 0) {
        CHECK((uint32_t)sl.smem_off + sl.span <= st.smem_entries);
        for (uint32_t i = 0; i < sl.span; ++i) {
          CHECK(!seen[sl.smem_off + i]);
          seen[sl.smem_off + i] = 1;
        }
        max_assigned = std::max(max_assigned, sl.span);
      } else {
        min_unassigned = std::min(min_unassigned, sl.span);
      }
    }
    CHECK(max_assigned <= min_unassigned);
    // order is a permutation of the dimensions, use masks only hold active slots
    int seen_dim = 0;
    for (uint32_t k = 0; k < 3; ++k) seen_dim |= 1 << st.order[k];
    CHECK(seen_dim == 7);
    for (int d = 0; d < 3; ++d) CHECK((st.use[d] & ~st.active) == 0);
  }
}

static void test_perms() {
  for (uint32_t n = 1; n <= 4; ++n) {
    uint32_t n_perm = 1;
    for (uint32_t i = 2; i <= n; ++i) n_perm *= i;
    std::vector<uint32_t> codes;
    for (uint32_t i = 0; i < n_perm; ++i) {
      uint32_t perm[SJ_MAX_DIMS];
      sjb_perm_of(i, n, perm);
      uint32_t seen = 0, code = 0;
      for (uint32_t k = 0; k < n; ++k) {
        CHECK(perm[k] < n && !((seen >> perm[k]) & 1u));
        seen |= 1u << perm[k];
        code = code * 4 + perm[k];
      }
      for (uint32_t c : codes) CHECK(c != code);
      codes.push_back(code);
    }
  }
}

// Filter layout of one dimension once its qualifying rows are counted (the
// per-dimension choice of bf_bits_per_key = SJ_BF_AUTO).
static void test_bf_effective() {
  uint32_t l2 = 99;
  // explicit modes are kept
  CHECK(bf_effective(kBfDirect, 20, 0, 100, 40960, &l2) == kBfDirect && l2 == 20);
  CHECK(bf_effective(kBfBlocked, 20, 8, 1000, 40960, &l2) == kBfBlocked && l2 == bf_blocked_log2(1000, 8, 20));
  // auto: a direct bitmap that fits the budget stays direct (2^16 bits = 8 KB)
  CHECK(bf_effective(kBfAuto, 16, 16, 40000, 40960, &l2) == kBfDirect && l2 == 16);
  // auto: 2^20 bits = 128 KB over the budget, 1,000 keys x 16 bits -> 256 words of 64 bits
  CHECK(bf_effective(kBfAuto, 20, 16, 1000, 40960, &l2) == kBfBlocked && l2 == 8);
  // auto: blocked would not be smaller than the direct bitmap -> direct
  CHECK(bf_effective(kBfAuto, 20, 16, 65536, 40960, &l2) == kBfDirect && l2 == 20);
  // auto: no qualifying key -> one 64-bit word (rejects every row)
  CHECK(bf_effective(kBfAuto, 20, 16, 0, 40960, &l2) == kBfBlocked && l2 == 0);
  // the blocked filter always fits the direct bitmap's allocation
  for (uint32_t lg = 7; lg <= 28; ++lg)
    for (uint32_t ins : {0u, 1u, 100u, 5000u, 1u << 20, 1u << 26})
      if (bf_effective(kBfAuto, lg, 16, ins, 0, &l2) == kBfBlocked) CHECK((8ull << l2) < (1ull << lg) / 8);
}

// A filter created by acquire() but never built leaves the index when it is
// discarded: the next acquire of the same predicate builds it anew.
static void test_filter_cache_discard() {
  std::vector<uint8_t> arena(256 * 4);
  std::vector<SjbEntryStats> stats(4);
  FilterCache c;
  c.init(arena.data(), arena.size(), stats.data(), 4);
  bool is_new = false;
  const int a = c.acquire(range_pred(0, 1, 5), 64, true, &is_new);
  CHECK(a >= 0 && is_new);
  c.discard_new(a);
  const int b = c.acquire(range_pred(0, 1, 5), 64, true, &is_new);
  CHECK(b >= 0 && is_new);  // not served from the cache
  c.at(b).built = true;
  c.release(b);
  const int b2 = c.acquire(range_pred(0, 1, 5), 64, true, &is_new);
  CHECK(b2 == b && !is_new);  // a built, released filter is cached
  // the discarded entry's arena range and id were freed: three more fit
  c.release(b2);
  for (int k = 1; k <= 3; ++k) CHECK(c.acquire(range_pred(k, 0, 0), 64, true, &is_new) >= 0 && is_new);
}

int main() {
  test_bf_effective();
  test_filter_cache_discard();
  test_perms();
  test_range_alloc();
  test_filter_cache();
  test_coverage();
  test_layouts();
  std::printf("OK\n");
  return 0;
}
