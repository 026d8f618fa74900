// sj_cache.h -- host-side bookkeeping of the shared-scan forms: a first-fit
// range allocator over a device arena, and the filter cache keyed by
// (dimension, predicate).
#pragma once

#include <stdint.h>

#include <algorithm>
#include <climits>
#include <map>
#include <string>
#include <unordered_map>
#include <vector>

#include "sj_shared.h"

namespace sj {

// First-fit allocator of [0, capacity) in `align`-sized units; frees coalesce.
class RangeAlloc {
 public:
  explicit RangeAlloc(uint64_t capacity = 0, uint64_t align = 1) { reset(capacity, align); }
  void reset(uint64_t capacity, uint64_t align) {
    align_ = align ? align : 1;
    cap_ = capacity / align_ * align_;
    free_.clear();
    if (cap_) free_[0] = cap_;
    used_ = 0;
  }
  // Offset of a block of `size` (rounded up to the alignment), or ~0 if none fits.
  uint64_t alloc(uint64_t size) {
    size = round(size);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < size) continue;
      const uint64_t off = it->first, rest = it->second - size;
      free_.erase(it);
      if (rest) free_[off + size] = rest;
      used_ += size;
      return off;
    }
    return ~0ull;
  }
  void release(uint64_t off, uint64_t size) {
    size = round(size);
    used_ -= size;
    auto nx = free_.lower_bound(off);
    if (nx != free_.end() && off + size == nx->first) {
      size += nx->second;
      nx = free_.erase(nx);
    }
    if (nx != free_.begin()) {
      auto pv = std::prev(nx);
      if (pv->first + pv->second == off) {
        pv->second += size;
        return;
      }
    }
    free_[off] = size;
  }
  uint64_t largest_free() const {
    uint64_t m = 0;
    for (auto& kv : free_) m = std::max(m, kv.second);
    return m;
  }
  uint64_t used() const { return used_; }
  uint64_t capacity() const { return cap_; }
  uint64_t round(uint64_t s) const { return (s + align_ - 1) / align_ * align_; }

 private:
  uint64_t align_ = 1, cap_ = 0, used_ = 0;
  std::map<uint64_t, uint64_t> free_;
};

// Coverage bookkeeping of a query on the circular scan: the fact rows it still
// needs, as at most two disjoint intervals (the part of [b, e) after its attach
// point, then the part before it, reached after the scan wraps).
struct Interval {
  int64_t b, e;
};

// Rows [b, e) intersected with the rows still to scan, one piece (a scan step
// never wraps, so at most one piece is non-empty).
inline Interval take(const std::vector<Interval>& remaining, int64_t b, int64_t e) {
  for (const Interval& iv : remaining) {
    const int64_t lo = std::max(iv.b, b), hi = std::min(iv.e, e);
    if (lo < hi) return {lo, hi};
  }
  return {0, 0};
}

// Remove the scanned rows c from the remaining intervals.
inline void cover(std::vector<Interval>& remaining, Interval c) {
  std::vector<Interval> out;
  for (const Interval& iv : remaining) {
    if (c.e <= iv.b || c.b >= iv.e) {
      out.push_back(iv);
      continue;
    }
    if (iv.b < c.b) out.push_back({iv.b, c.b});
    if (c.e < iv.e) out.push_back({c.e, iv.e});
  }
  remaining.swap(out);
}

// The intervals a query attaching at scan position p needs for [b, e): rows
// [p, e) first, then [b, p) after the wrap.
inline std::vector<Interval> attach(int64_t b, int64_t e, int64_t p) {
  if (e <= b) return {};
  if (p > b && p < e) return {{p, e}, {b, p}};
  return {{b, e}};
}

// First row at or after `pos` (cyclically over [0, n)) in the intervals, and
// its cyclic distance from pos; -1 when nothing is left.
inline int64_t first_needed(const std::vector<Interval>& remaining, int64_t pos, int64_t n, int64_t* dist) {
  int64_t best = -1, best_dist = INT64_MAX;
  for (const Interval& iv : remaining) {
    int64_t cand, d;
    if (pos >= iv.b && pos < iv.e) {
      cand = pos;
      d = 0;
    } else if (iv.b >= pos) {
      cand = iv.b;
      d = iv.b - pos;
    } else {
      cand = iv.b;
      d = iv.b + n - pos;
    }
    if (d < best_dist) {
      best_dist = d;
      best = cand;
    }
  }
  *dist = best_dist;
  return best;
}

// Filter bitmaps (one bit per PHT slot) and their statistics, resident on the
// device and shared by every query with the same dimension predicate.
struct FilterEntry {
  std::string key;
  uint32_t dim = 0;
  int32_t kind = 0, attr = -1, lo = 0, hi = 0;
  std::vector<int32_t> codes;
  uint64_t off = 0, bytes = 0;   // bitmap in the arena
  uint32_t stats_idx = 0;        // record in the stats array
  int refs = 0;
  uint64_t last_use = 0;
  bool built = false;
  bool live = false;
  SjbEntryStats host{};          // copy read back after the build (serving)
  bool host_valid = false;
  uint32_t stats_have = 0;       // attributes whose min/max the statistics hold
};

class FilterCache {
 public:
  void init(uint8_t* arena, uint64_t arena_bytes, SjbEntryStats* stats, uint32_t max_entries) {
    arena_ = arena;
    stats_ = stats;
    alloc_.reset(arena_bytes, 256);
    entries_.assign(max_entries, FilterEntry());
    free_ids_.clear();
    for (uint32_t i = max_entries; i-- > 0;) free_ids_.push_back(i);
    index_.clear();
  }

  static std::string make_key(const sjb_pred& p, std::vector<int32_t>* codes_out) {
    std::string k = std::to_string(p.dim) + "|" + std::to_string(p.kind);
    if (p.kind == SJ_PRED_RANGE) {
      k += "|" + std::to_string(p.attr) + "|" + std::to_string(p.lo) + "|" + std::to_string(p.hi);
    } else if (p.kind == SJ_PRED_IN) {
      std::vector<int32_t> c(p.in_codes, p.in_codes + p.in_count);
      std::sort(c.begin(), c.end());
      c.erase(std::unique(c.begin(), c.end()), c.end());
      k += "|" + std::to_string(p.attr);
      for (int32_t v : c) k += "," + std::to_string(v);
      if (codes_out) *codes_out = c;
    }
    return k;
  }

  // Entry id for the predicate (refcount taken), building a new entry when
  // needed; -1 when neither the arena nor the entry table has room even after
  // evicting every unreferenced entry.  *is_new tells the caller to build it.
  int acquire(const sjb_pred& p, uint32_t words, bool keep, bool* is_new) {
    std::vector<int32_t> codes;
    const std::string key = make_key(p, &codes);
    *is_new = false;
    auto it = index_.find(key);
    if (it != index_.end()) {
      FilterEntry& e = entries_[it->second];
      ++e.refs;
      e.last_use = ++clock_;
      ++hits_;
      return it->second;
    }
    const uint64_t bytes = (uint64_t)words * 4u;
    uint64_t off = alloc_.alloc(bytes);
    while ((off == ~0ull || free_ids_.empty()) && evict_one()) {
      if (off == ~0ull) off = alloc_.alloc(bytes);
    }
    if (off == ~0ull || free_ids_.empty()) {
      if (off != ~0ull) alloc_.release(off, bytes);
      return -1;
    }
    const uint32_t id = free_ids_.back();
    free_ids_.pop_back();
    FilterEntry& e = entries_[id];
    e = FilterEntry();
    e.key = key;
    e.dim = (uint32_t)p.dim;
    e.kind = p.kind;
    e.attr = p.attr;
    e.lo = p.lo;
    e.hi = p.hi;
    e.codes = codes;
    e.off = off;
    e.bytes = bytes;
    e.stats_idx = id;
    e.refs = 1;
    e.last_use = ++clock_;
    e.live = true;
    e.built = false;
    if (keep) index_[key] = (int)id;
    *is_new = true;
    ++misses_;
    return (int)id;
  }

  // Drop one reference; entries outside the index (cache disabled) are freed
  // when unreferenced.
  void release(int id) {
    FilterEntry& e = entries_[id];
    if (--e.refs > 0) return;
    auto it = index_.find(e.key);
    if (it == index_.end() || it->second != id) drop(id);
  }

  // Drop one reference to an entry acquire() just created and that will not be
  // built (its job did not fit, or the call failed first): it leaves the index,
  // so no later acquire finds an unbuilt filter.
  void discard_new(int id) {
    FilterEntry& e = entries_[id];
    if (--e.refs > 0) return;
    auto it = index_.find(e.key);
    if (it != index_.end() && it->second == id) index_.erase(it);
    drop(id);
  }

  void clear_unreferenced() {
    while (evict_one()) {
    }
  }

  FilterEntry& at(int id) { return entries_[id]; }
  uint32_t* bitmap(int id) { return reinterpret_cast<uint32_t*>(arena_ + entries_[id].off); }
  SjbEntryStats* stats(int id) { return stats_ + entries_[id].stats_idx; }
  uint64_t bytes_used() const { return alloc_.used(); }
  uint64_t bytes_capacity() const { return alloc_.capacity(); }
  uint64_t hits() const { return hits_; }
  uint64_t misses() const { return misses_; }

 private:
  bool evict_one() {
    int victim = -1;
    for (auto& kv : index_) {
      const FilterEntry& e = entries_[kv.second];
      if (e.refs == 0 && (victim < 0 || e.last_use < entries_[victim].last_use)) victim = kv.second;
    }
    if (victim < 0) return false;
    index_.erase(entries_[victim].key);
    drop(victim);
    return true;
  }
  void drop(int id) {
    FilterEntry& e = entries_[id];
    if (!e.live) return;
    alloc_.release(e.off, e.bytes);
    e.live = false;
    free_ids_.push_back((uint32_t)id);
  }

  uint8_t* arena_ = nullptr;
  SjbEntryStats* stats_ = nullptr;
  RangeAlloc alloc_;
  std::vector<FilterEntry> entries_;
  std::vector<uint32_t> free_ids_;
  std::unordered_map<std::string, int> index_;
  uint64_t clock_ = 0, hits_ = 0, misses_ = 0;
};

}  // namespace sj

struct sj_engine;

namespace sj {

// A registered schema: device-side per-slot tables shared by every query, plus
// host copies of each attribute's range over the dimension rows (for the
// worst-case group spans that admission and capacity checks use).
struct SchemaState {
  sjb_schema schema{};
  SjbSchemaRt rt{};
  uint64_t* masks = nullptr;      // all dimensions' 64-bit slot words
  size_t masks_bytes = 0;
  int32_t* slot_attr = nullptr;   // all dimensions' slot-attribute tables
  int64_t attr_min[SJ_MAX_DIMS][SJB_MAX_ATTRS]{};
  int64_t attr_max[SJ_MAX_DIMS][SJB_MAX_ATTRS]{};
  uint32_t words[SJ_MAX_DIMS]{};  // filter bitmap words per dimension
};

sj_status schema_register(sj_engine* eng, const sjb_schema* sc, SchemaState& st);
void schema_release(SchemaState& st);
// Validates one query against the schema; *worst = product of the full ranges
// of its grouped attributes (accumulator entries it may need).
sj_status validate_query(const SchemaState& S, const sjb_query& q, uint64_t* worst);
sj_status cuda_fail(cudaError_t e, const char* what);
sj_status fail_fmt(sj_status s, const char* fmt, ...);

}  // namespace sj
