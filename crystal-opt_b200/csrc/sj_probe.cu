// sj_probe.cu -- the fused star-join probe: fact scan -> LIP Bloom filters -> PHT
// probes -> group-by SUM, one persistent warp-specialized kernel per query.
//
// Replaces the reference's probe<128,4> kernels (src/ssb-jo/q33/0-lip.cu:28-112,
// src/ssb-jo/q33/0-naive.cu:28-91, src/ssb-jo/q41/0-lip.cu:28-131).  Same answer,
// different machine mapping:
//   * Persistent grid of one CTA per SM: one producer warp and NWC consumer warps.
//     Only the column tested first is read densely.  The producer streams each
//     chunk of it with one CTA-local TMA bulk copy (cp.async.bulk, no multicast)
//     into a ring of shared-memory stages; "full" mbarriers signal the consumers,
//     "empty" mbarriers (one arrival per consumer warp) give the stage back.
//     There is no block-wide barrier in the steady state.
//   * Each consumer warp tests its slice of the stage against the first filter
//     (held in shared memory) and compacts the survivors (warp ballot + popc) into
//     its own ring queue Q1 of row offsets.  Later columns are read only at
//     survivor rows (sector-sparse reads, prefetched into L2 at enqueue time).
//     Survivors of the second test are compacted again into the warp's Q2; the
//     remaining tests, the PHT probes and the aggregate run densely on Q2.  Queue
//     heads/tails are warp-uniform registers.  Values of earlier steps are not
//     carried in the queues: the rare survivors recompute them from L2.
//   * Filters are evaluated on the PHT slot of each key, so a filter never rejects
//     a row the PHT would accept; filters that fit the budget live in shared memory.
//   * Group partials (dense dictionary codes) live in shared memory and are
//     flushed once per CTA with 64-bit atomics; group spaces that do not fit
//     aggregate straight into global memory.
//   * Adaptive LIP: consumer warps count probes/passes per filter; every few chunks
//     the producer re-ranks the filter order for the chunks it issues next.  A warp
//     drains its queues before the first chunk of a new order, so the result never
//     depends on the order, only the work does.
#include "sj_internal.h"
#include "sj_ptx.cuh"

namespace sj {

enum : uint32_t { kStepBF = 0, kStepPHT = 1 };
enum : int { kModeDirectSmem = 0, kModeBlockedSmem = 1, kModeBfAny = 2, kModePht = 3 };

struct SmemLayout {
  uint32_t stage_off, full_off, empty_off, bf_off, q1_off, q2_off, gsum_off, gcnt_off, ctl_off, total;
};

struct Ctl {
  uint32_t abort;
  uint32_t n_steps[2];
  uint32_t steps[2][kMaxSteps];  // (dim | kind << 4)
  uint32_t order[2][kMaxDims];
  uint32_t stage_ver[16];
  uint32_t bf_in_smem[kMaxDims];  // byte offset within the filter region, or ~0u
  uint32_t bf_log2[kMaxDims];
  uint32_t bf_mode[kMaxDims];     // layout each dimension's filter was built in
  uint32_t group_stride[kMaxDims];
  uint32_t n_groups;
  uint32_t groups_in_smem;
  uint32_t probes[kMaxDims], passes[kMaxDims];
  uint32_t step_in[kMaxSteps], step_out[kMaxSteps];
  uint32_t rows_scanned;
  uint32_t reorders;
};

__host__ __device__ inline uint32_t align_up(uint32_t x, uint32_t a) { return (x + a - 1) / a * a; }

__host__ __device__ inline SmemLayout probe_layout(const SjProbeGeom& g) {
  const uint32_t nwc = g.threads / 32 - 1;
  SmemLayout L;
  uint32_t o = 0;
  L.stage_off = o;
  o += g.stages * g.chunk_rows * 4u;
  o = align_up(o, 16);
  L.full_off = o;
  o += g.stages * 8u;
  L.empty_off = o;
  o += g.stages * 8u;
  o = align_up(o, 16);
  L.bf_off = o;
  o += g.bf_smem_bytes;
  o = align_up(o, 16);
  L.q1_off = o;
  o += nwc * g.q1_cap * 4u;
  L.q2_off = o;
  o += nwc * g.q2_cap * 4u;
  o = align_up(o, 16);
  L.gsum_off = o;
  o += g.group_smem_cap * 8u;
  L.gcnt_off = o;
  o += g.group_smem_cap * 4u;
  o = align_up(o, 16);
  L.ctl_off = o;
  o += (uint32_t)sizeof(Ctl);
  L.total = align_up(o, 128);
  return L;
}

__device__ __forceinline__ uint32_t lds_u32(uint32_t saddr) {
  uint32_t v;
  asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"(saddr));
  return v;
}
__device__ __forceinline__ uint64_t lds_u64(uint32_t saddr) {
  uint64_t v;
  asm volatile("ld.shared.u64 %0, [%1];" : "=l"(v) : "r"(saddr));
  return v;
}
__device__ __forceinline__ uint2 lds_u32x2(uint32_t saddr) {
  uint2 v;
  asm volatile("ld.shared.v2.u32 {%0, %1}, [%2];" : "=r"(v.x), "=r"(v.y) : "r"(saddr));
  return v;
}
__device__ __forceinline__ int4 lds_v4(uint32_t saddr) {
  int4 v;
  asm volatile("ld.shared.v4.s32 {%0, %1, %2, %3}, [%4];" : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "r"(saddr));
  return v;
}
__device__ __forceinline__ uint32_t ld_volatile_u32(const uint32_t* p) {
  return *reinterpret_cast<const volatile uint32_t*>(p);
}

// Slot of a fact key with the common in-range case first; the remainder path
// (keys outside [key_min, key_min + len)) is a rarely taken branch.
__device__ __forceinline__ uint32_t slot_fast(int32_t k, int32_t kmin, uint32_t len, uint64_t m) {
  const uint32_t d = (uint32_t)k - (uint32_t)kmin;
  if (__builtin_expect(d < len, 1)) return d;
  return (uint32_t)__umul64hi(m * (uint64_t)d, (uint64_t)len);
}

// Per-dimension filter view held in registers.
struct BfView {
  uint32_t smem;     // shared address of the filter, or 0 if it stays in global memory
  const void* gptr;  // global filter
  uint32_t mode, k, log2;
};

__device__ __forceinline__ bool bf_test(const BfView& f, uint32_t slot, uint64_t pol_keep) {
  if (f.mode == kBfDirect) {
    const uint32_t w = slot >> 5;
    const uint32_t word = f.smem ? lds_u32(f.smem + w * 4u)
                                 : ld_keep_u32(reinterpret_cast<const uint32_t*>(f.gptr) + w, pol_keep);
    return (word >> (slot & 31u)) & 1u;
  }
  const uint32_t w = bf_word(slot, f.log2);
  const uint64_t m = bf_mask(slot, f.k);
  const uint64_t word = f.smem ? lds_u64(f.smem + w * 8u)
                               : ld_keep_u64(reinterpret_cast<const uint64_t*>(f.gptr) + w, pol_keep);
  return (word & m) == m;
}

// Step list of one join order.  LIP: every filter first, then the PHT probes that
// still matter (grouped dimensions need the code; the direct bitmap is exact over
// PHT slots, so an ungrouped dimension that has one needs no PHT probe).  Naive:
// PHT probes only, in join order (src/ssb-jo/q33/0-naive.cu:50-72).
__device__ inline uint32_t make_steps(const SjPlanRt& P, const uint32_t* bf_mode, const uint32_t* order,
                                      uint32_t* steps) {
  uint32_t n = 0;
  if (P.lip) {
    for (uint32_t p = 0; p < P.n_dims; ++p) steps[n++] = order[p] | (kStepBF << 4);
    for (uint32_t p = 0; p < P.n_dims; ++p) {
      const SjDimRt& D = P.dim[order[p]];
      if (D.grouped || bf_mode[order[p]] != kBfDirect) steps[n++] = order[p] | (kStepPHT << 4);
    }
  } else {
    for (uint32_t p = 0; p < P.n_dims; ++p) steps[n++] = order[p] | (kStepPHT << 4);
  }
  return n;
}

// Expected filter tests per row of an order under the observed pass rates.
// Expected filter-test cost per fact row of a LIP order: each test costs 1 when
// its filter is in shared memory and kL2TestCost when it is read from L2, and
// a row reaches position p with the product of the earlier pass rates.
constexpr float kL2TestCost = 4.f;

__device__ inline float order_cost(const float* rate, const float* weight, const uint32_t* order, uint32_t n) {
  float c = 0.f, live = 1.f;
  for (uint32_t p = 0; p < n; ++p) {
    c += live * weight[order[p]];
    live *= rate[order[p]];
  }
  return c;
}

// Four per-dimension values held in registers, selected by a runtime dimension
// index without local memory.
struct Vals4 {
  uint32_t v0, v1, v2, v3;
  __device__ __forceinline__ uint32_t get(uint32_t d) const {
    return d == 0 ? v0 : (d == 1 ? v1 : (d == 2 ? v2 : v3));
  }
  __device__ __forceinline__ void set(uint32_t d, uint32_t x) {
    v0 = d == 0 ? x : v0;
    v1 = d == 1 ? x : v1;
    v2 = d == 2 ? x : v2;
    v3 = d == 3 ? x : v3;
  }
};

// The streamed dimension's parameters, in registers for one chunk.
struct First {
  const int32_t* fk;
  const int2* ht;
  int32_t kmin;
  uint32_t len;
  uint64_t fm;
  BfView bf;
};

// State of one consumer warp.  Every field is identical in all 32 lanes.
// PAIR: Q1 rounds may take two survivors per lane (q1_pair); off where the
// CTA's register budget has no room for the second survivor's state.
template <bool PAIR>
struct Warp {
  const SjPlanRt& P;
  Ctl& c;
  uint32_t* q1;
  uint32_t* q2;
  uint32_t q1m, q2m;
  unsigned long long* s_sum;
  uint32_t* s_cnt;
  uint32_t bf_base;
  const uint8_t* bf_ptr;  // the same filter region as a shared-memory pointer
  uint64_t base_row;
  uint64_t pol_first, pol_keep;
  uint32_t lane;
  uint32_t t1, h1, t2, h2;

  __device__ __forceinline__ BfView bfview(uint32_t d) const {
    BfView f;
    const SjDimRt& D = P.dim[d];
    f.mode = c.bf_mode[d];
    f.k = D.bf_k;
    f.log2 = c.bf_log2[d];
    f.gptr = D.bf;
    const uint32_t off = c.bf_in_smem[d];
    f.smem = off == ~0u ? 0u : bf_base + off;
    return f;
  }

  __device__ __forceinline__ uint32_t slot_at(uint32_t d, uint32_t rel) const {
    const SjDimRt& D = P.dim[d];
    return slot_fast(ld_stream(D.fact_fk + base_row + rel, pol_first), D.key_min, D.ht_len, D.fastmod_m);
  }

  __device__ __forceinline__ void aggregate(int64_t m, const Vals4& cv) {
    uint32_t g = 0;
    if (0 < P.n_dims && P.dim[0].grouped) g += cv.v0 * c.group_stride[0];
    if (1 < P.n_dims && P.dim[1].grouped) g += cv.v1 * c.group_stride[1];
    if (2 < P.n_dims && P.dim[2].grouped) g += cv.v2 * c.group_stride[2];
    if (3 < P.n_dims && P.dim[3].grouped) g += cv.v3 * c.group_stride[3];
    if (c.groups_in_smem) {
      atomicAdd(&s_sum[g], (unsigned long long)m);
      atomicAdd(&s_cnt[g], 1u);
    } else {
      atomicAdd(&P.g_sum[g], (unsigned long long)m);
      atomicAdd(&P.g_cnt[g], 1ull);
    }
  }

  // Steps [first, n) for the warp's live lanes, then the aggregate.  Every lane
  // takes part (warp-synchronous).  The loads a row still needs go out together
  // instead of one dependent chain per step: first the fact keys of every
  // dimension still to be looked up and the measure, then every remaining
  // filter word and PHT slot.  The tests are then evaluated in step order and
  // each step's entries and passes counted with two ballots (one shared-memory
  // atomic per warp and step), exactly as a step-by-step walk counts them; a row
  // passes only if every step passes, so loading ahead changes the work, never
  // the answer.
  __device__ __forceinline__ void finish(uint32_t ver, uint32_t first, bool alive, uint32_t rel, uint32_t have,
                                         uint32_t coded, Vals4 sv, Vals4 cv) {
    const uint32_t n = c.n_steps[ver];
    if (!__ballot_sync(0xffffffffu, alive)) return;
    // 1. fact keys of the dimensions still needed (steps and grouping), and the measure
    uint32_t need = 0;
    for (uint32_t p = first; p < n; ++p) need |= 1u << (c.steps[ver][p] & 15u);
    for (uint32_t d = 0; d < P.n_dims; ++d)
      if (P.dim[d].grouped && !((coded >> d) & 1u)) need |= 1u << d;
    need &= ~have;
    int64_t mv = 0;
    if (alive) {
#pragma unroll
      for (uint32_t d = 0; d < kMaxDims; ++d)
        if ((need >> d) & 1u) sv.set(d, slot_at(d, rel));
      mv = (int64_t)ld_stream(P.measure + base_row + rel, pol_first);
      if (P.measure_sub) mv -= (int64_t)ld_stream(P.measure_sub + base_row + rel, pol_first);
    }
    // 2. every remaining filter word / PHT slot
    uint64_t raw[kMaxSteps];
#pragma unroll
    for (uint32_t p = 0; p < kMaxSteps; ++p) {
      raw[p] = 0;
      if (alive && p >= first && p < n) {
        const uint32_t st = c.steps[ver][p], d = st & 15u;
        const uint32_t sl = sv.get(d);
        if ((st >> 4) == kStepBF) {
          const BfView f = bfview(d);
          if (f.mode == kBfDirect) {
            const uint32_t w = sl >> 5;
            raw[p] = f.smem ? lds_u32(f.smem + w * 4u)
                            : ld_keep_u32(reinterpret_cast<const uint32_t*>(f.gptr) + w, pol_keep);
          } else {
            const uint32_t w = bf_word(sl, f.log2);
            raw[p] = f.smem ? lds_u64(f.smem + w * 8u)
                            : ld_keep_u64(reinterpret_cast<const uint64_t*>(f.gptr) + w, pol_keep);
          }
        } else {
          const int2 e = ld_slot(P.dim[d].ht + sl, pol_keep);
          raw[p] = ((uint64_t)(uint32_t)e.y << 32) | (uint32_t)e.x;
        }
      }
    }
    // 3. the tests in step order, counted as the plan walks them
#pragma unroll
    for (uint32_t p = 0; p < kMaxSteps; ++p) {
      if (p < first || p >= n) continue;
      const uint32_t in = __ballot_sync(0xffffffffu, alive);
      if (!in) return;
      const uint32_t st = c.steps[ver][p], d = st & 15u;
      const bool is_bf = (st >> 4) == kStepBF;
      bool pass = false;
      if (alive) {
        const uint32_t sl = sv.get(d);
        if (is_bf) {
          if (c.bf_mode[d] == kBfDirect) {
            pass = ((uint32_t)raw[p] >> (sl & 31u)) & 1u;
          } else {
            const uint64_t m = bf_mask(sl, P.dim[d].bf_k);
            pass = (raw[p] & m) == m;
          }
        } else {
          pass = (uint32_t)raw[p] != 0u;
          cv.set(d, (uint32_t)(raw[p] >> 32));
          coded |= 1u << d;
        }
      }
      const uint32_t out = __ballot_sync(0xffffffffu, pass);
      if (lane == 0) {
        atomicAdd(&c.step_in[p], (uint32_t)__popc(in));
        atomicAdd(&c.step_out[p], (uint32_t)__popc(out));
        if (is_bf) {
          atomicAdd(&c.probes[d], (uint32_t)__popc(in));
          atomicAdd(&c.passes[d], (uint32_t)__popc(out));
        }
      }
      alive = pass;
    }
    if (!alive) return;
    // codes of grouped dimensions whose PHT probe passed in an earlier step
    for (uint32_t d = 0; d < P.n_dims; ++d) {
      if (!P.dim[d].grouped || ((coded >> d) & 1u)) continue;
      cv.set(d, (uint32_t)ld_slot(P.dim[d].ht + sv.get(d), pol_keep).y);
    }
    aggregate(mv, cv);
  }

  // Q1 entries [h1, h1 + cnt): step 1, then finish (plans of <= 2 steps) or
  // compact the survivors into Q2.
  __device__ __forceinline__ void q1_round(uint32_t ver, uint32_t cnt) {
    __syncwarp();
    const uint32_t n = c.n_steps[ver];
    const uint32_t st1 = c.steps[ver][n > 1 ? 1 : 0];
    const uint32_t d1 = st1 & 15u;
    const bool bf1 = (st1 >> 4) == kStepBF;
    bool pass = false;
    uint32_t rel = 0, have = 0, coded = 0;
    Vals4 sv{0, 0, 0, 0}, cv{0, 0, 0, 0};
    if (lane < cnt) {
      rel = q1[(h1 + lane) & q1m];
      if (n == 1) {
        pass = true;
      } else {
        const uint32_t s1 = slot_at(d1, rel);
        sv.set(d1, s1);
        have = 1u << d1;
        if (bf1) {
          pass = bf_test(bfview(d1), s1, pol_keep);
        } else {
          const int2 e = ld_slot(P.dim[d1].ht + s1, pol_keep);
          pass = e.x != 0;
          cv.set(d1, (uint32_t)e.y);
          coded = 1u << d1;
        }
      }
    }
    const uint32_t m = __ballot_sync(0xffffffffu, pass);
    if (n <= 2) {
      finish(ver, 2, pass, rel, have, coded, sv, cv);
    } else {
      if (pass) {
        q2[(t2 + __popc(m & lanemask_lt())) & q2m] = rel;
        const uint32_t d2 = c.steps[ver][2] & 15u;
        if (d2 != d1) prefetch_l2(P.dim[d2].fact_fk + base_row + rel);
      }
      t2 += __popc(m);
    }
    if (lane == 0 && n > 1) {
      atomicAdd(&c.step_in[1], cnt);
      atomicAdd(&c.step_out[1], (uint32_t)__popc(m));
      if (bf1) {
        atomicAdd(&c.probes[d1], cnt);
        atomicAdd(&c.passes[d1], (uint32_t)__popc(m));
      }
    }
    h1 += cnt;
  }

  // Q1 entries [h1, h1 + 64) of a plan with more than two steps: q1_round on
  // two survivors per lane, with both lanes' step-1 loads (the next FK column,
  // then its filter word or PHT slot) in flight together, the survivors queued
  // in Q2.  The caller leaves 64 free Q2 entries.
  __device__ __forceinline__ void q1_pair(uint32_t ver) {
    __syncwarp();
    const uint32_t st1 = c.steps[ver][1];
    const uint32_t d1 = st1 & 15u;
    const bool bf1 = (st1 >> 4) == kStepBF;
    const uint32_t ra = q1[(h1 + lane) & q1m], rb = q1[(h1 + 32u + lane) & q1m];
    const uint32_t s_a = slot_at(d1, ra), s_b = slot_at(d1, rb);
    bool pa, pb;
    if (bf1) {
      const BfView f = bfview(d1);
      pa = bf_test(f, s_a, pol_keep);
      pb = bf_test(f, s_b, pol_keep);
    } else {
      pa = ld_slot(P.dim[d1].ht + s_a, pol_keep).x != 0;
      pb = ld_slot(P.dim[d1].ht + s_b, pol_keep).x != 0;
    }
    const uint32_t ma = __ballot_sync(0xffffffffu, pa), mb = __ballot_sync(0xffffffffu, pb);
    const uint32_t d2 = c.steps[ver][2] & 15u;
    if (pa) {
      q2[(t2 + __popc(ma & lanemask_lt())) & q2m] = ra;
      if (d2 != d1) prefetch_l2(P.dim[d2].fact_fk + base_row + ra);
    }
    t2 += __popc(ma);
    if (pb) {
      q2[(t2 + __popc(mb & lanemask_lt())) & q2m] = rb;
      if (d2 != d1) prefetch_l2(P.dim[d2].fact_fk + base_row + rb);
    }
    t2 += __popc(mb);
    if (lane == 0) {
      const uint32_t out = (uint32_t)(__popc(ma) + __popc(mb));
      atomicAdd(&c.step_in[1], 64u);
      atomicAdd(&c.step_out[1], out);
      if (bf1) {
        atomicAdd(&c.probes[d1], 64u);
        atomicAdd(&c.passes[d1], out);
      }
    }
    h1 += 64;
  }

  __device__ __forceinline__ void q2_round(uint32_t ver, uint32_t cnt) {
    __syncwarp();
    finish(ver, 2, lane < cnt, q2[(h2 + lane) & q2m], 0u, 0u, Vals4{0, 0, 0, 0}, Vals4{0, 0, 0, 0});
    h2 += cnt;
  }

  // Queue rounds: full rounds only while streaming, everything when draining.
  __device__ __forceinline__ void pump(uint32_t ver, bool drain) {
    for (;;) {
      const uint32_t a1 = t1 - h1, a2 = t2 - h2;
      if (a2 >= 32 || (drain && a2 > 0 && a1 == 0)) {
        q2_round(ver, min(a2, 32u));
      } else if (PAIR && a1 >= 64 && a2 + 64u <= q2m + 1u && c.n_steps[ver] > 2) {
        q1_pair(ver);
      } else if (a1 >= 32 || (drain && a1 > 0)) {
        q1_round(ver, min(a1, 32u));
      } else {
        break;
      }
    }
  }

  // Test the rows [off, off + rows) of a staged chunk against the first step and
  // queue the survivors.  FULL: every row of the chunk is valid and staged.
  // Per lane and pass: RPL independent rows; the pass bits collect in a register
  // mask, and one warp prefix scan of the mask popcounts places the survivors.
  template <int RPL, int MODE, int K, bool FULL>
  __device__ __forceinline__ uint32_t scan(uint32_t ver, const int32_t* sbuf, const First& f, uint32_t off,
                                           uint32_t rows, uint64_t cstart, uint32_t crows, uint32_t tma_rows,
                                           uint32_t skip, uint32_t rel0, const int32_t* pf) {
    static_assert(RPL <= 32, "pass mask is 32 bits");
    const uint32_t t_begin = t1;
    // plain shared-memory loads (not volatile asm), so the compiler can schedule a
    // pass's staged loads and filter lookups together; the mbarrier waits and
    // arrives around a stage carry memory clobbers
    const uint8_t* fbase = (MODE == kModeDirectSmem || MODE == kModeBlockedSmem) ? bf_ptr + (f.bf.smem - bf_base)
                                                                                  : nullptr;
    for (uint32_t i0 = off; i0 < off + rows; i0 += 32u * RPL) {
      uint32_t d[RPL];
      uint32_t valid = ~0u;  // bit j: row j of this lane lies in the scanned range
      bool oor = false;      // some key outside [key_min, key_min + len)
#pragma unroll
      for (uint32_t j4 = 0; j4 < RPL / 4; ++j4) {
        const uint32_t r4 = i0 + (j4 * 32u + lane) * 4u;
        const int4 v = *reinterpret_cast<const int4*>(sbuf + r4);
        int32_t fk[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (uint32_t j = 0; j < 4; ++j) {
          if (!FULL) {
            const uint32_t r = r4 + j;
            const bool ok = (r < crows) && (r >= skip);
            if (!ok) valid &= ~(1u << (j4 * 4 + j));
            if (ok && r >= tma_rows) fk[j] = ld_stream(f.fk + cstart + r, pol_first);
          }
          d[j4 * 4 + j] = (uint32_t)fk[j] - (uint32_t)f.kmin;
          oor |= d[j4 * 4 + j] >= f.len;
        }
      }
      if (__any_sync(0xffffffffu, oor)) {  // rare: reduce out-of-range keys modulo len
#pragma unroll
        for (uint32_t j = 0; j < RPL; ++j)
          if (d[j] >= f.len) d[j] = (uint32_t)__umul64hi(f.fm * (uint64_t)d[j], (uint64_t)f.len);
      }
      uint32_t mask = 0;
#pragma unroll
      for (uint32_t j = 0; j < RPL; ++j) {
        const uint32_t sl = d[j];
        bool ok;
        if (MODE == kModeDirectSmem) {
          const uint32_t wd = reinterpret_cast<const uint32_t*>(fbase)[sl >> 5];
          ok = __funnelshift_r(wd, wd, sl) & 1u;  // rotate right: bit (sl mod 32) to bit 0
        } else if (MODE == kModeBlockedSmem) {
          const uint32_t h1 = bf_h1(sl);
          const uint32_t w = __funnelshift_rc(h1, 0u, 32u - f.bf.log2);  // h1 >> (32 - log2), 0 for log2 = 0
          const uint2 wv = reinterpret_cast<const uint2*>(fbase)[w];
          ok = bf_test_word<K>(wv.x, wv.y, bf_g(h1));
        } else if (MODE == kModeBfAny) {
          ok = bf_test(f.bf, sl, pol_keep);
        } else {
          ok = ld_slot(f.ht + sl, pol_keep).x != 0;
        }
        mask |= (ok ? 1u : 0u) << j;
      }
      if (!FULL) mask &= valid;
      const uint32_t lanes = __ballot_sync(0xffffffffu, mask != 0);
      if (lanes) {
        uint32_t pos, total;
        if (__any_sync(0xffffffffu, mask & (mask - 1u))) {
          // some lane has several survivors: warp prefix scan of the counts
          const uint32_t cnt = __popc(mask);
          uint32_t incl = cnt;
#pragma unroll
          for (uint32_t o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
          }
          total = __shfl_sync(0xffffffffu, incl, 31);
          pos = t1 + incl - cnt;
        } else {
          // at most one survivor per lane: the lane ballot is the prefix
          total = __popc(lanes);
          pos = t1 + __popc(lanes & lanemask_lt());
        }
        while (mask) {
          const uint32_t j = __ffs(mask) - 1u;
          mask &= mask - 1u;
          const uint32_t rr = rel0 + i0 + ((j >> 2) * 32u + lane) * 4u + (j & 3u);
          q1[pos++ & q1m] = rr;
          if (pf) prefetch_l2(pf + rr);
        }
        t1 += total;
        if (t1 - h1 > q1m + 1 - 32u * RPL) pump(ver, false);  // keep room for one more pass
      }
    }
    return t1 - t_begin;
  }
};

// NWC consumer warps + 1 producer warp; RPL fact rows per lane per scan pass.
template <int NWC, int RPL>
__global__ void __launch_bounds__((NWC + 1) * 32, 1) sj_probe_kernel(const __grid_constant__ SjPlanRt P,
                                                                     const __grid_constant__ SjProbeGeom G) {
  static_assert(RPL % 4 == 0, "rows per lane must be a multiple of 4");
  constexpr uint32_t NT = (NWC + 1) * 32;
  pdl_launch_dependents();
  extern __shared__ __align__(128) uint8_t smem[];
  const SmemLayout L = probe_layout(G);
  int32_t* stage = reinterpret_cast<int32_t*>(smem + L.stage_off);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + L.full_off);
  uint64_t* empty = reinterpret_cast<uint64_t*>(smem + L.empty_off);
  uint8_t* bfmem = smem + L.bf_off;
  Ctl& c = *reinterpret_cast<Ctl*>(smem + L.ctl_off);
  const SjDesc* desc = P.desc;
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  const uint32_t S = G.stages, CH = G.chunk_rows;

  const uint64_t base_row = P.row_begin & ~3ull;
  const uint64_t span = P.row_end - base_row;
  const uint32_t n_chunks = (uint32_t)((span + CH - 1) / CH);
  const uint32_t my_iters = (blockIdx.x < n_chunks) ? (n_chunks - blockIdx.x + gridDim.x - 1) / gridDim.x : 0u;

  // ---- setup (thread 0): mbarriers; while the build may still run (programmatic
  // dependent launch), an L2 prefetch of this CTA's first chunks of the column
  // the plan's order tests first (the fact columns are inputs, never written);
  // then, the build complete, the plan steps and filter placement ------------
  if (tid == 0) {
    memset(&c, 0, sizeof(Ctl));
    for (uint32_t s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], NWC);
    }
    mbar_fence_init();
    const int32_t* col0 = P.dim[P.order[0]].fact_fk;
    for (uint32_t it = 0; it < S && it < my_iters; ++it) {
      const uint64_t start = base_row + (uint64_t)(blockIdx.x + it * gridDim.x) * CH;
      const uint32_t bytes = (uint32_t)(min((uint64_t)CH, P.row_end - start) & ~3ull) * 4u;
      if (bytes) bulk_prefetch_l2(col0 + start, bytes);
    }
  }
  pdl_wait();  // the build's descriptor, hash tables and filters are complete
  if (tid == 0) {
    for (uint32_t d = 0; d < P.n_dims; ++d) {
      c.bf_log2[d] = desc->dim[d].bf_log2;
      c.bf_mode[d] = desc->dim[d].bf_mode;
    }
    // starting order and filter placement, chosen once per query by sj_dim_insert
    uint32_t ord[kMaxDims];
    for (uint32_t d = 0; d < kMaxDims; ++d) {
      ord[d] = desc->start_order[d];
      c.bf_in_smem[d] = desc->bf_smem_off[d];
    }
    for (uint32_t d = 0; d < kMaxDims; ++d) c.order[0][d] = c.order[1][d] = (d < P.n_dims) ? ord[d] : 0u;
    c.n_steps[0] = c.n_steps[1] = make_steps(P, c.bf_mode, ord, c.steps[0]);
    for (uint32_t p = 0; p < kMaxSteps; ++p) c.steps[1][p] = c.steps[0][p];
    for (uint32_t d = 0; d < P.n_dims; ++d) c.group_stride[d] = desc->dim[d].group_stride;
    c.n_groups = desc->n_groups;
    c.groups_in_smem = c.n_groups <= G.group_smem_cap;
  }
  __syncthreads();

  // ---- filters into shared memory, zero the group partials ----------------
  for (uint32_t d = 0; d < P.n_dims; ++d) {
    if (c.bf_in_smem[d] == ~0u) continue;
    const SjDimRt& D = P.dim[d];
    const uint32_t bytes = (c.bf_mode[d] == kBfDirect) ? max(8u, (1u << c.bf_log2[d]) / 8u) : (8u << c.bf_log2[d]);
    if (bytes >= 16u) {
      const uint4* src = reinterpret_cast<const uint4*>(D.bf);
      uint4* dst = reinterpret_cast<uint4*>(bfmem + c.bf_in_smem[d]);
      for (uint32_t i = tid; i < bytes / 16u; i += NT) dst[i] = src[i];
    } else if (tid == 0) {
      *reinterpret_cast<uint2*>(bfmem + c.bf_in_smem[d]) = *reinterpret_cast<const uint2*>(D.bf);
    }
  }
  unsigned long long* s_sum = reinterpret_cast<unsigned long long*>(smem + L.gsum_off);
  uint32_t* s_cnt = reinterpret_cast<uint32_t*>(smem + L.gcnt_off);
  if (c.groups_in_smem) {
    for (uint32_t g = tid; g < c.n_groups; g += NT) {
      s_sum[g] = 0ull;
      s_cnt[g] = 0u;
    }
  }
  __syncthreads();

  const uint64_t pol_first = policy_evict_first();
  const uint64_t pol_keep = policy_evict_last();

  if (warp == NWC) {
    // ---- producer: one lane issues every chunk's TMA copy -------------------
    if (lane == 0) {
      uint32_t issue_ver = 0, last_switch = 0, it = 0;
      bool aborted = false;
      for (; it < my_iters; ++it) {
        const uint32_t s = it % S;
        if (it >= S && !mbar_wait_bounded(&empty[s], ((it / S) - 1u) & 1u, kMaxPolls)) {
          aborted = true;
          break;
        }
        if (ld_volatile_u32(&c.abort)) {
          aborted = true;
          break;
        }
        const uint32_t chunk = blockIdx.x + it * gridDim.x;
        const uint32_t d = c.order[issue_ver][0];
        c.stage_ver[s] = issue_ver;
        const uint64_t start = base_row + (uint64_t)chunk * CH;
        const uint64_t rows = min((uint64_t)CH, P.row_end - start);
        const uint32_t bytes = (uint32_t)(rows & ~3ull) * 4u;
        fence_proxy_async_smem();
        if (bytes) {
          mbar_arrive_expect_tx(&full[s], bytes);
          bulk_g2s(stage + (size_t)s * CH, P.dim[d].fact_fk + start, bytes, &full[s], pol_first);
        } else {
          mbar_arrive(&full[s]);
        }
        // adaptive re-ranking of the filter order for the chunks issued after this one:
        // evaluated once this chunk's copy is in flight, so the evaluation overlaps
        // the wait for the next free stage instead of delaying a copy
        if (P.lip && P.adaptive && P.n_dims > 1 && it >= last_switch + 2 * S &&
            (it == 2 * S || it % G.reorder_period == 0)) {
          float rate[kMaxDims];
          for (uint32_t d = 0; d < kMaxDims; ++d) {
            const float pr = (float)ld_volatile_u32(&c.probes[d]);
            const float pa = (float)ld_volatile_u32(&c.passes[d]);
            rate[d] = (d < P.n_dims) ? (pa + 1.f) / (pr + 2.f) : 1.f;
          }
          float weight[kMaxDims];
          for (uint32_t d = 0; d < kMaxDims; ++d) weight[d] = (c.bf_in_smem[d] == ~0u) ? kL2TestCost : 1.f;
          // candidate: sorted by observed pass rate (cheap on the issuing lane); taken
          // when it cuts the placement-weighted cost by more than 10%
          uint32_t cand[kMaxDims];
          const uint32_t* cur = c.order[issue_ver];
          for (uint32_t d = 0; d < P.n_dims; ++d) cand[d] = cur[d];
          for (uint32_t a = 1; a < P.n_dims; ++a)
            for (uint32_t b = a; b > 0 && rate[cand[b]] < rate[cand[b - 1]]; --b) {
              const uint32_t t = cand[b];
              cand[b] = cand[b - 1];
              cand[b - 1] = t;
            }
          if (order_cost(rate, weight, cand, P.n_dims) < 0.9f * order_cost(rate, weight, cur, P.n_dims)) {
            const uint32_t nv = issue_ver ^ 1u;
            for (uint32_t d = 0; d < kMaxDims; ++d) c.order[nv][d] = (d < P.n_dims) ? cand[d] : 0u;
            c.n_steps[nv] = make_steps(P, c.bf_mode, c.order[nv], c.steps[nv]);
            issue_ver = nv;
            last_switch = it;
            c.reorders++;
          }
        }
      }
      if (aborted) {
        c.abort = 1;
        // let copies still in flight land before the CTA's shared memory goes away
        const uint32_t lo = it > S ? it - S : 0u;
        for (uint32_t j = lo; j < it; ++j) mbar_wait_bounded(&full[j % S], (j / S) & 1u, kMaxPolls);
      }
    }
  } else {
    // ---- consumer warps ------------------------------------------------------
    Warp<(NWC <= 15)> w{P, c,
           reinterpret_cast<uint32_t*>(smem + L.q1_off) + warp * G.q1_cap,
           reinterpret_cast<uint32_t*>(smem + L.q2_off) + warp * G.q2_cap,
           G.q1_cap - 1, G.q2_cap - 1, s_sum, s_cnt, smem_addr(bfmem), bfmem, base_row, pol_first, pol_keep, lane,
           0, 0, 0, 0};
    const uint32_t slice = CH / NWC;
    const uint32_t my_off = warp * slice;
    uint32_t exec_ver = 0;
    bool aborted = false;
    for (uint32_t it = 0; it < my_iters; ++it) {
      const uint32_t s = it % S;
      if (!mbar_wait_bounded(&full[s], (it / S) & 1u, kMaxPolls)) {
        c.abort = 1;
        aborted = true;
        break;
      }
      if (ld_volatile_u32(&c.abort)) {
        aborted = true;
        break;
      }
      const uint32_t sver = c.stage_ver[s];
      if (sver != exec_ver) {
        w.pump(exec_ver, true);  // first chunk of a new filter order
        exec_ver = sver;
      }
      const uint32_t ver = exec_ver;
      const uint32_t st0 = c.steps[ver][0];
      const uint32_t d0 = st0 & 15u;
      First f;
      f.fk = P.dim[d0].fact_fk;
      f.ht = P.dim[d0].ht;
      f.kmin = P.dim[d0].key_min;
      f.len = P.dim[d0].ht_len;
      f.fm = P.dim[d0].fastmod_m;
      f.bf = w.bfview(d0);
      const bool is_bf = (st0 >> 4) == kStepBF;
      const int mode = !is_bf ? kModePht
                              : (!f.bf.smem ? kModeBfAny : (f.bf.mode == kBfDirect ? kModeDirectSmem : kModeBlockedSmem));
      const uint32_t chunk = blockIdx.x + it * gridDim.x;
      const uint64_t cstart = base_row + (uint64_t)chunk * CH;
      const uint32_t crows = (uint32_t)min((uint64_t)CH, P.row_end - cstart);
      const uint32_t tma_rows = crows & ~3u;
      const uint32_t skip = (cstart < P.row_begin) ? (uint32_t)(P.row_begin - cstart) : 0u;
      const uint32_t rel0 = (uint32_t)(cstart - base_row);
      const int32_t* pf = nullptr;  // column read at survivor rows by step 1
      if (c.n_steps[ver] > 1) {
        const uint32_t d1 = c.steps[ver][1] & 15u;
        if (d1 != d0) pf = P.dim[d1].fact_fk + base_row;
      }
      const int32_t* sbuf = stage + (size_t)s * CH;
      const bool fullc = (crows == CH) && (skip == 0);
      uint32_t passed;
#define SJ_SCAN(M, K)                                                                                        \
  passed = fullc                                                                                             \
               ? w.template scan<RPL, M, K, true>(ver, sbuf, f, my_off, slice, cstart, crows, tma_rows, skip, \
                                                  rel0, pf)                                                   \
               : w.template scan<RPL, M, K, false>(ver, sbuf, f, my_off, slice, cstart, crows, tma_rows, skip, \
                                                   rel0, pf)
      if (mode == kModeDirectSmem) SJ_SCAN(kModeDirectSmem, 0);
      else if (mode == kModeBlockedSmem) {
        if (f.bf.k == 1) SJ_SCAN(kModeBlockedSmem, 1);
        else if (f.bf.k == 2) SJ_SCAN(kModeBlockedSmem, 2);
        else if (f.bf.k == 3) SJ_SCAN(kModeBlockedSmem, 3);
        else SJ_SCAN(kModeBlockedSmem, 4);
      } else if (mode == kModeBfAny) SJ_SCAN(kModeBfAny, 0);
      else SJ_SCAN(kModePht, 0);
#undef SJ_SCAN
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(&empty[s]);  // this warp is done reading the stage
        const uint32_t lo = max(my_off, skip), hi = min(my_off + slice, crows);
        const uint32_t valid = hi > lo ? hi - lo : 0u;
        atomicAdd(&c.rows_scanned, valid);
        atomicAdd(&c.step_in[0], valid);
        atomicAdd(&c.step_out[0], passed);
        if (is_bf) {
          atomicAdd(&c.probes[d0], valid);
          atomicAdd(&c.passes[d0], passed);
        }
      }
      w.pump(ver, false);
    }
    if (!aborted) w.pump(exec_ver, true);
  }
  __syncthreads();

  // ---- flush group partials and counters -----------------------------------
  const bool aborted = ld_volatile_u32(&c.abort) != 0;
  if (!aborted && c.groups_in_smem) {
    for (uint32_t g = tid; g < c.n_groups; g += NT) {
      const uint32_t cnt = s_cnt[g];
      if (cnt) {
        atomicAdd(&P.g_sum[g], s_sum[g]);
        atomicAdd(&P.g_cnt[g], (unsigned long long)cnt);
      }
    }
  }
  if (tid == 0) {
    SjDesc* dw = P.desc;
    if (aborted) atomicOr(&dw->error_flags, kErrWaitTimeout);
    atomicAdd(&dw->rows_scanned, (unsigned long long)c.rows_scanned);
    for (uint32_t p = 0; p < kMaxSteps; ++p) {
      if (c.step_in[p]) atomicAdd(&dw->step_in[p], (unsigned long long)c.step_in[p]);
      if (c.step_out[p]) atomicAdd(&dw->step_out[p], (unsigned long long)c.step_out[p]);
    }
    for (uint32_t d = 0; d < P.n_dims; ++d) {
      if (c.probes[d]) atomicAdd(&dw->bf_probes[d], (unsigned long long)c.probes[d]);
      if (c.passes[d]) atomicAdd(&dw->bf_passes[d], (unsigned long long)c.passes[d]);
    }
    if (c.reorders) atomicAdd(&dw->reorders, (unsigned long long)c.reorders);
  }
}

// Compact the non-empty groups into result rows, decoding dictionary codes back
// to payload values, and clear each group it reads: the group sums are zero
// again for the next probe, so no build has to clear the whole group space.
__global__ void __launch_bounds__(256) sj_finalize_kernel(const __grid_constant__ SjPlanRt P) {
  pdl_wait();  // the probe's group sums are complete
  SjDesc* desc = P.desc;
  const uint32_t n_groups = desc->n_groups;
  uint32_t n_codes[kMaxDims], stride[kMaxDims];  // read once, beside n_groups
#pragma unroll
  for (uint32_t d = 0; d < kMaxDims; ++d) {
    const bool grouped = d < P.n_dims && P.dim[d].grouped;
    n_codes[d] = grouped && desc->dim[d].n_codes ? desc->dim[d].n_codes : 1u;
    stride[d] = grouped ? desc->dim[d].group_stride : 1u;
  }
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < n_groups; g += gridDim.x * blockDim.x) {
    const unsigned long long cnt = P.g_cnt[g];
    if (!cnt) continue;
    const uint32_t pos = atomicAdd(&desc->groups_out, 1u);
    if (pos >= P.group_capacity) continue;  // cannot happen: at most n_groups rows
    sj_group_row r;
#pragma unroll
    for (uint32_t d = 0; d < kMaxDims; ++d) {
      r.attr[d] = 0;
      if (d < P.n_dims && P.dim[d].grouped) r.attr[d] = P.dim[d].dict[(g / stride[d]) % n_codes[d]];
    }
    r.count = cnt;
    r.sum = P.g_sum[g];
    P.rows_out[pos] = r;
    P.g_sum[g] = 0ull;
    P.g_cnt[g] = 0ull;
  }
}

// ---- host-side launchers ---------------------------------------------------
uint32_t probe_smem_bytes(const SjProbeGeom& g) { return probe_layout(g).total; }

template <int NWC, int RPL>
static cudaError_t launch_probe_t(const SjPlanRt& P, const SjProbeGeom& G, uint32_t smem, cudaStream_t st,
                                  const L2Window& w, bool pdl) {
  cudaError_t e = cudaFuncSetAttribute(sj_probe_kernel<NWC, RPL>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  return launch_windowed(sj_probe_kernel<NWC, RPL>, dim3(G.grid), dim3((NWC + 1) * 32), smem, st, w, pdl, P, G);
}

// G.threads = 32 * (consumer warps + 1); rows_per_lane: rows each lane tests per pass;
// w: L2 window over the query's hash tables and filters (may be empty); pdl: the
// previous kernel of the stream is the build's sj_dim_insert (programmatic
// dependent launch).
cudaError_t launch_probe(const SjPlanRt& P, const SjProbeGeom& G, uint32_t rows_per_lane, cudaStream_t st,
                         const L2Window& w, bool pdl) {
  const uint32_t smem = probe_layout(G).total;
  const uint32_t nwc = G.threads / 32 - 1;
#define SJ_CASE(W, R) \
  if (nwc == W && rows_per_lane == R) return launch_probe_t<W, R>(P, G, smem, st, w, pdl);
  SJ_CASE(7, 8)
  SJ_CASE(7, 16)
  SJ_CASE(15, 8)
  SJ_CASE(15, 16)
  SJ_CASE(23, 4)
  SJ_CASE(23, 8)
#undef SJ_CASE
  return cudaErrorInvalidValue;
}

// pdl: the previous kernel of the stream is the probe (programmatic dependent launch).
cudaError_t launch_finalize(const SjPlanRt& P, uint32_t group_capacity, cudaStream_t st, bool pdl) {
  uint32_t blocks = (group_capacity + 255) / 256;
  if (blocks > 296) blocks = 296;  // grid-stride over the dense groups (24 for Q3.3)
  if (blocks < 1) blocks = 1;
  return launch_windowed(sj_finalize_kernel, dim3(blocks), dim3(256), 0, st, L2Window{}, pdl, P);
}

}  // namespace sj
