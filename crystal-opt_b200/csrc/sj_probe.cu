// sj_probe.cu -- the fused star-join probe: fact scan -> LIP Bloom filters -> PHT
// probes -> group-by SUM, one persistent kernel per query; optionally the whole
// query (build prologue, probe, group compaction) in one cooperative launch.
//
// Replaces the reference's probe<128,4> kernels (src/ssb-jo/q33/0-lip.cu:28-112,
// src/ssb-jo/q33/0-naive.cu:28-91, src/ssb-jo/q41/0-lip.cu:28-131) and, in the
// fused form, its whole runQuery (src/ssb-jo/q33/0-lip.cu:205-302).  Same answer,
// different machine mapping:
//   * One CTA per SM, every warp a scanner.  Only the column tested first is read
//     densely: each warp streams its share of it with 128-bit loads (U per lane
//     in flight) straight into registers.  Warps share no staging buffer, so a
//     warp that stops to serve its survivors holds up no other warp's stream.
//   * Each warp tests its rows against the first filter (in shared memory) and
//     compacts the survivors (ballot / warp scan) into its own ring queue Q1 of
//     row offsets.  Later columns are read only at survivor rows (sector-sparse
//     reads, prefetched into L2 when the row is queued).  Survivors of the second
//     test are compacted again into the warp's Q2; the remaining tests, the PHT
//     probes and the aggregate run densely on Q2.  Values of earlier steps are not
//     carried in the queues: the rare survivors recompute them from L2.
//   * Filters are evaluated on the PHT slot of each key, so a filter never rejects
//     a row the PHT would accept; filters that fit the budget live in shared memory.
//   * Group partials (dense dictionary codes) live in shared memory and are
//     flushed once per CTA with 64-bit atomics; group spaces that do not fit
//     aggregate straight into global memory.
//   * Counters are summed per warp (ballot / popc) and added to shared memory by
//     one lane per round.
//   * Adaptive LIP: warp 0 re-ranks the filter order from the CTA's probe/pass
//     counters every few passes.  A warp drains its queues before it runs a new
//     order, so the result never depends on the order, only the work does.
//   * Fused form: the build of sj_build.cuh runs as a prologue (zero the tables,
//     scan the dimensions | grid barrier | geometry and order per CTA, insert |
//     grid barrier), and after the probe a third barrier lets every CTA compact
//     its share of the dense groups into result rows.  The barriers are bounded
//     waits: on expiry the kernel records an error bit and returns.
#include "sj_build.cuh"

#include <algorithm>
#include <cstring>

namespace sj {

enum : uint32_t { kStepBF = 0, kStepPHT = 1 };
enum : int { kModeDirectSmem = 0, kModeBlockedSmem = 1, kModeBfAny = 2, kModePht = 3 };

constexpr uint32_t kMaxWarps = 32;

struct SmemLayout {
  uint32_t bf_off, q1_off, q2_off, gsum_off, gcnt_off, ctl_off, total;
};

struct Ctl {
  uint32_t ver;    // order version the warps run next (0 or 1)
  uint32_t abort;  // a grid barrier expired
  uint32_t n_steps[2];
  uint32_t steps[2][kMaxSteps];  // (dim | kind << 4)
  uint32_t order[2][kMaxDims];
  uint32_t warp_ver[kMaxWarps];   // version each warp runs
  uint32_t bf_in_smem[kMaxDims];  // byte offset within the filter region, or ~0u
  uint32_t bf_log2[kMaxDims];
  uint32_t bf_mode[kMaxDims];     // layout each dimension's filter was built in
  uint32_t group_stride[kMaxDims];
  uint32_t n_codes[kMaxDims];
  uint32_t n_groups;
  uint32_t groups_in_smem;
  uint32_t probes[kMaxDims], passes[kMaxDims];
  uint32_t step_in[kMaxSteps], step_out[kMaxSteps];
  uint32_t rows_scanned;
  uint32_t reorders;
  uint32_t scan_count[kMaxDims];  // fused prologue: this CTA's qualifying counts
  uint32_t inserted[kMaxDims];    // fused prologue: every CTA's counts
};

__host__ __device__ inline uint32_t align_up(uint32_t x, uint32_t a) { return (x + a - 1) / a * a; }

// The Q1 region doubles as the fused prologue's payload-prefix scratch.
__host__ __device__ inline SmemLayout probe_layout(const SjProbeGeom& g) {
  const uint32_t nw = g.threads / 32;
  SmemLayout L;
  uint32_t o = 0;
  L.bf_off = o;
  o += g.bf_smem_bytes;
  o = align_up(o, 16);
  L.q1_off = o;
  const uint32_t q1_bytes = nw * g.q1_cap * 4u;
  o += q1_bytes > g.prefix_words * 4u ? q1_bytes : g.prefix_words * 4u;
  L.q2_off = o;
  o += nw * g.q2_cap * 4u;
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
__device__ __forceinline__ uint32_t ld_volatile_u32(const uint32_t* p) {
  return *reinterpret_cast<const volatile uint32_t*>(p);
}
__device__ __forceinline__ int4 ldg4_stream(const int4* p, uint64_t pol) {
  int4 v;
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.s32 {%0, %1, %2, %3}, [%4], %5;"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ uint32_t ld_acquire_gpu(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_gpu(uint32_t* p, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Grid-wide barrier of the fused kernel (all CTAs resident: cooperative launch).
// Thread 0 of each CTA arrives on a counter; the last one resets it and bumps the
// generation the others wait on.  The wait is bounded: on expiry the CTA records
// kErrWaitTimeout and sets c.abort.  Returns false when the kernel must stop.
__device__ __forceinline__ bool grid_barrier(SjDesc* desc, Ctl& c) {
  __syncthreads();
  if (threadIdx.x == 0 && !c.abort) {
    const uint32_t gen = ld_acquire_gpu(&desc->bar_gen);
    __threadfence();
    bool ok = true;
    if (atomicAdd(&desc->bar_count, 1u) == gridDim.x - 1) {
      atomicExch(&desc->bar_count, 0u);
      __threadfence();
      st_release_gpu(&desc->bar_gen, gen + 1u);
    } else {
      uint32_t polls = 0;
      while (ld_acquire_gpu(&desc->bar_gen) == gen) {
        if (++polls > kMaxPolls) {
          ok = false;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    if (!ok) {
      atomicOr(&desc->error_flags, kErrWaitTimeout);
      c.abort = 1;
    }
  }
  __syncthreads();
  return !c.abort;
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

// The same k bits as bf_test_word with k known at run time (1..4).
__device__ __forceinline__ uint32_t bf_test_word_k(uint32_t lo, uint32_t hi, uint32_t g, uint32_t k) {
  uint32_t r = __funnelshift_r(lo, lo, g >> 27);
  if (k > 1) r &= __funnelshift_r(hi, hi, g >> 22);
  if (k > 2) r &= __funnelshift_r(lo, lo, g >> 17);
  if (k > 3) r &= __funnelshift_r(hi, hi, g >> 12);
  return r & 1u;
}

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

// The streamed dimension's parameters, in registers while a warp runs an order.
struct First {
  const int4* col4;  // its fact column, as 16-byte groups from the base row
  const int32_t* fk;
  const int2* ht;
  int32_t kmin;
  uint32_t len;
  uint64_t fm;
  BfView bf;
};

// State of one scanning warp.  Every field is identical in all 32 lanes.
template <int U>
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

  __device__ __forceinline__ void aggregate(uint32_t rel, const Vals4& cv) {
    uint32_t g = 0;
    if (0 < P.n_dims && P.dim[0].grouped) g += cv.v0 * c.group_stride[0];
    if (1 < P.n_dims && P.dim[1].grouped) g += cv.v1 * c.group_stride[1];
    if (2 < P.n_dims && P.dim[2].grouped) g += cv.v2 * c.group_stride[2];
    if (3 < P.n_dims && P.dim[3].grouped) g += cv.v3 * c.group_stride[3];
    int64_t m = (int64_t)ld_stream(P.measure + base_row + rel, pol_first);
    if (P.measure_sub) m -= (int64_t)ld_stream(P.measure_sub + base_row + rel, pol_first);
    if (c.groups_in_smem) {
      atomicAdd(&s_sum[g], (unsigned long long)m);
      atomicAdd(&s_cnt[g], 1u);
    } else {
      atomicAdd(&P.g_sum[g], (unsigned long long)m);
      atomicAdd(&P.g_cnt[g], 1ull);
    }
  }

  // Steps [first, n) for the warp's live lanes, then the aggregate.  Every lane
  // takes part (warp-synchronous): each step's entries and passes are counted
  // with two ballots.  Slots / codes a step needs and that earlier steps did not
  // leave in registers are recomputed.
  __device__ __forceinline__ void finish(uint32_t ver, uint32_t first, bool alive, uint32_t rel, uint32_t have,
                                         uint32_t coded, Vals4 sv, Vals4 cv) {
    const uint32_t n = c.n_steps[ver];
    for (uint32_t p = first; p < n; ++p) {
      const uint32_t in = __ballot_sync(0xffffffffu, alive);
      if (!in) return;
      const uint32_t st = c.steps[ver][p];
      const uint32_t d = st & 15u;
      const bool is_bf = (st >> 4) == kStepBF;
      bool pass = false;
      if (alive) {
        if (!((have >> d) & 1u)) {
          sv.set(d, slot_at(d, rel));
          have |= 1u << d;
        }
        if (is_bf) {
          pass = bf_test(bfview(d), sv.get(d), pol_keep);
        } else {
          const int2 e = ld_slot(P.dim[d].ht + sv.get(d), pol_keep);
          pass = e.x != 0;
          cv.set(d, (uint32_t)e.y);
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
      const uint32_t s = ((have >> d) & 1u) ? sv.get(d) : slot_at(d, rel);
      cv.set(d, (uint32_t)ld_slot(P.dim[d].ht + s, pol_keep).y);
    }
    aggregate(rel, cv);
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
    const bool live = lane < cnt;
    const uint32_t rel = q2[(h2 + lane) & q2m];
    finish(ver, 2, live, rel, 0u, 0u, Vals4{0, 0, 0, 0}, Vals4{0, 0, 0, 0});
    h2 += cnt;
  }

  // Queue rounds: full rounds only while streaming, everything when draining.
  __device__ __forceinline__ void pump(uint32_t ver, bool drain) {
    for (;;) {
      const uint32_t a1 = t1 - h1, a2 = t2 - h2;
      if (a2 >= 32 || (drain && a2 > 0 && a1 == 0)) {
        q2_round(ver, min(a2, 32u));
      } else if (a1 >= 64 && a2 + 64u <= q2m + 1u && c.n_steps[ver] > 2) {
        q1_pair(ver);
      } else if (a1 >= 32 || (drain && a1 > 0)) {
        q1_round(ver, min(a1, 32u));
      } else {
        break;
      }
    }
  }

  // Queue this lane's survivors of one 16-byte group (mask bit j: row rel0 + j),
  // warp-wide: ballot prefix when no lane has two, else a warp scan of the counts.
  // Q1 has room for 128 more entries after a pump.
  __device__ __forceinline__ void push4(uint32_t ver, uint32_t m, uint32_t rel0, const int32_t* pf) {
    const uint32_t lanes = __ballot_sync(0xffffffffu, m != 0);
    if (!lanes) return;
    uint32_t pos, total;
    if (__any_sync(0xffffffffu, m & (m - 1u))) {
      const uint32_t cnt = __popc(m);
      uint32_t incl = cnt;
#pragma unroll
      for (uint32_t o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
      }
      total = __shfl_sync(0xffffffffu, incl, 31);
      pos = incl - cnt;
    } else {
      total = __popc(lanes);
      pos = __popc(lanes & lanemask_lt());
    }
    if (t1 - h1 + total > q1m + 1u) pump(ver, false);
    pos += t1;
    while (m) {
      const uint32_t j = __ffs(m) - 1u;
      m &= m - 1u;
      const uint32_t rr = rel0 + j;
      q1[pos++ & q1m] = rr;
      if (pf) prefetch_l2(pf + rr);
    }
    t1 += total;
  }

  // One pass over this warp's 16-byte groups rel4 + u * 32 + lane (u < U), whose
  // loaded values are v[u] (valid bit u): test every row against the first step
  // and queue the survivors.  Returns this lane's survivor count.
  template <int MODE>
  __device__ __forceinline__ uint32_t pass(uint32_t ver, const int4 (&v)[U], uint32_t valid, uint32_t rel4,
                                           const First& f, const int32_t* pf) {
    const uint8_t* fbase = (MODE == kModeDirectSmem || MODE == kModeBlockedSmem) ? bf_ptr + (f.bf.smem - bf_base)
                                                                                  : nullptr;
    uint32_t mask = 0;
    // one 16-byte group at a time keeps four slots live instead of 4U
#pragma unroll
    for (int u = 0; u < U; ++u) {
      uint32_t d[4] = {(uint32_t)v[u].x - (uint32_t)f.kmin, (uint32_t)v[u].y - (uint32_t)f.kmin,
                       (uint32_t)v[u].z - (uint32_t)f.kmin, (uint32_t)v[u].w - (uint32_t)f.kmin};
      const uint32_t mx = max(max(d[0], d[1]), max(d[2], d[3]));
      if (__any_sync(0xffffffffu, mx >= f.len)) {  // rare: reduce out-of-range keys modulo len
#pragma unroll
        for (int j = 0; j < 4; ++j)
          if (d[j] >= f.len) d[j] = (uint32_t)__umul64hi(f.fm * (uint64_t)d[j], (uint64_t)f.len);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const uint32_t sl = d[j];
        bool ok;
        if (MODE == kModeDirectSmem) {
          const uint32_t wd = reinterpret_cast<const uint32_t*>(fbase)[sl >> 5];
          ok = __funnelshift_r(wd, wd, sl) & 1u;  // rotate right: bit (sl mod 32) to bit 0
        } else if (MODE == kModeBlockedSmem) {
          const uint32_t h = bf_h1(sl);
          const uint32_t w = __funnelshift_rc(h, 0u, 32u - f.bf.log2);  // h >> (32 - log2), 0 for log2 = 0
          const uint2 wv = reinterpret_cast<const uint2*>(fbase)[w];
          ok = bf_test_word_k(wv.x, wv.y, bf_g(h), f.bf.k);
        } else if (MODE == kModeBfAny) {
          ok = bf_test(f.bf, sl, pol_keep);
        } else {
          ok = ld_slot(f.ht + sl, pol_keep).x != 0;
        }
        mask |= (ok ? 1u : 0u) << (4 * u + j);
      }
    }
    uint32_t vm = 0;
#pragma unroll
    for (int u = 0; u < U; ++u) vm |= ((valid >> u) & 1u) ? (0xFu << (4 * u)) : 0u;
    mask &= vm;
    if (__ballot_sync(0xffffffffu, mask != 0)) {
#pragma unroll
      for (int u = 0; u < U; ++u) push4(ver, (mask >> (4 * u)) & 0xFu, 4u * (rel4 + u * 32u + lane), pf);
    }
    return __popc(mask);
  }
};

// ---- fused prologue: the build of sj_build.cuh on every CTA --------------------

// Zero `bytes` (a multiple of 16) at p, grid-strided.
__device__ __forceinline__ void zero_grid(void* p, size_t bytes) {
  uint4* q = reinterpret_cast<uint4*>(p);
  const size_t n = bytes / 16u;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    q[i] = make_uint4(0u, 0u, 0u, 0u);
}

__device__ __forceinline__ size_t bf_alloc_bytes(const SjDimRt& D) {
  const size_t b = (D.bf_mode == kBfBlocked) ? ((size_t)8 << D.bf_max_log2) : (((size_t)1 << D.bf_max_log2) / 8);
  return b < 16 ? 16 : b;
}

// Returns false when a grid barrier expired.  On return every CTA's Ctl holds the
// filter layouts, group strides, the starting order and the filter placement,
// and the tables are built.  `scratch` (shared) receives the payload prefixes.
__device__ bool fused_build(const SjPlanRt& P, Ctl& c, uint32_t* scratch) {
  SjDesc* desc = P.desc;
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  // (a) zero the hash tables and filters; scan the dimensions.  The payload
  // bitmaps and desc->scan_count start at zero: the previous run left them so (or
  // the host cleared the arena).  The run's statistics start from zero here; they
  // are written only after the second barrier.
  if (blockIdx.x == 0 && tid == 0) {
    desc->rows_scanned = 0;
    desc->reorders = 0;
    desc->groups_out = 0;
    for (uint32_t p = 0; p < kMaxSteps; ++p) desc->step_in[p] = desc->step_out[p] = 0;
    for (uint32_t d = 0; d < kMaxDims; ++d) desc->bf_probes[d] = desc->bf_passes[d] = 0;
  }
  for (uint32_t d = 0; d < P.n_dims; ++d) {
    const SjDimRt& D = P.dim[d];
    zero_grid(D.ht, ((size_t)D.ht_len * 8u + 15u) & ~(size_t)15u);
    zero_grid(D.bf, bf_alloc_bytes(D));
  }
  for (uint32_t d = 0; d < P.n_dims; ++d) {
    const uint32_t cnt = dim_scan_rows(P, d, blockIdx.x, gridDim.x, &desc->error_flags);
    if (lane == 0 && cnt) atomicAdd(&c.scan_count[d], cnt);
  }
  __syncthreads();
  if (tid < P.n_dims && c.scan_count[tid]) atomicAdd(&desc->scan_count[tid], c.scan_count[tid]);
  if (!grid_barrier(desc, c)) return false;

  // (b) every CTA derives the same geometry from the counts and the bitmaps
  uint32_t poff[kMaxDims];
  {
    uint32_t o = 0;
    for (uint32_t d = 0; d < P.n_dims; ++d) {
      poff[d] = o;
      if (P.dim[d].grouped) o += (P.dim[d].payload_span + 31u) / 32u;
    }
  }
  if (tid < P.n_dims) c.inserted[tid] = ld_acquire_gpu(&desc->scan_count[tid]);
  if (warp < P.n_dims && P.dim[warp].grouped)
    warp_bitmap_prefix(P.dim[warp].payload_bitmap, (P.dim[warp].payload_span + 31u) / 32u, scratch + poff[warp],
                       &c.n_codes[warp], lane);
  __syncthreads();
  if (tid == 0) {
    for (uint32_t d = 0; d < P.n_dims; ++d) {
      const SjDimRt& D = P.dim[d];
      uint32_t l2;
      c.bf_mode[d] = bf_effective(D.bf_mode, D.bf_max_log2, D.bf_bits_per_key, c.inserted[d], P.bf_smem_budget, &l2);
      c.bf_log2[d] = l2;
      if (!D.grouped) c.n_codes[d] = 0;
    }
    c.n_groups = group_strides(P, c.n_codes, c.group_stride);
    choose_start(P, c.inserted, c.order[0], c.bf_in_smem);
  }
  __syncthreads();
  if (blockIdx.x == 0) {  // the descriptor the host reads, and the dictionaries
    if (tid < P.n_dims) {
      desc->dim[tid].n_inserted = c.inserted[tid];
      desc->dim[tid].bf_log2 = c.bf_log2[tid];
      desc->dim[tid].bf_mode = c.bf_mode[tid];
      desc->dim[tid].n_codes = c.n_codes[tid];
      desc->dim[tid].group_stride = c.group_stride[tid];
    }
    if (tid < kMaxDims) {
      desc->start_order[tid] = c.order[0][tid];
      desc->bf_smem_off[tid] = c.bf_in_smem[tid];
    }
    if (tid == 0) desc->n_groups = c.n_groups;
    for (uint32_t d = 0; d < P.n_dims; ++d)
      if (P.dim[d].grouped) write_dict(P.dim[d], scratch + poff[d], (P.dim[d].payload_span + 31u) / 32u);
  }
  // group accumulators of this run's dense groups start at zero
  zero_grid(P.g_sum, ((size_t)c.n_groups * 8u + 15u) & ~(size_t)15u);
  zero_grid(P.g_cnt, ((size_t)c.n_groups * 8u + 15u) & ~(size_t)15u);
  for (uint32_t d = 0; d < P.n_dims; ++d)
    dim_insert_rows(P, d, c.bf_mode[d], c.bf_log2[d], scratch + poff[d], blockIdx.x, gridDim.x);
  if (!grid_barrier(desc, c)) return false;

  // (c) leave the scan's inputs at zero for the next run: nothing reads the
  // payload bitmaps or the counts after the second barrier
  if (blockIdx.x == 0) {
    for (uint32_t d = 0; d < P.n_dims; ++d) {
      if (!P.dim[d].grouped) continue;
      const uint32_t words = (P.dim[d].payload_span + 31u) / 32u;
      for (uint32_t w = tid; w < words; w += blockDim.x) P.dim[d].payload_bitmap[w] = 0u;
    }
    if (tid < kMaxDims) desc->scan_count[tid] = 0u;
  }
  return true;
}

// NW scanning warps; U 16-byte groups (4U fact rows) per lane per pass.
// fused: run the build prologue and the group compaction in this launch
// (cooperative launch); else the build kernels ran before (programmatic
// dependent launch) and sj_finalize_kernel follows.
template <int NW, int U>
__global__ void __launch_bounds__(NW * 32, 1) sj_probe_kernel(const __grid_constant__ SjPlanRt P,
                                                              const __grid_constant__ SjProbeGeom G,
                                                              const uint32_t fused) {
  constexpr uint32_t NT = NW * 32;
  extern __shared__ __align__(128) uint8_t smem[];
  const SmemLayout L = probe_layout(G);
  uint8_t* bfmem = smem + L.bf_off;
  Ctl& c = *reinterpret_cast<Ctl*>(smem + L.ctl_off);
  SjDesc* desc = P.desc;
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;

  if (!fused) {
    pdl_launch_dependents();
    pdl_wait();  // the build's descriptor, hash tables and filters are complete
  }
  for (uint32_t i = tid; i < (uint32_t)sizeof(Ctl) / 4u; i += NT) reinterpret_cast<uint32_t*>(&c)[i] = 0u;
  __syncthreads();

  bool run = true;
  if (fused) {
    run = fused_build(P, c, reinterpret_cast<uint32_t*>(smem + L.q1_off));
  } else if (tid == 0) {
    for (uint32_t d = 0; d < P.n_dims; ++d) {
      c.bf_log2[d] = desc->dim[d].bf_log2;
      c.bf_mode[d] = desc->dim[d].bf_mode;
      c.group_stride[d] = desc->dim[d].group_stride;
      c.n_codes[d] = desc->dim[d].n_codes;
    }
    for (uint32_t d = 0; d < kMaxDims; ++d) {
      c.order[0][d] = desc->start_order[d];
      c.bf_in_smem[d] = desc->bf_smem_off[d];
    }
    c.n_groups = desc->n_groups;
  }

  unsigned long long* s_sum = reinterpret_cast<unsigned long long*>(smem + L.gsum_off);
  uint32_t* s_cnt = reinterpret_cast<uint32_t*>(smem + L.gcnt_off);
  const uint64_t pol_first = policy_evict_first();
  const uint64_t pol_keep = policy_evict_last();

  if (run) {
    // ---- plan steps, filters into shared memory, zero the group partials ------
    if (tid == 0) {
      for (uint32_t d = P.n_dims; d < kMaxDims; ++d) c.order[0][d] = 0u;
      for (uint32_t d = 0; d < kMaxDims; ++d) c.order[1][d] = c.order[0][d];
      c.n_steps[0] = c.n_steps[1] = make_steps(P, c.bf_mode, c.order[0], c.steps[0]);
      for (uint32_t p = 0; p < kMaxSteps; ++p) c.steps[1][p] = c.steps[0][p];
      c.groups_in_smem = c.n_groups <= G.group_smem_cap;
    }
    __syncthreads();
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
    if (c.groups_in_smem) {
      for (uint32_t g = tid; g < c.n_groups; g += NT) {
        s_sum[g] = 0ull;
        s_cnt[g] = 0u;
      }
    }
    __syncthreads();

    // ---- the scan ------------------------------------------------------------
    const uint64_t rb = P.row_begin, re = P.row_end;
    const uint64_t base_row = rb & ~3ull;
    const uint64_t body_b = (rb + 3ull) & ~3ull;                    // first row of the 16-byte groups
    const uint64_t body_e = max((uint64_t)(re & ~3ull), body_b);    // end of the 16-byte groups
    const uint32_t start4 = (uint32_t)((body_b - base_row) / 4u);
    const uint32_t end4 = (uint32_t)((body_e - base_row) / 4u);
    Warp<U> w{P, c,
              reinterpret_cast<uint32_t*>(smem + L.q1_off) + warp * G.q1_cap,
              reinterpret_cast<uint32_t*>(smem + L.q2_off) + warp * G.q2_cap,
              G.q1_cap - 1, G.q2_cap - 1, s_sum, s_cnt, smem_addr(bfmem), bfmem, base_row, pol_first, pol_keep, lane,
              0, 0, 0, 0};
    uint32_t exec_ver = 0;
    First f;
    int mode = kModeDirectSmem;
    const int32_t* pf = nullptr;
    bool is_bf = true;
    uint32_t d0 = 0;
    auto setup = [&](uint32_t ver) {
      const uint32_t st0 = c.steps[ver][0];
      d0 = st0 & 15u;
      const SjDimRt& D = P.dim[d0];
      f.fk = D.fact_fk;
      f.col4 = reinterpret_cast<const int4*>(D.fact_fk + base_row);
      f.ht = D.ht;
      f.kmin = D.key_min;
      f.len = D.ht_len;
      f.fm = D.fastmod_m;
      f.bf = w.bfview(d0);
      is_bf = (st0 >> 4) == kStepBF;
      mode = !is_bf ? kModePht
                    : (!f.bf.smem ? kModeBfAny : (f.bf.mode == kBfDirect ? kModeDirectSmem : kModeBlockedSmem));
      pf = nullptr;
      if (c.n_steps[ver] > 1) {
        const uint32_t d1 = c.steps[ver][1] & 15u;
        if (d1 != d0) pf = P.dim[d1].fact_fk + base_row;
      }
    };
    setup(0);

    // rows outside the 16-byte groups (at most 3 at each end): warp 0 of CTA 0
    if (blockIdx.x == 0 && warp == 0) {
      const uint64_t head_e = min(body_b, re), tail_b = max((uint64_t)(re & ~3ull), body_b);
      uint64_t row = 0;
      bool have = false;
      if (lane < 3) {
        row = rb + lane;
        have = row < head_e;
      } else if (lane < 6) {
        row = tail_b + (lane - 3);
        have = row < re;
      }
      bool ok = false;
      if (have) {
        const uint32_t sl = slot_fast(ld_stream(f.fk + row, pol_first), f.kmin, f.len, f.fm);
        ok = is_bf ? bf_test(f.bf, sl, pol_keep) : (ld_slot(f.ht + sl, pol_keep).x != 0);
      }
      const uint32_t hm = __ballot_sync(0xffffffffu, have), pm = __ballot_sync(0xffffffffu, ok);
      if (ok) {
        const uint32_t rel = (uint32_t)(row - base_row);
        w.q1[(w.t1 + __popc(pm & lanemask_lt())) & w.q1m] = rel;
        if (pf) prefetch_l2(pf + rel);
      }
      w.t1 += __popc(pm);
      if (lane == 0 && hm) {
        atomicAdd(&c.rows_scanned, (uint32_t)__popc(hm));
        atomicAdd(&c.step_in[0], (uint32_t)__popc(hm));
        atomicAdd(&c.step_out[0], (uint32_t)__popc(pm));
        if (is_bf) {
          atomicAdd(&c.probes[d0], (uint32_t)__popc(hm));
          atomicAdd(&c.passes[d0], (uint32_t)__popc(pm));
        }
      }
    }

    const uint32_t gw = blockIdx.x * NW + warp;
    const uint32_t stride4 = gridDim.x * NW * 32u * U;
    const bool adaptive = P.lip && P.adaptive && P.n_dims > 1;
    uint32_t passes_done = 0;
    for (uint32_t rel4 = start4 + gw * 32u * U;; rel4 += stride4) {
      // lane 0 may have just re-ranked: every lane takes its view of the version
      const uint32_t cv = __shfl_sync(0xffffffffu, ld_volatile_u32(&c.ver), 0);
      if (cv != exec_ver) {  // a new filter order: drain the queues under the old one
        __threadfence_block();
        w.pump(exec_ver, true);
        exec_ver = cv;
        if (lane == 0) c.warp_ver[warp] = cv;
        setup(cv);
      }
      if (rel4 >= end4) break;
      int4 v[U];
      uint32_t valid = 0;
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const uint32_t i4 = rel4 + u * 32u + lane;
        const bool ok = i4 < end4;
        v[u] = ok ? ldg4_stream(f.col4 + i4, pol_first) : make_int4(f.kmin, f.kmin, f.kmin, f.kmin);
        valid |= (ok ? 1u : 0u) << u;
      }
      uint32_t passed;
      if (mode == kModeDirectSmem) passed = w.template pass<kModeDirectSmem>(exec_ver, v, valid, rel4, f, pf);
      else if (mode == kModeBlockedSmem) passed = w.template pass<kModeBlockedSmem>(exec_ver, v, valid, rel4, f, pf);
      else if (mode == kModeBfAny) passed = w.template pass<kModeBfAny>(exec_ver, v, valid, rel4, f, pf);
      else passed = w.template pass<kModePht>(exec_ver, v, valid, rel4, f, pf);
      const uint32_t rows = __reduce_add_sync(0xffffffffu, 4u * __popc(valid));
      const uint32_t outs = __reduce_add_sync(0xffffffffu, passed);
      if (lane == 0) {
        atomicAdd(&c.rows_scanned, rows);
        atomicAdd(&c.step_in[0], rows);
        atomicAdd(&c.step_out[0], outs);
        if (is_bf) {
          atomicAdd(&c.probes[d0], rows);
          atomicAdd(&c.passes[d0], outs);
        }
      }
      w.pump(exec_ver, false);
      ++passes_done;
      // adaptive re-ranking, by warp 0 for the CTA, once every warp runs the
      // current order (so the version about to be rewritten is in no warp's use)
      if (adaptive && warp == 0 && lane == 0 && (passes_done == 8 || passes_done % G.reorder_period == 0)) {
        const uint32_t cur = c.ver;
        bool settled = true;
        for (uint32_t x = 0; x < NW; ++x) settled = settled && ld_volatile_u32(&c.warp_ver[x]) == cur;
        if (settled) {
          float rate[kMaxDims];
          for (uint32_t d = 0; d < kMaxDims; ++d) {
            const float pr = (float)ld_volatile_u32(&c.probes[d]);
            const float pa = (float)ld_volatile_u32(&c.passes[d]);
            rate[d] = (d < P.n_dims) ? (pa + 1.f) / (pr + 2.f) : 1.f;
          }
          float weight[kMaxDims];
          for (uint32_t d = 0; d < kMaxDims; ++d) weight[d] = (c.bf_in_smem[d] == ~0u) ? kL2TestCost : 1.f;
          uint32_t cand[kMaxDims];
          const uint32_t* ord = c.order[cur];
          for (uint32_t d = 0; d < P.n_dims; ++d) cand[d] = ord[d];
          for (uint32_t a = 1; a < P.n_dims; ++a)
            for (uint32_t b = a; b > 0 && rate[cand[b]] < rate[cand[b - 1]]; --b) {
              const uint32_t t = cand[b];
              cand[b] = cand[b - 1];
              cand[b - 1] = t;
            }
          if (order_cost(rate, weight, cand, P.n_dims) < 0.9f * order_cost(rate, weight, ord, P.n_dims)) {
            const uint32_t nv = cur ^ 1u;
            for (uint32_t d = 0; d < kMaxDims; ++d) c.order[nv][d] = (d < P.n_dims) ? cand[d] : 0u;
            c.n_steps[nv] = make_steps(P, c.bf_mode, c.order[nv], c.steps[nv]);
            c.reorders++;
            __threadfence_block();
            *reinterpret_cast<volatile uint32_t*>(&c.ver) = nv;
          }
        }
      }
    }
    w.pump(exec_ver, true);
    __syncthreads();

    // ---- flush group partials and counters ----------------------------------
    if (c.groups_in_smem) {
      for (uint32_t g = tid; g < c.n_groups; g += NT) {
        const uint32_t cnt = s_cnt[g];
        if (cnt) {
          atomicAdd(&P.g_sum[g], s_sum[g]);
          atomicAdd(&P.g_cnt[g], (unsigned long long)cnt);
        }
      }
    }
    if (tid == 0) {
      atomicAdd(&desc->rows_scanned, (unsigned long long)c.rows_scanned);
      for (uint32_t p = 0; p < kMaxSteps; ++p) {
        if (c.step_in[p]) atomicAdd(&desc->step_in[p], (unsigned long long)c.step_in[p]);
        if (c.step_out[p]) atomicAdd(&desc->step_out[p], (unsigned long long)c.step_out[p]);
      }
      for (uint32_t d = 0; d < P.n_dims; ++d) {
        if (c.probes[d]) atomicAdd(&desc->bf_probes[d], (unsigned long long)c.probes[d]);
        if (c.passes[d]) atomicAdd(&desc->bf_passes[d], (unsigned long long)c.passes[d]);
      }
      if (c.reorders) atomicAdd(&desc->reorders, (unsigned long long)c.reorders);
    }
  }
  if (!fused || !grid_barrier(desc, c)) return;

  // ---- fused: compact the non-empty groups into result rows ------------------
  for (uint32_t g = blockIdx.x * NT + tid; g < c.n_groups; g += gridDim.x * NT) {
    const unsigned long long cnt = P.g_cnt[g];
    if (!cnt) continue;
    const uint32_t pos = atomicAdd(&desc->groups_out, 1u);
    sj_group_row r;
    for (uint32_t d = 0; d < kMaxDims; ++d) {
      r.attr[d] = 0;
      if (d < P.n_dims && P.dim[d].grouped) {
        const uint32_t n = c.n_codes[d] ? c.n_codes[d] : 1u;
        r.attr[d] = P.dim[d].dict[(g / c.group_stride[d]) % n];
      }
    }
    r.count = cnt;
    r.sum = P.g_sum[g];
    P.rows_out[pos] = r;
  }
}

// Compact the non-empty groups into result rows, decoding dictionary codes back
// to payload values (after a probe launched without `fused`).
__global__ void __launch_bounds__(256) sj_finalize_kernel(const __grid_constant__ SjPlanRt P) {
  pdl_wait();  // the probe's group sums are complete
  SjDesc* desc = P.desc;
  const uint32_t n_groups = desc->n_groups;
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < n_groups; g += gridDim.x * blockDim.x) {
    const unsigned long long cnt = P.g_cnt[g];
    if (!cnt) continue;
    const uint32_t pos = atomicAdd(&desc->groups_out, 1u);
    sj_group_row r;
    for (uint32_t d = 0; d < kMaxDims; ++d) {
      r.attr[d] = 0;
      if (d < P.n_dims && P.dim[d].grouped) {
        const uint32_t n = desc->dim[d].n_codes ? desc->dim[d].n_codes : 1u;
        const uint32_t code = (g / desc->dim[d].group_stride) % n;
        r.attr[d] = P.dim[d].dict[code];
      }
    }
    r.count = cnt;
    r.sum = P.g_sum[g];
    P.rows_out[pos] = r;
  }
}

// ---- host-side launchers ---------------------------------------------------
uint32_t probe_smem_bytes(const SjProbeGeom& g) { return probe_layout(g).total; }

template <int NW, int U>
static cudaError_t launch_probe_t(const SjPlanRt& P, const SjProbeGeom& G, uint32_t smem, cudaStream_t st,
                                  const L2Window& w, bool pdl, bool fused) {
  cudaError_t e = cudaFuncSetAttribute(sj_probe_kernel<NW, U>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  if (fused)
    return launch_cooperative(sj_probe_kernel<NW, U>, dim3(G.grid), dim3(NW * 32), smem, st, w, P, G, 1u);
  return launch_windowed(sj_probe_kernel<NW, U>, dim3(G.grid), dim3(NW * 32), smem, st, w, pdl, P, G, 0u);
}

// G.threads = 32 * scanning warps; G.rows_per_lane = 4 * U; w: L2 window over
// the query's hash tables and filters (may be empty); pdl: the previous kernel of
// the stream is the build's sj_dim_insert (programmatic dependent launch);
// fused: build, probe and compaction in this one cooperative launch.
cudaError_t launch_probe(const SjPlanRt& P, const SjProbeGeom& G, cudaStream_t st, const L2Window& w, bool pdl,
                         bool fused) {
  const uint32_t smem = probe_layout(G).total;
  const uint32_t nw = G.threads / 32;
#define SJ_CASE(W, R) \
  if (nw == W && G.rows_per_lane == R) return launch_probe_t<W, R / 4>(P, G, smem, st, w, pdl, fused);
  SJ_CASE(16, 8)
  SJ_CASE(16, 16)
  SJ_CASE(24, 8)
  SJ_CASE(24, 16)
  SJ_CASE(32, 8)
  SJ_CASE(32, 16)
#undef SJ_CASE
  return cudaErrorInvalidValue;
}

static bool probe_shape_built(uint32_t threads, uint32_t rows_per_lane) {
  return (threads == 512 || threads == 768 || threads == 1024) && (rows_per_lane == 8 || rows_per_lane == 16);
}

// Probe geometry from a plan's tuning (zero fields take the defaults): 1,024
// threads, 16 rows per lane per pass, one CTA per SM, and the shared memory the
// queues and group partials leave -- up to 192 KB -- for filters.
// prefix_words: payload-bitmap words of the grouped dimensions (fused build).
// Returns an error text, or nullptr.
const char* make_probe_geom(const sj_tuning& t, uint32_t sm_count, size_t smem_optin, uint32_t prefix_words,
                            SjProbeGeom* out) {
  SjProbeGeom g;
  memset(&g, 0, sizeof(g));
  g.threads = t.threads ? (uint32_t)t.threads : 1024u;
  g.rows_per_lane = t.compact_threshold ? (uint32_t)t.compact_threshold : 16u;
  if (!probe_shape_built(g.threads, g.rows_per_lane))
    return "probe shape not built (threads 512/768/1024, 8 or 16 rows per lane)";
  if (t.ctas_per_sm > 1) return "the probe runs one CTA per SM";
  g.grid = sm_count;
  g.group_smem_cap = 1024;
  g.q1_cap = 256;  // a push queues at most 128 rows, after a pump leaves fewer than 32
  g.q2_cap = 128;  // room for a two-survivors-per-lane Q1 round (64) over a partial Q2
  g.reorder_period = 16;
  g.prefix_words = prefix_words;
  g.bf_smem_bytes = 0;
  const uint32_t base = probe_layout(g).total;
  if (base > smem_optin) return "queues and group partials exceed the device's shared memory";
  uint32_t room = (uint32_t)((smem_optin - base) & ~(size_t)127);
  if (room > 192u * 1024u) room = 192u * 1024u;
  g.bf_smem_bytes = t.bf_smem_bytes > 0 ? std::min<uint32_t>((uint32_t)t.bf_smem_bytes, room) : room;
  g.bf_smem_bytes &= ~15u;
  g.smem_bytes = probe_layout(g).total;
  if (g.smem_bytes > smem_optin) return "probe shared memory exceeds the device limit";
  *out = g;
  return nullptr;
}

// pdl: the previous kernel of the stream is the probe (programmatic dependent launch).
cudaError_t launch_finalize(const SjPlanRt& P, uint32_t group_capacity, cudaStream_t st, bool pdl) {
  uint32_t blocks = (group_capacity + 255) / 256;
  if (blocks > 1184) blocks = 1184;
  if (blocks < 1) blocks = 1;
  return launch_windowed(sj_finalize_kernel, dim3(blocks), dim3(256), 0, st, L2Window{}, pdl, P);
}

}  // namespace sj
