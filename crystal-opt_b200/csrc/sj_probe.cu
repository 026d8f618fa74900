// sj_probe.cu -- the fused star-join probe: fact scan -> LIP Bloom filters -> PHT
// probes -> group-by SUM, one persistent kernel per query.
//
// Replaces the reference's probe<128,4> kernels (src/ssb-jo/q33/0-lip.cu:28-112,
// src/ssb-jo/q33/0-naive.cu:28-91, src/ssb-jo/q41/0-lip.cu:28-131).  Same answer,
// different machine mapping:
//   * Persistent grid (a multiple of the SM count).  Each CTA walks fact chunks
//     round-robin.  Only the column tested first is read densely: its chunk is
//     streamed by a CTA-local TMA bulk copy (cp.async.bulk, no multicast) into a
//     ring of shared-memory stages, each completing on its own mbarrier.
//   * Filters are evaluated on the PHT slot of each key; the filters that fit the
//     budget are copied into shared memory once per CTA.
//   * Survivors of the first test are compacted (warp ballot + popc, one shared
//     atomic per warp) into ring queue Q1 with their row and slot.  Later columns
//     are read only at survivor rows (sector-sparse reads, prefetched into L2 at
//     enqueue time).  Survivors of the second test are compacted again into Q2;
//     the remaining tests, the PHT probes and the aggregate run densely on Q2.
//     Queue tails are monotonic counters read back after the sub-block barrier,
//     so every thread holds the same head/tail values in registers and queue
//     decisions need no extra barrier.
//   * Group partials (dense dictionary codes) live in shared memory and are
//     flushed once per CTA with 64-bit atomics; group spaces that do not fit
//     aggregate straight into global memory.
//   * Adaptive LIP: each CTA counts probes/passes per filter and re-ranks the
//     filter order every few chunks.  A new order applies to chunks issued after
//     the decision; queues are drained before the first chunk of the new order is
//     consumed, so the result never depends on the order, only the work does.
#include "sj_internal.h"
#include "sj_ptx.cuh"

namespace sj {

enum : uint32_t { kStepBF = 0, kStepPHT = 1 };

struct SmemLayout {
  uint32_t stage_off, bar_off, bf_off, q1_row_off, q1_val_off, q2_row_off, q2_v0_off, q2_v1_off, gsum_off,
      gcnt_off, ctl_off, total;
};

struct Ctl {
  uint32_t cnt1[2], cnt2[2];      // monotonic append counters (double-buffered)
  uint32_t abort;
  uint32_t issue_ver;
  uint32_t n_steps[2];
  uint32_t steps[2][kMaxSteps];  // (dim | kind << 4)
  uint32_t order[2][kMaxDims];
  uint32_t stage_ver[16];
  uint32_t bf_in_smem[kMaxDims];  // byte offset within the filter region, or ~0u
  uint32_t bf_log2[kMaxDims];
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
  SmemLayout L;
  uint32_t o = 0;
  L.stage_off = o;
  o += g.stages * g.chunk_rows * 4u;
  o = align_up(o, 16);
  L.bar_off = o;
  o += g.stages * 8u;
  o = align_up(o, 16);
  L.bf_off = o;
  o += g.bf_smem_bytes;
  o = align_up(o, 16);
  L.q1_row_off = o;
  o += g.q1_cap * 4u;
  L.q1_val_off = o;
  o += g.q1_cap * 4u;
  L.q2_row_off = o;
  o += g.q2_cap * 4u;
  L.q2_v0_off = o;
  o += g.q2_cap * 4u;
  L.q2_v1_off = o;
  o += g.q2_cap * 4u;
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
__device__ inline uint32_t make_steps(const SjPlanRt& P, const uint32_t* order, uint32_t* steps) {
  uint32_t n = 0;
  if (P.lip) {
    for (uint32_t p = 0; p < P.n_dims; ++p) steps[n++] = order[p] | (kStepBF << 4);
    for (uint32_t p = 0; p < P.n_dims; ++p) {
      const SjDimRt& D = P.dim[order[p]];
      if (D.grouped || D.bf_mode != kBfDirect) steps[n++] = order[p] | (kStepPHT << 4);
    }
  } else {
    for (uint32_t p = 0; p < P.n_dims; ++p) steps[n++] = order[p] | (kStepPHT << 4);
  }
  return n;
}

// Expected filter tests per row of an order under the observed pass rates.
__device__ inline float order_cost(const float* rate, const uint32_t* order, uint32_t n) {
  float c = 0.f, live = 1.f;
  for (uint32_t p = 0; p < n; ++p) {
    c += live;
    live *= rate[order[p]];
  }
  return c;
}

struct Probe {
  const SjPlanRt& P;
  const SjProbeGeom& G;
  Ctl& c;
  uint32_t* q1_row;
  int32_t* q1_val;
  uint32_t* q2_row;
  int32_t* q2_v0;
  int32_t* q2_v1;
  unsigned long long* s_sum;
  uint32_t* s_cnt;
  BfView bf[kMaxDims];
  uint64_t base_row;  // row of queue offset 0 (row_begin rounded down to 4)
  uint64_t pol_first, pol_keep;
  // queue state, identical in every thread of the CTA
  uint32_t t1, h1, t2, h2;
  uint32_t seen1[2], seen2[2];
  uint32_t b1, b2;

  __device__ __forceinline__ uint32_t slot_at(uint32_t d, uint32_t rel) const {
    const SjDimRt& D = P.dim[d];
    return slot_of(ld_stream(D.fact_fk + base_row + rel, pol_first), D.key_min, D.ht_len, D.fastmod_m);
  }

  __device__ void aggregate(uint32_t rel, const uint32_t* cv) {
    uint32_t g = 0;
#pragma unroll
    for (uint32_t d = 0; d < kMaxDims; ++d)
      if (d < P.n_dims && P.dim[d].grouped) g += cv[d] * c.group_stride[d];
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

  // Restore what steps [0, upto) produced: a slot (filter step) or a code (PHT step).
  __device__ __forceinline__ void load_state(uint32_t ver, uint32_t upto, int32_t v0, int32_t v1, uint32_t& have,
                                             uint32_t* sv, uint32_t* cv) {
    have = 0;
#pragma unroll
    for (uint32_t p = 0; p < 2; ++p) {
      if (p >= upto) break;
      const uint32_t st = c.steps[ver][p];
      const uint32_t d = st & 15u;
      const uint32_t v = (uint32_t)(p ? v1 : v0);
      if ((st >> 4) == kStepBF) sv[d] = v;
      else cv[d] = v;
      have |= 1u << d;
    }
  }

  // Steps [2, n) for one Q2 survivor, then the aggregate.
  __device__ void finish_row(uint32_t ver, uint32_t rel, uint32_t have, uint32_t* sv, uint32_t* cv) {
    const uint32_t n = c.n_steps[ver];
    for (uint32_t p = 2; p < n; ++p) {
      const uint32_t st = c.steps[ver][p];
      const uint32_t d = st & 15u;
      atomicAdd(&c.step_in[p], 1u);
      if (!((have >> d) & 1u)) {
        sv[d] = slot_at(d, rel);
        have |= 1u << d;
      }
      if ((st >> 4) == kStepBF) {
        atomicAdd(&c.probes[d], 1u);
        if (!bf_test(bf[d], sv[d], pol_keep)) return;
        atomicAdd(&c.passes[d], 1u);
      } else {
        const int2 e = ld_slot(P.dim[d].ht + sv[d], pol_keep);
        if (e.x == 0) return;
        cv[d] = (uint32_t)e.y;
      }
      atomicAdd(&c.step_out[p], 1u);
    }
    aggregate(rel, cv);
  }

  // Q1 entries [h1, h1 + cnt): step 1, then aggregate (plans of <= 2 steps) or
  // compact the survivors into Q2.  Called by every thread with the same cnt.
  __device__ void q1_round(uint32_t ver, uint32_t cnt) {
    const uint32_t tid = threadIdx.x, lane = tid & 31u;
    const uint32_t n = c.n_steps[ver];
    const uint32_t st0 = c.steps[ver][0], st1 = c.steps[ver][n > 1 ? 1 : 0];
    const uint32_t d0 = st0 & 15u, d1 = st1 & 15u;
    bool pass = false;
    uint32_t rel = 0;
    int32_t v0 = 0, v1 = 0;
    if (tid < cnt) {
      const uint32_t e = (h1 + tid) & (G.q1_cap - 1);
      rel = q1_row[e];
      v0 = q1_val[e];
      if (n == 1) {
        pass = true;
      } else {
        const uint32_t s1 = (d1 == d0 && (st0 >> 4) == kStepBF) ? (uint32_t)v0 : slot_at(d1, rel);
        if ((st1 >> 4) == kStepBF) {
          pass = bf_test(bf[d1], s1, pol_keep);
          v1 = (int32_t)s1;
        } else {
          const int2 e2 = ld_slot(P.dim[d1].ht + s1, pol_keep);
          pass = e2.x != 0;
          v1 = e2.y;
        }
      }
    }
    const uint32_t mo = __ballot_sync(0xffffffffu, pass);
    if (n <= 2) {
      if (pass) {
        uint32_t sv[kMaxDims] = {0, 0, 0, 0}, cv[kMaxDims] = {0, 0, 0, 0}, have;
        load_state(ver, n, v0, v1, have, sv, cv);
        aggregate(rel, cv);
      }
      if (n == 2 && lane == 0 && mo) atomicAdd(&c.step_out[1], (uint32_t)__popc(mo));
    } else {
      uint32_t base = 0;
      if (lane == 0 && mo) base = atomicAdd(&c.cnt2[b2], (uint32_t)__popc(mo));
      base = __shfl_sync(0xffffffffu, base, 0);
      if (pass) {
        const uint32_t e = (t2 + (base - seen2[b2]) + __popc(mo & lanemask_lt())) & (G.q2_cap - 1);
        q2_row[e] = rel;
        q2_v0[e] = v0;
        q2_v1[e] = v1;
        // the column the next step reads at this row
        const uint32_t d2 = c.steps[ver][2] & 15u;
        if (d2 != d0 && d2 != d1) prefetch_l2(P.dim[d2].fact_fk + base_row + rel);
      }
    }
    __syncthreads();
    if (n > 2) {
      const uint32_t cur = ld_volatile_u32(&c.cnt2[b2]);
      const uint32_t added = cur - seen2[b2];
      t2 += added;
      seen2[b2] = cur;
      b2 ^= 1u;
      if (tid == 0) c.step_out[1] += added;
    }
    if (tid == 0 && n > 1) {
      c.step_in[1] += cnt;
      if ((st1 >> 4) == kStepBF) c.probes[d1] += cnt;
    }
    if (n > 1 && (st1 >> 4) == kStepBF && lane == 0 && mo) atomicAdd(&c.passes[d1], (uint32_t)__popc(mo));
    h1 += cnt;
  }

  __device__ void q2_round(uint32_t ver, uint32_t cnt) {
    const uint32_t tid = threadIdx.x;
    if (tid < cnt) {
      const uint32_t e = (h2 + tid) & (G.q2_cap - 1);
      uint32_t sv[kMaxDims] = {0, 0, 0, 0}, cv[kMaxDims] = {0, 0, 0, 0}, have;
      load_state(ver, 2, q2_v0[e], q2_v1[e], have, sv, cv);
      finish_row(ver, q2_row[e], have, sv, cv);
    }
    __syncthreads();
    h2 += cnt;
  }

  // Run queue rounds: full rounds only while streaming, everything when draining.
  __device__ void pump(uint32_t ver, bool drain) {
    const uint32_t nt = blockDim.x;
    for (;;) {
      const uint32_t a1 = t1 - h1, a2 = t2 - h2;
      if (a2 >= nt || (drain && a2 > 0 && a1 == 0)) {
        q2_round(ver, min(a2, nt));
      } else if (a1 >= nt || (drain && a1 > 0)) {
        q1_round(ver, min(a1, nt));
      } else {
        break;
      }
    }
  }
};

// NT threads per CTA; RPT fact rows per thread per sub-block (multiple of 4).
template <int NT, int RPT>
__global__ void __launch_bounds__(NT, 1) sj_probe_kernel(const __grid_constant__ SjPlanRt P,
                                                         const __grid_constant__ SjProbeGeom G) {
  static_assert(RPT % 4 == 0, "rows per thread must be a multiple of 4");
  constexpr uint32_t SB = NT * RPT;  // rows per sub-block
  extern __shared__ __align__(128) uint8_t smem[];
  const SmemLayout L = probe_layout(G);
  int32_t* stage = reinterpret_cast<int32_t*>(smem + L.stage_off);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + L.bar_off);
  uint8_t* bfmem = smem + L.bf_off;
  Ctl& c = *reinterpret_cast<Ctl*>(smem + L.ctl_off);
  const SjDesc* desc = P.desc;
  const uint32_t tid = threadIdx.x, lane = tid & 31u;
  const uint32_t S = G.stages, CH = G.chunk_rows;

  const uint64_t base_row = P.row_begin & ~3ull;
  const uint64_t span = P.row_end - base_row;
  const uint32_t n_chunks = (uint32_t)((span + CH - 1) / CH);

  // ---- setup (thread 0): plan steps, filter placement, mbarriers ----------
  if (tid == 0) {
    memset(&c, 0, sizeof(Ctl));
    for (uint32_t d = 0; d < kMaxDims; ++d) c.order[0][d] = c.order[1][d] = P.order[d];
    c.n_steps[0] = c.n_steps[1] = make_steps(P, P.order, c.steps[0]);
    for (uint32_t p = 0; p < kMaxSteps; ++p) c.steps[1][p] = c.steps[0][p];
    uint32_t used = 0;
    for (uint32_t p = 0; p < P.n_dims; ++p) {
      const uint32_t d = P.order[p];
      const SjDimRt& D = P.dim[d];
      const uint32_t l2 = desc->dim[d].bf_log2;
      c.bf_log2[d] = l2;
      const uint32_t bytes = (D.bf_mode == kBfDirect) ? max(8u, (1u << l2) / 8u) : (8u << l2);
      if (P.lip && used + bytes <= G.bf_smem_bytes) {
        c.bf_in_smem[d] = used;
        used += align_up(bytes, 16);
      } else {
        c.bf_in_smem[d] = ~0u;
      }
    }
    for (uint32_t d = 0; d < P.n_dims; ++d) c.group_stride[d] = desc->dim[d].group_stride;
    c.n_groups = desc->n_groups;
    c.groups_in_smem = c.n_groups <= G.group_smem_cap;
    for (uint32_t s = 0; s < S; ++s) mbar_init(&bar[s], 1);
    mbar_fence_init();
  }
  __syncthreads();

  // ---- copy filters into shared memory, zero group partials ---------------
  for (uint32_t d = 0; d < P.n_dims; ++d) {
    if (c.bf_in_smem[d] == ~0u) continue;
    const SjDimRt& D = P.dim[d];
    const uint32_t bytes = (D.bf_mode == kBfDirect) ? max(8u, (1u << c.bf_log2[d]) / 8u) : (8u << c.bf_log2[d]);
    if (bytes >= 16u) {
      const uint4* src = reinterpret_cast<const uint4*>(D.bf);
      uint4* dst = reinterpret_cast<uint4*>(bfmem + c.bf_in_smem[d]);
      for (uint32_t i = tid; i < bytes / 16u; i += NT) dst[i] = src[i];
    } else if (tid == 0) {
      *reinterpret_cast<uint2*>(bfmem + c.bf_in_smem[d]) = *reinterpret_cast<const uint2*>(D.bf);
    }
  }
  Probe pr{P, G, c,
           reinterpret_cast<uint32_t*>(smem + L.q1_row_off),
           reinterpret_cast<int32_t*>(smem + L.q1_val_off),
           reinterpret_cast<uint32_t*>(smem + L.q2_row_off),
           reinterpret_cast<int32_t*>(smem + L.q2_v0_off),
           reinterpret_cast<int32_t*>(smem + L.q2_v1_off),
           reinterpret_cast<unsigned long long*>(smem + L.gsum_off),
           reinterpret_cast<uint32_t*>(smem + L.gcnt_off)};
  if (c.groups_in_smem) {
    for (uint32_t g = tid; g < c.n_groups; g += NT) {
      pr.s_sum[g] = 0ull;
      pr.s_cnt[g] = 0u;
    }
  }
#pragma unroll
  for (uint32_t d = 0; d < kMaxDims; ++d) {
    pr.bf[d].mode = kBfDirect;
    pr.bf[d].k = 1;
    pr.bf[d].log2 = 0;
    pr.bf[d].gptr = nullptr;
    pr.bf[d].smem = 0;
    if (d < P.n_dims) {
      const SjDimRt& D = P.dim[d];
      pr.bf[d].mode = D.bf_mode;
      pr.bf[d].k = D.bf_k;
      pr.bf[d].log2 = c.bf_log2[d];
      pr.bf[d].gptr = D.bf;
      pr.bf[d].smem = (c.bf_in_smem[d] == ~0u) ? 0u : smem_addr(bfmem + c.bf_in_smem[d]);
    }
  }
  pr.base_row = base_row;
  pr.pol_first = policy_evict_first();
  pr.pol_keep = policy_evict_last();
  pr.t1 = pr.h1 = pr.t2 = pr.h2 = 0;
  pr.seen1[0] = pr.seen1[1] = pr.seen2[0] = pr.seen2[1] = 0;
  pr.b1 = pr.b2 = 0;
  __syncthreads();

  // ---- TMA producer (thread 0) --------------------------------------------
  const uint32_t my_iters = (blockIdx.x < n_chunks) ? (n_chunks - blockIdx.x + gridDim.x - 1) / gridDim.x : 0u;
  uint32_t issued = 0;  // meaningful in thread 0
  auto issue = [&](uint32_t it) {
    const uint32_t s = it % S;
    const uint32_t chunk = blockIdx.x + it * gridDim.x;
    const uint32_t ver = c.issue_ver;
    const uint32_t d = c.order[ver][0];
    c.stage_ver[s] = ver;
    const uint64_t start = base_row + (uint64_t)chunk * CH;
    const uint64_t rows = min((uint64_t)CH, P.row_end - start);
    const uint32_t bytes = (uint32_t)(rows & ~3ull) * 4u;
    fence_proxy_async_smem();
    if (bytes) {
      mbar_arrive_expect_tx(&bar[s], bytes);
      bulk_g2s(stage + (size_t)s * CH, P.dim[d].fact_fk + start, bytes, &bar[s], pr.pol_first);
    } else {
      mbar_arrive(&bar[s]);
    }
  };
  if (tid == 0) {
    for (; issued < S && issued < my_iters; ++issued) issue(issued);
  }

  // ---- main loop -----------------------------------------------------------
  uint32_t exec_ver = 0;
  uint32_t it = 0;
  for (; it < my_iters; ++it) {
    const uint32_t s = it % S;
    const uint32_t chunk = blockIdx.x + it * gridDim.x;
    if (!mbar_wait_bounded(&bar[s], (it / S) & 1u, kMaxPolls)) c.abort = 1;
    __syncthreads();
    if (c.abort) break;
    const uint32_t sver = c.stage_ver[s];
    if (sver != exec_ver) {
      // first chunk of a new filter order: drain the queues under the old one
      pr.pump(exec_ver, true);
      exec_ver = sver;
    }
    const uint32_t ver = exec_ver;
    const uint32_t st0 = c.steps[ver][0];
    const uint32_t d0 = st0 & 15u;
    const SjDimRt& D0 = P.dim[d0];
    const BfView f0 = pr.bf[d0];
    const bool is_bf = (st0 >> 4) == kStepBF;
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
    const uint32_t t1_before = pr.t1;

    for (uint32_t sb = 0; sb < CH; sb += SB) {
      bool pass[RPT];
      int32_t val[RPT];
#pragma unroll
      for (uint32_t k = 0; k < RPT / 4; ++k) {
        const uint32_t r4 = sb + (k * NT + tid) * 4u;  // first row of this int4
        int4 v = *reinterpret_cast<const int4*>(sbuf + r4);
        int32_t fk[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (uint32_t j = 0; j < 4; ++j) {
          const uint32_t r = r4 + j;
          const bool valid = (r < crows) && (r >= skip);
          if (valid && r >= tma_rows) fk[j] = ld_stream(D0.fact_fk + cstart + r, pr.pol_first);
          const uint32_t sl = slot_of(fk[j], D0.key_min, D0.ht_len, D0.fastmod_m);
          bool ok;
          int32_t vv;
          if (is_bf) {
            ok = valid && bf_test(f0, sl, pr.pol_keep);
            vv = (int32_t)sl;
          } else {
            int2 e = valid ? ld_slot(D0.ht + sl, pr.pol_keep) : make_int2(0, 0);
            ok = e.x != 0;
            vv = e.y;
          }
          pass[k * 4 + j] = ok;
          val[k * 4 + j] = vv;
        }
      }
      uint32_t m[RPT], tot = 0;
#pragma unroll
      for (uint32_t j = 0; j < RPT; ++j) {
        m[j] = __ballot_sync(0xffffffffu, pass[j]);
        tot += __popc(m[j]);
      }
      uint32_t base = 0;
      if (lane == 0 && tot) base = atomicAdd(&c.cnt1[pr.b1], tot);
      base = __shfl_sync(0xffffffffu, base, 0);
      uint32_t pos = pr.t1 + (base - pr.seen1[pr.b1]);
      const uint32_t lt = lanemask_lt();
#pragma unroll
      for (uint32_t j = 0; j < RPT; ++j) {
        if (pass[j]) {
          const uint32_t rrow = rel0 + sb + ((j / 4) * NT + tid) * 4u + (j & 3u);
          const uint32_t e = (pos + __popc(m[j] & lt)) & (G.q1_cap - 1);
          pr.q1_row[e] = rrow;
          pr.q1_val[e] = val[j];
          if (pf) prefetch_l2(pf + rrow);
        }
        pos += __popc(m[j]);
      }
      __syncthreads();  // entries visible; counter final for this sub-block
      const uint32_t cur = ld_volatile_u32(&c.cnt1[pr.b1]);
      pr.t1 += cur - pr.seen1[pr.b1];
      pr.seen1[pr.b1] = cur;
      pr.b1 ^= 1u;
      pr.pump(ver, false);
    }
    // The stage has been read by every thread (barrier in the last sub-block).
    if (tid == 0) {
      const uint32_t valid_rows = crows - skip;
      const uint32_t passed = pr.t1 - t1_before;
      c.rows_scanned += valid_rows;
      c.step_in[0] += valid_rows;
      c.step_out[0] += passed;
      if (is_bf) {
        c.probes[d0] += valid_rows;
        c.passes[d0] += passed;
      }
      // adaptive re-ranking of the filter order
      if (P.lip && P.adaptive && P.n_dims > 1 && exec_ver == c.issue_ver && ((it + 1) % G.reorder_period) == 0) {
        float rate[kMaxDims];
        for (uint32_t d = 0; d < kMaxDims; ++d)
          rate[d] = (d < P.n_dims) ? ((float)c.passes[d] + 1.f) / ((float)c.probes[d] + 2.f) : 1.f;
        uint32_t cand[kMaxDims];
        const uint32_t* cur = c.order[c.issue_ver];
        for (uint32_t d = 0; d < P.n_dims; ++d) cand[d] = cur[d];
        for (uint32_t a = 1; a < P.n_dims; ++a)  // insertion sort by rate
          for (uint32_t b = a; b > 0 && rate[cand[b]] < rate[cand[b - 1]]; --b) {
            const uint32_t t = cand[b];
            cand[b] = cand[b - 1];
            cand[b - 1] = t;
          }
        if (order_cost(rate, cand, P.n_dims) < 0.9f * order_cost(rate, cur, P.n_dims)) {
          const uint32_t nv = c.issue_ver ^ 1u;
          for (uint32_t d = 0; d < kMaxDims; ++d) c.order[nv][d] = (d < P.n_dims) ? cand[d] : 0u;
          c.n_steps[nv] = make_steps(P, c.order[nv], c.steps[nv]);
          c.issue_ver = nv;
          c.reorders++;
        }
      }
      if (issued < my_iters) {
        issue(issued);
        ++issued;
      }
    }
  }
  const bool aborted = c.abort != 0;
  if (!aborted) {
    pr.pump(exec_ver, true);
  } else if (tid == 0) {
    // let copies still in flight land before the CTA's shared memory goes away
    for (uint32_t j = it; j < issued; ++j) mbar_wait_bounded(&bar[j % S], (j / S) & 1u, kMaxPolls);
  }
  __syncthreads();

  // ---- flush group partials and counters -----------------------------------
  if (!aborted && c.groups_in_smem) {
    for (uint32_t g = tid; g < c.n_groups; g += NT) {
      const uint32_t cnt = pr.s_cnt[g];
      if (cnt) {
        atomicAdd(&P.g_sum[g], pr.s_sum[g]);
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
// to payload values.
__global__ void __launch_bounds__(256) sj_finalize_kernel(const __grid_constant__ SjPlanRt P) {
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

template <int NT, int RPT>
static cudaError_t launch_probe_t(const SjPlanRt& P, const SjProbeGeom& G, uint32_t smem, cudaStream_t st) {
  cudaError_t e = cudaFuncSetAttribute(sj_probe_kernel<NT, RPT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  sj_probe_kernel<NT, RPT><<<G.grid, NT, smem, st>>>(P, G);
  return cudaGetLastError();
}

// rows_per_thread: 4, 8 or 16 rows per thread per sub-block.
cudaError_t launch_probe(const SjPlanRt& P, const SjProbeGeom& G, uint32_t rows_per_thread, cudaStream_t st) {
  const uint32_t smem = probe_layout(G).total;
#define SJ_CASE(N, R) \
  if (G.threads == N && rows_per_thread == R) return launch_probe_t<N, R>(P, G, smem, st);
  SJ_CASE(256, 4)
  SJ_CASE(256, 8)
  SJ_CASE(256, 16)
  SJ_CASE(512, 4)
  SJ_CASE(512, 8)
  SJ_CASE(512, 16)
  SJ_CASE(1024, 4)
  SJ_CASE(1024, 8)
#undef SJ_CASE
  return cudaErrorInvalidValue;
}

cudaError_t launch_finalize(const SjPlanRt& P, uint32_t group_capacity, cudaStream_t st) {
  uint32_t blocks = (group_capacity + 255) / 256;
  if (blocks > 1184) blocks = 1184;
  if (blocks < 1) blocks = 1;
  sj_finalize_kernel<<<blocks, 256, 0, st>>>(P);
  return cudaGetLastError();
}

}  // namespace sj
