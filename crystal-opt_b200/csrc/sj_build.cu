// sj_build.cu -- dimension-side kernels: predicate evaluation, payload dictionary,
// perfect-hash-table insert and Bloom-filter insert.
//
// Replaces the reference's build_hashtable_{s,c,d} kernels
// (src/ssb-jo/q33/0-lip.cu:114-203): BlockLoad(dim_val) -> BlockPred* ->
// BlockLoad(dim_key) -> BlockBuildBloomFilter -> BlockBuildSelectivePHT_2.
//
// Two launches per query, each covering every dimension (blockIdx.y = dim):
//   sj_dim_scan   counts qualifying rows and marks their payloads in a bitmap over
//                 the payload domain (the group-key dictionary);
//   sj_dim_insert sizes the filter from the count (bits per inserted key), ranks
//                 payloads into dense group codes, and inserts qualifying rows into
//                 the PHT ([key, code] slots, the reference's 2 x int32 layout) and
//                 the filter.
// Everything the probe needs (filter geometry, code counts, group strides) is
// written to the query descriptor on the device: no host round trip, so a whole
// query can be captured in a CUDA graph.
#include "sj_internal.h"
#include "sj_ptx.cuh"

namespace sj {

// Predicate of dimension row i (BlockPredEQ/BlockPredOrEQ chains and the
// BlockPredGTE/BlockPredLTE range, crystal/pred.cuh:237-356).
__device__ __forceinline__ bool dim_pred(const SjDimRt& D, uint64_t i) {
  if (D.pred_kind == SJ_PRED_ALL) return true;
  int32_t a = D.filter_attr[i];
  if (D.pred_kind == SJ_PRED_RANGE) return a >= D.pred_lo && a <= D.pred_hi;
  if ((uint32_t)a >= (uint32_t)SJ_MAX_IN_CODES) return false;
  return (D.in_bitmap[(uint32_t)a >> 5] >> ((uint32_t)a & 31u)) & 1u;
}

__global__ void __launch_bounds__(256) sj_dim_scan(const __grid_constant__ SjPlanRt P) {
  pdl_launch_dependents();  // sj_dim_insert may be scheduled; it waits for this grid
  const uint32_t d = blockIdx.y;
  if (d >= P.n_dims) return;
  const SjDimRt& D = P.dim[d];
  SjDesc* desc = P.desc;
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t count = 0;
  for (uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x; i0 < D.rows; i0 += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t i = i0 + threadIdx.x;
    bool q = (i < D.rows) && dim_pred(D, i);
    if (q && D.grouped) {
      uint32_t off = (uint32_t)(D.payload[i] - D.payload_min);
      if (off >= D.payload_span) {
        atomicOr(&desc->error_flags, kErrPayloadDomain);
      } else {
        uint32_t bit = 1u << (off & 31u);
        uint32_t* w = D.payload_bitmap + (off >> 5);
        if (!(*w & bit)) atomicOr(w, bit);
      }
    }
    count += __popc(__ballot_sync(0xffffffffu, q));
  }
  if (lane == 0 && count) atomicAdd(&desc->dim[d].n_inserted, count);
}

// Exclusive prefix of the popcounts of `words` bitmap words into pre[] (and their
// total), by warp 0 with shuffles: payload bitmaps are at most 2,048 words
// (SJ_MAX_PAYLOAD_SPAN bits), 1-32 for the SSB attributes.  One block barrier.
__device__ void bitmap_prefix(const uint32_t* bm, uint32_t words, uint32_t* pre, uint32_t* total) {
  if (threadIdx.x < 32) {
    const uint32_t lane = threadIdx.x;
    const uint32_t per = (words + 31) / 32;
    const uint32_t b = lane * per, e = min(words, b + per);
    uint32_t s = 0;
    for (uint32_t w = b; w < e; ++w) s += __popc(bm[w]);
    uint32_t incl = s;
#pragma unroll
    for (uint32_t o = 1; o < 32; o <<= 1) {
      const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    uint32_t run = incl - s;  // exclusive
    for (uint32_t w = b; w < e; ++w) {
      pre[w] = run;
      run += __popc(bm[w]);
    }
    if (total && lane == 31) *total = incl;
  }
  __syncthreads();
}

// Expected filter-test cost per fact row of a LIP order: a test costs 1 when its
// filter is in the probe's shared memory and kL2TestCost when it is read from
// L2; a row reaches position p with the product of the earlier pass rates.
constexpr float kL2TestCost = 4.f;

// Starting LIP order and filter placement for the probe.  Filters take the
// probe's shared memory in LIP order while they fit.  With adaptive LIP the
// order is the cheapest one over all permutations, with each dimension's
// qualifying fraction as its pass-rate estimate; otherwise the plan's order.
__device__ void choose_start(const SjPlanRt& P, SjDesc* desc) {
  const uint32_t n = P.n_dims;
  uint32_t bytes[kMaxDims] = {0, 0, 0, 0};
  float rate[kMaxDims] = {1.f, 1.f, 1.f, 1.f};
  for (uint32_t d = 0; d < n; ++d) {
    const SjDimRt& D = P.dim[d];
    const uint32_t ins = desc->dim[d].n_inserted;
    uint32_t l2;
    const uint32_t mode = bf_effective(D.bf_mode, D.bf_max_log2, D.bf_bits_per_key, ins, P.bf_smem_budget, &l2);
    bytes[d] = (mode == kBfDirect) ? max(8u, (1u << l2) / 8u) : (8u << l2);
    rate[d] = ((float)ins + 1.f) / ((float)D.rows + 2.f);
  }
  auto place = [&](const uint32_t* ord, uint32_t* off, float* weight) {
    uint32_t used = 0;
    for (uint32_t p = 0; p < n; ++p) {
      const uint32_t d = ord[p];
      const bool fits = P.lip && used + bytes[d] <= P.bf_smem_budget;
      off[d] = fits ? used : ~0u;
      weight[d] = fits ? 1.f : kL2TestCost;
      if (fits) used += (bytes[d] + 15u) & ~15u;
    }
  };
  uint32_t best[kMaxDims] = {0, 1, 2, 3};
  for (uint32_t p = 0; p < n; ++p) best[p] = P.order[p];
  if (P.lip && P.adaptive && n > 1) {
    uint32_t perm[kMaxDims] = {0, 1, 2, 3};
    float best_cost = 3.4e38f;
    for (;;) {
      uint32_t off[kMaxDims];
      float weight[kMaxDims];
      place(perm, off, weight);
      float cost = 0.f, live = 1.f;
      for (uint32_t p = 0; p < n; ++p) {
        cost += live * weight[perm[p]];
        live *= rate[perm[p]];
      }
      if (cost < best_cost) {
        best_cost = cost;
        for (uint32_t p = 0; p < n; ++p) best[p] = perm[p];
      }
      int i = (int)n - 2;  // next permutation (lexicographic)
      while (i >= 0 && perm[i] >= perm[i + 1]) --i;
      if (i < 0) break;
      int j = (int)n - 1;
      while (perm[j] <= perm[i]) --j;
      uint32_t t = perm[i];
      perm[i] = perm[j];
      perm[j] = t;
      for (int a = i + 1, b = (int)n - 1; a < b; ++a, --b) {
        t = perm[a];
        perm[a] = perm[b];
        perm[b] = t;
      }
    }
  }
  uint32_t off[kMaxDims] = {~0u, ~0u, ~0u, ~0u};
  float weight[kMaxDims];
  place(best, off, weight);
  for (uint32_t d = 0; d < kMaxDims; ++d) {
    desc->start_order[d] = d < n ? best[d] : 0u;
    desc->bf_smem_off[d] = d < n ? off[d] : ~0u;
  }
}

__global__ void __launch_bounds__(256) sj_dim_insert(const __grid_constant__ SjPlanRt P) {
  pdl_launch_dependents();  // the probe may be scheduled; it waits for this grid
  pdl_wait();               // sj_dim_scan's counts and payload bitmaps are complete
  extern __shared__ uint32_t prefix[];  // payload-bitmap prefix popcounts
  __shared__ uint32_t s_total;
  const uint32_t d = blockIdx.y;
  if (d >= P.n_dims) return;
  const SjDimRt& D = P.dim[d];
  SjDesc* desc = P.desc;

  const uint32_t n_ins = desc->dim[d].n_inserted;
  uint32_t log2;
  const uint32_t mode = bf_effective(D.bf_mode, D.bf_max_log2, D.bf_bits_per_key, n_ins, P.bf_smem_budget, &log2);
  const uint32_t pwords = D.grouped ? (D.payload_span + 31u) / 32u : 0u;
  if (D.grouped) bitmap_prefix(D.payload_bitmap, pwords, prefix, &s_total);

  if (blockIdx.x == 0) {
    if (threadIdx.x == 0) {
      desc->dim[d].bf_log2 = log2;
      desc->dim[d].bf_mode = mode;
    }
    if (D.grouped) {
      // dictionary: code -> payload value
      for (uint32_t w = threadIdx.x; w < pwords; w += blockDim.x) {
        uint32_t bits = D.payload_bitmap[w];
        uint32_t code = prefix[w];
        while (bits) {
          uint32_t b = __ffs(bits) - 1u;
          D.dict[code++] = D.payload_min + (int32_t)(w * 32u + b);
          bits &= bits - 1u;
        }
      }
      if (threadIdx.x == 0) desc->dim[d].n_codes = s_total;
    }
    if (d == 0 && threadIdx.x == 0) {
      // group strides over the dense codes, dimension 0 most significant
      uint32_t groups = 1;
      for (int dd = (int)P.n_dims - 1; dd >= 0; --dd) {
        const SjDimRt& E = P.dim[dd];
        if (!E.grouped) {
          desc->dim[dd].group_stride = 0;
          continue;
        }
        uint32_t n = 0;
        const uint32_t ew = (E.payload_span + 31u) / 32u;
        for (uint32_t w = 0; w < ew; ++w) n += __popc(E.payload_bitmap[w]);
        desc->dim[dd].group_stride = groups;
        groups *= (n ? n : 1u);
      }
      desc->n_groups = groups;
      choose_start(P, desc);
    }
  }

  const uint64_t pol = policy_evict_last();
  (void)pol;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < D.rows;
       i += (uint64_t)gridDim.x * blockDim.x) {
    if (!dim_pred(D, i)) continue;
    const int32_t key = D.key[i];
    const uint32_t s = slot_of(key, D.key_min, D.ht_len, D.fastmod_m);
    int32_t val = 0;
    if (D.grouped) {
      uint32_t off = (uint32_t)(D.payload[i] - D.payload_min);
      if (off >= D.payload_span) continue;  // flagged by sj_dim_scan
      val = (int32_t)(prefix[off >> 5] + __popc(D.payload_bitmap[off >> 5] & ((1u << (off & 31u)) - 1u)));
    } else if (D.payload) {
      val = D.payload[i];
    }
    // BlockBuildSelectivePHT_2: claim the slot's key once, then store the value.
    atomicCAS(&D.ht[s].x, 0, key);
    D.ht[s].y = val;
    // Filter insert keyed by the PHT slot, so the filter never rejects a row the
    // PHT would accept.
    if (mode == kBfDirect) {
      uint32_t* w = reinterpret_cast<uint32_t*>(D.bf) + (s >> 5);
      uint32_t bit = 1u << (s & 31u);
      if (!(*w & bit)) atomicOr(w, bit);
    } else {
      unsigned long long* w = reinterpret_cast<unsigned long long*>(D.bf) + bf_word(s, log2);
      const unsigned long long m = bf_mask(s, D.bf_k);
      if ((*w & m) != m) atomicOr(w, m);
    }
  }
}

}  // namespace sj
