// sj_build.cuh -- device-side pieces of the dimension build (sj_build.cu's
// kernels): the predicate, the scan and insert loops over a dimension, the
// payload-bitmap prefix and dictionary, group strides and the starting LIP order.
//
// They restate the reference's build_hashtable_{s,c,d} kernels
// (src/ssb-jo/q33/0-lip.cu:114-203): BlockLoad(dim_val) -> BlockPred* ->
// BlockLoad(dim_key) -> BlockBuildBloomFilter -> BlockBuildSelectivePHT_2, split
// into a scan (qualifying count and the payload bitmap that becomes the
// group-key dictionary) and an insert (PHT slots [key, dense code] and the
// filter, keyed by the PHT slot).
#pragma once
#include "sj_internal.h"
#include "sj_ptx.cuh"

namespace sj {

// Expected filter-test cost per fact row of a LIP order: a test costs 1 when its
// filter is in the probe's shared memory and kL2TestCost when it is read from
// L2; a row reaches position p with the product of the earlier pass rates.
constexpr float kL2TestCost = 4.f;

// Predicate of dimension row i (BlockPredEQ/BlockPredOrEQ chains and the
// BlockPredGTE/BlockPredLTE range, crystal/pred.cuh:237-356).
__device__ __forceinline__ bool dim_pred(const SjDimRt& D, uint64_t i) {
  if (D.pred_kind == SJ_PRED_ALL) return true;
  int32_t a = D.filter_attr[i];
  if (D.pred_kind == SJ_PRED_RANGE) return a >= D.pred_lo && a <= D.pred_hi;
  if ((uint32_t)a >= (uint32_t)SJ_MAX_IN_CODES) return false;
  return (D.in_bitmap[(uint32_t)a >> 5] >> ((uint32_t)a & 31u)) & 1u;
}

// Scan of dimension d by block `blk` of `nblk` (block-strided over the rows):
// marks the payload of every qualifying row in the payload bitmap and appends
// the row's index to D.qual_rows, counted in *n_qual (one atomic per warp).
__device__ __forceinline__ void dim_scan_rows(const SjPlanRt& P, uint32_t d, uint32_t blk, uint32_t nblk,
                                              uint32_t* error_flags, uint32_t* n_qual) {
  const SjDimRt& D = P.dim[d];
  const uint32_t lane = threadIdx.x & 31u;
  for (uint64_t i0 = (uint64_t)blk * blockDim.x; i0 < D.rows; i0 += (uint64_t)nblk * blockDim.x) {
    const uint64_t i = i0 + threadIdx.x;
    const bool q = (i < D.rows) && dim_pred(D, i);
    if (q && D.grouped) {
      const uint32_t off = (uint32_t)(D.payload[i] - D.payload_min);
      if (off >= D.payload_span) {
        atomicOr(error_flags, kErrPayloadDomain);
      } else {
        const uint32_t bit = 1u << (off & 31u);
        uint32_t* w = D.payload_bitmap + (off >> 5);
        if (!(*w & bit)) atomicOr(w, bit);
      }
    }
    const uint32_t m = __ballot_sync(0xffffffffu, q);
    if (m) {
      uint32_t base = 0;
      if (lane == 0) base = atomicAdd(n_qual, (uint32_t)__popc(m));
      base = __shfl_sync(0xffffffffu, base, 0);
      if (q) D.qual_rows[base + __popc(m & lanemask_lt())] = (uint32_t)i;
    }
  }
}

// Exclusive prefix of the popcounts of `words` bitmap words into pre[] (and their
// total), by one warp with shuffles: payload bitmaps are at most 2,048 words
// (SJ_MAX_PAYLOAD_SPAN bits), 1-32 for the SSB attributes.  `lane` is the
// calling warp's lane; no block barrier.
__device__ __forceinline__ void warp_bitmap_prefix(const uint32_t* bm, uint32_t words, uint32_t* pre,
                                                   uint32_t* total, uint32_t lane) {
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
  const uint32_t t = __shfl_sync(0xffffffffu, incl, 31);
  if (total && lane == 0) *total = t;
}

// Dictionary of dimension d (code -> payload value), block-strided over the
// bitmap words, from the prefix `pre`.
__device__ __forceinline__ void write_dict(const SjDimRt& D, const uint32_t* pre, uint32_t words) {
  for (uint32_t w = threadIdx.x; w < words; w += blockDim.x) {
    uint32_t bits = D.payload_bitmap[w];
    uint32_t code = pre[w];
    while (bits) {
      const uint32_t b = __ffs(bits) - 1u;
      D.dict[code++] = D.payload_min + (int32_t)(w * 32u + b);
      bits &= bits - 1u;
    }
  }
}

// Group strides over the dense codes, dimension 0 most significant; returns the
// number of dense groups.
__device__ __forceinline__ uint32_t group_strides(const SjPlanRt& P, const uint32_t* n_codes, uint32_t* stride) {
  uint32_t groups = 1;
  for (int d = (int)P.n_dims - 1; d >= 0; --d) {
    if (!P.dim[d].grouped) {
      stride[d] = 0;
      continue;
    }
    stride[d] = groups;
    groups *= (n_codes[d] ? n_codes[d] : 1u);
  }
  return groups;
}

// Element i (0..3) of a 4-entry array held in registers.
template <typename T>
__device__ __forceinline__ T sel4(const T (&a)[kMaxDims], uint32_t i) {
  return i == 0 ? a[0] : i == 1 ? a[1] : i == 2 ? a[2] : a[3];
}

// Permutation number p (0 <= p < n!) of 0..n-1 in lexicographic order; entries
// from n on are their index.  The permutations are packed one byte each (entry
// i in bits 2i..2i+1), eight to a 64-bit word, so lane p reads its own with two
// shifts instead of factorial-base divisions.
__device__ __forceinline__ void nth_perm(uint32_t p, uint32_t n, uint32_t (&perm)[kMaxDims]) {
  uint64_t w;
  if (n == 4) w = p < 8 ? 0xb1e16c9c78d8b4e4ull : (p < 16 ? 0x36c672d22d8d39c9ull : 0x1b4b278763931e4eull);
  else if (n == 3) w = 0xc6d2c9e1d8e4ull;
  else if (n == 2) w = 0xe1e4ull;
  else w = 0xe4ull;  // identity
  const uint32_t code = (uint32_t)(w >> (8u * (p & 7u))) & 0xFFu;
#pragma unroll
  for (uint32_t i = 0; i < kMaxDims; ++i) perm[i] = (code >> (2u * i)) & 3u;
}

// Starting LIP order and filter placement for the probe, by one warp (`lane`).
// Filters take the probe's shared memory in LIP order while they fit.  With
// adaptive LIP the order is the cheapest over all permutations (lane p prices
// permutation p; ties go to the first in lexicographic order), with each
// dimension's qualifying fraction as its pass-rate estimate; otherwise the
// plan's order.
__device__ __forceinline__ void choose_start(const SjPlanRt& P, const uint32_t (&inserted)[kMaxDims],
                                             uint32_t* start_order, uint32_t* smem_off, uint32_t lane) {
  const uint32_t n = P.n_dims;
  uint32_t bytes[kMaxDims] = {0, 0, 0, 0};
  float rate[kMaxDims] = {1.f, 1.f, 1.f, 1.f};
#pragma unroll
  for (uint32_t d = 0; d < kMaxDims; ++d) {
    if (d >= n) continue;
    const SjDimRt& D = P.dim[d];
    uint32_t l2;
    const uint32_t mode = bf_effective(D.bf_mode, D.bf_max_log2, D.bf_bits_per_key, inserted[d], P.bf_smem_budget, &l2);
    bytes[d] = (mode == kBfDirect) ? max(8u, (1u << l2) / 8u) : (8u << l2);
    rate[d] = ((float)inserted[d] + 1.f) / ((float)D.rows + 2.f);
  }
  // placement of the filters for order `ord`: byte offsets and test weights
  auto place = [&](const uint32_t (&ord)[kMaxDims], uint32_t (&off)[kMaxDims], float (&weight)[kMaxDims]) {
    uint32_t used = 0;
#pragma unroll
    for (uint32_t d = 0; d < kMaxDims; ++d) {
      off[d] = ~0u;
      weight[d] = kL2TestCost;
    }
#pragma unroll
    for (uint32_t p = 0; p < kMaxDims; ++p) {
      if (p >= n) continue;
      const uint32_t d = ord[p], b = sel4(bytes, d);
      const bool fits = P.lip && used + b <= P.bf_smem_budget;
#pragma unroll
      for (uint32_t e = 0; e < kMaxDims; ++e)
        if (e == d) {
          off[e] = fits ? used : ~0u;
          weight[e] = fits ? 1.f : kL2TestCost;
        }
      if (fits) used += (b + 15u) & ~15u;
    }
  };
  uint32_t best[kMaxDims] = {0, 1, 2, 3};
#pragma unroll
  for (uint32_t p = 0; p < kMaxDims; ++p)
    if (p < n) best[p] = P.order[p];
  if (P.lip && P.adaptive && n > 1) {
    const uint32_t n_perm = n == 4 ? 24u : n == 3 ? 6u : 2u;
    uint32_t perm[kMaxDims];
    nth_perm(lane < n_perm ? lane : 0u, n, perm);
    uint32_t off[kMaxDims];
    float weight[kMaxDims];
    place(perm, off, weight);
    float cost = 0.f, live = 1.f;
#pragma unroll
    for (uint32_t p = 0; p < kMaxDims; ++p) {
      if (p >= n) continue;
      cost += live * sel4(weight, perm[p]);
      live *= sel4(rate, perm[p]);
    }
    if (lane >= n_perm) cost = 3.4e38f;
    uint32_t arg = lane;
#pragma unroll
    for (uint32_t o = 16; o; o >>= 1) {
      const float c2 = __shfl_xor_sync(0xffffffffu, cost, o);
      const uint32_t a2 = __shfl_xor_sync(0xffffffffu, arg, o);
      if (c2 < cost || (c2 == cost && a2 < arg)) {
        cost = c2;
        arg = a2;
      }
    }
    nth_perm(arg, n, best);
  }
  uint32_t off[kMaxDims];
  float weight[kMaxDims];
  place(best, off, weight);
  if (lane < kMaxDims) {
    start_order[lane] = lane < n ? sel4(best, lane) : 0u;
    smem_off[lane] = lane < n ? sel4(off, lane) : ~0u;
  }
}

// Insert of dimension d by block `blk` of `nblk`, over the n_qual rows the scan
// listed: each claims its PHT slot (BlockBuildSelectivePHT_2: the key once, then
// the value -- here the payload's dense code, its rank in the payload bitmap)
// and sets its filter bits, keyed by the PHT slot so the filter never rejects a
// row the PHT accepts.
__device__ __forceinline__ void dim_insert_rows(const SjPlanRt& P, uint32_t d, uint32_t mode, uint32_t log2,
                                                const uint32_t* prefix, uint32_t n_qual, uint32_t blk,
                                                uint32_t nblk) {
  const SjDimRt& D = P.dim[d];
  for (uint32_t k = blk * blockDim.x + threadIdx.x; k < n_qual; k += nblk * blockDim.x) {
    const uint32_t i = D.qual_rows[k];
    const int32_t key = D.key[i];
    const uint32_t s = slot_of(key, D.key_min, D.ht_len, D.fastmod_m);
    int32_t val = 0;
    if (D.grouped) {
      const uint32_t off = (uint32_t)(D.payload[i] - D.payload_min);
      if (off >= D.payload_span) continue;  // flagged by the scan
      val = (int32_t)(prefix[off >> 5] + __popc(D.payload_bitmap[off >> 5] & ((1u << (off & 31u)) - 1u)));
    } else if (D.payload) {
      val = D.payload[i];
    }
    atomicCAS(&D.ht[s].x, 0, key);
    D.ht[s].y = val;
    if (mode == kBfDirect) {
      uint32_t* w = reinterpret_cast<uint32_t*>(D.bf) + (s >> 5);
      const uint32_t bit = 1u << (s & 31u);
      if (!(*w & bit)) atomicOr(w, bit);
    } else {
      unsigned long long* w = reinterpret_cast<unsigned long long*>(D.bf) + bf_word(s, log2);
      const unsigned long long m = bf_mask(s, D.bf_k);
      if ((*w & m) != m) atomicOr(w, m);
    }
  }
}

}  // namespace sj
