// sj_batch.cu -- the shared-scan star join: many queries, one pass over the fact table.
//
// Design (the shared-pipeline idea of CJOIN, Candea et al., VLDB 2009, mapped to
// B200): every dimension keeps one 64-bit word per PHT slot whose bit q says
// whether query slot q's predicate accepts the dimension row stored in that
// slot.  A fact row starts with the set of query slots whose row range covers it
// and ANDs in one word per dimension lookup; the survivors are (row, query)
// pairs, aggregated into per-query group accumulators.  One fact scan and at
// most one L2 lookup per (row, dimension) serve every query of the batch.
//
// Per query this computes exactly what the reference's probe computes for one
// query (src/ssb-jo/q33/0-lip.cu:28-112 with the uint64 sum of
// src/ssb-jo/q31/0-lip.cu:98-113): PHT slot (fk - key_min) mod ht_len
// (crystal/join.cuh:27), a hit iff the slot holds a qualifying row, the group
// key from that row's attributes.
//
// Kernels
//   sjb_register_kernel  slot uniqueness check + per-slot attribute tables
//   sjb_zero_jobs_kernel / sjb_build_kernel
//                        filter bitmap (one bit per slot) + count/min/max
//                        statistics for each (dimension, predicate) to build
//   sjb_layout_kernel    group layout and lookup order on the device (batch)
//   sjb_zero_groups_kernel, sjb_compose_kernel (bitmaps -> 64-bit slot words)
//   sjb_probe_kernel     the shared scan
//   sjb_finalize_kernel  non-empty accumulators -> result rows
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <climits>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "sj_cache.h"
#include "sj_internal.h"
#include "sj_shared.h"

namespace sj {

constexpr uint32_t kFull = 0xffffffffu;

// ------------------------------------------------------- registration ----
__global__ void __launch_bounds__(256) sjb_register_kernel(const __grid_constant__ SjbSchemaRt S, uint32_t d,
                                                           uint32_t* slot_rows, SjbCounters* ctr) {
  const SjbDimRt& R = S.dim[d];
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < R.rows;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t s = slot_of(R.key[i], R.key_min, R.len, R.fastmod_m);
    if (atomicAdd(&slot_rows[s], 1u) != 0u) atomicOr(&ctr->error, kBErrCollision);
    for (uint32_t a = 0; a < R.n_attrs; ++a) const_cast<int32_t*>(R.slot_attr[a])[s] = R.attr[a][i];
  }
}

cudaError_t sjb_launch_register(const SjbSchemaRt& S, uint32_t* slot_rows, SjbCounters* ctr, cudaStream_t st) {
  for (uint32_t d = 0; d < S.n_dims; ++d) {
    const int64_t rows = S.dim[d].rows;
    if (rows <= 0) continue;
    const uint32_t blocks = (uint32_t)std::min<int64_t>((rows + 255) / 256, 4096);
    uint64_t off = 0;
    for (uint32_t e = 0; e < d; ++e) off += S.dim[e].len;
    sjb_register_kernel<<<blocks, 256, 0, st>>>(S, d, slot_rows + off, ctr);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// --------------------------------------------------------- filter build ----
__global__ void __launch_bounds__(256) sjb_zero_jobs_kernel(const SjbBatchDesc* __restrict__ D) {
  const uint32_t j = blockIdx.y;
  if (j >= D->n_jobs) return;
  const SjbJob& J = D->jobs[j];
  if (J.stats_mask & kJobStatsOnly) return;  // its filter is built and in use
  for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < J.words; w += gridDim.x * blockDim.x)
    J.bitmap[w] = 0u;
  if (blockIdx.x == 0 && threadIdx.x < sizeof(SjbEntryStats) / 4)
    reinterpret_cast<uint32_t*>(J.stats)[threadIdx.x] = 0u;
}

// One pass per dimension serves all of that dimension's jobs: each row's key
// and attributes are read once, then every job's predicate is evaluated on them
// (blockIdx.y = dimension).  Per job and warp: one ballot, one atomicOr per
// distinct bitmap word, and the statistics only when some row qualified, kept
// in shared memory and flushed once per block.  The min/max of an attribute is
// reduced only when the job's stats_mask names it (the attributes its queries
// group by); statistics-only jobs skip the bitmap and the count.
constexpr uint32_t kBuildThreads = 256;

__global__ void __launch_bounds__(kBuildThreads) sjb_build_kernel(const __grid_constant__ SjbSchemaRt S,
                                                                  const SjbBatchDesc* __restrict__ D) {
  __shared__ SjbJob s_job[kBMaxJobs];
  __shared__ uint32_t s_cnt[kBMaxJobs];
  __shared__ uint32_t s_umax[kBMaxJobs][SJB_MAX_ATTRS], s_nmin[kBMaxJobs][SJB_MAX_ATTRS];
  __shared__ uint32_t s_nj, s_warp_base[kBuildThreads / 32];
  const uint32_t d = blockIdx.y;
  if (d >= S.n_dims) return;
  const uint32_t tid = threadIdx.x, lane = tid & 31u, wid = tid >> 5;
  const uint32_t nj_all = min(D->n_jobs, (uint32_t)kBMaxJobs);
  // this dimension's jobs, compacted in job order
  const bool mine = tid < nj_all && D->jobs[tid].dim == d;
  const uint32_t bal = __ballot_sync(kFull, mine);
  if (lane == 0) s_warp_base[wid] = __popc(bal);
  __syncthreads();
  if (tid == 0) {
    uint32_t run = 0;
    for (uint32_t w = 0; w < kBuildThreads / 32; ++w) {
      const uint32_t c = s_warp_base[w];
      s_warp_base[w] = run;
      run += c;
    }
    s_nj = run;
  }
  __syncthreads();
  if (mine) {
    const uint32_t k = s_warp_base[wid] + __popc(bal & ((1u << lane) - 1u));
    s_job[k] = D->jobs[tid];
    s_cnt[k] = 0;
    for (uint32_t a = 0; a < SJB_MAX_ATTRS; ++a) s_umax[k][a] = s_nmin[k][a] = 0;
  }
  __syncthreads();
  const uint32_t nj = s_nj;
  if (nj == 0) return;
  const SjbDimRt& R = S.dim[d];
  const uint32_t na = R.n_attrs;
  // the loop bound is uniform across the warp, so full-warp collectives are safe inside
  for (int64_t i0 = (int64_t)blockIdx.x * kBuildThreads; i0 < R.rows; i0 += (int64_t)gridDim.x * kBuildThreads) {
    const int64_t i = i0 + tid;
    const bool in = i < R.rows;
    const int32_t key = in ? R.key[i] : 0;
    int32_t av[SJB_MAX_ATTRS];
#pragma unroll
    for (uint32_t a = 0; a < SJB_MAX_ATTRS; ++a) av[a] = (in && a < na) ? R.attr[a][i] : 0;
    const bool live = in && key != 0;  // CAS(slot, 0, 0) never claims a slot (crystal/join.cuh:270)
    const uint32_t s = live ? slot_of(key, R.key_min, R.len, R.fastmod_m) : 0u;
    const uint32_t wd = s >> 5, bit = 1u << (s & 31u);
    uint32_t uv[SJB_MAX_ATTRS];
#pragma unroll
    for (uint32_t a = 0; a < SJB_MAX_ATTRS; ++a) uv[a] = (uint32_t)av[a] ^ 0x80000000u;
    for (uint32_t k = 0; k < nj; ++k) {
      const SjbJob& J = s_job[k];
      bool ok = live;
      if (ok && J.kind != SJ_PRED_ALL) {
        int32_t a = av[0];
#pragma unroll
        for (uint32_t x = 1; x < SJB_MAX_ATTRS; ++x) a = (uint32_t)J.attr == x ? av[x] : a;
        if (J.kind == SJ_PRED_RANGE)
          ok = a >= J.lo && a <= J.hi;
        else
          ok = (uint32_t)a < (uint32_t)SJ_MAX_IN_CODES &&
               ((D->in_bits[J.in_index][(uint32_t)a >> 5] >> ((uint32_t)a & 31u)) & 1u);
      }
      uint32_t pend = __ballot_sync(kFull, ok);
      if (!pend) continue;  // warp-uniform
      const uint32_t n_ok = __popc(pend);
      if (J.stats_mask & kJobStatsOnly) pend = 0;  // the bitmap is built already
      while (pend) {  // one atomicOr per distinct bitmap word in the warp
        const uint32_t leader = __ffs(pend) - 1u;
        const uint32_t lw = __shfl_sync(kFull, wd, leader);
        const bool hit = ((pend >> lane) & 1u) && wd == lw;
        const uint32_t bits = __reduce_or_sync(kFull, hit ? bit : 0u);
        if (lane == leader) atomicOr(J.bitmap + lw, bits);
        pend &= ~__ballot_sync(kFull, hit);
      }
      if (lane == 0) atomicAdd(&s_cnt[k], n_ok);
#pragma unroll
      for (uint32_t a = 0; a < SJB_MAX_ATTRS; ++a) {
        if (a < na && ((J.stats_mask >> a) & 1u)) {
          const uint32_t mx = __reduce_max_sync(kFull, ok ? uv[a] : 0u);
          const uint32_t mn = __reduce_max_sync(kFull, ok ? ~uv[a] : 0u);
          if (lane == 0) {
            atomicMax(&s_umax[k][a], mx);
            atomicMax(&s_nmin[k][a], mn);
          }
        }
      }
    }
  }
  __syncthreads();
  for (uint32_t k = tid; k < nj; k += kBuildThreads) {
    if (!s_cnt[k]) continue;
    const uint32_t mask = s_job[k].stats_mask;
    SjbEntryStats* st = s_job[k].stats;
    if (!(mask & kJobStatsOnly)) atomicAdd(&st->count, s_cnt[k]);
    for (uint32_t a = 0; a < na; ++a) {
      if (!((mask >> a) & 1u)) continue;
      atomicMax(&st->umax[a], s_umax[k][a]);
      atomicMax(&st->nmin[a], s_nmin[k][a]);
    }
  }
}

cudaError_t sjb_launch_build(const SjbSchemaRt& S, const SjbBatchDesc* desc, uint32_t max_jobs,
                             uint32_t jobs_hint, int sm_count, cudaStream_t st) {
  (void)jobs_hint;
  if (max_jobs == 0) return cudaSuccess;
  uint64_t max_len = 1, max_rows = 1;
  for (uint32_t d = 0; d < S.n_dims; ++d) {
    max_len = std::max<uint64_t>(max_len, S.dim[d].len);
    max_rows = std::max<uint64_t>(max_rows, (uint64_t)S.dim[d].rows);
  }
  const uint32_t zblocks = (uint32_t)std::min<uint64_t>((max_len / 32 + 256) / 256, 64);
  sjb_zero_jobs_kernel<<<dim3(zblocks, max_jobs), 256, 0, st>>>(desc);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  // enough blocks to fill the GPU on the largest dimension: eight per SM, so the
  // jobs' per-warp ballots and reductions of other blocks hide each other's
  // latency (1% of a 64-query batch over four per SM)
  const uint32_t bx = (uint32_t)std::max<uint64_t>(
      1, std::min<uint64_t>((max_rows + kBuildThreads - 1) / kBuildThreads, (uint64_t)sm_count * 8));
  sjb_build_kernel<<<dim3(bx, S.n_dims), kBuildThreads, 0, st>>>(S, desc);
  return cudaGetLastError();
}

// --------------------------------------------------------------- layout ----
// One thread per query slot (two warps).  Each thread computes its query's group
// layout; accumulator offsets are a warp scan of the spans, the dimension use
// masks are ballots, and the shared-memory partials go to the smallest spans
// first (each candidate's offset is the sum of the spans ranked before it).
__global__ void __launch_bounds__(kBq) sjb_layout_kernel(const __grid_constant__ SjbSchemaRt S,
                                                         const SjbBatchDesc* __restrict__ D,
                                                         SjbStep* __restrict__ out, SjbCounters* ctr) {
  __shared__ SjbStep st;
  __shared__ uint32_t s_err;
  __shared__ unsigned long long s_wsum[2], s_wact[2], s_wuse[2][SJ_MAX_DIMS];
  __shared__ float s_cover[kBq], s_pcost[24];
  __shared__ long long s_wlo[2], s_whi[2];
  __shared__ uint32_t s_span[kBq], s_smax[2];
  __shared__ uint8_t s_pos[SJ_MAX_DIMS];
  const uint32_t q = threadIdx.x, lane = q & 31u, wp = q >> 5;
  if (q == 0) s_err = 0;
  __syncthreads();
  SjbSlot& sl = st.slot[q];
  for (uint32_t d = 0; d < SJ_MAX_DIMS; ++d) {
    st.bm[q][d] = nullptr;
    st.sel[q][d] = 1.f;
  }
  sl.b = 0;
  sl.e = 0;
  sl.group_base = 0;
  sl.span = 0;
  sl.n_g = 0;
  sl.smem_off = -1;
  if (q < D->n_queries) {
    const SjbBatchQuery& Q = D->q[q];
    const SjbEntryStats* stp[SJ_MAX_DIMS];
    for (uint32_t k = 0; k < Q.n_preds; ++k) stp[k] = Q.stats[k];
    const uint32_t err = sjb_group_layout(S, Q, stp, sl, st.sel[q], D->group_capacity);
    if (err) atomicOr(&s_err, err);
    for (uint32_t k = 0; k < Q.n_preds; ++k) st.bm[q][Q.dim[k]] = Q.bitmap[k];
    sl.b = Q.b;
    sl.e = Q.e;
  }
  const bool act = q < D->n_queries && sl.span > 0 && sl.e > sl.b;
  // accumulator offsets: exclusive scan of the active spans in slot order
  unsigned long long incl = act ? sl.span : 0ull;
  for (uint32_t off = 1; off < 32; off <<= 1) {
    const unsigned long long v = __shfl_up_sync(kFull, incl, off);
    if (lane >= off) incl += v;
  }
  const unsigned long long wtot = __shfl_sync(kFull, incl, 31);
  const uint32_t ab = __ballot_sync(kFull, act);
  uint32_t ub[SJ_MAX_DIMS];
  for (uint32_t d = 0; d < SJ_MAX_DIMS; ++d) ub[d] = __ballot_sync(kFull, act && st.bm[q][d] != nullptr);
  long long lo = act ? sl.b : LLONG_MAX, hi = act ? sl.e : 0;
  for (uint32_t off = 16; off; off >>= 1) {
    lo = min(lo, __shfl_xor_sync(kFull, lo, off));
    hi = max(hi, __shfl_xor_sync(kFull, hi, off));
  }
  if (lane == 0) {
    s_wsum[wp] = wtot;
    s_wact[wp] = ab;
    s_wlo[wp] = lo;
    s_whi[wp] = hi;
    for (uint32_t d = 0; d < SJ_MAX_DIMS; ++d) s_wuse[wp][d] = ub[d];
  }
  __syncthreads();
  const unsigned long long total = s_wsum[0] + s_wsum[1];
  const bool over = total > D->group_capacity;
  sl.group_base = incl - (act ? sl.span : 0ull) + (wp ? s_wsum[0] : 0ull);
  const uint64_t active = over ? 0ull : (s_wact[0] | (s_wact[1] << 32));
  const bool a2 = (active >> q) & 1ull;
  if (q == 0) {
    if (over) s_err |= kBErrGroupCapacity;
    st.active = active;
    st.seg_b = active ? min(s_wlo[0], s_wlo[1]) : 0;
    st.seg_e = active ? max(s_whi[0], s_whi[1]) : 0;
    st.n_dims = S.n_dims;
    for (uint32_t d = 0; d < SJ_MAX_DIMS; ++d) st.use[d] = over ? 0ull : (s_wuse[0][d] | (s_wuse[1][d] << 32));
    st.error = s_err;
    if (s_err) atomicOr(&ctr->error, s_err);
  }
  __syncthreads();
  // lookup order: each of the first n! threads prices one order, thread 0 takes the cheapest
  s_cover[q] = ((st.active >> q) & 1ull)
                   ? (float)((double)(sl.e - sl.b) / (double)max(1ll, (long long)(st.seg_e - st.seg_b)))
                   : 0.f;
  __syncthreads();
  uint32_t n_perm = 1;
  for (uint32_t i = 2; i <= S.n_dims; ++i) n_perm *= i;
  if (q < n_perm) {
    uint32_t perm[SJ_MAX_DIMS];
    sjb_perm_of(q, S.n_dims, perm);
    s_pcost[q] = sjb_order_lookups(st, s_cover, perm, S.n_dims);
  }
  __syncthreads();
  if (q == 0) {
    uint32_t bi = 0;
    for (uint32_t i = 1; i < n_perm; ++i)
      if (s_pcost[i] < s_pcost[bi]) bi = i;
    uint32_t perm[SJ_MAX_DIMS] = {0, 1, 2, 3};
    sjb_perm_of(bi, S.n_dims, perm);
    for (uint32_t d = 0; d < SJ_MAX_DIMS; ++d) st.order[d] = d < S.n_dims ? perm[d] : d;
    for (uint32_t k = 0; k < S.n_dims; ++k) s_pos[st.order[k]] = (uint8_t)k;
  }
  const bool cand = a2 && sl.span <= 2048u;
  s_span[q] = cand ? sl.span : 0u;
  __syncthreads();
  for (int g = 0; g < sl.n_g; ++g) sl.gpos[g] = s_pos[sl.gd[g]];
  uint32_t end = 0;
  if (cand) {  // offset = spans of the candidates ranked before this one (smaller span, then lower slot)
    uint32_t off = 0;
    for (uint32_t r = 0; r < (uint32_t)kBq; ++r) {
      const uint32_t sr = s_span[r];
      if (sr && (sr < sl.span || (sr == sl.span && r < q))) off += sr;
    }
    if (off + sl.span <= D->smem_capacity) {
      sl.smem_off = (int32_t)off;
      end = off + sl.span;
    }
  }
  for (uint32_t o = 16; o; o >>= 1) end = max(end, __shfl_xor_sync(kFull, end, o));
  if (lane == 0) s_smax[wp] = end;
  __syncthreads();
  if (q == 0) st.smem_entries = max(s_smax[0], s_smax[1]);
  __syncthreads();
  const uint32_t* src = reinterpret_cast<const uint32_t*>(&st);
  uint32_t* dst = reinterpret_cast<uint32_t*>(out);
  for (uint32_t i = threadIdx.x; i < sizeof(SjbStep) / 4; i += blockDim.x) dst[i] = src[i];
}

cudaError_t sjb_launch_layout(const SjbSchemaRt& S, const SjbBatchDesc* desc, SjbStep* step, SjbCounters* ctr,
                              cudaStream_t st) {
  sjb_layout_kernel<<<1, kBq, 0, st>>>(S, desc, step, ctr);
  return cudaGetLastError();
}

// ---------------------------------------------------- zero / compose ----
__global__ void __launch_bounds__(256) sjb_zero_groups_kernel(const SjbStep* __restrict__ G, uint64_t mask,
                                                              SjbAcc* __restrict__ acc) {
  const uint32_t q = blockIdx.y;
  if (!((G->active & mask) >> q & 1ull)) return;
  const SjbSlot& s = G->slot[q];
  ulonglong2* a = reinterpret_cast<ulonglong2*>(acc + s.group_base);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < s.span; i += gridDim.x * blockDim.x)
    a[i] = make_ulonglong2(0ull, 0ull);
}

cudaError_t sjb_launch_zero_groups(const SjbStep* step, uint64_t zero_mask, SjbAcc* acc, int sm_count,
                                   cudaStream_t st) {
  sjb_zero_groups_kernel<<<dim3((uint32_t)std::max(1, sm_count / 8), kBq), 256, 0, st>>>(step, zero_mask, acc);
  return cudaGetLastError();
}

// Lane j of a warp owns slot 32*w + j.  Lanes first load the bitmap word w of
// query slots j and j + 32 in parallel; each query's word then reaches every
// lane by shuffle, and its bit j lands in bit q of lane j's mask word.
// 32 x 32 bit transpose across a warp: lane l holds row l (bit c = element
// [l][c]) and returns column l (bit q = element [q][l]).  Five butterfly stages;
// stage j swaps the off-diagonal j x j blocks between lanes l and l ^ j, the
// shuffle-network form of the recursive block transpose (Warren, Hacker's
// Delight, 7-3).
__device__ __forceinline__ uint32_t warp_transpose32(uint32_t x, uint32_t lane) {
#pragma unroll
  for (uint32_t j = 16, m = 0x0000FFFFu; j; j >>= 1, m ^= m << j) {
    const uint32_t y = __shfl_xor_sync(kFull, x, j);
    x = (lane & j) ? ((x & ~m) | ((y & ~m) >> j)) : ((x & m) | ((y & m) << j));
  }
  return x;
}

__global__ void __launch_bounds__(256) sjb_compose_kernel(const __grid_constant__ SjbSchemaRt S,
                                                          const SjbStep* __restrict__ G) {
  const uint32_t d = blockIdx.y;
  if (d >= S.n_dims) return;
  const SjbDimRt& R = S.dim[d];
  const uint64_t use = G->use[d];
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t words = (R.len + 31u) / 32u;
  const uint32_t warps = gridDim.x * (blockDim.x / 32u);
  const uint32_t* bm_lo = ((use >> lane) & 1ull) ? G->bm[lane][d] : nullptr;
  const uint32_t* bm_hi = ((use >> (lane + 32)) & 1ull) ? G->bm[lane + 32][d] : nullptr;
  for (uint32_t w = blockIdx.x * (blockDim.x / 32u) + (threadIdx.x >> 5); w < words; w += warps) {
    const uint32_t m_lo = warp_transpose32(bm_lo ? __ldg(bm_lo + w) : 0u, lane);
    const uint32_t m_hi = warp_transpose32(bm_hi ? __ldg(bm_hi + w) : 0u, lane);
    const uint32_t s = w * 32u + lane;
    if (s < R.len) R.mask[s] = (uint64_t)m_lo | ((uint64_t)m_hi << 32);
  }
}

cudaError_t sjb_launch_compose(const SjbSchemaRt& S, const SjbStep* step, int sm_count, cudaStream_t st) {
  uint32_t max_len = 1;
  for (uint32_t d = 0; d < S.n_dims; ++d) max_len = std::max(max_len, S.dim[d].len);
  const uint32_t warps = (max_len + 31) / 32;
  const uint32_t blocks = std::min<uint32_t>((warps + 7) / 8, (uint32_t)sm_count * 8);
  sjb_compose_kernel<<<dim3(blocks, S.n_dims), 256, 0, st>>>(S, step);
  return cudaGetLastError();
}

// ----------------------------------------------------------------- probe ----
constexpr int kTileRows = 128;  // 32 lanes x 4 rows

struct TileCols {
  int4 fk[SJ_MAX_DIMS];
  int4 m;
  int4 sub;
};

struct PosDim {  // dimension parameters by lookup position
  const int32_t* col;
  const uint64_t* mask;
  uint64_t fastmod_m;
  uint64_t use;
  int32_t key_min;
  uint32_t len;
};

__device__ __forceinline__ int4 ld_col4(const int32_t* __restrict__ c, int64_t r, int64_t n) {
  if (r + 4 <= n) return __ldcs(reinterpret_cast<const int4*>(c + r));
  int4 v = make_int4(0, 0, 0, 0);
  if (r < n) v.x = __ldcs(c + r);
  if (r + 1 < n) v.y = __ldcs(c + r + 1);
  if (r + 2 < n) v.z = __ldcs(c + r + 2);
  return v;
}

__device__ __forceinline__ int32_t pick(const int4& v, int j) {
  return j == 0 ? v.x : j == 1 ? v.y : j == 2 ? v.z : v.w;
}

__device__ __forceinline__ uint32_t pick4(uint32_t a, uint32_t b, uint32_t c, uint32_t d, uint32_t k) {
  return k == 0 ? a : k == 1 ? b : k == 2 ? c : d;
}

__device__ __forceinline__ void tile_masks(const int64_t* s_b, const int64_t* s_e, int64_t r0, uint32_t lane,
                                           uint64_t& act, uint64_t& full) {
  const int64_t r1 = r0 + kTileRows;
  const int64_t b0 = s_b[lane], e0 = s_e[lane], b1 = s_b[lane + 32], e1 = s_e[lane + 32];
  act = (uint64_t)__ballot_sync(kFull, b0 < r1 && e0 > r0) |
        ((uint64_t)__ballot_sync(kFull, b1 < r1 && e1 > r0) << 32);
  full = (uint64_t)__ballot_sync(kFull, b0 <= r0 && e0 >= r1) |
         ((uint64_t)__ballot_sync(kFull, b1 <= r0 && e1 >= r1) << 32);
}

// PF: load the next tile's columns into registers while this tile is processed
// (for CTAs of 8 or 16 warps); without it, 32 warps per SM hide the latency.
template <int NW, bool PF>
__global__ void __launch_bounds__(NW * 32, 1)
    sjb_probe_kernel(const __grid_constant__ SjbSchemaRt S, const SjbStep* __restrict__ G,
                     SjbAcc* __restrict__ acc, SjbCounters* __restrict__ ctr) {
  extern __shared__ __align__(16) uint8_t smem[];
  SjbSlot* s_slot = reinterpret_cast<SjbSlot*>(smem);
  int64_t* s_b = reinterpret_cast<int64_t*>(smem + sizeof(SjbSlot) * kBq);
  int64_t* s_e = s_b + kBq;
  SjbAcc* s_acc = reinterpret_cast<SjbAcc*>(s_e + kBq);
  __shared__ PosDim s_dim[SJ_MAX_DIMS];
  __shared__ unsigned long long s_rows;

  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  const uint64_t active = G->active;
  const uint32_t n_smem = G->smem_entries;
  const uint32_t nd = G->n_dims;
  {
    const uint4* src = reinterpret_cast<const uint4*>(G->slot);
    uint4* dst = reinterpret_cast<uint4*>(s_slot);
    for (uint32_t i = tid; i < sizeof(SjbSlot) * kBq / 16; i += blockDim.x) dst[i] = src[i];
    if (tid < kBq) {
      const bool a = (active >> tid) & 1ull;
      s_b[tid] = a ? G->slot[tid].b : INT64_MAX;
      s_e[tid] = a ? G->slot[tid].e : INT64_MIN;
    }
    for (uint32_t i = tid; i < n_smem; i += blockDim.x) s_acc[i] = SjbAcc{0ull, 0ull};
    if (tid < SJ_MAX_DIMS) {
      PosDim p{nullptr, nullptr, 0ull, 0ull, 0, 1u};
      if (tid < nd) {
        const uint32_t d = G->order[tid];
        p.col = S.dim[d].fact_fk;
        p.mask = S.dim[d].mask;
        p.fastmod_m = S.dim[d].fastmod_m;
        p.use = G->use[d];
        p.key_min = S.dim[d].key_min;
        p.len = S.dim[d].len;
      }
      s_dim[tid] = p;
    }
    if (tid == 0) s_rows = 0;
  }
  __syncthreads();

  const int64_t seg_b = G->seg_b, seg_e = G->seg_e, n = S.fact_rows;
  const int32_t* __restrict__ meas = S.measure;
  const int32_t* __restrict__ msub = S.measure_sub;
  unsigned long long rows_seen = 0;
  if (active != 0 && seg_e > seg_b) {
    const int64_t tb = seg_b & ~(int64_t)(kTileRows - 1);
    const int64_t n_tiles = (seg_e - tb + kTileRows - 1) / kTileRows;
    const int64_t gw = (int64_t)blockIdx.x * NW + warp, GW = (int64_t)gridDim.x * NW;

    auto load = [&](int64_t t, uint64_t act, TileCols& c) {
      const int64_t r = tb + t * kTileRows + lane * 4;
#pragma unroll
      for (int k = 0; k < SJ_MAX_DIMS; ++k)
        if (k < (int)nd && (act & s_dim[k].use)) c.fk[k] = ld_col4(s_dim[k].col, r, n);
      c.m = ld_col4(meas, r, n);
      if (msub) c.sub = ld_col4(msub, r, n);
    };

    int64_t t = gw;
    uint64_t act = 0, full = 0;
    TileCols cur;
    cur.m = cur.sub = make_int4(0, 0, 0, 0);
#pragma unroll
    for (int k = 0; k < SJ_MAX_DIMS; ++k) cur.fk[k] = make_int4(0, 0, 0, 0);
    if (t < n_tiles) {
      tile_masks(s_b, s_e, tb + t * kTileRows, lane, act, full);
      if (act) load(t, act, cur);
    }
    while (t < n_tiles) {
      const int64_t tn = t + GW;
      uint64_t actn = 0, fulln = 0;
      TileCols nxt;
      if (PF) {
        nxt = cur;
        if (tn < n_tiles) {
          tile_masks(s_b, s_e, tb + tn * kTileRows, lane, actn, fulln);
          if (actn) load(tn, actn, nxt);
        }
      }
      if (act) {
        const int64_t r0 = tb + t * kTileRows;
        rows_seen += (unsigned long long)(min(r0 + kTileRows, min(seg_e, n)) - max(r0, seg_b));
        const int64_t rb = r0 + lane * 4;
        const uint64_t part = act & ~full;
        uint64_t m[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) m[j] = full;
        if (part) {
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            uint64_t p = part;
            while (p) {
              const int q = __ffsll((long long)p) - 1;
              p &= p - 1;
              if (s_b[q] <= rb + j && rb + j < s_e[q]) m[j] |= 1ull << q;
            }
          }
        }
        // Lookups in order, most selective dimension first; a row stops at the
        // first dimension that leaves it no query.
#pragma unroll
        for (int k = 0; k < SJ_MAX_DIMS; ++k) {
          if (k < (int)nd) {
            const PosDim P = s_dim[k];
            uint64_t w[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              w[j] = ~0ull;
              if (m[j] & P.use) {
                const uint32_t sk = slot_of(pick(cur.fk[k], j), P.key_min, P.len, P.fastmod_m);
                w[j] = __ldg(reinterpret_cast<const unsigned long long*>(P.mask) + sk) | ~P.use;
              }
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) m[j] &= w[j];
          }
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          uint64_t mm = m[j];
          if (!mm) continue;
          const int64_t v = (int64_t)pick(cur.m, j) - (msub ? (int64_t)pick(cur.sub, j) : 0);
          while (mm) {
            const int q = __ffsll((long long)mm) - 1;
            mm &= mm - 1;
            const SjbSlot& Q = s_slot[q];
            uint32_t g = 0;
            for (int gi = 0; gi < Q.n_g; ++gi) {
              // the slot is recomputed here (survivors only) rather than kept per row
              const uint32_t pos = Q.gpos[gi];
              const int32_t fk = (int32_t)pick4((uint32_t)pick(cur.fk[0], j), (uint32_t)pick(cur.fk[1], j),
                                                (uint32_t)pick(cur.fk[2], j), (uint32_t)pick(cur.fk[3], j), pos);
              const PosDim& P = s_dim[pos];
              const uint32_t s = slot_of(fk, P.key_min, P.len, P.fastmod_m);
              const int32_t a = __ldg(Q.gtab[gi] + s);
              g += (uint32_t)(a - Q.pmin[gi]) * Q.stride[gi];
            }
            SjbAcc* dst = Q.smem_off >= 0 ? s_acc + Q.smem_off + g : acc + Q.group_base + g;
            atomicAdd(&dst->cnt, 1ull);
            atomicAdd(&dst->sum, (unsigned long long)v);
          }
        }
      }
      if (PF) {
        cur = nxt;
        act = actn;
        full = fulln;
      } else if (tn < n_tiles) {
        tile_masks(s_b, s_e, tb + tn * kTileRows, lane, act, full);
        if (act) load(tn, act, cur);
      }
      t = tn;
    }
  }
  if (lane == 0 && rows_seen) atomicAdd(&s_rows, rows_seen);
  __syncthreads();
  // flush the shared partials
  uint64_t fl = active;
  while (fl) {
    const int q = __ffsll((long long)fl) - 1;
    fl &= fl - 1;
    const SjbSlot& Q = s_slot[q];
    if (Q.smem_off < 0) continue;
    for (uint32_t i = tid; i < Q.span; i += blockDim.x) {
      const SjbAcc a = s_acc[Q.smem_off + i];
      if (a.cnt) {
        atomicAdd(&acc[Q.group_base + i].cnt, a.cnt);
        atomicAdd(&acc[Q.group_base + i].sum, a.sum);
      }
    }
  }
  if (tid == 0 && s_rows) atomicAdd(&ctr->rows_scanned, s_rows);
}

uint32_t sjb_probe_smem_bytes(uint32_t smem_entries) {
  return (uint32_t)(sizeof(SjbSlot) * kBq + 2 * sizeof(int64_t) * kBq + sizeof(SjbAcc) * smem_entries);
}

template <int NW, bool PF>
static cudaError_t launch_probe_nw(const SjbSchemaRt& S, const SjbStep* step, SjbAcc* acc, SjbCounters* ctr,
                                   uint32_t smem_entries, int sm_count, cudaStream_t st, const L2Window& w) {
  const uint32_t smem = sjb_probe_smem_bytes(smem_entries);
  cudaError_t e = cudaFuncSetAttribute(sjb_probe_kernel<NW, PF>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  return launch_windowed(sjb_probe_kernel<NW, PF>, dim3(sm_count), dim3(NW * 32), smem, st, w, false, S, step, acc,
                         ctr);
}

cudaError_t sjb_launch_probe(const SjbSchemaRt& S, const SjbStep* step, SjbAcc* acc, SjbCounters* ctr,
                             uint32_t threads, uint32_t smem_entries, int sm_count, cudaStream_t st,
                             const L2Window& w) {
  switch (threads) {
    case 256: return launch_probe_nw<8, true>(S, step, acc, ctr, smem_entries, sm_count, st, w);
    case 512: return launch_probe_nw<16, true>(S, step, acc, ctr, smem_entries, sm_count, st, w);
    case 1024: return launch_probe_nw<32, false>(S, step, acc, ctr, smem_entries, sm_count, st, w);
  }
  return cudaErrorInvalidValue;
}

// -------------------------------------------------------------- finalize ----
__global__ void __launch_bounds__(256) sjb_finalize_kernel(const SjbStep* __restrict__ G, uint64_t mask,
                                                           const SjbAcc* __restrict__ acc, sjb_row* __restrict__ out,
                                                           uint64_t cap, SjbCounters* ctr,
                                                           const int32_t* __restrict__ slot_query) {
  const uint32_t q = blockIdx.y;
  // slot_query given: `mask` alone names the slots (serving); else the step's active slots
  const uint64_t sel = slot_query ? mask : (G->active & mask);
  if (!((sel >> q) & 1ull)) return;
  const SjbSlot& s = G->slot[q];
  const uint32_t lane = threadIdx.x & 31u;
  const int32_t qid = slot_query ? slot_query[q] : (int32_t)q;
  const uint32_t span = s.span;
  // `base` is warp-uniform, so the ballot below sees every lane
  for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < span;
       base += gridDim.x * blockDim.x) {
    const uint32_t i = base + lane;
    SjbAcc a{0ull, 0ull};
    if (i < span) a = acc[s.group_base + i];
    const bool keep = a.cnt != 0ull;
    const uint32_t bal = __ballot_sync(kFull, keep);
    if (!bal) continue;
    unsigned long long first = 0;
    if (lane == 0) first = atomicAdd(&ctr->out_rows, (unsigned long long)__popc(bal));
    first = __shfl_sync(kFull, first, 0);
    if (!keep) continue;
    const uint64_t idx = first + __popc(bal & ((1u << lane) - 1u));
    if (idx >= cap) continue;
    sjb_row r;
    r.query = qid;
    r.attr[0] = r.attr[1] = r.attr[2] = r.attr[3] = 0;
    r.pad_ = 0;
    for (int g = 0; g < s.n_g; ++g)
      r.attr[s.gk[g]] = s.pmin[g] + (int32_t)((i / s.stride[g]) % s.width[g]);
    r.count = a.cnt;
    r.sum = a.sum;
    out[idx] = r;
  }
}

cudaError_t sjb_launch_finalize(const SjbStep* step, uint64_t mask, const SjbAcc* acc, sjb_row* out, uint64_t cap,
                                SjbCounters* ctr, const int32_t* slot_query, int sm_count, cudaStream_t st) {
  sjb_finalize_kernel<<<dim3((uint32_t)std::max(1, sm_count / 4), kBq), 256, 0, st>>>(step, mask, acc, out, cap,
                                                                                       ctr, slot_query);
  return cudaGetLastError();
}

}  // namespace sj
