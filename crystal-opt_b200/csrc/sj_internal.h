// sj_internal.h -- device-side data structures shared by the build, probe and
// finalize kernels and the host orchestration (not part of the C ABI).
#pragma once
#include <cstdint>

#include "../../include/starjoin.h"

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include "sj_l2.h"

// Named range on the host timeline for each stage (NVTX v3, header-only: free
// unless a profiler is attached).
struct SjNvtxRange {
  explicit SjNvtxRange(const char* name) { nvtxRangePushA(name); }
  ~SjNvtxRange() { nvtxRangePop(); }
  SjNvtxRange(const SjNvtxRange&) = delete;
  SjNvtxRange& operator=(const SjNvtxRange&) = delete;
};

// Engine handle of the C ABI (include/starjoin.h): one device, one memory pool.
struct sj_engine {
  int device = 0;
  int sm_count = 148;
  size_t smem_optin = 232448;
  cudaMemPool_t pool = nullptr;
  cudaStream_t copy_stream = nullptr;  // host->device staging of streamed columns
  size_t l2_persist_bytes = 0;         // persisting-L2 set-aside held for the probes (0: none)
  size_t l2_window_max = 0;            // largest access-policy window the device takes
};

namespace sj {

// Sets the calling thread's sj_last_error() text and returns s.
sj_status set_error(sj_status s, const char* msg);


constexpr int kMaxDims = SJ_MAX_DIMS;
constexpr int kMaxSteps = 2 * SJ_MAX_DIMS;
constexpr uint32_t kMaxPolls = 1u << 22;  // bounded mbarrier waits (~0.5 s with backoff)

// Device error bits (SjDesc::error_flags).
enum : uint32_t {
  kErrPayloadDomain = 1u << 0,  // a grouped payload fell outside [payload_min, payload_max]
  kErrWaitTimeout = 1u << 1,    // a bounded mbarrier wait expired
  kErrQueueOverflow = 1u << 2,  // internal survivor queue overflow (must never happen)
};

// Filter layouts.
enum : uint32_t {
  kBfDirect = 0,   // one bit per PHT slot, 32-bit words (crystal/bloom.cuh layout)
  kBfBlocked = 1,  // k bits inside one 64-bit word per key (register-blocked)
  kBfAuto = 2,     // plan only: the build picks direct or blocked per dimension
};

// Bits per inserted key of the blocked filter that kBfAuto falls back to.
constexpr uint32_t kAutoBitsPerKey = 16;

// Per-dimension state the build kernels compute on the device.
struct SjDimDev {
  uint32_t n_inserted;     // qualifying dimension rows
  uint32_t bf_log2;        // blocked: log2(#64-bit words); direct: log2(#bits)
  uint32_t n_codes;        // distinct payload values of qualifying rows (grouped dims)
  uint32_t group_stride;   // multiplier of the dim's code in the group index
  uint32_t bf_mode;        // layout the build wrote (kBfDirect or kBfBlocked)
  uint32_t pad_;
};

// Per-query device descriptor (build writes, probe/finalize read, host fetches).
struct SjDesc {
  SjDimDev dim[kMaxDims];
  uint32_t start_order[kMaxDims];  // LIP order the probe starts with
  uint32_t bf_smem_off[kMaxDims];  // filter offset in the probe's shared memory, ~0u: read from L2
  uint32_t n_groups;
  uint32_t error_flags;
  uint32_t groups_out;     // finalize: number of rows written
  uint32_t pad0;
  unsigned long long rows_scanned;
  unsigned long long step_in[kMaxSteps];
  unsigned long long step_out[kMaxSteps];
  unsigned long long bf_probes[kMaxDims];
  unsigned long long bf_passes[kMaxDims];
  unsigned long long reorders;
};

// Runtime parameters of one dimension in the kernels.
struct SjDimRt {
  const int32_t* fact_fk;
  const int32_t* key;
  const int32_t* filter_attr;
  const int32_t* payload;
  const uint32_t* in_bitmap;  // SJ_PRED_IN: bitmap over [0, SJ_MAX_IN_CODES)
  int2* ht;                   // [key, value] slots
  void* bf;                   // filter words
  uint32_t* payload_bitmap;   // grouped: bitmap over the payload domain
  int32_t* dict;              // grouped: code -> payload
  uint32_t* qual_rows;        // indices of the qualifying dimension rows (the scan appends, the insert reads)
  uint64_t rows;
  uint64_t fastmod_m;         // ceil(2^64 / ht_len) for the slot reduction
  int32_t key_min;
  uint32_t ht_len;
  int32_t pred_kind, pred_lo, pred_hi;
  int32_t payload_min;
  uint32_t payload_span;
  uint32_t grouped;
  uint32_t bf_mode;
  uint32_t bf_k;
  uint32_t bf_bits_per_key;
  uint32_t bf_max_log2;       // capacity of the allocated filter
};

struct SjPlanRt {
  SjDimRt dim[kMaxDims];
  SjDesc* desc;
  uint8_t* zero_tables;        // hash tables and filters, cleared by the scan kernel (16-byte multiple)
  uint64_t zero_tables_bytes;  // 0: the caller cleared them
  const int32_t* measure;
  const int32_t* measure_sub;
  unsigned long long* g_sum;
  unsigned long long* g_cnt;
  sj_group_row* rows_out;
  uint64_t row_begin, row_end;
  uint32_t n_dims;
  uint32_t lip;
  uint32_t adaptive;
  uint32_t order[kMaxDims];
  uint32_t group_capacity;    // allocated dense group slots
  uint32_t bf_smem_budget;    // shared-memory bytes the probe holds filters in
};

// Launch geometry of the probe kernel.
struct SjProbeGeom {
  uint32_t threads;
  uint32_t chunk_rows;
  uint32_t stages;
  uint32_t grid;
  uint32_t bf_smem_bytes;
  uint32_t group_smem_cap;    // groups kept in shared memory when n_groups <= this
  uint32_t q1_cap, q2_cap;    // power-of-two survivor ring sizes
  uint32_t reorder_period;    // chunks between adaptive re-rankings
  uint32_t smem_bytes;        // total dynamic shared memory
};

// Slot of key k: (k - key_min) mod ht_len, computed as an unsigned 32-bit
// offset (HASH, crystal/join.cuh:27).  In-range keys take the subtraction
// only; others use Lemire-Kaser-Kurz direct remainder with M = ceil(2^64/d).
__host__ __device__ __forceinline__ uint32_t slot_of(int32_t k, int32_t kmin, uint32_t len, uint64_t m) {
  uint32_t d = (uint32_t)k - (uint32_t)kmin;
  if (d < len) return d;
#ifdef __CUDA_ARCH__
  uint64_t low = m * (uint64_t)d;
  return (uint32_t)__umul64hi(low, (uint64_t)len);
#else
  return d % len;
#endif
}

// Register-blocked filter geometry of PHT slot s: one 64-bit word chosen by the
// top bits of h = s * 0x9E3779B1 (Fibonacci multiplicative hashing, Knuth TAOCP
// vol. 3, 6.4), and k bits inside that word.  Bit j lies in the low 32-bit half
// for even j and in the high half for odd j (a split-block layout: the probe
// tests each bit with one 32-bit rotate), at a 5-bit position taken from the top
// of g = (h ^ (h >> 15)) * 0x846CA68B, a multiply-xorshift-multiply mix that
// decorrelates the positions from the word index on sequential slot numbers.
// Keying on the slot (not the raw key) makes the filter agree with the PHT: it
// never rejects a row whose slot is occupied.
__host__ __device__ __forceinline__ uint32_t bf_h1(uint32_t slot) { return slot * 0x9E3779B1u; }
__host__ __device__ __forceinline__ uint32_t bf_g(uint32_t h1) { return (h1 ^ (h1 >> 15)) * 0x846CA68Bu; }
__host__ __device__ __forceinline__ uint32_t bf_word(uint32_t slot, uint32_t log2w) {
  return log2w ? (bf_h1(slot) >> (32 - log2w)) : 0u;
}
// position (0..31) of bit j within its half
__host__ __device__ __forceinline__ uint32_t bf_pos(uint32_t g, uint32_t j) { return (g >> (27 - 5 * j)) & 31u; }
__host__ __device__ __forceinline__ uint64_t bf_mask(uint32_t slot, uint32_t k) {
  const uint32_t g = bf_g(bf_h1(slot));
  uint64_t m = 0;
  for (uint32_t j = 0; j < k; ++j) m |= (1ull << bf_pos(g, j)) << (32 * (j & 1u));
  return m;
}
// Probe-side test of the same k bits on a word held as two 32-bit halves.
template <int K>
__host__ __device__ __forceinline__ uint32_t bf_test_word(uint32_t lo, uint32_t hi, uint32_t g) {
#ifdef __CUDA_ARCH__
  uint32_t r = __funnelshift_r(lo, lo, g >> 27);  // rotate: uses the shift modulo 32
  if (K > 1) r &= __funnelshift_r(hi, hi, g >> 22);
  if (K > 2) r &= __funnelshift_r(lo, lo, g >> 17);
  if (K > 3) r &= __funnelshift_r(hi, hi, g >> 12);
  return r & 1u;
#else
  uint32_t r = 1u;
  for (int j = 0; j < K; ++j) r &= (((j & 1) ? hi : lo) >> bf_pos(g, (uint32_t)j)) & 1u;
  return r;
#endif
}

__host__ __device__ __forceinline__ uint32_t ceil_log2(uint64_t x) {
  uint32_t l = 0;
  while ((1ull << l) < x) ++l;
  return l;
}

// Filter geometry chosen from the number of inserted keys (blocked layout):
// 64-bit words = next power of two of ceil(n * bits_per_key / 64), clamped.
__host__ __device__ __forceinline__ uint32_t bf_blocked_log2(uint64_t n_inserted, uint32_t bits_per_key,
                                                             uint32_t max_log2) {
  uint64_t bits = n_inserted * (uint64_t)bits_per_key;
  uint64_t words = (bits + 63) / 64;
  if (words < 1) words = 1;
  uint32_t l = ceil_log2(words);
  return l > max_log2 ? max_log2 : l;
}

// Filter layout and size of one dimension once its qualifying rows are counted.
// kBfDirect: one bit per PHT slot (log2 = bf_max_log2 bits).  kBfBlocked:
// words sized from the inserted keys.  kBfAuto: the direct bitmap while it fits
// the probe's shared-memory filter budget, else the blocked layout at
// kAutoBitsPerKey bits per inserted key when that is smaller than the direct
// bitmap (the allocation is the direct bitmap's, so it always fits).
__host__ __device__ __forceinline__ uint32_t bf_effective(uint32_t mode, uint32_t max_log2, uint32_t bits_per_key,
                                                          uint32_t n_inserted, uint32_t smem_budget, uint32_t* log2) {
  if (mode == kBfBlocked) {
    *log2 = bf_blocked_log2(n_inserted, bits_per_key, max_log2);
    return kBfBlocked;
  }
  *log2 = max_log2;
  const uint32_t direct_bytes = max_log2 >= 6 ? (1u << max_log2) / 8u : 8u;
  if (mode == kBfDirect || direct_bytes <= smem_budget || max_log2 < 7) return kBfDirect;
  const uint32_t bl = bf_blocked_log2(n_inserted, kAutoBitsPerKey, max_log2 - 6);
  if ((8u << bl) >= direct_bytes) return kBfDirect;
  *log2 = bl;
  return kBfBlocked;
}

}  // namespace sj
