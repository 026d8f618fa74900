// detail.cuh -- shared machinery of the block-wide device functions.
//
// Every primitive works on a register tile of ITEMS_PER_THREAD items per thread
// in the striped arrangement the reference uses (crystal/load.cuh:25-116): item i
// of thread t is element t + i * BLOCK_THREADS of the tile.  A tile with
// BLOCK_THREADS * ITEMS_PER_THREAD == num_items takes the unguarded path; a
// partial tile skips every item at or beyond num_items.
#pragma once
#include <cstdint>

namespace crystal_b200 {

// Apply f(i) to every item index i of this thread that lies inside the tile.
template <int BT, int IPT, typename F>
__device__ __forceinline__ void for_items(int num_items, F&& f) {
  if (BT * IPT == num_items) {
#pragma unroll
    for (int i = 0; i < IPT; ++i) f(i);
  } else {
    const int t = (int)threadIdx.x;
#pragma unroll
    for (int i = 0; i < IPT; ++i)
      if (t + i * BT < num_items) f(i);
  }
}

// Same, for the tid-explicit "Direct" entry points.
template <int BT, int IPT, typename F>
__device__ __forceinline__ void for_items_tid(int tid, int num_items, bool guarded, F&& f) {
#pragma unroll
  for (int i = 0; i < IPT; ++i)
    if (!guarded || tid + i * BT < num_items) f(i);
}

// Column loads: read-once data, streamed with the evict-first (.cs) hint when
// the type has a cache-streaming intrinsic; plain loads otherwise.
template <typename T>
__device__ __forceinline__ T ld_stream(const T* p) { return *p; }
template <> __device__ __forceinline__ int ld_stream<int>(const int* p) { return __ldcs(p); }
template <> __device__ __forceinline__ unsigned ld_stream<unsigned>(const unsigned* p) { return __ldcs(p); }
template <> __device__ __forceinline__ float ld_stream<float>(const float* p) { return __ldcs(p); }
template <> __device__ __forceinline__ long long ld_stream<long long>(const long long* p) { return __ldcs(p); }
template <> __device__ __forceinline__ unsigned long long ld_stream<unsigned long long>(const unsigned long long* p) {
  return __ldcs(p);
}
template <> __device__ __forceinline__ double ld_stream<double>(const double* p) { return __ldcs(p); }

// (x - min) mod m for the reference's HASH / HASH1 (crystal/join.cuh:27,
// crystal/bloom.cuh:7), with the power-of-two modulus (every filter size the
// drivers use) reduced to a mask.  For keys >= min the value is identical to
// the reference's signed expression; keys below min, where the reference would
// index out of bounds, wrap as unsigned 32-bit offsets and stay in range.
__device__ __forceinline__ int mod_offset(long long x, long long mn, int m) {
  const unsigned d = (unsigned)(x - mn);
  const unsigned um = (unsigned)m;
  return (int)(((um & (um - 1u)) == 0u) ? (d & (um - 1u)) : (d % um));
}

}  // namespace crystal_b200
