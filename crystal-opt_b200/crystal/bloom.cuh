// bloom.cuh -- single-hash Bloom filter over a tile (crystal/bloom.cuh of the
// reference): a key sets / tests bit (key - keys_min) mod (bloom_filter_size * 32)
// of a zero-initialised array of bloom_filter_size 32-bit words.  With at least
// as many bits as the key range (the drivers size it as roundUpToPowerOfTwo(len))
// the filter is exact.  Build skips the atomic when the bit is already set.
// (The engine's own kernels use a register-blocked k-bit filter instead; these
// entry points keep the reference layout so reference drivers run unchanged.)
#pragma once
#include <cstdint>

#include "detail.cuh"

// The reference's hash macro, kept for code that names it.
#define HASH1(X, Y, Z) ((X - Z) % (Y))

namespace crystal_b200 {
template <typename K>
__device__ __forceinline__ void bloom_set(uint32_t* bf, int words, K key, K kmin) {
  const int bit = mod_offset((long long)key, (long long)kmin, words * 32);
  uint32_t* w = bf + (bit >> 5);
  const uint32_t m = 1u << (bit & 31);
  if (!(*w & m)) atomicOr(w, m);
}
template <typename K>
__device__ __forceinline__ int bloom_get(const uint32_t* bf, int words, K key, K kmin) {
  const int bit = mod_offset((long long)key, (long long)kmin, words * 32);
  return (int)((bf[bit >> 5] >> (bit & 31)) & 1u);
}
}  // namespace crystal_b200

template <typename K, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockBuildDirectBloomFilter(int tid, K (&items)[ITEMS_PER_THREAD],
                                                            int (&selection_flags)[ITEMS_PER_THREAD],
                                                            uint32_t* bloom_filter, int bloom_filter_size,
                                                            K keys_min) {
  crystal_b200::for_items_tid<BLOCK_THREADS, ITEMS_PER_THREAD>(tid, 0, false, [&](int i) {
    if (selection_flags[i]) crystal_b200::bloom_set(bloom_filter, bloom_filter_size, items[i], keys_min);
  });
}

template <typename K, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockBuildDirectBloomFilter(int tid, K (&items)[ITEMS_PER_THREAD],
                                                            int (&selection_flags)[ITEMS_PER_THREAD],
                                                            uint32_t* bloom_filter, int bloom_filter_size,
                                                            K keys_min, int num_items) {
  crystal_b200::for_items_tid<BLOCK_THREADS, ITEMS_PER_THREAD>(tid, num_items, true, [&](int i) {
    if (selection_flags[i]) crystal_b200::bloom_set(bloom_filter, bloom_filter_size, items[i], keys_min);
  });
}

template <typename K, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockBuildBloomFilter(K (&keys)[ITEMS_PER_THREAD],
                                                      int (&selection_flags)[ITEMS_PER_THREAD],
                                                      uint32_t* bloom_filter, int bloom_filter_size, K keys_min,
                                                      int num_items) {
  crystal_b200::for_items<BLOCK_THREADS, ITEMS_PER_THREAD>(num_items, [&](int i) {
    if (selection_flags[i]) crystal_b200::bloom_set(bloom_filter, bloom_filter_size, keys[i], keys_min);
  });
}

template <typename K, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockBuildBloomFilter(K (&keys)[ITEMS_PER_THREAD],
                                                      int (&selection_flags)[ITEMS_PER_THREAD],
                                                      uint32_t* bloom_filter, int bloom_filter_size, int num_items) {
  BlockBuildBloomFilter<K, BLOCK_THREADS, ITEMS_PER_THREAD>(keys, selection_flags, bloom_filter, bloom_filter_size,
                                                            (K)0, num_items);
}

template <typename K, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockProbeDirectBloomFilter(int tid, K (&items)[ITEMS_PER_THREAD],
                                                            int (&selection_flags)[ITEMS_PER_THREAD],
                                                            const uint32_t* bloom_filter, int bloom_filter_size,
                                                            K keys_min) {
  crystal_b200::for_items_tid<BLOCK_THREADS, ITEMS_PER_THREAD>(tid, 0, false, [&](int i) {
    if (selection_flags[i])
      selection_flags[i] = crystal_b200::bloom_get(bloom_filter, bloom_filter_size, items[i], keys_min);
  });
}

template <typename K, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockProbeDirectBloomFilter(int tid, K (&items)[ITEMS_PER_THREAD],
                                                            int (&selection_flags)[ITEMS_PER_THREAD],
                                                            const uint32_t* bloom_filter, int bloom_filter_size,
                                                            K keys_min, int num_items) {
  crystal_b200::for_items_tid<BLOCK_THREADS, ITEMS_PER_THREAD>(tid, num_items, true, [&](int i) {
    if (selection_flags[i])
      selection_flags[i] = crystal_b200::bloom_get(bloom_filter, bloom_filter_size, items[i], keys_min);
  });
}

template <typename K, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockProbeBloomFilter(K (&keys)[ITEMS_PER_THREAD],
                                                      int (&selection_flags)[ITEMS_PER_THREAD],
                                                      const uint32_t* bloom_filter, int bloom_filter_size, K keys_min,
                                                      int num_items) {
  crystal_b200::for_items<BLOCK_THREADS, ITEMS_PER_THREAD>(num_items, [&](int i) {
    if (selection_flags[i])
      selection_flags[i] = crystal_b200::bloom_get(bloom_filter, bloom_filter_size, keys[i], keys_min);
  });
}

template <typename K, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockProbeBloomFilter(K (&keys)[ITEMS_PER_THREAD],
                                                      int (&selection_flags)[ITEMS_PER_THREAD],
                                                      const uint32_t* bloom_filter, int bloom_filter_size,
                                                      int num_items) {
  BlockProbeBloomFilter<K, BLOCK_THREADS, ITEMS_PER_THREAD>(keys, selection_flags, bloom_filter, bloom_filter_size,
                                                            (K)0, num_items);
}
