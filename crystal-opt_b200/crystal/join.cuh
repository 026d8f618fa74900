// join.cuh -- selective perfect hash tables over a tile (crystal/join.cuh of the
// reference).  Slot of key x: (x - keys_min) mod ht_len.  _1 tables hold one K per
// slot (key only); _2 tables hold a [key, value] pair per slot, read back with
// one 64-bit load.  A probe hits iff the slot is nonzero; the _2 probe returns
// the value (the high 32 bits of the slot).  Build claims the slot's key with
// atomicCAS from 0, then (_2) stores the value.
#pragma once
#include <cstdint>

#include "detail.cuh"

// The reference's hash macro, kept for code that names it.
#define HASH(X, Y, Z) ((X - Z) % Y)

namespace crystal_b200 {
template <typename K>
__device__ __forceinline__ int pht_slot(K key, int len, K kmin) {
  return mod_offset((long long)key, (long long)kmin, len);
}
}  // namespace crystal_b200

template <typename K, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockProbeDirectAndPHT_1(int tid, K (&items)[ITEMS_PER_THREAD],
                                                         int (&selection_flags)[ITEMS_PER_THREAD], K* ht, int ht_len,
                                                         K keys_min) {
  crystal_b200::for_items_tid<BLOCK_THREADS, ITEMS_PER_THREAD>(tid, 0, false, [&](int i) {
    if (selection_flags[i]) selection_flags[i] = ht[crystal_b200::pht_slot(items[i], ht_len, keys_min)] != 0;
  });
}

template <typename K, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockProbeDirectAndPHT_1(int tid, K (&items)[ITEMS_PER_THREAD],
                                                         int (&selection_flags)[ITEMS_PER_THREAD], K* ht, int ht_len,
                                                         K keys_min, int num_items) {
  crystal_b200::for_items_tid<BLOCK_THREADS, ITEMS_PER_THREAD>(tid, num_items, true, [&](int i) {
    if (selection_flags[i]) selection_flags[i] = ht[crystal_b200::pht_slot(items[i], ht_len, keys_min)] != 0;
  });
}

template <typename K, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockProbeAndPHT_1(K (&items)[ITEMS_PER_THREAD],
                                                   int (&selection_flags)[ITEMS_PER_THREAD], K* ht, int ht_len,
                                                   K keys_min, int num_items) {
  crystal_b200::for_items<BLOCK_THREADS, ITEMS_PER_THREAD>(num_items, [&](int i) {
    if (selection_flags[i]) selection_flags[i] = ht[crystal_b200::pht_slot(items[i], ht_len, keys_min)] != 0;
  });
}

template <typename K, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockProbeAndPHT_1(K (&items)[ITEMS_PER_THREAD],
                                                   int (&selection_flags)[ITEMS_PER_THREAD], K* ht, int ht_len,
                                                   int num_items) {
  BlockProbeAndPHT_1<K, BLOCK_THREADS, ITEMS_PER_THREAD>(items, selection_flags, ht, ht_len, (K)0, num_items);
}

namespace crystal_b200 {
template <typename K, typename V>
__device__ __forceinline__ void pht2_probe(const K* ht, int slot, V& res, int& flag) {
  const uint64_t s = *reinterpret_cast<const uint64_t*>(&ht[slot << 1]);
  if (s != 0) res = (V)(s >> 32);
  else flag = 0;
}
}  // namespace crystal_b200

template <typename K, typename V, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockProbeDirectAndPHT_2(int tid, K (&keys)[ITEMS_PER_THREAD],
                                                         V (&res)[ITEMS_PER_THREAD],
                                                         int (&selection_flags)[ITEMS_PER_THREAD], K* ht, int ht_len,
                                                         K keys_min) {
  crystal_b200::for_items_tid<BLOCK_THREADS, ITEMS_PER_THREAD>(tid, 0, false, [&](int i) {
    if (selection_flags[i])
      crystal_b200::pht2_probe(ht, crystal_b200::pht_slot(keys[i], ht_len, keys_min), res[i], selection_flags[i]);
  });
}

template <typename K, typename V, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockProbeDirectAndPHT_2(int tid, K (&items)[ITEMS_PER_THREAD],
                                                         V (&res)[ITEMS_PER_THREAD],
                                                         int (&selection_flags)[ITEMS_PER_THREAD], K* ht, int ht_len,
                                                         K keys_min, int num_items) {
  crystal_b200::for_items_tid<BLOCK_THREADS, ITEMS_PER_THREAD>(tid, num_items, true, [&](int i) {
    if (selection_flags[i])
      crystal_b200::pht2_probe(ht, crystal_b200::pht_slot(items[i], ht_len, keys_min), res[i], selection_flags[i]);
  });
}

template <typename K, typename V, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockProbeAndPHT_2(K (&keys)[ITEMS_PER_THREAD], V (&res)[ITEMS_PER_THREAD],
                                                   int (&selection_flags)[ITEMS_PER_THREAD], K* ht, int ht_len,
                                                   K keys_min, int num_items) {
  crystal_b200::for_items<BLOCK_THREADS, ITEMS_PER_THREAD>(num_items, [&](int i) {
    if (selection_flags[i])
      crystal_b200::pht2_probe(ht, crystal_b200::pht_slot(keys[i], ht_len, keys_min), res[i], selection_flags[i]);
  });
}

template <typename K, typename V, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockProbeAndPHT_2(K (&keys)[ITEMS_PER_THREAD], V (&res)[ITEMS_PER_THREAD],
                                                   int (&selection_flags)[ITEMS_PER_THREAD], K* ht, int ht_len,
                                                   int num_items) {
  BlockProbeAndPHT_2<K, V, BLOCK_THREADS, ITEMS_PER_THREAD>(keys, res, selection_flags, ht, ht_len, (K)0, num_items);
}

template <typename K, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockBuildDirectSelectivePHT_1(int tid, K (&keys)[ITEMS_PER_THREAD],
                                                               int (&selection_flags)[ITEMS_PER_THREAD], K* ht,
                                                               int ht_len, K keys_min) {
  crystal_b200::for_items_tid<BLOCK_THREADS, ITEMS_PER_THREAD>(tid, 0, false, [&](int i) {
    if (selection_flags[i]) atomicCAS(&ht[crystal_b200::pht_slot(keys[i], ht_len, keys_min)], (K)0, keys[i]);
  });
}

template <typename K, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockBuildDirectSelectivePHT_1(int tid, K (&items)[ITEMS_PER_THREAD],
                                                               int (&selection_flags)[ITEMS_PER_THREAD], K* ht,
                                                               int ht_len, K keys_min, int num_items) {
  crystal_b200::for_items_tid<BLOCK_THREADS, ITEMS_PER_THREAD>(tid, num_items, true, [&](int i) {
    if (selection_flags[i]) atomicCAS(&ht[crystal_b200::pht_slot(items[i], ht_len, keys_min)], (K)0, items[i]);
  });
}

template <typename K, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockBuildSelectivePHT_1(K (&keys)[ITEMS_PER_THREAD],
                                                         int (&selection_flags)[ITEMS_PER_THREAD], K* ht, int ht_len,
                                                         K keys_min, int num_items) {
  crystal_b200::for_items<BLOCK_THREADS, ITEMS_PER_THREAD>(num_items, [&](int i) {
    if (selection_flags[i]) atomicCAS(&ht[crystal_b200::pht_slot(keys[i], ht_len, keys_min)], (K)0, keys[i]);
  });
}

template <typename K, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockBuildSelectivePHT_1(K (&keys)[ITEMS_PER_THREAD],
                                                         int (&selection_flags)[ITEMS_PER_THREAD], K* ht, int ht_len,
                                                         int num_items) {
  BlockBuildSelectivePHT_1<K, BLOCK_THREADS, ITEMS_PER_THREAD>(keys, selection_flags, ht, ht_len, (K)0, num_items);
}

namespace crystal_b200 {
template <typename K, typename V>
__device__ __forceinline__ void pht2_insert(K* ht, int slot, K key, V val) {
  atomicCAS(&ht[slot << 1], (K)0, key);
  ht[(slot << 1) + 1] = (K)val;
}
}  // namespace crystal_b200

template <typename K, typename V, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockBuildDirectSelectivePHT_2(int tid, K (&keys)[ITEMS_PER_THREAD],
                                                               V (&res)[ITEMS_PER_THREAD],
                                                               int (&selection_flags)[ITEMS_PER_THREAD], K* ht,
                                                               int ht_len, K keys_min) {
  crystal_b200::for_items_tid<BLOCK_THREADS, ITEMS_PER_THREAD>(tid, 0, false, [&](int i) {
    if (selection_flags[i])
      crystal_b200::pht2_insert(ht, crystal_b200::pht_slot(keys[i], ht_len, keys_min), keys[i], res[i]);
  });
}

template <typename K, typename V, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockBuildDirectSelectivePHT_2(int tid, K (&keys)[ITEMS_PER_THREAD],
                                                               V (&res)[ITEMS_PER_THREAD],
                                                               int (&selection_flags)[ITEMS_PER_THREAD], K* ht,
                                                               int ht_len, K keys_min, int num_items) {
  crystal_b200::for_items_tid<BLOCK_THREADS, ITEMS_PER_THREAD>(tid, num_items, true, [&](int i) {
    if (selection_flags[i])
      crystal_b200::pht2_insert(ht, crystal_b200::pht_slot(keys[i], ht_len, keys_min), keys[i], res[i]);
  });
}

template <typename K, typename V, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockBuildSelectivePHT_2(K (&keys)[ITEMS_PER_THREAD], V (&res)[ITEMS_PER_THREAD],
                                                         int (&selection_flags)[ITEMS_PER_THREAD], K* ht, int ht_len,
                                                         K keys_min, int num_items) {
  crystal_b200::for_items<BLOCK_THREADS, ITEMS_PER_THREAD>(num_items, [&](int i) {
    if (selection_flags[i])
      crystal_b200::pht2_insert(ht, crystal_b200::pht_slot(keys[i], ht_len, keys_min), keys[i], res[i]);
  });
}

template <typename K, typename V, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockBuildSelectivePHT_2(K (&keys)[ITEMS_PER_THREAD], V (&res)[ITEMS_PER_THREAD],
                                                         int (&selection_flags)[ITEMS_PER_THREAD], K* ht, int ht_len,
                                                         int num_items) {
  BlockBuildSelectivePHT_2<K, V, BLOCK_THREADS, ITEMS_PER_THREAD>(keys, res, selection_flags, ht, ht_len, (K)0,
                                                                  num_items);
}
