// store.cuh -- striped tile store (crystal/store.cuh of the reference).
#pragma once
#include "detail.cuh"

template <typename T, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockStoreDirect(int tid, T* block_itr, T (&items)[ITEMS_PER_THREAD]) {
  T* p = block_itr + tid;
  crystal_b200::for_items_tid<BLOCK_THREADS, ITEMS_PER_THREAD>(tid, 0, false,
                                                               [&](int i) { p[i * BLOCK_THREADS] = items[i]; });
}

template <typename T, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockStoreDirect(int tid, T* block_itr, T (&items)[ITEMS_PER_THREAD], int num_items) {
  T* p = block_itr + tid;
  crystal_b200::for_items_tid<BLOCK_THREADS, ITEMS_PER_THREAD>(tid, num_items, true,
                                                               [&](int i) { p[i * BLOCK_THREADS] = items[i]; });
}

template <typename T, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockStore(T* out, T (&items)[ITEMS_PER_THREAD], int num_items) {
  T* p = out + threadIdx.x;
  crystal_b200::for_items<BLOCK_THREADS, ITEMS_PER_THREAD>(num_items,
                                                           [&](int i) { p[i * BLOCK_THREADS] = items[i]; });
}
