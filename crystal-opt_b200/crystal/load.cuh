// load.cuh -- striped tile loads (crystal/load.cuh:25-116 of the reference):
// item i of thread t <- ptr[t + i * BLOCK_THREADS]; BlockPredLoad loads only
// items whose selection flag is set.  The caller passes the tile base pointer.
#pragma once
#include "detail.cuh"

template <typename T, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockPredLoadDirect(const unsigned int tid, T* block_itr,
                                                    T (&items)[ITEMS_PER_THREAD],
                                                    int (&selection_flags)[ITEMS_PER_THREAD]) {
  const T* p = block_itr + tid;
  crystal_b200::for_items_tid<BLOCK_THREADS, ITEMS_PER_THREAD>((int)tid, 0, false, [&](int i) {
    if (selection_flags[i]) items[i] = crystal_b200::ld_stream(p + i * BLOCK_THREADS);
  });
}

template <typename T, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockPredLoadDirect(const unsigned int tid, T* block_itr,
                                                    T (&items)[ITEMS_PER_THREAD], int num_items,
                                                    int (&selection_flags)[ITEMS_PER_THREAD]) {
  const T* p = block_itr + tid;
  crystal_b200::for_items_tid<BLOCK_THREADS, ITEMS_PER_THREAD>((int)tid, num_items, true, [&](int i) {
    if (selection_flags[i]) items[i] = crystal_b200::ld_stream(p + i * BLOCK_THREADS);
  });
}

template <typename T, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockPredLoad(T* inp, T (&items)[ITEMS_PER_THREAD], int num_items,
                                              int (&selection_flags)[ITEMS_PER_THREAD]) {
  const T* p = inp + threadIdx.x;
  crystal_b200::for_items<BLOCK_THREADS, ITEMS_PER_THREAD>(num_items, [&](int i) {
    if (selection_flags[i]) items[i] = crystal_b200::ld_stream(p + i * BLOCK_THREADS);
  });
}

template <typename T, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockLoadDirect(const unsigned int tid, T* block_itr, T (&items)[ITEMS_PER_THREAD]) {
  const T* p = block_itr + tid;
  crystal_b200::for_items_tid<BLOCK_THREADS, ITEMS_PER_THREAD>(
      (int)tid, 0, false, [&](int i) { items[i] = crystal_b200::ld_stream(p + i * BLOCK_THREADS); });
}

template <typename T, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockLoadDirect(const unsigned int tid, T* block_itr, T (&items)[ITEMS_PER_THREAD],
                                                int num_items) {
  const T* p = block_itr + tid;
  crystal_b200::for_items_tid<BLOCK_THREADS, ITEMS_PER_THREAD>(
      (int)tid, num_items, true, [&](int i) { items[i] = crystal_b200::ld_stream(p + i * BLOCK_THREADS); });
}

template <typename T, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockLoad(T* inp, T (&items)[ITEMS_PER_THREAD], int num_items) {
  const T* p = inp + threadIdx.x;
  crystal_b200::for_items<BLOCK_THREADS, ITEMS_PER_THREAD>(
      num_items, [&](int i) { items[i] = crystal_b200::ld_stream(p + i * BLOCK_THREADS); });
}
