// reduce.cuh -- block-wide sum (crystal/reduce.cuh of the reference): every
// thread contributes its value (or the sum of its items); thread 0 receives the
// block total.  `shared` must hold 32 elements.  32-bit integers reduce within a
// warp with one redux.sync; other types with a shuffle tree.
#pragma once

namespace crystal_b200 {
template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
template <> __device__ __forceinline__ int warp_sum<int>(int v) { return __reduce_add_sync(0xffffffffu, v); }
template <> __device__ __forceinline__ unsigned warp_sum<unsigned>(unsigned v) {
  return __reduce_add_sync(0xffffffffu, v);
}
}  // namespace crystal_b200

template <typename T, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ T BlockSum(T item, T* shared) {
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  T v = crystal_b200::warp_sum(item);
  if (lane == 0) shared[wid] = v;
  __syncthreads();
  v = ((int)threadIdx.x < (int)(blockDim.x >> 5)) ? shared[lane] : (T)0;
  if (wid == 0) v = crystal_b200::warp_sum(v);
  return v;
}

template <typename T, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ T BlockSum(T (&items)[ITEMS_PER_THREAD], T* shared) {
  T s = 0;
#pragma unroll
  for (int i = 0; i < ITEMS_PER_THREAD; ++i) s += items[i];
  return BlockSum<T, BLOCK_THREADS, ITEMS_PER_THREAD>(s, shared);
}
