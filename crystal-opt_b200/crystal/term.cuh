// term.cuh -- per-thread early exit test (crystal/term.cuh of the reference):
// true when none of this thread's items is still selected.
#pragma once

template <typename T, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ bool IsTerm(int (&selection_flags)[ITEMS_PER_THREAD]) {
  int any = 0;
#pragma unroll
  for (int i = 0; i < ITEMS_PER_THREAD; ++i) any |= selection_flags[i];
  return any == 0;
}
