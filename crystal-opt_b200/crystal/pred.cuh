// pred.cuh -- selection flags over register tiles (crystal/pred.cuh of the
// reference): InitFlags sets every flag; BlockPred* overwrites the flags with the
// predicate; BlockPredAnd* / BlockPredOr* combine it with the current flags.
#pragma once
#include "detail.cuh"

template <int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void InitFlags(int (&selection_flags)[ITEMS_PER_THREAD]) {
#pragma unroll
  for (int i = 0; i < ITEMS_PER_THREAD; ++i) selection_flags[i] = 1;
}

namespace crystal_b200 {
enum class Combine { Set, And, Or };

template <Combine C, typename T, typename Op>
__device__ __forceinline__ void combine(int& flag, const T& item, const Op& op) {
  if (C == Combine::Set) flag = op(item) ? 1 : 0;
  else if (C == Combine::And) flag = (flag && op(item)) ? 1 : 0;
  else flag = (flag || op(item)) ? 1 : 0;
}
}  // namespace crystal_b200

#define CRYSTAL_B200_PRED_FAMILY(NAME, MODE)                                                                      \
  template <typename T, typename SelectOp, int BLOCK_THREADS, int ITEMS_PER_THREAD>                               \
  __device__ __forceinline__ void NAME##Direct(int tid, T (&items)[ITEMS_PER_THREAD], SelectOp select_op,        \
                                               int (&selection_flags)[ITEMS_PER_THREAD]) {                       \
    crystal_b200::for_items_tid<BLOCK_THREADS, ITEMS_PER_THREAD>(tid, 0, false, [&](int i) {                     \
      crystal_b200::combine<MODE>(selection_flags[i], items[i], select_op);                                      \
    });                                                                                                           \
  }                                                                                                               \
  template <typename T, typename SelectOp, int BLOCK_THREADS, int ITEMS_PER_THREAD>                               \
  __device__ __forceinline__ void NAME##Direct(int tid, T (&items)[ITEMS_PER_THREAD], SelectOp select_op,        \
                                               int (&selection_flags)[ITEMS_PER_THREAD], int num_items) {        \
    crystal_b200::for_items_tid<BLOCK_THREADS, ITEMS_PER_THREAD>(tid, num_items, true, [&](int i) {              \
      crystal_b200::combine<MODE>(selection_flags[i], items[i], select_op);                                      \
    });                                                                                                           \
  }                                                                                                               \
  template <typename T, typename SelectOp, int BLOCK_THREADS, int ITEMS_PER_THREAD>                               \
  __device__ __forceinline__ void NAME(T (&items)[ITEMS_PER_THREAD], SelectOp select_op,                          \
                                       int (&selection_flags)[ITEMS_PER_THREAD], int num_items) {                \
    crystal_b200::for_items<BLOCK_THREADS, ITEMS_PER_THREAD>(num_items, [&](int i) {                             \
      crystal_b200::combine<MODE>(selection_flags[i], items[i], select_op);                                      \
    });                                                                                                           \
  }

CRYSTAL_B200_PRED_FAMILY(BlockPred, crystal_b200::Combine::Set)
CRYSTAL_B200_PRED_FAMILY(BlockPredAnd, crystal_b200::Combine::And)
CRYSTAL_B200_PRED_FAMILY(BlockPredOr, crystal_b200::Combine::Or)
#undef CRYSTAL_B200_PRED_FAMILY

// Comparison functors (public: drivers may pass them to BlockPred directly).
#define CRYSTAL_B200_CMP(NAME, OP)                                                  \
  template <typename T>                                                             \
  struct NAME {                                                                     \
    T compare;                                                                      \
    __device__ __forceinline__ NAME(T compare) : compare(compare) {}                \
    __device__ __forceinline__ bool operator()(const T& a) const { return a OP compare; } \
  };
CRYSTAL_B200_CMP(LessThan, <)
CRYSTAL_B200_CMP(GreaterThan, >)
CRYSTAL_B200_CMP(LessThanEq, <=)
CRYSTAL_B200_CMP(GreaterThanEq, >=)
CRYSTAL_B200_CMP(Eq, ==)
#undef CRYSTAL_B200_CMP

// Named comparison wrappers: BlockPred{LT,GT,LTE,GTE,EQ}, BlockPredAnd{...}, BlockPredOrEQ.
#define CRYSTAL_B200_NAMED(NAME, FAMILY, FUNCTOR)                                                       \
  template <typename T, int BLOCK_THREADS, int ITEMS_PER_THREAD>                                        \
  __device__ __forceinline__ void NAME(T (&items)[ITEMS_PER_THREAD], T compare,                         \
                                       int (&selection_flags)[ITEMS_PER_THREAD], int num_items) {      \
    FAMILY<T, FUNCTOR<T>, BLOCK_THREADS, ITEMS_PER_THREAD>(items, FUNCTOR<T>(compare), selection_flags, \
                                                           num_items);                                  \
  }
CRYSTAL_B200_NAMED(BlockPredLT, BlockPred, LessThan)
CRYSTAL_B200_NAMED(BlockPredAndLT, BlockPredAnd, LessThan)
CRYSTAL_B200_NAMED(BlockPredGT, BlockPred, GreaterThan)
CRYSTAL_B200_NAMED(BlockPredAndGT, BlockPredAnd, GreaterThan)
CRYSTAL_B200_NAMED(BlockPredLTE, BlockPred, LessThanEq)
CRYSTAL_B200_NAMED(BlockPredAndLTE, BlockPredAnd, LessThanEq)
CRYSTAL_B200_NAMED(BlockPredGTE, BlockPred, GreaterThanEq)
CRYSTAL_B200_NAMED(BlockPredAndGTE, BlockPredAnd, GreaterThanEq)
CRYSTAL_B200_NAMED(BlockPredEQ, BlockPred, Eq)
CRYSTAL_B200_NAMED(BlockPredAndEQ, BlockPredAnd, Eq)
CRYSTAL_B200_NAMED(BlockPredOrEQ, BlockPredOr, Eq)
#undef CRYSTAL_B200_NAMED
