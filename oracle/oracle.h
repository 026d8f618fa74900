/*
 * oracle.h -- CPU restatement of the reference star join.  TEST INFRASTRUCTURE:
 * only the tests, the smoke check and the benchmark's CPU-baseline leg use it,
 * as the checker.  The engine never calls it.
 *
 * It restates, in plain C, what the reference computes on the GPU:
 *   - dimension build (src/ssb-jo/q33/0-lip.cu:114-203): predicate on a
 *     dimension attribute, then BlockBuildSelectivePHT_2 (crystal/join.cuh:260-335):
 *     slot h = (key - key_min) % ht_len, slot key set once (atomicCAS from 0),
 *     slot value = payload;
 *   - probe (src/ssb-jo/q33/0-lip.cu:28-112, 0-naive.cu:28-91):
 *     BlockProbeAndPHT_2 (crystal/join.cuh:108-131): a row joins dimension d iff
 *     slot (fk - key_min) % ht_len holds a nonzero key, and then picks up the
 *     slot value; Bloom filters only remove rows a PHT probe would remove, so
 *     the oracle does not model them;
 *   - aggregation (src/ssb-jo/q31/0-lip.cu:98-113 uint64 form): group by the
 *     payloads of the grouped dimensions, SUM as two's-complement uint64.
 */
#ifndef SJ_ORACLE_H
#define SJ_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OR_MAX_DIMS 4

typedef struct or_dim {
  const int32_t* fact_fk;
  const int32_t* key;
  const int32_t* filter_attr;
  const int32_t* payload;   /* NULL: key-only table */
  int64_t rows;
  int32_t key_min;
  int32_t ht_len;
  int32_t pred_kind;        /* 0 all, 1 IN, 2 RANGE */
  int32_t pred_lo, pred_hi;
  int32_t in_count;
  const int32_t* in_codes;
  int32_t group;
  int32_t payload_min, payload_max;
} or_dim;

typedef struct or_plan {
  int32_t n_dims;
  or_dim dims[OR_MAX_DIMS];
  const int32_t* measure;
  const int32_t* measure_sub;
  int64_t row_begin, row_end;
  int32_t order[OR_MAX_DIMS];
} or_plan;

typedef struct or_group_row {
  int32_t attr[OR_MAX_DIMS];
  uint64_t count;
  uint64_t sum;
} or_group_row;

/* Error codes. */
#define OR_OK 0
#define OR_ERR_INVALID 1
#define OR_ERR_CAPACITY 5
#define OR_ERR_PAYLOAD_DOMAIN 9

/* Run the plan over host arrays with `threads` worker threads (0 = all cores
 * this process may use).  Rows come out sorted by the grouped payloads in
 * dimension order.  Returns OR_ERR_CAPACITY with *n_out = groups if cap is short. */
int or_starjoin(const or_plan* plan, int threads, or_group_row* out, int64_t cap, int64_t* n_out);

/* Build only: fill ht (2 * ht_len int32, zeroed by the callee) for dimension d. */
int or_build_pht(const or_dim* d, int32_t* ht);

/* Cores the process may run on. */
int or_available_cores(void);

/* Column `col` of the seeded synthetic schema (crystal-opt_b200/csrc/sj_datagen.h:
 * SplitMix64 stream per column, value a pure function of (seed, col, row)) into
 * dst[0, n), on `threads` host threads (<= 0: all cores).  Lets the benchmark's
 * CPU legs generate their inputs without loading the engine's library. */
void or_gen_column(int32_t* dst, int64_t n, uint64_t seed, int32_t col, int32_t kind, int32_t lo, int32_t hi,
                   int threads);
/* Rows [row0, row0 + n) of the same column into dst[0, n). */
void or_gen_rows(int32_t* dst, int64_t row0, int64_t n, uint64_t seed, int32_t col, int32_t kind, int32_t lo,
                 int32_t hi, int threads);

#ifdef __cplusplus
}
#endif
#endif
