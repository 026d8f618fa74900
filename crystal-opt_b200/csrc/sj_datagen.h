/*
 * Seeded synthetic star-schema generator (host C/C++ and CUDA device).
 *
 * Stands in for SSB dbgen output (the reference reads raw int32 column files
 * written by its loader, src/ssb/ssb_utils.h:161-171).  Every value is a pure
 * function of (seed, column id, row index), so a column can be produced in any
 * order, on the host or on the GPU, in parallel, and always bit-identically.
 *
 * Random stream: SplitMix64 (Steele, Lea, Flood, "Fast splittable
 * pseudorandom number generators", OOPSLA 2014).  Draw i of a column is the
 * i-th SplitMix64 output for that column's stream key.  A draw maps to a
 * closed integer range [lo, hi] by the multiply-shift reduction
 * lo + ((draw >> 32) * (hi - lo + 1)) >> 32 (Lemire 2019).
 *
 * Distributions follow the star-join workload: fact foreign keys uniform over
 * the dimension key range, revenue uniform in [1, 10^7], city codes uniform over
 * 250 codes (SSB city = nation*10 + digit, test/ssb/loader/convert.py:55,74),
 * part category over 25 codes, a per-dimension "sel" attribute uniform over
 * [0, 1000) for fine-grained selectivity sweeps, and a date dimension of the 2556
 * consecutive SSB days 1992-01-01 .. 1998-12-30 in yyyymmdd form (the reference's
 * date hash table covers exactly 19920101..19981230,
 * src/ssb-jo/q33/0-lip.cu:219).
 */
#ifndef SJ_DATAGEN_H
#define SJ_DATAGEN_H

#include <stdint.h>

#if defined(__CUDACC__)
#define SJ_HD static __host__ __device__ __forceinline__
#else
#define SJ_HD static inline
#endif

/* Column ids: one independent stream per generated column. */
enum {
  SJ_COL_FK_CUST = 1,
  SJ_COL_FK_SUPP = 2,
  SJ_COL_FK_PART = 3,
  SJ_COL_FK_DATE = 4,
  SJ_COL_REVENUE = 5,
  SJ_COL_SUPPLYCOST = 6,
  SJ_COL_CUST_CITY = 11,
  SJ_COL_CUST_SEL = 12,
  SJ_COL_SUPP_CITY = 21,
  SJ_COL_SUPP_SEL = 22,
  SJ_COL_PART_CATEGORY = 31,
  SJ_COL_PART_SEL = 32,
  SJ_COL_PART_BRAND = 33,
  SJ_COL_DATE_SEL = 42
};

/* Number of days in the SSB date dimension (19920101 .. 19981230). */
#define SJ_DATE_DAYS 2556
#define SJ_DATE_MIN 19920101
#define SJ_DATE_MAX 19981230

/* SplitMix64 output function applied to state z (adds the golden gamma first). */
SJ_HD uint64_t sj_mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

/* Stream key of column `col` under `seed`. */
SJ_HD uint64_t sj_stream_key(uint64_t seed, uint32_t col) {
  return sj_mix64(seed ^ ((uint64_t)col << 40));
}

/* Draw i of the stream with key `key`: the i-th SplitMix64 output. */
SJ_HD uint64_t sj_draw(uint64_t key, uint64_t i) {
  return sj_mix64(key + i * 0x9E3779B97F4A7C15ull);
}

/* Map a draw onto the closed range [lo, hi] (hi - lo + 1 <= 2^32). */
SJ_HD int32_t sj_uniform(uint64_t draw, int32_t lo, int32_t hi) {
  uint64_t range = (uint64_t)((int64_t)hi - (int64_t)lo + 1);
  return (int32_t)((int64_t)lo + (int64_t)(((draw >> 32) * range) >> 32));
}

/* yyyymmdd of day `day` (0-based) counted from 1992-01-01. */
SJ_HD int32_t sj_date_key(int32_t day) {
  int32_t y = 1992;
  for (;;) {
    int32_t len = (y % 4 == 0) ? 366 : 365; /* 1992..1998: century rule not needed */
    if (day < len) break;
    day -= len;
    ++y;
  }
  int32_t feb = (y % 4 == 0) ? 29 : 28;
  int32_t m = 1;
  for (;;) {
    int32_t ml = (m == 2) ? feb : ((m == 4 || m == 6 || m == 9 || m == 11) ? 30 : 31);
    if (day < ml) break;
    day -= ml;
    ++m;
  }
  return y * 10000 + m * 100 + day + 1;
}

/* Kinds of generated column (how a draw becomes a value). */
enum {
  SJ_GEN_UNIFORM = 0,  /* uniform in [lo, hi] */
  SJ_GEN_DATEKEY = 1,  /* date key of a uniform day in [0, SJ_DATE_DAYS) */
  SJ_GEN_SEQ = 2,      /* lo + row (dimension primary keys 1..N) */
  SJ_GEN_DATE_SEQ = 3, /* date key of day `row` (date dimension key column) */
  SJ_GEN_DATE_YEAR = 4 /* year of day `row` (date dimension d_year) */
};

/* Value at `row` of a generated column. */
SJ_HD int32_t sj_gen_value(uint64_t key, int32_t kind, int32_t lo, int32_t hi, uint64_t row) {
  switch (kind) {
    case SJ_GEN_DATEKEY:
      return sj_date_key(sj_uniform(sj_draw(key, row), 0, SJ_DATE_DAYS - 1));
    case SJ_GEN_SEQ:
      return (int32_t)((int64_t)lo + (int64_t)row);
    case SJ_GEN_DATE_SEQ:
      return sj_date_key((int32_t)row);
    case SJ_GEN_DATE_YEAR:
      return sj_date_key((int32_t)row) / 10000;
    default:
      return sj_uniform(sj_draw(key, row), lo, hi);
  }
}

#endif /* SJ_DATAGEN_H */
