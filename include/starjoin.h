/*
 * starjoin.h -- C ABI of the B200 star-join engine (sm_100a).
 *
 * One query = a streaming scan of int32 fact columns, per-dimension Bloom
 * pre-filters applied in Lookahead-Information-Passing (LIP) order, probes into
 * selective perfect hash tables (PHTs) built from the filtered dimension
 * tables, and an exact uint64 group-by SUM.
 *
 * Reference interfaces this ABI replaces (yliang412/crystal-opt):
 *   - runQuery(...)            src/ssb-jo/q33/0-lip.cu:205-302 (LIP drivers) and
 *                              src/ssb-jo/q33/0-naive.cu:178-257 (naive drivers):
 *                              alloc -> memset -> dimension builds -> probe -> D2H.
 *                              Replaced by sj_run_plain() / sj_ssb_q33_run().
 *   - build_hashtable_{s,c,d} src/ssb-jo/q33/0-lip.cu:114-203 (predicate ->
 *                              BlockBuildBloomFilter -> BlockBuildSelectivePHT_2).
 *                              Replaced by sj_query_build().
 *   - probe<128,4>             src/ssb-jo/q33/0-lip.cu:28-112 (BF probes in LIP
 *                              order, PHT probes, group atomicAdd).
 *                              Replaced by sj_query_probe().
 *   - the reference's Q4.1 4-dimension LIP driver (src/ssb-jo/q41/0-lip.cu:28-131)
 *                              is the n_dims == 4 form of the same plan.
 *
 * Conventions
 *   - Every entry point returns an sj_status; nothing calls exit() (the
 *     reference aborts through CubDebugExit, src/ssb-jo/q33/0-lip.cu:224-242).
 *     sj_last_error() gives a human-readable detail for the calling thread.
 *   - Column pointers are caller-owned.  Unless a call says otherwise they are
 *     device pointers, int32, 16-byte aligned (cudaMalloc gives 256).
 *   - Streams are passed as `void*` holding a cudaStream_t (NULL = legacy
 *     default stream, as the reference uses).
 *   - Handles are not shared between threads without external locking; distinct
 *     handles may be used concurrently.
 *   - Key hashing follows the reference exactly: a dimension key K occupies PHT
 *     slot (K - key_min) mod ht_len (crystal/join.cuh:27, HASH).  Keys below
 *     key_min are reduced as unsigned 32-bit offsets (the reference would index
 *     out of bounds there).
 */
#ifndef STARJOIN_H
#define STARJOIN_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SJ_MAX_DIMS 4
#define SJ_MAX_IN_CODES 4096   /* IN-list predicates: codes in [0, 4096) */
#define SJ_MAX_PAYLOAD_SPAN 65536 /* payload_max - payload_min + 1 for grouped dims */
#define SJ_BF_AUTO (-1)          /* sj_plan.bf_bits_per_key: filter layout chosen per dimension */

typedef enum sj_status {
  SJ_OK = 0,
  SJ_ERR_INVALID_ARGUMENT = 1,
  SJ_ERR_UNSUPPORTED = 2,
  SJ_ERR_OUT_OF_MEMORY = 3,
  SJ_ERR_CUDA = 4,
  SJ_ERR_CAPACITY = 5,   /* caller's result buffer is too small; *n_out holds the need */
  SJ_ERR_TIMEOUT = 6,    /* a bounded device-side wait expired; context stays usable */
  SJ_ERR_NO_DEVICE = 7,  /* no CUDA device / extension built without one */
  SJ_ERR_REJECTED = 8,   /* admission control refused the request (serving form) */
  SJ_ERR_CANCELLED = 9   /* the request was cancelled, or its server shut down (serving form) */
} sj_status;

/* Dimension predicate kinds (the reference's BlockPred* chains in the build
 * kernels, src/ssb-jo/q33/0-lip.cu:130-135 and :187-190). */
typedef enum sj_pred_kind {
  SJ_PRED_ALL = 0,   /* every row qualifies (InitFlags) */
  SJ_PRED_IN = 1,    /* attr IN {codes}   (BlockPredEQ + BlockPredOrEQ ...) */
  SJ_PRED_RANGE = 2  /* lo <= attr <= hi (BlockPredGTE / BlockPredLTE) */
} sj_pred_kind;

typedef struct sj_dim {
  /* fact side */
  const int32_t* fact_fk;     /* fact foreign-key column (fact_rows entries) */
  /* dimension table (rows entries per column) */
  const int32_t* key;         /* primary key column (e.g. s_suppkey) */
  const int32_t* filter_attr; /* attribute tested by the predicate (e.g. s_city) */
  const int32_t* payload;     /* value stored in the PHT and used as group key
                                 (e.g. s_city, d_year); NULL -> key-only table
                                 (BlockBuildSelectivePHT_1 form) */
  int64_t rows;
  int32_t key_min;            /* keys_min of HASH (19920101 for the date table) */
  int32_t ht_len;             /* PHT slots (reference: dim rows, or
                                 19981230-19920101+1 = 61130 for dates) */
  int32_t pred_kind;          /* sj_pred_kind */
  int32_t pred_lo, pred_hi;   /* SJ_PRED_RANGE bounds (inclusive) */
  int32_t in_count;           /* SJ_PRED_IN: number of codes */
  const int32_t* in_codes;    /* SJ_PRED_IN: HOST array of codes in [0, SJ_MAX_IN_CODES) */
  int32_t group;              /* 1: payload is part of the group-by key */
  int32_t payload_min;        /* grouped dims: payload domain [min, max] */
  int32_t payload_max;
} sj_dim;

/* Launch geometry; 0 fields are chosen by the engine (or the autotuner cache). */
typedef struct sj_tuning {
  int32_t threads;            /* threads per CTA of the probe kernel (128..1024) */
  int32_t chunk_rows;         /* fact rows per TMA stage (multiple of 4*threads) */
  int32_t stages;             /* TMA ring depth (2..8) */
  int32_t ctas_per_sm;        /* persistent CTAs per SM (1..4) */
  int32_t compact_threshold;  /* survivors queued before a compaction round (0 = threads) */
  int32_t bf_smem_bytes;      /* shared-memory budget for Bloom filters */
  int32_t record_events;      /* 1: CUDA events around each build and probe, for the build_ms /
                                 probe_ms of sj_query_get_stats (0: none; an event between the
                                 build and the probe holds the probe's launch until the build ends) */
} sj_tuning;

typedef struct sj_plan {
  int32_t n_dims;                 /* 1..SJ_MAX_DIMS */
  sj_dim dims[SJ_MAX_DIMS];
  const int32_t* measure;         /* SUM(measure) (e.g. lo_revenue) */
  const int32_t* measure_sub;     /* optional: SUM(measure - measure_sub) (Q4.x) */
  int64_t fact_rows;              /* length of every fact column */
  int64_t row_begin;              /* scanned range [row_begin, row_end) */
  int64_t row_end;                /* -1 -> fact_rows */
  int32_t order[SJ_MAX_DIMS];     /* join order: dim indices, first = outermost */
  int32_t lip;                    /* 1: all Bloom probes first (LIP), 0: naive */
  int32_t adaptive;               /* 1: re-rank the LIP order from observed pass rates */
  int32_t bf_bits_per_key;        /* 0: direct bitmap, one bit per key slot
                                     (crystal/bloom.cuh layout); >0: register-blocked
                                     filter with this many bits per inserted key;
                                     SJ_BF_AUTO: per dimension, the direct bitmap while it
                                     fits the probe's shared-memory filter budget, else the
                                     blocked filter at 16 bits per inserted key (bf_hashes
                                     bits set) when that is smaller */
  int32_t bf_hashes;              /* blocked filter: bits set per key in one 64-bit word (1..4) */
  sj_tuning tune;
} sj_plan;

/* One result group.  attr[d] is the payload of dimension d when that dimension
 * is grouped, else 0.  sum is the two's-complement uint64 sum of the measure
 * (the reference's uint64 accumulation, src/ssb-jo/q31/0-lip.cu:102-110);
 * its low 32 bits equal the reference's int32 sums of Q3.3
 * (src/ssb-jo/q33/0-lip.cu:108). */
typedef struct sj_group_row {
  int32_t attr[SJ_MAX_DIMS];
  uint64_t count;
  uint64_t sum;
} sj_group_row;

/* Per-query counters read back after a probe. */
typedef struct sj_query_stats {
  uint64_t rows_scanned;
  uint64_t step_in[2 * SJ_MAX_DIMS];   /* rows entering plan step i */
  uint64_t step_out[2 * SJ_MAX_DIMS];  /* rows leaving plan step i */
  uint64_t bf_inserted[SJ_MAX_DIMS];   /* keys inserted into each dimension's filter */
  uint64_t bf_words[SJ_MAX_DIMS];      /* filter size in 32-bit words */
  uint64_t groups;                     /* non-empty groups */
  uint64_t reorders;                   /* adaptive LIP re-rankings (all CTAs) */
  uint32_t error_flags;                /* device-side error bits (0 = none) */
  float build_ms, probe_ms;            /* CUDA-event times of the last run (tune.record_events) */
  int32_t bf_blocked[SJ_MAX_DIMS];     /* 1: the dimension's filter was built blocked, 0: direct */
} sj_query_stats;

typedef struct sj_engine sj_engine;
typedef struct sj_query sj_query;

/* ---- engine ------------------------------------------------------------ */
sj_status sj_engine_create(int device, sj_engine** out);
void sj_engine_destroy(sj_engine* e);
const char* sj_status_string(sj_status s);
const char* sj_last_error(void);
int sj_device_sm_count(sj_engine* e);

/* ---- plain single query (drop-in for runQuery) ------------------------- */
/* Validate the plan and reserve device state (PHTs, filters, groups). */
sj_status sj_query_prepare(sj_engine* e, const sj_plan* plan, sj_query** out);
/* Dimension builds: predicate -> filter insert -> PHT insert (async on stream). */
sj_status sj_query_build(sj_query* q, void* stream);
/* Fused scan -> LIP filters -> PHT probes -> group SUM (async on stream). */
sj_status sj_query_probe(sj_query* q, void* stream);
/* Wait for the stream, copy the groups out (sorted by the grouped attrs in
 * dimension order).  SJ_ERR_CAPACITY if cap < groups (*n_out = groups). */
sj_status sj_query_fetch(sj_query* q, sj_group_row* out, int64_t cap, int64_t* n_out, void* stream);
sj_status sj_query_get_stats(sj_query* q, sj_query_stats* out);
void sj_query_release(sj_query* q);

/* prepare + build + probe + fetch + release in one call; *ms gets the CUDA-event
 * time from the first build launch to the end of the probe (the span the
 * reference's time_query covers, src/ssb-jo/q33/0-lip.cu:216-278).
 * If host_columns is nonzero every column pointer in the plan is HOST memory:
 * the engine stages the fact columns to the device itself, inside *ms. */
sj_status sj_run_plain(sj_engine* e, const sj_plan* plan, int host_columns,
                       sj_group_row* out, int64_t cap, int64_t* n_out, float* ms, void* stream);

/* The reference's Q3.3 call, argument for argument (src/ssb-jo/q33/0-lip.cu:205):
 * predicates s_city IN {231,235}, c_city IN {231,235}, d_year <= 1997, group by
 * (d_year, c_city, s_city), SUM(lo_revenue).  order[3] lists the join order
 * over {0 = supplier, 1 = customer, 2 = date} (the six drivers
 * src/ssb-jo/q33/{0..5}-{lip,naive}.cu); lip selects the LIP or naive driver;
 * bf_bits_per_key = 0 keeps the reference's direct bitmap filter.
 * Rows come back as attr[0] = s_city, attr[1] = c_city, attr[2] = d_year. */
sj_status sj_ssb_q33_run(sj_engine* e,
                         const int32_t* lo_orderdate, const int32_t* lo_custkey,
                         const int32_t* lo_suppkey, const int32_t* lo_revenue, int64_t lo_len,
                         const int32_t* d_datekey, const int32_t* d_year, int64_t d_len,
                         const int32_t* s_suppkey, const int32_t* s_city, int64_t s_len,
                         const int32_t* c_custkey, const int32_t* c_city, int64_t c_len,
                         const int32_t order[3], int32_t lip, int32_t bf_bits_per_key,
                         sj_group_row* out, int64_t cap, int64_t* n_out, float* time_query_ms);

/* The same Q3.3 call for callers that cannot allocate device memory while a
 * query runs (a fixed device-memory budget handed out up front, an allocator-free
 * latency path -- cudaMalloc may synchronize the device -- or a runtime that owns
 * every allocation).  No counterpart in the reference.  It allocates nothing: all
 * scratch (hash tables, filters, group partials, result rows) lives in one
 * 48 MiB file-scope device array that every GPU loading this library holds until
 * the process exits; queries needing more return SJ_ERR_CAPACITY (the
 * customer and supplier tables together up to about 2.3M rows fit).  Column pointers are
 * device memory; `out` is a host buffer of `cap` rows.  Every call looks up
 * the array's device address with `device` current (the lookup allocates
 * nothing and stays valid across cudaDeviceReset); the first call on a device
 * also loads the library's device code there, so make it before any stream
 * capture.  Calls share the array and keep the last call's contents (each call
 * clears what must start at zero); calls that overlap on the GPU race, so
 * serialize them.  Errors: sj_noalloc_last_error(). */
sj_status sj_ssb_q33_run_noalloc(int device,
                                 const int32_t* lo_orderdate, const int32_t* lo_custkey,
                                 const int32_t* lo_suppkey, const int32_t* lo_revenue, int64_t lo_len,
                                 const int32_t* d_datekey, const int32_t* d_year, int64_t d_len,
                                 const int32_t* s_suppkey, const int32_t* s_city, int64_t s_len,
                                 const int32_t* c_custkey, const int32_t* c_city, int64_t c_len,
                                 const int32_t order[3], int32_t lip, int32_t bf_bits_per_key,
                                 sj_group_row* out, int64_t cap, int64_t* n_out, void* stream);
const char* sj_noalloc_last_error(void);

/* ---- autotuner ----------------------------------------------------------
 * Chooses the probe's launch geometry (threads per CTA, rows per lane, rows per
 * stage, stage count) and, when asked, the filter kind (direct bitmap,
 * SJ_BF_AUTO with 2 or 3 bits set per key, or blocked Bloom filter with 4/8/16
 * bits per key and 1..4 bits set per key) and
 * the join order, by timing candidates on the plan's own columns (coordinate
 * descent: filter, then geometry, then order).  Every candidate's groups must
 * equal the first candidate's, bit for bit.  With a cache file, the winner is
 * stored under a signature of the plan (table sizes, grouping, and each
 * dimension's selectivity rounded to a power of 2) and later plans with the
 * same signature take it without a search.  No counterpart in the reference,
 * whose geometry is fixed at compile time (src/ssb-jo/q33/0-lip.cu:46-52). */
typedef struct sj_autotune_opts {
  int32_t reps;            /* timed probes per candidate (0 = 5) */
  int32_t tune_filter;     /* 1: also choose bf_bits_per_key / bf_hashes */
  int32_t tune_order;      /* 0: keep the plan's order, 1: most selective first, 2: time every order */
  int32_t verify;          /* 1: compare every candidate's groups with the first's */
  const char* cache_path;  /* tuning cache file, or NULL */
} sj_autotune_opts;

typedef struct sj_autotune_report {
  int32_t candidates;      /* plans timed */
  int32_t cache_hit;       /* 1: taken from the cache, nothing timed */
  int32_t mismatches;      /* candidates whose groups differed (0 unless the engine is wrong) */
  float default_ms;        /* probe time of the plan as given */
  float best_ms;           /* probe time of the chosen plan */
  double selectivity[SJ_MAX_DIMS];  /* qualifying fraction of each dimension's rows */
} sj_autotune_report;

/* plan is in/out: on success its tune, bf_bits_per_key, bf_hashes and order
 * hold the choice.  Device columns only. */
sj_status sj_autotune(sj_engine* e, sj_plan* plan, const sj_autotune_opts* opts, sj_autotune_report* report,
                      void* stream);

/* ---- Bloom filter unit interface (tests; the reference's src/ops/bloom.cu) -- */
/* Build a filter over keys[flags != 0] and probe probe_keys; out_flags[i] = 1 if
 * probe_keys[i] may be present.  All pointers are device pointers.
 * bits_per_key = 0 selects the direct bitmap of `direct_words` 32-bit words. */
sj_status sj_bloom_test(const int32_t* keys, const int32_t* flags, int64_t n_keys,
                        const int32_t* probe_keys, int32_t* out_flags, int64_t n_probe,
                        int32_t bits_per_key, int32_t hashes, int32_t key_min,
                        int32_t direct_words, void* stream);

/* ---- the reference's column files (src/ssb/ssb_utils.h:106-171) ----------
 * One headerless file of native little-endian int32 values per SSB column,
 * named by table and by the column's position in SSB's column list
 * ("lo_custkey" -> "LINEORDER2", "d_year" -> "DDATE4").  With these, SSB data
 * in the reference's data directory loads into the engine, and synthetic
 * columns can be written for the reference's own drivers to read. */
/* The file name of an SSB column (NUL-terminated into out[cap]). */
sj_status sj_ssb_column_file(const char* column, char* out, int64_t cap);
/* Read n values of `column` from directory dir into host memory. */
sj_status sj_ssb_load_column(const char* dir, const char* column, int64_t n, int32_t* out);
/* Write n host values as `column`'s file in directory dir. */
sj_status sj_ssb_store_column(const char* dir, const char* column, int64_t n, const int32_t* data);

/* ---- synthetic data on the device (same values as the host generator) ---- */
/* Fill dst[0..n) with generated column values (see sj_datagen.h kinds). */
sj_status sj_gen_column_device(int32_t* dst, int64_t n, uint64_t seed, int32_t col,
                               int32_t kind, int32_t lo, int32_t hi, void* stream);
/* Rows [row0, row0 + n) of the same column into dst[0..n): one shard of a table
 * that several GPUs split by rows, each generating only its own part. */
sj_status sj_gen_rows_device(int32_t* dst, int64_t row0, int64_t n, uint64_t seed, int32_t col,
                             int32_t kind, int32_t lo, int32_t hi, void* stream);
/* Host form of the same generator (needs no GPU); threads <= 0 uses all cores. */
void sj_gen_column_host(int32_t* dst, int64_t n, uint64_t seed, int32_t col,
                        int32_t kind, int32_t lo, int32_t hi, int threads);

#ifdef __cplusplus
}
#endif
#endif /* STARJOIN_H */
