/*
 * starjoin_batch.h -- shared-scan forms of the star join: many queries, one fact scan.
 *
 * The plain engine (starjoin.h) answers one query per scan of the fact table, as
 * the reference's runQuery does (src/ssb-jo/q33/0-lip.cu:205-302).  The two forms
 * here answer up to SJB_MAX_QUERIES queries per scan:
 *
 *   batch   sjb_batch_run(): a batch of queries with different predicates,
 *           groupings and fact row ranges in one persistent probe launch; the
 *           whole device pipeline (filter builds, mask composition, layout,
 *           probe, group compaction, read-back) replays as one CUDA graph.
 *   serving sjs_server_*(): a request loop over a resident fact table; queries
 *           are admitted as slots and device memory free up, attach to a
 *           circular shared scan at its current position and leave after one
 *           pass over their row range, so queries that arrive while others run
 *           share the scan with them (continuous batching).
 *
 * Semantics per query are those of the plain engine with a direct (exact)
 * filter: a fact row contributes to query q iff, for every dimension q uses,
 * PHT slot (fk - key_min) mod ht_len holds a dimension row that passes q's
 * predicate on that dimension (crystal/join.cuh:27,108-131); the group key is
 * that row's grouped attribute; SUM is the two's-complement uint64 sum of
 * measure - measure_sub.  The shared forms need each slot to hold at most one
 * dimension row (true for SSB's keys 1..N and date key ranges); schema
 * registration checks it and refuses dimensions with colliding keys.
 *
 * How the scan is shared: per dimension d, one 64-bit word per PHT slot holds
 * bit q iff query q's predicate accepts the row in that slot.  A fact row's
 * candidate set starts as the queries whose range covers it, and each
 * dimension lookup ANDs it with that slot's word (queries not using d pass
 * through).  Per (dimension, predicate) filter bitmaps are cached on the device
 * and composed into the mask words whenever the set of running queries changes.
 */
#ifndef STARJOIN_BATCH_H
#define STARJOIN_BATCH_H

#include "starjoin.h"

#ifdef __cplusplus
extern "C" {
#endif

#define SJB_MAX_QUERIES 64
#define SJB_MAX_ATTRS 4

/* A dimension shared by every query of a batch / server. */
typedef struct sjb_dim {
  const int32_t* fact_fk;            /* device, fact_rows entries, 16-byte aligned */
  const int32_t* key;                /* device, rows entries */
  int64_t rows;
  int32_t key_min;                   /* HASH keys_min (19920101 for the date table) */
  int32_t ht_len;                    /* PHT slots */
  int32_t n_attrs;                   /* attribute columns (0..SJB_MAX_ATTRS) */
  const int32_t* attr[SJB_MAX_ATTRS];/* device, rows entries: predicate / group-by attributes */
} sjb_dim;

typedef struct sjb_schema {
  int32_t n_dims;                    /* 1..SJ_MAX_DIMS */
  sjb_dim dims[SJ_MAX_DIMS];
  const int32_t* measure;            /* device, 16-byte aligned */
  const int32_t* measure_sub;        /* optional (SUM(measure - measure_sub)) */
  int64_t fact_rows;
} sjb_schema;

/* One dimension of one query. */
typedef struct sjb_pred {
  int32_t dim;                       /* schema dimension index */
  int32_t kind;                      /* sj_pred_kind */
  int32_t attr;                      /* attribute tested (ignored for SJ_PRED_ALL) */
  int32_t lo, hi;                    /* SJ_PRED_RANGE: lo <= attr <= hi */
  int32_t in_count;                  /* SJ_PRED_IN */
  const int32_t* in_codes;           /* SJ_PRED_IN: HOST array, codes in [0, SJ_MAX_IN_CODES) */
  int32_t group_attr;                /* attribute grouped by, -1: not grouped */
} sjb_pred;

typedef struct sjb_query {
  int32_t n_preds;                   /* 1..SJ_MAX_DIMS, distinct dims */
  sjb_pred preds[SJ_MAX_DIMS];
  int64_t row_begin, row_end;        /* fact rows [row_begin, row_end) */
} sjb_query;

/* One result group.  attr[k] is the grouped attribute of preds[k] (0 when
 * preds[k] is not grouped). */
typedef struct sjb_row {
  int32_t query;                     /* index of the query in its batch (or 0 for a ticket) */
  int32_t attr[SJ_MAX_DIMS];
  int32_t pad_;
  uint64_t count;
  uint64_t sum;
} sjb_row;

typedef struct sjb_limits {
  int64_t group_entries;             /* group accumulator entries (16 B each); 0 = 1<<24 */
  int64_t result_rows;               /* result rows per batch; 0 = 1<<20 */
  int64_t filter_cache_bytes;        /* device bytes for cached filter bitmaps; 0 = 1 GiB */
  int32_t use_graph;                 /* 1: replay the batch pipeline as one CUDA graph */
  int32_t cache_filters;             /* 1: keep filter bitmaps across batches, keyed by predicate */
  int32_t threads;                   /* probe CTA size: 256, 512 or 1024 (0 = 1024) */
  int32_t smem_group_entries;        /* per-CTA shared-memory group partials (0 = 6144) */
} sjb_limits;

typedef struct sjb_batch sjb_batch;

typedef struct sjb_stats {
  float ms_total;                    /* device time of the last batch / step */
  float ms_probe;                    /* shared-scan probe kernel alone */
  uint64_t rows_scanned;             /* fact rows read by the last probe */
  uint64_t filters_built;            /* filter bitmaps built by the last call */
  uint64_t filters_cached;           /* filter bitmaps served from the cache */
  uint64_t group_entries;            /* accumulator entries laid out */
  uint64_t error_flags;
} sjb_stats;

/* Register the schema (checks slot uniqueness, builds per-slot attribute
 * tables) and reserve device memory for the limits. */
sj_status sjb_batch_create(sj_engine* eng, const sjb_schema* schema, const sjb_limits* limits, sjb_batch** out);
void sjb_batch_destroy(sjb_batch* b);

/* Run n queries (1..SJB_MAX_QUERIES) in one shared scan and return their groups,
 * sorted by nothing in particular (row.query names the query).  Synchronous on
 * `stream`.  SJ_ERR_CAPACITY: *n_out holds the rows needed. */
sj_status sjb_batch_run(sjb_batch* b, const sjb_query* queries, int32_t n, sjb_row* out, int64_t cap,
                        int64_t* n_out, void* stream);
sj_status sjb_batch_get_stats(sjb_batch* b, sjb_stats* out);

/* Autotuner of the batched form's probe shape (no counterpart in the
 * reference, which fixes its launch shapes at compile time,
 * src/ssb-jo/q33/0-lip.cu:245,268): runs `sample` (n queries) on a batch of
 * each candidate shape -- CTA size 1024 / 512 / 256 threads x shared-memory
 * group partials 6144 / 2048 / 12288 entries, the other limits from `base` --
 * times the probe (median of `reps` runs after one warm-up) and returns the
 * fastest shape's limits in *chosen.  Every candidate's groups must equal the
 * first candidate's (SJ_ERR_CUDA otherwise).  Synchronous; the default stream. */
typedef struct sjb_tune_report {
  int32_t candidates;                /* shapes timed */
  int32_t mismatches;                /* shapes whose groups differed (must be 0) */
  int32_t threads;                   /* chosen CTA size */
  int32_t smem_group_entries;        /* chosen shared-memory group partials */
  float best_probe_ms;               /* chosen shape's median probe time */
  float default_probe_ms;            /* the default shape's (1024 threads, 6144 entries) */
} sjb_tune_report;
sj_status sjb_batch_tune(sj_engine* eng, const sjb_schema* schema, const sjb_limits* base,
                         const sjb_query* sample, int32_t n, int32_t reps, sjb_limits* chosen,
                         sjb_tune_report* report);

/* ------------------------------------------------------------- serving ---- */
typedef struct sjs_server sjs_server;

typedef struct sjs_config {
  sjb_limits limits;
  int64_t step_rows;                 /* fact rows per scan step (0 = fact_rows / 8) */
  int32_t max_active;                /* queries sharing the scan (1..SJB_MAX_QUERIES, 0 = 64) */
  int32_t plain;                     /* 1: one query at a time through the plain engine (the baseline loop) */
  int64_t hbm_reserve_bytes;         /* device memory left free for others (0 = 2 GiB) */
  int32_t fault_admit_every;         /* fault injection (tests): every k-th admission fails as if its
                                        device allocation had failed (SJ_ERR_OUT_OF_MEMORY); 0 = off */
  int32_t solo_plain;                /* 1: while no query is scanning and exactly one waits, that query runs
                                        through the plain engine (low-load latency; same answer) when its row
                                        range fits in one scan step and its group space fits the plain engine;
                                        0 = every query joins the shared scan */
} sjs_config;

typedef struct sjs_ticket_info {
  int32_t done;                      /* 1: finished (rows available) */
  int32_t status;                    /* sj_status of the query */
  int64_t n_rows;
  double submit_s, admit_s, finish_s;/* host monotonic clock, seconds */
} sjs_ticket_info;

typedef struct sjs_stats {
  uint64_t submitted, admitted, finished, rejected;
  uint64_t steps;                    /* scan steps run */
  uint64_t rows_scanned;             /* fact rows read */
  uint64_t filters_built, filters_cached;
  uint64_t peak_active;
  double busy_s;                     /* wall time the loop spent with work */
  double admit_s;                    /* ... of which admitting (filter builds, layout) */
  double scan_s;                     /* ... of which scan steps (probe, results) */
  double probe_device_s;             /* device time of the shared-scan probes (CUDA events) */
  uint64_t solo;                     /* queries the idle server ran through the plain engine (solo_plain) */
} sjs_stats;

sj_status sjs_server_create(sj_engine* eng, const sjb_schema* schema, const sjs_config* cfg, sjs_server** out);
/* Enqueue a query; thread-safe.  The query (and its IN codes) is copied. */
sj_status sjs_submit(sjs_server* s, const sjb_query* q, uint64_t* ticket);
/* Non-blocking status; when done and out != NULL, copies up to cap rows and
 * releases the ticket (SJ_ERR_CAPACITY keeps it, with info->n_rows the need). */
sj_status sjs_poll(sjs_server* s, uint64_t ticket, sjs_ticket_info* info, sjb_row* out, int64_t cap);
/* Block until the ticket is done (timeout_s <= 0: no limit), then as sjs_poll. */
sj_status sjs_wait(sjs_server* s, uint64_t ticket, double timeout_s, sjs_ticket_info* info, sjb_row* out,
                   int64_t cap);
/* Cancel a ticket: a queued query is dropped, a running one leaves the scan at
 * the next step boundary; either way the ticket completes with SJ_ERR_CANCELLED.
 * Cancelling a finished ticket changes nothing. */
sj_status sjs_cancel(sjs_server* s, uint64_t ticket);
sj_status sjs_get_stats(sjs_server* s, sjs_stats* out);
double sjs_now(void);                /* the clock of sjs_ticket_info, seconds */
/* Stops the loop; open tickets complete with SJ_ERR_CANCELLED and threads
 * blocked in sjs_wait return before the server is freed. */
void sjs_server_destroy(sjs_server* s);

#ifdef __cplusplus
}
#endif
#endif
