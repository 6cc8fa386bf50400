/*
 * Seeded synthetic workloads and page encoding (libb200join_workloads.so).
 *
 * The reference measures on JOB/IMDB, which is not available here; these
 * generators build tables of the benchmark shapes instead (seeded, so every
 * process that asks for the same name/seed/scale gets identical pages):
 *
 *   "join2"     two-table equi-join. R: 1M rows, INT32 key = permutation of
 *               0..1M-1, INT64 payload uniform in [0, 2^40). S: 8M rows, INT32
 *               fk uniform over R's keys with 10% NULL, INT32 payload uniform in
 *               [0, 1e6). Output R.payload, S.payload, S.fk.
 *   "snowflake" fact table of 50M rows with four INT32 foreign keys, each
 *               Zipf(s=1.1) over its dimension's keys (rank->key by a seeded
 *               permutation); dimensions of 5M / 1M / 200K / 20K rows with a
 *               unique INT32 key, an INT32 attribute uniform in [0,1000) and a
 *               VARCHAR of uniform length 1..64 (printable ASCII). The
 *               dimensions are pre-filtered on attr < 10 / 50 / 300 / 600
 *               (1% / 5% / 30% / 60%) before they reach the plan, as the
 *               contest applies SQL filters at load time. Output: two
 *               dimension strings and two fact keys.
 *
 *   "schema20"  20 tables in a random PK-FK tree (10K-40M rows before a
 *               per-table filter of selectivity log-uniform in [0.1%, 100%];
 *               FKs uniform or Zipf(0.8-1.5) over the parent's keys; columns:
 *               INT32 key, INT32 FK, INT32 / FP64 / VARCHAR payloads) and 256
 *               random acyclic queries of 2-12 tables over them
 *               (bjw_workload_query); the workload's plan is query 0.
 *   "schema20w" the same tables and queries with INT64 join keys on every
 *               other table (odd ids key their rows, and their children
 *               reference them, by INT64 values whose low 32 bits are the
 *               INT32 key's and whose high halves vary from -4 to 3); no
 *               reference counterpart (the reference reads join keys as 32
 *               bits), so results are checked against the oracle only.
 *
 * `scale` multiplies every row count (1.0 = the sizes above).
 */
#ifndef B200JOIN_WORKLOADS_H
#define B200JOIN_WORKLOADS_H

#include "../../include/b200join.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct bjw_workload bjw_workload;
typedef struct bjw_pages bjw_pages;

/* Builds a named workload; returns 0 on success. */
BJ_API int bjw_workload_create(const char* name, uint64_t seed, double scale, bjw_workload** out);
/* The same with `nqueries` queries for "schema20" (query k depends only on
 * the seed, the scale and k, so the first 256 equal the default workload's);
 * other names ignore nqueries. */
BJ_API int bjw_workload_create_queries(const char* name, uint64_t seed, double scale, uint64_t nqueries,
                                       bjw_workload** out);
/* Rows of input `table` before the filter applied at load time (schema20),
 * else its row count. */
BJ_API uint64_t bjw_workload_base_rows(bjw_workload* w, uint64_t table);
/* Loads a plan written by bjw_save_plan. */
BJ_API int bjw_workload_load(const char* path, bjw_workload** out);
/* The plan view (valid until bjw_workload_free). */
BJ_API const bj_plan* bjw_workload_plan(bjw_workload* w);
/* Snowflake only: the fact table joined with its first `dims` dimensions
 * (1..4), over the workload's first dims + 1 tables (pages shared); output: the
 * four fact keys and the joined dimensions' names. NULL for other workloads.
 * Valid until bjw_workload_free. */
BJ_API const bj_plan* bjw_workload_variant(bjw_workload* w, int dims);
/* Queries of the workload (1 except for "schema20") and query k (valid until
 * bjw_workload_free; NULL when k is out of range). */
BJ_API uint64_t bjw_workload_num_queries(bjw_workload* w);
BJ_API const bj_plan* bjw_workload_query(bjw_workload* w, uint64_t k);
/* Total bytes of input pages the plan's scans read. */
BJ_API uint64_t bjw_workload_scan_bytes(bjw_workload* w);
BJ_API void bjw_workload_free(bjw_workload* w);

/* Writes a plan (with its pages) to a file; returns 0 on success. */
BJ_API int bjw_save_plan(const char* path, const bj_plan* plan);
/* Writes a table to a file; returns 0 on success. */
BJ_API int bjw_save_table(const char* path, const bj_table* table);

/* Encodes one column from flat arrays with the contest's packing rules.
 * INT32: values is int32_t[n]; INT64: int64_t[n]; FP64: double[n];
 * VARCHAR: values is ignored, str_offsets[n+1] index str_bytes.
 * valid may be NULL (no NULLs); else valid[i] != 0 marks a non-null row. */
BJ_API int bjw_encode_column(int32_t type, uint64_t n, const void* values, const uint8_t* valid,
                      const uint64_t* str_offsets, const char* str_bytes, bjw_pages** out);
BJ_API uint64_t bjw_pages_count(const bjw_pages* p);
BJ_API const void* const* bjw_pages_ptrs(const bjw_pages* p);
BJ_API void bjw_pages_free(bjw_pages* p);

#ifdef __cplusplus
}
#endif

#endif
