/*
 * CPU oracle for the join engine -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain C++ restatement of what the reference engine computes for a plan,
 * used by tests/ and by bench.py's CPU-baseline leg to check the CUDA path.
 * The product never links, loads or calls anything here.
 *
 * Parity is pinned two ways: against the golden cases of the reference's own
 * API tests (tests/unit_tests.cpp:19-663, fixtures in tests/golden/), and
 * against the reference engine itself, built from its sources by
 * oracle/Makefile into oracle/_ref/ and run on the same plan files.
 */
#ifndef B200JOIN_ORACLE_H
#define B200JOIN_ORACLE_H

#include "../include/b200join.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_table oracle_table;
typedef struct oracle_rows oracle_rows;

/* Runs `plan` on the CPU; the result is a table of contest pages. */
int oracle_execute(const bj_plan* plan, oracle_table** out, char* err, uint64_t err_len);
const bj_table* oracle_table_view(const oracle_table* t);
void oracle_table_free(oracle_table* t);

/* Checks the page format of a table (row counts, bitmaps, offsets, long
 * strings). Returns 0 if valid, else writes a message. */
int oracle_validate_table(const bj_table* t, char* err, uint64_t err_len);

/* Decodes a table into a sorted row multiset for exact comparison. */
int oracle_rows_from_table(const bj_table* t, oracle_rows** out, char* err, uint64_t err_len);
uint64_t oracle_rows_count(const oracle_rows* r);
/* 1 if both multisets hold the same rows (same values, same NULLs, same
 * column types), else 0; `first_diff` gets the sorted position of the first
 * difference (or the shorter count). */
int oracle_rows_equal(const oracle_rows* a, const oracle_rows* b, uint64_t* first_diff);
/* Order-independent digest: out[0] = rows, out[1] = sum of row hashes,
 * out[2] = xor of row hashes (64-bit, wrapping). */
void oracle_rows_digest(const oracle_rows* r, uint64_t out[3]);
/* Text of sorted row i ("NULL", integers, %.17g doubles, quoted strings). */
int oracle_rows_format(const oracle_rows* r, uint64_t i, char* buf, uint64_t len);
void oracle_rows_free(oracle_rows* r);

#ifdef __cplusplus
}
#endif

#endif
