/*
 * CPU restatement of parallel-RA's semi-naive fixed point (the oracle).
 *
 * TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py as the checker.  The product library never
 * links, loads or calls it.
 *
 * The call sequence mirrors the B200 library's C ABI (include/ra_engine.h):
 * relations, SCCs, rules, dependencies, execute, then per-relation dumps and
 * the per-SCC history of (sum |delta|, sum |full|) pairs.
 */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_prog oracle_prog;

/* versions (src/relation/balanced_hash_relation.h:13) */
#define ORACLE_DELTA 0
#define ORACLE_FULL 1
/* copy kinds */
#define ORACLE_COPY 0
#define ORACLE_ACOPY 1
#define ORACLE_COPY_FILTER 2
/* predicates on input columns 0 and 1 (values equal include/ra_engine.h RA_PRED_*) */
#define ORACLE_PRED_TRUE 0
#define ORACLE_PRED_FALSE 1
#define ORACLE_PRED_EQ 2
#define ORACLE_PRED_NE 3
#define ORACLE_PRED_LT 4
#define ORACLE_PRED_GT 5
#define ORACLE_PRED_LE 6
#define ORACLE_PRED_GE 7

oracle_prog* oracle_create(void);
void oracle_destroy(oracle_prog* p);
int oracle_relation(oracle_prog* p, uint32_t jcc, uint32_t arity, uint32_t tag, const char* name, int version);
int oracle_load_rows(oracle_prog* p, int rel, const uint64_t* rows, uint64_t nrows);
int oracle_scc(oracle_prog* p, int fixpoint, int id);
int oracle_scc_add_relation(oracle_prog* p, int scc, int rel, int init_status);
int oracle_scc_add_join(oracle_prog* p, int scc, int out, int in0, int ver0, int in1, int ver1,
                        const int* proj, int nproj);
int oracle_scc_add_copy(oracle_prog* p, int scc, int kind, int out, int in, int ver,
                        const int* proj, int nproj, int pred);
int oracle_depend(oracle_prog* p, int src_scc, int dst_scc);
/* runs every SCC in scheduler order; returns 0 on success */
int oracle_execute(oracle_prog* p, int batch_size);
/* history: flattened [scc_id, n_batches, (sum_delta, sum_full) * n_batches] per executed SCC */
uint64_t oracle_history_len(oracle_prog* p);
uint64_t oracle_history(oracle_prog* p, uint64_t* out, uint64_t cap);
uint64_t oracle_full_count(oracle_prog* p, int rel);
/* full relation rows (arity+1 u64 each, trie order); returns rows written */
uint64_t oracle_dump_full(oracle_prog* p, int rel, uint64_t* out, uint64_t cap_rows);
double oracle_fixpoint_seconds(oracle_prog* p);
/* Shortest-path-length histogram of a directed graph over every source
 * (independent check of transitive closure's per-iteration deltas). */
uint64_t oracle_tc_distance_histogram(const uint64_t* src, const uint64_t* dst, uint64_t m, uint64_t n,
                                      uint64_t* hist, uint64_t cap, int threads);

#ifdef __cplusplus
}
#endif
