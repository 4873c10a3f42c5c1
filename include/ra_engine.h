/*
 * parallel-RA on B200: C ABI of the device engine.
 *
 * One ra_program holds the relations, SCCs (strongly connected components,
 * the reference's RAM tasks) and rules of one Datalog program, all resident on
 * one GPU.  The C++ classes relation / RAM / parallel_join / parallel_copy /
 * parallel_copy_filter / LIE in parallel-ra_b200/cxx are thin builders over
 * these calls, so programs written against parallel-RA's C++ API
 * (e.g. tests/transitive_closure.cpp) compile unchanged.
 *
 * Conventions: every call returns an ra_status (0 = RA_OK).  Relations and
 * SCCs are small integer handles local to their program.  Tuples cross the
 * ABI as rows of arity+1 uint64 (data columns, then the intern id column),
 * the layout of the reference's binary relation files
 * (utility/tsv_to_bin.cpp:38-64, src/IO/parallel_io.cpp:115-213).
 * Calls on one program must come from one host thread at a time.
 */
#ifndef RA_ENGINE_H
#define RA_ENGINE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum ra_status {
    RA_OK = 0,
    RA_E_BADARG = 1,      /* invalid handle, arity, projection, version ... */
    RA_E_IO = 2,          /* relation file or its .size metadata unreadable */
    RA_E_OOM = 3,         /* device allocation failed */
    RA_E_CUDA = 4,        /* a CUDA runtime call failed (message via ra_last_error) */
    RA_E_UNSUPPORTED = 5, /* program shape outside what the engine implements */
    RA_E_TIMEOUT = 6,     /* a bounded device-side wait gave up */
    RA_E_STATE = 7        /* call made in the wrong phase (e.g. dump before execute) */
} ra_status;

/* relation versions, src/relation/balanced_hash_relation.h:13 */
#define RA_DELTA 0
#define RA_FULL 1

/* copy rule kinds: parallel_copy (src/RA/parallel_copy.h:28),
 * parallel_acopy (src/RA/parallel_acopy.h:45),
 * parallel_copy_filter (src/RA/parallel_copy_filter.h:29) */
#define RA_COPY 0
#define RA_ACOPY 1
#define RA_COPY_FILTER 2

/* Device-evaluable copy_filter predicates over input columns 0 and 1 (the
 * only columns the reference passes to the filter lambda,
 * src/relation/shmap_relation_exp.cpp:233-236). */
#define RA_PRED_TRUE 0
#define RA_PRED_FALSE 1
#define RA_PRED_EQ 2
#define RA_PRED_NE 3
#define RA_PRED_LT 4
#define RA_PRED_GT 5
#define RA_PRED_LE 6
#define RA_PRED_GE 7

/* Intern-id numbering of derived tuples (ra_program_set_id_order).  Ids are
 * (tag << 46) | counter, counter per intern tag, as in RAM::local_insert_in_newt
 * (src/RAM/RA_tasks.cpp:861-875).  The order in which new tuples take counter
 * values:
 *   RA_IDS_EMISSION  -- this engine's deterministic candidate order (default;
 *                       deltas are not kept sorted between iterations);
 *   RA_IDS_REFERENCE -- the single-rank reference's order: every new delta is
 *                       radix-sorted into trie order so the next iteration
 *                       enumerates candidates exactly as the reference does.
 * Relation contents on the data columns and every per-iteration delta size
 * are identical in both modes; only the id column differs. */
#define RA_IDS_EMISSION 0
#define RA_IDS_REFERENCE 1

typedef struct ra_program ra_program;

/* Per-run statistics of the last ra_program_execute. */
typedef struct ra_stats {
    uint64_t iterations;        /* fixed-point iterations over all SCCs */
    uint64_t join_candidates;   /* sum over iterations of join/copy outputs */
    uint64_t new_tuples;        /* sum over iterations of tuples added to delta */
    uint64_t kernel_launches;   /* engine kernels launched by the run */
    double fixpoint_ms;         /* device time of the SCC loops (CUDA events) */
    double dedup_ms;            /* device time of the fused join+dedup kernels */
    uint64_t dedup_launches;    /* launches of those kernels */
    uint64_t dedup_bytes;       /* algorithmic bytes moved by those kernels */
    uint32_t value_bits;        /* bits per packed column chosen for the run */
    uint32_t reserved;
    /* Device time per phase of the device-driven iterations: from the
     * persistent SCC kernel's own clocks (barrier to barrier: [2] claims incl.
     * heavy rows, [3] select + iteration end), or, for the per-launch kernels,
     * only with per-launch events (RA_KERNEL_EVENTS=1; no graph):
     * [0] join scan, [1] plan, [2] expand + claim, [3] select, [4] sort,
     * [5] iteration end. */
    double phase_ms[6];
    uint64_t graph_builds;      /* CUDA graphs captured + instantiated by the run */
    double graph_build_ms;      /* host time spent building them */
    uint64_t regrows;           /* buffer regrowths (iteration retried) */
    uint64_t device_bytes;      /* device memory the program holds after the run */
    uint64_t device_bytes_peak; /* most device memory it held during the run */
    uint64_t dense_sccs;        /* SCCs run by the dense row-closure evaluator */
    /* Dense evaluator, with per-launch events only (ra_program_set_launch_timing):
     * device time of the row searches and of the emission of new tuples. */
    double dense_search_ms;
    double dense_emit_ms;
    uint64_t bitmap_relations;  /* output relations of device-driven SCCs that used a bitmap seen set */
    uint64_t persistent_launches; /* cooperative launches of the persistent SCC kernel (one per SCC run,
                                     plus one per replay after a buffer grew) */
    uint64_t reach_sccs;        /* SCCs run by the reachability evaluator (composed reachable sets) */
    uint64_t reach_levels;      /* levels it swept (longest path over nodes that reach no cycle, + 1) */
    double reach_ms;            /* host wall time of those evaluations (synchronised, launches included) */
    double reach_phase_ms[4];   /* of which: [0] graph set-up and checks, [1] the level sweep,
                                   [2] nodes that reach a cycle, [3] emission of the new tuples */
    uint64_t sliced_iterations; /* iterations run in slices of outer rows: their candidates did not fit
                                   the candidate buffer the memory cap (ra_program_set_memory_cap) allows */
    uint64_t sliced_passes;     /* join + select passes of those iterations */
    uint64_t heavy_items;       /* work items (2048 candidates each) that join rows with more than 4096
                                   matches were split into, expanded by every block of the launch */
    uint64_t tail_iterations;   /* iterations run by the tail kernel: small iterations back to back in
                                   one thread-block cluster, inside the SCC's CUDA graph */
} ra_stats;

/* Runtime tuning of one program (no counterpart in the reference, whose
 * B-tree/shmap indexes have no load factor).  Picked per machine by the
 * autotuner (parallel-ra_b200/autotune.py); the defaults are its B200 choice.
 *   seen_load_max       hash load factor: a relation's seen set (open addressing,
 *                       power-of-two slots) is rebuilt larger before an
 *                       iteration could push its load past this (0.1 .. 0.9)
 *   seen_grow           a rebuilt seen set is sized for seen_grow x the tuples
 *                       stored and arriving (1.1 .. 8): fewer rebuilds vs memory
 *   log_growth          capacity factor when a relation's tuple log grows (1.1 .. 4)
 *   join_blocks_per_sm  CTAs per SM of the fused join kernel (1 .. 16)
 *   select_blocks_per_sm  CTAs per SM of the winner-selection kernel (1 .. 16)
 *   dense_max_bytes     device bytes the dense row-closure evaluator may use for
 *                       its bit matrices (0 switches it off).  A fixed-point SCC
 *                       whose one rule has the transitive-closure shape
 *                       R(z,x) :- R_delta(y,x), S_full(y,z) over values (per
 *                       instance) below 65,536 runs as one breadth-first search
 *                       per row of R in shared memory instead of the hash-set
 *                       path (emission id order, batch size 1). */
typedef struct ra_tuning {
    double seen_load_max;
    double seen_grow;
    double log_growth;
    uint32_t join_blocks_per_sm;
    uint32_t select_blocks_per_sm;
    double dense_max_bytes;
} ra_tuning;

/* Create a program on CUDA device `device`.  Replaces the per-rank set-up of
 * mpi_comm::create + LIE::LIE (src/comm/comm.cpp:22-30, src/lie/lie.h:67-81). */
int ra_program_create(int device, ra_program** out);
int ra_program_destroy(ra_program* p);
/* Bind the program to an existing CUDA stream (cudaStream_t); 0 = engine's own. */
int ra_program_set_stream(ra_program* p, void* stream);
/* Checkpoint dumps, LIE::enable_IO + set_output_dir + set_cp_iteration (+
 * enable_separate_io) (src/lie/lie.h:81-105, lie.cpp:154-193): after every
 * every_batches-th batch of each SCC (0 = never), the directory
 * <output_dir>/checkpoint-<scc id>-<batch> receives scc_metadata (executed SCC
 * ids) and every relation's <name>_full / <name>_delta rows in trie order with
 * their .size files, as relation::parallel_IO writes them (separate_files:
 * per-rank names <name>_full_0, ...).  Fixed-point SCCs then run one iteration
 * per host round trip. */
int ra_program_set_checkpoint(ra_program* p, const char* output_dir, uint32_t every_batches, int separate_files);
/* Restart from a dump directory, LIE::set_restart_flag + set_restart_dir_name
 * (lie.cpp:260-330): the SCCs listed in its scc_metadata are not run again, and
 * every SCC that runs takes each relation's delta from <dir>/<name>_delta
 * (<name>_delta_0 with separate_files) instead of moving full into delta.
 * The relations' full versions come from their own files (the dump's
 * <name>_full), as the program loads them.  dump_dir NULL or "" = no restart. */
int ra_program_set_restart(ra_program* p, const char* dump_dir, int separate_files);
/* Cap on the device memory the program may hold (0 = none): an allocation past
 * it fails the run with RA_E_OOM, leaving the program reusable -- how a server
 * keeps a program inside its share of the device, and how tests inject an
 * out-of-memory failure from the host.  No reference counterpart. */
int ra_program_set_memory_cap(ra_program* p, uint64_t bytes);
/* Failure-path self-test of the device-side bounded waits: runs the engine's
 * look-back wait on device `device` against a predecessor that never
 * publishes, with a limit of max_polls polls (1 .. the engine's own limit).
 * Returns RA_E_TIMEOUT when the wait gave up and reported it, as every engine
 * wait does instead of spinning forever; the context stays usable.  No
 * reference counterpart (the reference has no device waits). */
int ra_selftest_bounded_wait(int device, uint64_t max_polls);
/* Measures this GPU's random-access ceiling that bounds the seen-set claims of
 * the semi-naive join: `ops` 16-byte compare-and-swaps, then `ops` 8-byte
 * loads, at uniformly random slots of a fresh table of `slots` 16-byte slots
 * (a claim's own access pattern, at the size of the workload's seen set).
 * Writes the rates in operations per second to out_rates[0] (CAS) and
 * out_rates[1] (loads).  Allocates and frees the table itself.  No reference
 * counterpart (a measurement aid for the roofline of the claim kernels). */
int ra_calibrate_random_access(int device, uint64_t slots, uint64_t ops, double* out_rates);
/* Read / replace the program's tuning (RA_E_BADARG outside the ranges above;
 * RA_E_STATE during a run). */
int ra_program_get_tuning(ra_program* p, ra_tuning* out);
int ra_program_set_tuning(ra_program* p, const ra_tuning* t);
/* Iterations per fixed-point check, LIE::set_batch_size (src/lie/lie.h:111). */
int ra_program_set_batch_size(ra_program* p, uint32_t batch_size);
/* RA_IDS_EMISSION or RA_IDS_REFERENCE (no counterpart in the reference, whose
 * ids depend on its rank count). */
int ra_program_set_id_order(ra_program* p, int mode);
/* Per-launch CUDA events around every iteration kernel (fills ra_stats.phase_ms
 * and dedup_ms); iterations are then launched from the host instead of a CUDA
 * graph.  A profiling aid: the reference's counterpart is the per-phase
 * MPI_Wtime table of RAM::execute_in_batches (src/RAM/RA_tasks.cpp:1138-1253). */
int ra_program_set_launch_timing(ra_program* p, int on);
/* No counterpart in the reference (whose only evaluator is the semi-naive loop
 * of RAM::execute_in_batches).  Chooses how the engine runs its SCCs, with the
 * same results either way:
 *   reach       closure-shaped SCCs (R(z,x) :- R_delta(y,x), S_full(y,z), R
 *               initially S reversed) by composing reachable sets (default 0;
 *               RA_REACH=1 in the environment sets 1 at creation);
 *   persistent  every other device-driven SCC as one cooperative launch of the
 *               persistent iteration kernel instead of a CUDA graph of
 *               per-iteration launches (default 0; RA_PERSIST=1 sets 1). */
int ra_program_set_evaluators(ra_program* p, int reach, int persistent);

/* relation(jcc, is_canonical, arity, tag, name, file, version),
 * src/relation/balanced_hash_relation.h:97.  0 <= jcc <= arity <= 63.  A program
 * whose tuples pack into one 63-bit key (arity <= 8, 1 <= jcc, join keys within
 * 30 bits, no intern id copied into a data column) runs on the packed path;
 * any other runs with every relation as rows of arity + 1 u64 in trie order
 * (the wide path, ids numbered as the single-rank reference numbers them), which
 * takes no batched instances (RA_E_UNSUPPORTED). */
int ra_relation_create(ra_program* p, uint32_t jcc, uint32_t arity, uint32_t tag,
                       const char* name, int version, int* rel_out);
/* Initial tuples from host rows (arity+1 u64 each).  Replaces
 * relation::load_data_from_file + populate_full (balanced_hash_relation.cpp:609-793)
 * and the load-time all_to_all (src/IO/parallel_io.cpp:239-297). */
int ra_relation_load_rows(ra_program* p, int rel, const uint64_t* host_rows, uint64_t nrows);
/* Same, from rows already in device memory (copied; the caller keeps ownership). */
int ra_relation_load_rows_device(ra_program* p, int rel, const uint64_t* dev_rows, uint64_t nrows);
/* Same, from a file in the reference's binary format plus "<path>.size"
 * (parallel_io::parallel_read_input_relation_from_file_to_local_buffer,
 * src/IO/parallel_io.cpp:115-213). */
int ra_relation_load_file(ra_program* p, int rel, const char* path);

/* RAM(bool fixpoint, int id), src/RAM/RA_tasks.h:52 */
int ra_scc_create(ra_program* p, int fixpoint, int scc_id, int* scc_out);
/* RAM::add_relation(relation*&, bool init_status), src/RAM/RA_tasks.h:75 */
int ra_scc_add_relation(ra_program* p, int scc, int rel, int init_status);
/* RAM::add_rule(new parallel_join(out, in0, ver0, in1, ver1, proj)),
 * src/RA/parallel_join.h:55 */
int ra_scc_add_join(ra_program* p, int scc, int out, int in0, int ver0, int in1, int ver1,
                    const int* proj, int nproj);
/* RAM::add_rule(new parallel_copy / parallel_acopy / parallel_copy_filter(...)),
 * src/RA/parallel_copy.h:28, parallel_acopy.h:45, parallel_copy_filter.h:29.
 * pred is an RA_PRED_* code (ignored unless kind == RA_COPY_FILTER). */
int ra_scc_add_copy(ra_program* p, int scc, int kind, int out, int in, int ver,
                    const int* proj, int nproj, int pred);
/* LIE::add_scc_dependance(src, dst), src/lie/lie.h:131 */
int ra_scc_depend(ra_program* p, int src_scc, int dst_scc);

/* LIE::execute (src/lie/lie.cpp:197-448): run every SCC in dependency order to
 * its fixed point on the device. */
int ra_program_execute(ra_program* p);
/* One step of LIE::execute's task loop (src/lie/lie.cpp:254-441): run the first
 * runnable SCC (LIE::one_runnable_tasks, lie.cpp:27-60) to its fixed point and
 * store its id in *scc_id, or store -1 when every SCC has run (that call ends the
 * run).  Between steps, relation counts are those LIE::execute prints after an
 * SCC: before that SCC's final delta -> full merge (lie.cpp:432). */
int ra_program_run_next_scc(ra_program* p, int* scc_id);
/* Return every relation to its loaded state so the program can run again. */
int ra_program_reset(ra_program* p);
/* Free the device memory a program keeps between runs (relation logs, seen
 * sets, indexes, iteration scratch, captured graphs) -- the memory-return
 * step of a long-lived server; loaded rows stay.  Ends the last run (its
 * results are gone); the next run allocates afresh.  No reference
 * counterpart: the reference frees its relations only at exit (~LIE). */
int ra_program_release(ra_program* p);

/* Per-SCC history in execution order, flattened as
 * [scc_id, n, (sum_delta, sum_full) x n] per SCC -- the values that
 * RAM::check_for_fixed_point pushes (src/RAM/RA_tasks.cpp:1072-1085). */
int ra_program_history(ra_program* p, uint64_t* out, uint64_t cap, uint64_t* len);
int ra_program_stats(ra_program* p, ra_stats* out);
/* Device time (microseconds) of every iteration of the last run that ran on
 * the device-driven path, SCCs in execution order -- the Total_time column of
 * RAM::execute_in_batches' per-iteration table (src/RAM/RA_tasks.cpp:1198-1235). */
int ra_program_iteration_times(ra_program* p, double* out_us, uint64_t cap, uint64_t* len);

/* relation::get_full_element_count / get_delta_element_count
 * (src/relation/balanced_hash_relation.h:183,206) */
int ra_relation_counts(ra_program* p, int rel, uint64_t* full, uint64_t* delta);
/* Full relation rows (arity+1 u64 each) in lexicographic order, the order in
 * which the reference's trie enumerates them (shmap_relation_exp.cpp:77-112).
 * Writes min(cap_rows, count) rows to host memory. */
int ra_relation_dump_full(ra_program* p, int rel, uint64_t* host_rows, uint64_t cap_rows,
                          uint64_t* rows_out);

/* Batched instances (an extension; the reference runs one program instance per
 * mpirun).  Several independent instances of one program run as a single
 * program over their disjoint union: the caller rebases instance i's values by
 * value_base[i] (strictly increasing; instance i owns the values
 * [value_base[i], value_base[i+1]), the last one everything above its base).
 * Joins match equal values only, so no tuple crosses instances and every
 * iteration of the union is the same iteration of each instance.  Set before a
 * run (n_instances = 0 switches accounting off); the engine then counts every
 * iteration's new tuples per instance, inside the device's winner selection. */
int ra_program_set_instances(ra_program* p, const uint64_t* value_base, uint32_t n_instances);
/* Per-instance new-tuple counts of every iteration of the last run, SCCs in
 * execution order: rows of n_instances counts, one row per iteration -- per
 * instance the sum_delta that RAM::check_for_fixed_point pushes
 * (src/RAM/RA_tasks.cpp:1072-1085) for batch size 1.  *rows = iterations
 * recorded; min(cap_rows, *rows) rows are written.  RA_E_UNSUPPORTED when an
 * SCC of the run took the host path, which keeps no per-instance counts. */
int ra_program_instance_history(ra_program* p, uint64_t* out, uint64_t cap_rows, uint64_t* rows);
/* Per-instance row count and order-independent digest of a relation's full
 * version: counts[i] and digests[i] (n_instances entries each, or one entry
 * when no instances are set) cover the rows whose column 0 lies in instance
 * i's range.  The digest is a sum over rows of a hash of the data columns
 * minus the instance base (ids excluded), so it does not depend on the packing
 * width, the row order or the other instances: a batched run's digest of
 * instance i equals a plain run's digest of that instance alone. */
int ra_relation_instance_summary(ra_program* p, int rel, uint64_t* counts, uint64_t* digests);

/* Largest row count ra_rows_distinct_noalloc accepts. */
#define RA_NOALLOC_MAX_ROWS (1u << 17)

/* No counterpart in the reference.  Sorts nrows rows of arity+1 u64 (data
 * columns, then the id column) lexicographically and drops exact duplicates --
 * the full version a relation holds after loading those rows -- without
 * allocating device memory, for callers that cannot call cudaMalloc (a runtime
 * that reserved the whole GPU up front, a latency-critical thread that must not
 * take cudaMalloc's implicit synchronisation, a host that forbids the CUDA
 * allocator).  dev_rows, dev_out_rows (room for nrows rows) and dev_out_nrows
 * are device pointers; stream is a cudaStream_t (0 = legacy default stream).
 * Returns RA_E_BADARG when nrows > RA_NOALLOC_MAX_ROWS.
 * Returns RA_E_UNSUPPORTED when the rows' data columns do not pack into 63
 * bits (arity x bits of the largest value).
 * Scratch is one fixed static device array (about 6 MB, held on every GPU
 * that loads the library until exit).  Every call looks up that array's
 * device address in the current context (no allocation); the first call on a
 * device also loads the library's device code there, so make it before any
 * stream capture on that device.  The call blocks the calling thread once (a
 * stream synchronisation that reads the largest value back); the rest is
 * stream-ordered, *dev_out_nrows included.  All calls share the array: calls
 * that overlap on the GPU (other streams, other host threads) race and must be
 * serialised by the caller. */
int ra_rows_distinct_noalloc(const uint64_t* dev_rows, uint64_t nrows, uint32_t arity,
                             uint64_t* dev_out_rows, uint64_t* dev_out_nrows, void* stream);

const char* ra_status_string(int status);
/* Message of the last failing call on this program ("" if none). */
const char* ra_last_error(ra_program* p);

#ifdef __cplusplus
}
#endif
#endif /* RA_ENGINE_H */
