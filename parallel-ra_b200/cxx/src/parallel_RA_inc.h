/*
 * parallel-RA's C++ program API over the B200 engine.
 *
 * Source-compatible with the classes a parallel-RA program uses -- mpi_comm,
 * relation, RAM, parallel_join, parallel_copy, parallel_acopy,
 * parallel_copy_filter, LIE -- so a program that does
 *     #include "../src/parallel_RA_inc.h"
 * (tests/transitive_closure.cpp:1 of the reference) compiles unchanged
 * against this directory.  The classes only record the program; LIE::execute
 * hands it to the device engine through the C ABI in include/ra_engine.h.
 * There is no MPI: the whole program runs on one GPU (RA_DEVICE, default 0).
 */
#pragma once

#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <assert.h>
#include <unistd.h>
#include <sys/stat.h>
#include <iostream>
#include <fstream>
#include <string>
#include <vector>
#include <map>
#include <set>

/* src/compat.h:29-39 */
typedef int8_t s8;
typedef int16_t s16;
typedef int32_t s32;
typedef int64_t s64;
typedef uint8_t u8;
typedef uint16_t u16;
typedef uint32_t u32;
typedef uint64_t u64;
typedef char c8;
typedef wchar_t c16;

/* src/relation/balanced_hash_relation.h:12-15 */
enum {LEFT = 0, RIGHT};
enum {DELTA = 0, FULL, FULL_AND_DELTA};
enum {COPY = 0, COPY_FILTER, COPY_GENERATE, ACOPY, JOIN};
enum {STATIC = 0, DYNAMIC};

/* The handful of MPI names a program itself touches (tests/transitive_closure.cpp
 * uses MPI_Abort on bad arguments).  One process drives one GPU. */
typedef int MPI_Comm;
#ifndef MPI_COMM_WORLD
#define MPI_COMM_WORLD 0
#endif
int MPI_Abort(MPI_Comm comm, int code);
double MPI_Wtime();

/* src/comm/comm.h:8-74, for a single process */
class mpi_comm
{
    int rank = 0, nprocs = 1, local_rank = 0, local_nprocs = 1;
    MPI_Comm world_comm = MPI_COMM_WORLD, local_comm = MPI_COMM_WORLD;

public:
    mpi_comm() {}
    MPI_Comm get_comm() { return world_comm; }
    int get_nprocs() { return nprocs; }
    int get_rank() { return rank; }
    int get_local_nprocs() { return local_nprocs; }
    int get_local_rank() { return local_rank; }
    MPI_Comm get_local_comm() { return local_comm; }
    void set_local_comm(MPI_Comm comm) { local_comm = comm; }
    void create(int argc, char** argv);
    void destroy();
};

struct ra_program;

/* src/relation/balanced_hash_relation.h:17-233 (program-facing part) */
class relation
{
    u32 join_column_count;
    bool is_canonical;
    u32 arity;
    u32 intern_tag;
    std::string debug_id;
    int initailization_type;
    std::string filename;

    ra_program* prog = nullptr;   /* set by LIE::execute */
    int handle = -1;

public:
    relation(u32 jcc, bool is_c, u32 ar, u32 tg, std::string fname, int version)
        : join_column_count(jcc), is_canonical(is_c), arity(ar), intern_tag(tg), initailization_type(version),
          filename(fname) {}
    relation(u32 jcc, bool is_c, u32 ar, u32 tg, std::string did, std::string fname, int version)
        : join_column_count(jcc), is_canonical(is_c), arity(ar), intern_tag(tg), debug_id(did),
          initailization_type(version), filename(fname) {}

    bool get_is_canonical() { return is_canonical; }
    u32 get_arity() { return arity; }
    int get_join_column_count() { return (int)join_column_count; }
    u32 get_intern_tag() { return intern_tag; }
    std::string get_debug_id() { return debug_id; }
    std::string get_filename() { return filename; }
    void set_filename(std::string file) { filename = file; }
    void set_initailization_type(int x) { initailization_type = x; }
    int get_initailization_type() { return initailization_type; }

    /* element counts after (or during) LIE::execute */
    int get_full_element_count();
    int get_delta_element_count();
    u32 get_global_full_element_count() { return (u32)get_full_element_count(); }
    u32 get_global_delta_element_count() { return (u32)get_delta_element_count(); }

    /* Extension: full rows (arity+1 u64 each, sorted) after LIE::execute. */
    std::vector<u64> dump_full();

    /* bound by LIE::execute */
    void bind(ra_program* p, int h) { prog = p; handle = h; }
    int get_handle() const { return handle; }
};

/* src/RA/parallel_RA.h:13-72 */
class parallel_RA
{
protected:
    u32 RA_type = JOIN;

public:
    parallel_RA() {}
    virtual ~parallel_RA() {}
    u32 get_RA_type() { return RA_type; }
};

/* src/RA/parallel_join.h:55 */
class parallel_join : public parallel_RA
{
public:
    relation *out, *in0, *in1;
    int ver0, ver1;
    std::vector<int> proj;
    parallel_join(relation* output, relation* G, int G_type, relation* T, int T_type, std::vector<int> projection)
        : out(output), in0(G), in1(T), ver0(G_type), ver1(T_type), proj(projection) { RA_type = JOIN; }
};

/* src/RA/parallel_copy.h:28 */
class parallel_copy : public parallel_RA
{
public:
    relation *out, *in;
    int ver;
    std::vector<int> reorder;
    parallel_copy(relation* dest, relation* src, int src_version, std::vector<int> reorder_index_array)
        : out(dest), in(src), ver(src_version), reorder(reorder_index_array) { RA_type = COPY; }
};

/* src/RA/parallel_acopy.h:45 */
class parallel_acopy : public parallel_RA
{
public:
    relation *out, *in;
    int ver;
    std::vector<int> reorder;
    parallel_acopy(relation* dest, relation* src, int src_version, std::vector<int> reorder_index_array)
        : out(dest), in(src), ver(src_version), reorder(reorder_index_array) { RA_type = ACOPY; }
};

/* src/RA/parallel_copy_filter.h:29.  The host predicate is fingerprinted at
 * LIE::execute into one of the device predicates RA_PRED_* (include/ra_engine.h);
 * a predicate that matches none of them is rejected with an error. */
class parallel_copy_filter : public parallel_RA
{
public:
    relation *out, *in;
    int ver;
    std::vector<int> reorder;
    bool (*lambda)(const u64* const);
    parallel_copy_filter(relation* dest, relation* src, int src_version, std::vector<int> reorder_index_array,
                         bool (*func)(const u64* const))
        : out(dest), in(src), ver(src_version), reorder(reorder_index_array), lambda(func) { RA_type = COPY_FILTER; }
};

/* src/RAM/RA_tasks.h:14-167 (program-facing part) */
class RAM
{
    int ram_id;
    bool fixpoint;
    std::vector<relation*> rels;
    std::vector<bool> status;
    std::vector<parallel_RA*> RA_list;

public:
    RAM(bool ic, int id) : ram_id(id), fixpoint(ic) {}
    ~RAM();
    int get_id() { return ram_id; }
    int get_iteration_count() { return fixpoint ? -1 : 1; }
    void add_relation(relation*& G, bool i_status) { rels.push_back(G); status.push_back(i_status); }
    void add_rule(parallel_RA* pj) { RA_list.push_back(pj); }
    u32 get_ram_relation_count() { return (u32)rels.size(); }
    void set_refinement_factor(double) {}
    void enable_logging() {}

    bool is_fixpoint() const { return fixpoint; }
    const std::vector<relation*>& relations() const { return rels; }
    const std::vector<bool>& relation_status() const { return status; }
    const std::vector<parallel_RA*>& rules() const { return RA_list; }
};

/* src/lie/lie.h:13-152 */
class LIE
{
    u32 batch_size = 10;
    double batch_time = 0;
    mpi_comm mcomm;
    std::string app_name;
    std::vector<relation*> lie_relations;
    std::vector<RAM*> lie_sccs;
    std::vector<std::pair<RAM*, RAM*>> deps;
    bool enable_io = false, restart_flag = false, share_io = false, offset_io = false, separate_io = false;
    bool all_to_all_meta_data_dump = false;
    std::string restart_dir_name, output_dir;
    int loop_counter = 0, cp_iteration = 0;
    std::vector<int> executed_scc_id;
    ra_program* prog = nullptr;

public:
    LIE() {}
    ~LIE();

    void set_cp_iteration(int iteration) { cp_iteration = iteration; }
    void set_output_dir(std::string output) { output_dir = output; }
    void set_executed_scc_id(std::vector<int> id) { executed_scc_id = id; }
    std::vector<int> get_executed_scc_id() { return executed_scc_id; }
    void set_loop_counter(int count) { loop_counter = count; }
    int get_loop_counter() { return loop_counter; }
    void enable_separate_io() { separate_io = true; }
    void enable_all_to_all_dump() { all_to_all_meta_data_dump = true; }
    void enable_offset_io() { offset_io = true; }
    void enable_share_io() { share_io = true; }
    void set_restart_dir_name(std::string path) { restart_dir_name = path; }
    void set_restart_flag(bool flag) { restart_flag = flag; }
    void enable_IO() { enable_io = true; }

    void print_all_relation_size();
    void set_comm(mpi_comm comm) { mcomm = comm; }
    void set_name(std::string name) { app_name = name; }
    void set_batch_size(u32 bs) { batch_size = bs; }
    u32 get_batch_size() { return batch_size; }
    void set_batch_time(double bt) { batch_time = bt; }
    double get_batch_time() { return batch_time; }

    void add_relation(relation* rel) { lie_relations.push_back(rel); }
    void add_scc(RAM* ra) { lie_sccs.push_back(ra); }
    void add_scc_dependance(RAM* src_task, RAM* destination_task);
    bool execute();

    /* Extension: the per-SCC history of (sum |delta|, sum |full|) after execute,
     * flattened [scc_id, n, pairs...] as ra_program_history returns it. */
    std::vector<u64> get_history();
};
