/*
 * Parity driver over the REFERENCE library (oracle/_ref/ref_driver).
 *
 * TEST INFRASTRUCTURE ONLY.  It builds a program from programs.h with the
 * reference's public API and replays the scheduling of LIE::execute
 * (src/lie/lie.cpp:197-448) itself, so that the per-iteration history vector
 * that RAM::execute_in_batches fills (src/RAM/RA_tasks.h:156, pushed by
 * RAM::check_for_fixed_point src/RAM/RA_tasks.cpp:1072-1085) can be recorded:
 *   - SCC order: first SCC, in add order, that is not the destination of an
 *     edge whose source has not run yet (LIE::one_runnable_tasks, lie.cpp:27-60);
 *   - init_status relations: insert_full_in_delta (lie.cpp:295-301);
 *   - non-fixpoint SCC: one execute_in_batches call (lie.cpp:355-383);
 *     fixpoint SCC: repeat until the last pushed delta sum is 0 (lie.cpp:390-423);
 *   - then RAM::insert_delta_in_full (lie.cpp:432).
 *
 * usage: ref_driver <tc|sg> <edge_file> <empty_file> <out_dir> [batch_size]
 *        ref_driver file <program.txt> <empty_file> <out_dir> <data_dir>
 *                   (a program description, its batch size from the file)
 * writes: <out_dir>/history.txt   "scc <id> <iters>" then "<sum_delta> <sum_full>" per batch
 *         <out_dir>/sizes.txt     "<name> <arity> <full_count>" per relation
 *         <out_dir>/<name>.bin    full relation rows (arity+1 u64, trie order = sorted),
 *                                 unless RA_REF_NODUMP=1 (timing runs)
 *         <out_dir>/time.txt      fixpoint seconds (sum over SCCs of execute_in_batches)
 */
#include "parallel_RA_inc.h"
#include "programs.h"

#include <set>
#include <sys/stat.h>

static void dump_relation(relation* r, const std::string& path)
{
    vector_buffer vb;
    vb.vector_buffer_create_empty();
    std::vector<u64> prefix = {};
    r->get_full()[0].as_vector_buffer_recursive(&vb, prefix);
    FILE* f = fopen(path.c_str(), "wb");
    if (vb.size) fwrite(vb.buffer, 1, vb.size, f);
    fclose(f);
    vb.vector_buffer_free();
}

int main(int argc, char** argv)
{
    if (argc < 5) {
        fprintf(stderr, "usage: %s <tc|sg> <edge_file> <empty_file> <out_dir> [batch_size]\n", argv[0]);
        return 2;
    }
    std::string prog = argv[1], edge = argv[2], empty = argv[3], out = argv[4];
    int batch = (argc > 5 && prog != "file") ? atoi(argv[5]) : 1;

    mpi_comm mcomm;
    mcomm.create(argc, argv);
    mcomm.set_local_comm(MPI_COMM_WORLD);

    ra_program_def p;
    if (prog == "tc") build_tc(p, edge, empty);
    else if (prog == "sg") build_sg(p, edge, empty);
    else if (prog == "file" && argc > 5) {
        build_from_description(p, edge, argv[5], empty);
        batch = pd_batch_size(edge);
    }
    else { fprintf(stderr, "unknown program %s\n", prog.c_str()); return 2; }

    for (relation* r : p.relations) {
        r->set_restart_flag(false);
        r->set_share_io(false);
        r->set_separate_io(false);
        r->set_offset_io(false);
        r->initialize_relation(mcomm);
    }

    mkdir(out.c_str(), 0755);
    FILE* hist = fopen((out + "/history.txt").c_str(), "w");
    std::map<u64, u64> intern_map;
    std::set<RAM*> done;
    double fixpoint_s = 0;

    for (;;) {
        RAM* task = nullptr;
        for (RAM* s : p.sccs) {
            if (done.count(s)) continue;
            bool blocked = false;
            for (auto& d : p.deps)
                if (d.second == s && !done.count(d.first)) blocked = true;
            if (!blocked) { task = s; break; }
        }
        if (!task) break;

        task->set_comm(mcomm);
        relation** rels = task->get_RAM_relations();
        bool* status = task->get_RAM_relations_status();
        for (u32 i = 0; i < task->get_ram_relation_count(); i++)
            if (status[i]) rels[i]->insert_full_in_delta();

        std::vector<u32> history;
        double t[9] = {0};
        int loop = 0;
        double t0 = MPI_Wtime();
        if (task->get_iteration_count() == 1) {
            task->execute_in_batches("ref", batch, history, intern_map, &t[0], &t[1], &t[2], &t[3], &t[4], &t[5], &t[6], &t[7], &t[8], loop, task->get_id(), out, false);
        } else {
            u64 delta = 0;
            do {
                task->execute_in_batches("ref", batch, history, intern_map, &t[0], &t[1], &t[2], &t[3], &t[4], &t[5], &t[6], &t[7], &t[8], loop, task->get_id(), out, false);
                delta = history[history.size() - 2];
                loop++;
            } while (delta != 0);
        }
        task->insert_delta_in_full();
        fixpoint_s += MPI_Wtime() - t0;

        fprintf(hist, "scc %d %zu\n", task->get_id(), history.size() / 2);
        for (size_t i = 0; i + 1 < history.size(); i += 2)
            fprintf(hist, "%u %u\n", history[i], history[i + 1]);
        done.insert(task);
    }
    fclose(hist);

    FILE* sz = fopen((out + "/sizes.txt").c_str(), "w");
    for (relation* r : p.relations) {
        fprintf(sz, "%s %u %d\n", r->get_debug_id().c_str(), r->get_arity(), r->get_full_element_count());
        if (!getenv("RA_REF_NODUMP")) dump_relation(r, out + "/" + r->get_debug_id() + ".bin");
    }
    fclose(sz);
    FILE* tf = fopen((out + "/time.txt").c_str(), "w");
    fprintf(tf, "%.9f\n", fixpoint_s);
    fclose(tf);

    mcomm.destroy();
    return 0;
}
