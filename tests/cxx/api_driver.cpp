/*
 * Parity driver over the B200 library's C++ API (test code).
 *
 * Builds tc or sg from oracle/programs.h -- the same builders ref_driver runs
 * on the reference library -- through the source-compatible classes in
 * parallel-ra_b200/cxx/src, runs LIE::execute, and writes the same files as
 * oracle/ref_driver.cpp: history.txt, sizes.txt and <relation>.bin.
 *
 * usage: api_driver <tc|sg> <edge_file> <empty_file> <out_dir> [batch_size]
 */
#include "parallel_RA_inc.h"
#include "../../oracle/programs.h"

int main(int argc, char** argv)
{
    if (argc < 5) {
        fprintf(stderr, "usage: %s <tc|sg> <edge_file> <empty_file> <out_dir> [batch_size]\n", argv[0]);
        return 2;
    }
    std::string prog = argv[1], edge = argv[2], empty = argv[3], out = argv[4];
    int batch = argc > 5 ? atoi(argv[5]) : 1;
    mpi_comm mcomm;
    mcomm.create(argc, argv);

    ra_program_def p;
    if (prog == "tc") build_tc(p, edge, empty);
    else if (prog == "sg") build_sg(p, edge, empty);
    else return 2;

    LIE* lie = new LIE();
    for (relation* r : p.relations) lie->add_relation(r);
    for (RAM* s : p.sccs) lie->add_scc(s);
    for (auto& d : p.deps) lie->add_scc_dependance(d.first, d.second);
    lie->set_comm(mcomm);
    lie->set_batch_size(batch);
    lie->execute();
    lie->print_all_relation_size();

    mkdir(out.c_str(), 0755);
    std::vector<u64> h = lie->get_history();
    FILE* hist = fopen((out + "/history.txt").c_str(), "w");
    for (size_t i = 0; i < h.size();) {
        u64 id = h[i], n = h[i + 1];
        fprintf(hist, "scc %llu %llu\n", (unsigned long long)id, (unsigned long long)n);
        for (u64 j = 0; j < n; j++)
            fprintf(hist, "%llu %llu\n", (unsigned long long)h[i + 2 + 2 * j], (unsigned long long)h[i + 3 + 2 * j]);
        i += 2 + 2 * n;
    }
    fclose(hist);
    FILE* sz = fopen((out + "/sizes.txt").c_str(), "w");
    for (relation* r : p.relations) {
        fprintf(sz, "%s %u %d\n", r->get_debug_id().c_str(), r->get_arity(), r->get_full_element_count());
        std::vector<u64> rows = r->dump_full();
        FILE* f = fopen((out + "/" + r->get_debug_id() + ".bin").c_str(), "wb");
        if (!rows.empty()) fwrite(rows.data(), 8, rows.size(), f);
        fclose(f);
    }
    fclose(sz);
    delete lie;
    mcomm.destroy();
    return 0;
}
