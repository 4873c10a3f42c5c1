/*
 * Implementation of the source-compatible C++ program API
 * (cxx/src/parallel_RA_inc.h) over the engine's C ABI (include/ra_engine.h).
 *
 * Ownership follows the reference: ~LIE deletes the relations it was given
 * (src/lie/lie.cpp:451-458), each RAM is deleted once it has run
 * (LIE::update_task_graph, lie.cpp:64-75), and ~RAM deletes its rules
 * (src/RAM/RA_tasks.cpp:10-15).  Errors the reference would abort on
 * (unreadable relation file, MPI_Abort) print a message and exit(1).
 */
#include "parallel_RA_inc.h"
#include "ra_engine.h"

#include <chrono>

namespace {

[[noreturn]] void die(ra_program* p, int st, const char* what)
{
    fprintf(stderr, "parallel-RA (B200): %s failed: %s%s%s\n", what, ra_status_string(st), p ? ": " : "",
            p ? ra_last_error(p) : "");
    fflush(stdout);
    exit(1);
}

#define RA_CK(p, call)                         \
    do {                                       \
        int st_ = (call);                      \
        if (st_ != RA_OK) die((p), st_, #call); \
    } while (0)

/* Map a host filter predicate onto a device predicate by evaluating it on a
 * fixed set of column pairs: the lambda sees input columns 0 and 1 only
 * (src/relation/shmap_relation_exp.cpp:233-236), so its behaviour over
 * ordered / equal pairs identifies it among the comparison predicates. */
int classify_predicate(bool (*f)(const u64* const))
{
    static const u64 vals[] = {0ull, 1ull, 2ull, 3ull, 7ull, 1000ull, 1ull << 40, (1ull << 62) + 5};
    const int n = (int)(sizeof vals / sizeof vals[0]);
    bool ok[8];
    for (int k = 0; k < 8; k++) ok[k] = true;
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) {
            u64 d[2] = {vals[i], vals[j]};
            bool r = f(d);
            const u64 a = vals[i], b = vals[j];
            const bool expect[8] = {true, false, a == b, a != b, a < b, a > b, a <= b, a >= b};
            for (int k = 0; k < 8; k++) ok[k] = ok[k] && (r == expect[k]);
        }
    for (int k = 0; k < 8; k++)
        if (ok[k]) return k;   /* RA_PRED_TRUE .. RA_PRED_GE share these codes */
    return -1;
}

}  // namespace

int MPI_Abort(MPI_Comm, int code)
{
    fflush(stdout);
    exit(code == 0 ? 1 : (code & 0xff));
}

double MPI_Wtime()
{
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

void mpi_comm::create(int, char**) {}
void mpi_comm::destroy() {}

int relation::get_full_element_count()
{
    if (!prog) return 0;
    uint64_t f = 0, d = 0;
    RA_CK(prog, ra_relation_counts(prog, handle, &f, &d));
    return (int)f;
}

int relation::get_delta_element_count()
{
    if (!prog) return 0;
    uint64_t f = 0, d = 0;
    RA_CK(prog, ra_relation_counts(prog, handle, &f, &d));
    return (int)d;
}

std::vector<u64> relation::dump_full()
{
    std::vector<u64> rows;
    if (!prog) return rows;
    uint64_t f = 0, d = 0, got = 0;
    RA_CK(prog, ra_relation_counts(prog, handle, &f, &d));
    rows.resize((size_t)f * (arity + 1));
    RA_CK(prog, ra_relation_dump_full(prog, handle, rows.data(), f, &got));
    rows.resize((size_t)got * (arity + 1));
    return rows;
}

RAM::~RAM()
{
    for (parallel_RA* r : RA_list) delete r;
}

void LIE::add_scc_dependance(RAM* src_task, RAM* destination_task)
{
    for (auto& d : deps)
        if (d.first == src_task && d.second == destination_task) return;
    deps.push_back({src_task, destination_task});
}

bool LIE::execute()
{
    int device = 0;
    if (const char* e = getenv("RA_DEVICE")) device = atoi(e);
    if (!prog) RA_CK(nullptr, ra_program_create(device, &prog));
    /* RA_ID_ORDER=reference numbers new tuples exactly as the single-rank
     * reference does (see ra_program_set_id_order); default: emission order */
    if (const char* e = getenv("RA_ID_ORDER"))
        RA_CK(prog, ra_program_set_id_order(prog, strcmp(e, "reference") == 0 ? RA_IDS_REFERENCE : RA_IDS_EMISSION));

    /* checkpoint dumps (lie.cpp:154-193, 356-420) and restart (lie.cpp:260-330) */
    RA_CK(prog, ra_program_set_checkpoint(prog, enable_io ? output_dir.c_str() : "",
                                          enable_io && cp_iteration > 0 ? (uint32_t)cp_iteration : 0,
                                          separate_io ? 1 : 0));
    RA_CK(prog, ra_program_set_restart(prog, restart_flag ? restart_dir_name.c_str() : "", separate_io ? 1 : 0));

    std::map<relation*, int> handle;
    for (relation* r : lie_relations) {
        int h = -1;
        RA_CK(prog, ra_relation_create(prog, (uint32_t)r->get_join_column_count(), r->get_arity(),
                                       r->get_intern_tag(), r->get_debug_id().c_str(),
                                       r->get_initailization_type() == DELTA ? RA_DELTA : RA_FULL, &h));
        r->bind(prog, h);
        handle[r] = h;
        /* relation::initialize_relation (balanced_hash_relation.cpp:744-756): a restart with
         * per-rank files reads <file>_<rank> */
        std::string file = r->get_filename();
        if (restart_flag && separate_io) file += "_0";
        RA_CK(prog, ra_relation_load_file(prog, h, file.c_str()));
    }
    auto rel = [&](relation* r) {
        auto it = handle.find(r);
        if (it == handle.end()) {
            fprintf(stderr, "parallel-RA (B200): relation %s was not added to the LIE\n", r->get_debug_id().c_str());
            exit(1);
        }
        return it->second;
    };

    std::map<RAM*, int> scc_handle;
    for (RAM* s : lie_sccs) {
        int h = -1;
        RA_CK(prog, ra_scc_create(prog, s->is_fixpoint() ? 1 : 0, s->get_id(), &h));
        scc_handle[s] = h;
        for (size_t i = 0; i < s->relations().size(); i++)
            RA_CK(prog, ra_scc_add_relation(prog, h, rel(s->relations()[i]), s->relation_status()[i] ? 1 : 0));
        for (parallel_RA* ra : s->rules()) {
            switch (ra->get_RA_type()) {
            case JOIN: {
                parallel_join* j = (parallel_join*)ra;
                RA_CK(prog, ra_scc_add_join(prog, h, rel(j->out), rel(j->in0), j->ver0, rel(j->in1), j->ver1,
                                            j->proj.data(), (int)j->proj.size()));
                break;
            }
            case COPY: {
                parallel_copy* c = (parallel_copy*)ra;
                RA_CK(prog, ra_scc_add_copy(prog, h, RA_COPY, rel(c->out), rel(c->in), c->ver, c->reorder.data(),
                                            (int)c->reorder.size(), RA_PRED_TRUE));
                break;
            }
            case ACOPY: {
                parallel_acopy* c = (parallel_acopy*)ra;
                RA_CK(prog, ra_scc_add_copy(prog, h, RA_ACOPY, rel(c->out), rel(c->in), c->ver, c->reorder.data(),
                                            (int)c->reorder.size(), RA_PRED_TRUE));
                break;
            }
            case COPY_FILTER: {
                parallel_copy_filter* c = (parallel_copy_filter*)ra;
                int pred = classify_predicate(c->lambda);
                if (pred < 0) {
                    fprintf(stderr,
                            "parallel-RA (B200): copy_filter predicate into %s is not one of the comparisons of "
                            "columns 0 and 1 the device evaluates (==, !=, <, >, <=, >=, true, false)\n",
                            c->out->get_debug_id().c_str());
                    exit(1);
                }
                RA_CK(prog, ra_scc_add_copy(prog, h, RA_COPY_FILTER, rel(c->out), rel(c->in), c->ver,
                                            c->reorder.data(), (int)c->reorder.size(), pred));
                break;
            }
            default:
                fprintf(stderr, "parallel-RA (B200): rule type %u is not supported\n", ra->get_RA_type());
                exit(1);
            }
        }
    }
    for (auto& d : deps) RA_CK(prog, ra_scc_depend(prog, scc_handle[d.first], scc_handle[d.second]));
    RA_CK(prog, ra_program_set_batch_size(prog, batch_size));

    std::cout << "Using the B200 engine (one GPU, device " << device << ")" << std::endl;
    std::cout << "----------------- Initialization Complete ---------------------" << std::endl << std::endl;

    for (;;) {
        int id = -1;
        RA_CK(prog, ra_program_run_next_scc(prog, &id));
        if (id < 0) break;
        RAM* ran = nullptr;
        for (RAM* s : lie_sccs)
            if (s && s->get_id() == id) ran = s;
        std::cout << "-------------------Executing SCC " << id << "------------------" << std::endl;
        if (ran && !ran->is_fixpoint()) print_all_relation_size();
        executed_scc_id.push_back(id);
        loop_counter++;
        /* LIE::update_task_graph deletes the task once it has run (lie.cpp:64-75) */
        for (RAM*& s : lie_sccs)
            if (s == ran) {
                delete s;
                s = nullptr;
            }
    }
    return true;
}

std::vector<u64> LIE::get_history()
{
    std::vector<u64> h;
    if (!prog) return h;
    uint64_t n = 0;
    RA_CK(prog, ra_program_history(prog, nullptr, 0, &n));
    h.resize(n);
    RA_CK(prog, ra_program_history(prog, h.data(), n, &n));
    return h;
}

/* src/lie/lie.cpp:128-150 */
void LIE::print_all_relation_size()
{
    u64 total_facts = 0;
    for (relation* r : lie_relations) {
        u64 n = (u64)r->get_full_element_count();
        std::cout << r->get_debug_id() << ": {" << r->get_arity() << "}. (" << n << " total facts)" << std::endl;
        total_facts += n;
    }
    std::cout << "Total facts across all relations " << total_facts << std::endl << std::endl;
}

LIE::~LIE()
{
    for (relation* r : lie_relations) {
        r->bind(nullptr, -1);
        delete r;
    }
    for (RAM* s : lie_sccs) delete s;
    if (prog) ra_program_destroy(prog);
}
