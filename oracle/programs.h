/*
 * Datalog programs written once against parallel-RA's public C++ API
 * (relation, RAM, parallel_join, parallel_copy, parallel_copy_filter), so the
 * same source builds on the reference library (oracle/_ref/ref_driver) and on
 * the B200 library's source-compatible headers (parallel-ra_b200/cxx).
 *
 * TEST INFRASTRUCTURE: these builders feed the parity drivers.
 *
 *  - tc: exactly the rule set of tests/transitive_closure.cpp:56-77 (T stored
 *        as (dst,src); copy G {1,0}; join T DELTA x G FULL {3,1}).
 *  - sg: same generation over a parent->child edge relation:
 *        SGB(x,y)  :- edge(p,x), edge(p,y).               (join E FULL x E FULL)
 *        SG(x,y)   :- SGB(x,y), x != y.                   (copy_filter)
 *        TMP(b,x)  :- SG(a,b), edge(a,x).                 (join SG DELTA x E FULL)
 *        SG(x,y)   :- TMP(b,x), edge(b,y).                (join TMP DELTA x E FULL)
 *        The reference's join carries no filter (src/RA/parallel_join.h:55), so
 *        the base rule is a join into SGB followed by a filtering copy.
 */
#pragma once
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>
#include <utility>

struct ra_program_def {
    std::vector<relation*> relations;
    std::vector<RAM*> sccs;                          /* in add_scc order */
    std::vector<std::pair<RAM*, RAM*>> deps;        /* (src, dst): src runs first */
};

/* tests/transitive_closure.cpp:56-77 */
inline void build_tc(ra_program_def& p, const std::string& edge_file, const std::string& empty_file)
{
    relation* T = new relation(1, true, 2, 257, "T", empty_file, FULL);
    relation* G = new relation(1, true, 2, 256, "G", edge_file, FULL);

    RAM* scc_join = new RAM(true, 1);
    scc_join->add_relation(G, false);
    scc_join->add_relation(T, true);
    scc_join->add_rule(new parallel_join(T, T, DELTA, G, FULL, {3, 1}));

    RAM* scc_copy = new RAM(false, 2);
    scc_copy->add_relation(G, false);
    scc_copy->add_relation(T, true);
    scc_copy->add_rule(new parallel_copy(T, G, FULL, {1, 0}));

    p.relations = {T, G};
    p.sccs = {scc_join, scc_copy};
    p.deps = {{scc_copy, scc_join}};
}

inline bool sg_distinct(const u64* const data) { return data[0] != data[1]; }

inline void build_sg(ra_program_def& p, const std::string& edge_file, const std::string& empty_file)
{
    relation* E   = new relation(1, true, 2, 300, "edge", edge_file, FULL);
    relation* SGB = new relation(1, true, 2, 301, "SGB", empty_file, FULL);
    relation* SG  = new relation(1, true, 2, 302, "SG", empty_file, FULL);
    relation* TMP = new relation(1, true, 2, 303, "TMP", empty_file, FULL);

    /* (p, x, idE, y, idE') -> (x, y) */
    RAM* scc_base = new RAM(false, 10);
    scc_base->add_relation(E, false);
    scc_base->add_relation(SGB, true);
    scc_base->add_rule(new parallel_join(SGB, E, FULL, E, FULL, {1, 3}));

    RAM* scc_filter = new RAM(false, 11);
    scc_filter->add_relation(SGB, false);
    scc_filter->add_relation(SG, true);
    scc_filter->add_rule(new parallel_copy_filter(SG, SGB, FULL, {0, 1}, sg_distinct));

    /* (a, b, idS, x, idE) -> (b, x);  (b, x, idT, y, idE) -> (x, y) */
    RAM* scc_rec = new RAM(true, 12);
    scc_rec->add_relation(E, false);
    scc_rec->add_relation(SG, true);
    scc_rec->add_relation(TMP, false);
    scc_rec->add_rule(new parallel_join(TMP, SG, DELTA, E, FULL, {1, 3}));
    scc_rec->add_rule(new parallel_join(SG, TMP, DELTA, E, FULL, {1, 3}));

    p.relations = {E, SGB, SG, TMP};
    p.sccs = {scc_base, scc_filter, scc_rec};
    p.deps = {{scc_base, scc_filter}, {scc_filter, scc_rec}};
}

/* copy_filter predicates of the program descriptions (the generated programs'
 * lambdas on columns 0 and 1). */
inline bool pd_eq(const u64* const d) { return d[0] == d[1]; }
inline bool pd_ne(const u64* const d) { return d[0] != d[1]; }
inline bool pd_lt(const u64* const d) { return d[0] < d[1]; }
inline bool pd_gt(const u64* const d) { return d[0] > d[1]; }
inline bool pd_le(const u64* const d) { return d[0] <= d[1]; }
inline bool pd_ge(const u64* const d) { return d[0] >= d[1]; }
inline bool pd_true(const u64* const) { return true; }
inline bool pd_false(const u64* const) { return false; }

/* A program description (tests/golden/<program>/program.txt, written by
 * tests/golden/make_slog_golden.py from a reference program source):
 *   batch <n>
 *   rel <jcc> <canonical 0|1> <arity> <tag> <FULL|DELTA> <name> <file|->
 *   scc <fixpoint 0|1> <id>                       (in LIE::add_scc order)
 *   member <scc> <rel> <init 0|1>
 *   join <scc> <out> <in0> <DELTA|FULL> <in1> <DELTA|FULL> <c,c,...>
 *   copy <scc> <copy|acopy|filter> <out> <in> <DELTA|FULL> <pred> <c,c,...>
 *   dep <src scc> <dst scc>
 * Relation files are read from data_dir; "-" is an empty relation. */
inline std::vector<int> pd_cols(const std::string& s)
{
    std::vector<int> v;
    std::stringstream ss(s);
    std::string t;
    while (std::getline(ss, t, ',')) v.push_back(atoi(t.c_str()));
    return v;
}

inline int pd_batch_size(const std::string& path)
{
    std::ifstream in(path);
    std::string kw;
    int b = 1;
    while (in >> kw) {
        if (kw == "batch") in >> b;
        std::string rest;
        std::getline(in, rest);
    }
    return b;
}

inline void build_from_description(ra_program_def& p, const std::string& path, const std::string& data_dir,
                                   const std::string& empty_file)
{
    std::ifstream in(path);
    if (!in) { fprintf(stderr, "cannot read %s\n", path.c_str()); exit(2); }
    std::string kw;
    while (in >> kw) {
        if (kw == "batch") {
            int b;
            in >> b;
        } else if (kw == "rel") {
            unsigned jcc, canon, arity, tag;
            std::string ver, name, file;
            in >> jcc >> canon >> arity >> tag >> ver >> name >> file;
            const std::string f = file == "-" ? empty_file : data_dir + "/" + file;
            p.relations.push_back(new relation(jcc, canon != 0, arity, tag, name, f, ver == "DELTA" ? DELTA : FULL));
        } else if (kw == "scc") {
            int fix, id;
            in >> fix >> id;
            p.sccs.push_back(new RAM(fix != 0, id));
        } else if (kw == "member") {
            int s, r, init;
            in >> s >> r >> init;
            p.sccs[s]->add_relation(p.relations[r], init != 0);
        } else if (kw == "join") {
            int s, o, a, b;
            std::string va, vb, cols;
            in >> s >> o >> a >> va >> b >> vb >> cols;
            p.sccs[s]->add_rule(new parallel_join(p.relations[o], p.relations[a], va == "DELTA" ? DELTA : FULL,
                                                  p.relations[b], vb == "DELTA" ? DELTA : FULL, pd_cols(cols)));
        } else if (kw == "copy") {
            int s, o, a;
            std::string kind, va, pred, cols;
            in >> s >> kind >> o >> a >> va >> pred >> cols;
            const int v = va == "DELTA" ? DELTA : FULL;
            if (kind == "copy") {
                p.sccs[s]->add_rule(new parallel_copy(p.relations[o], p.relations[a], v, pd_cols(cols)));
            } else if (kind == "acopy") {
                p.sccs[s]->add_rule(new parallel_acopy(p.relations[o], p.relations[a], v, pd_cols(cols)));
            } else {
                bool (*f)(const u64* const) = pred == "eq" ? pd_eq : pred == "ne" ? pd_ne : pred == "lt" ? pd_lt
                    : pred == "gt" ? pd_gt : pred == "le" ? pd_le : pred == "ge" ? pd_ge : pred == "true" ? pd_true
                    : pd_false;
                p.sccs[s]->add_rule(new parallel_copy_filter(p.relations[o], p.relations[a], v, pd_cols(cols), f));
            }
        } else if (kw == "dep") {
            int a, b;
            in >> a >> b;
            p.deps.push_back({p.sccs[a], p.sccs[b]});
        } else {
            std::string rest;
            std::getline(in, rest);   /* comments and unknown lines */
        }
    }
}
