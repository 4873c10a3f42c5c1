/*
 * CPU restatement of parallel-RA's semi-naive fixed point (the oracle).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline leg.  Never linked or loaded by the product.
 *
 * Relations are kept, as in the reference, as three sets of (arity+1)-column
 * tuples (full, delta, newt) in lexicographic ("trie") order -- the order in
 * which the reference's per-bucket tries of B-tree maps enumerate tuples
 * (src/relation/shmap_relation_exp.cpp:77-112).  Each function below cites
 * the reference code it restates.
 */
#include "ra_oracle.h"

#include <array>
#include <chrono>
#include <cstring>
#include <map>
#include <set>
#include <string>
#include <vector>
#include <thread>
#include <atomic>

namespace {

constexpr int kMaxCols = 64;                /* arity + 1 <= 64 */
constexpr uint64_t kJoinThreshold = 20000000;   /* src/RAM/RA_tasks.cpp:312 */

using tuple = std::array<uint64_t, kMaxCols>;   /* unused trailing columns are 0 */
using tset = std::set<tuple>;

struct relation_state {
    uint32_t jcc = 1, arity = 2, tag = 0;
    std::string name;
    tset full, delta, newt;
};

enum rule_kind { K_JOIN, K_COPY, K_ACOPY, K_FILTER };

struct rule {
    rule_kind kind;
    int out, in0, ver0, in1, ver1;
    std::vector<int> proj;
    int pred;
};

struct scc_state {
    bool fixpoint;
    int id;
    std::vector<int> rels;
    std::vector<bool> init_status;
    std::vector<rule> rules;
    bool done = false;
};

/* find_in_full / find_in_delta / find_in_newt: a tuple "exists" when some
 * stored tuple has the given first `len` columns
 * (src/relation/shmap_relation_exp.cpp:54-66; balanced_hash_relation.cpp:1015-1035). */
bool has_prefix(const tset& s, const uint64_t* t, int len)
{
    tuple key{};
    for (int i = 0; i < len; i++) key[i] = t[i];
    auto it = s.lower_bound(key);
    if (it == s.end()) return false;
    for (int i = 0; i < len; i++)
        if ((*it)[i] != t[i]) return false;
    return true;
}

bool eval_pred(int pred, uint64_t a, uint64_t b)
{
    switch (pred) {
    case ORACLE_PRED_TRUE: return true;
    case ORACLE_PRED_FALSE: return false;
    case ORACLE_PRED_EQ: return a == b;
    case ORACLE_PRED_NE: return a != b;
    case ORACLE_PRED_LT: return a < b;
    case ORACLE_PRED_GT: return a > b;
    case ORACLE_PRED_LE: return a <= b;
    case ORACLE_PRED_GE: return a >= b;
    }
    return false;
}

}  // namespace

struct oracle_prog {
    std::vector<relation_state> rels;
    std::vector<scc_state> sccs;
    std::vector<std::pair<int, int>> deps;
    std::map<uint64_t, uint64_t> intern_map;     /* LIE::intern_map, src/lie/lie.h:36 */
    std::vector<uint64_t> history;
    double fixpoint_s = 0;

    const tset& version(int rel, int ver) { return ver == ORACLE_DELTA ? rels[rel].delta : rels[rel].full; }

    /* Interning, src/RAM/RA_tasks.cpp:861-875 at one rank (bucket 0). */
    uint64_t intern(uint32_t tag)
    {
        uint64_t key = (uint64_t)tag << 46;
        auto it = intern_map.find(key);
        uint64_t v = (it == intern_map.end()) ? 0 : it->second + 1;
        intern_map[key] = v;
        return key | v;
    }

    /* One local_compute call over all rules of the SCC (src/RAM/RA_tasks.cpp:305-555)
     * followed by local_insert_in_newt (:824-905).  Returns true when every join
     * finished within the per-call output threshold (parallel_join.cpp:196-201). */
    bool compute_and_insert(scc_state& s, std::vector<uint64_t>& offsets)
    {
        bool completed = true;
        std::vector<std::vector<tuple>> streams(s.rules.size());
        for (size_t r = 0; r < s.rules.size(); r++) {
            const rule& ru = s.rules[r];
            auto& out = streams[r];
            if (ru.kind != K_JOIN) {
                /* copy emitters, src/relation/shmap_relation_exp.cpp:116-265 */
                for (const tuple& t : version(ru.in0, ru.ver0)) {
                    if (ru.kind == K_FILTER && !eval_pred(ru.pred, t[0], t[1])) continue;
                    tuple o{};
                    for (size_t j = 0; j < ru.proj.size(); j++) o[j] = t[ru.proj[j]];
                    out.push_back(o);
                }
                continue;
            }
            /* join dispatch, src/RAM/RA_tasks.cpp:452-520 */
            const relation_state& in0 = rels[ru.in0];
            const relation_state& in1 = rels[ru.in1];
            int jcc = (int)in0.jcc;
            bool left;
            const tset *outer, *inner;
            int outer_w, inner_w;
            if (ru.ver0 == ORACLE_DELTA) {
                left = true;
                outer = &in0.delta;
                inner = (ru.ver1 == ORACLE_DELTA) ? &in1.delta : &in1.full;
                outer_w = (int)in0.arity + 1;
                inner_w = (int)in1.arity + 1;
            } else {
                left = false;
                outer = (ru.ver1 == ORACLE_DELTA) ? &in1.delta : &in1.full;
                inner = &in0.full;
                outer_w = (int)in1.arity + 1;
                inner_w = (int)in0.arity + 1;
            }
            /* parallel_join::local_join, src/RA/parallel_join.cpp:157-230 */
            if (outer->empty() || inner->empty()) continue;
            if (offsets[r] > outer->size()) continue;
            tset local_dedup;
            uint64_t local_count = 0;
            uint64_t row = 0;
            auto it = outer->begin();
            std::advance(it, (long)offsets[r]);
            row = offsets[r];
            for (; it != outer->end(); ++it, ++row) {
                const tuple& o = *it;
                tuple key{};
                for (int i = 0; i < jcc; i++) key[i] = o[i];
                for (auto jt = inner->lower_bound(key); jt != inner->end(); ++jt) {
                    const tuple& u = *jt;
                    bool match = true;
                    for (int i = 0; i < jcc; i++) match = match && u[i] == o[i];
                    if (!match) break;
                    /* as_all_to_allv_{left,right}_join_buffer_helper,
                     * src/relation/shmap_relation_exp.cpp:335-349, 403-417 */
                    uint64_t re[2 * kMaxCols];
                    int n = 0;
                    if (left) {
                        for (int i = 0; i < outer_w; i++) re[n++] = o[i];
                        for (int i = jcc; i < inner_w; i++) re[n++] = u[i];
                    } else {
                        for (int i = 0; i < inner_w; i++) re[n++] = u[i];
                        for (int i = jcc; i < outer_w; i++) re[n++] = o[i];
                    }
                    tuple p{};
                    for (size_t j = 0; j < ru.proj.size(); j++) p[j] = re[ru.proj[j]];
                    if (local_dedup.insert(p).second) {
                        out.push_back(p);
                        local_count++;
                    }
                }
                if (local_count > kJoinThreshold) {
                    offsets[r] = row + 1;
                    completed = false;
                    break;
                }
            }
        }

        /* RAM::local_insert_in_newt, src/RAM/RA_tasks.cpp:824-905 */
        for (size_t r = 0; r < s.rules.size(); r++) {
            const rule& ru = s.rules[r];
            relation_state& out = rels[ru.out];
            if (ru.kind == K_ACOPY) {
                int w = (int)out.arity + 1;
                for (const tuple& t : streams[r])
                    if (!has_prefix(out.full, t.data(), w) && !has_prefix(out.delta, t.data(), w))
                        out.newt.insert(t);
            } else {
                int w = (int)out.arity;
                for (const tuple& t : streams[r]) {
                    if (has_prefix(out.full, t.data(), w) || has_prefix(out.delta, t.data(), w) ||
                        has_prefix(out.newt, t.data(), w))
                        continue;
                    tuple n = t;
                    n[w] = intern(out.tag);
                    out.newt.insert(n);
                }
            }
        }
        return completed;
    }

    /* RAM::execute_in_batches, src/RAM/RA_tasks.cpp:1121-1269 */
    void execute_in_batches(scc_state& s, int batch_size, std::vector<uint64_t>& hist)
    {
        std::vector<uint64_t> offsets(s.rules.size(), 0);
        while (batch_size != 0) {
            while (!compute_and_insert(s, offsets)) {}
            for (size_t i = 0; i < offsets.size(); i++) offsets[i] = 0;
            /* RAM::local_insert_in_full -> relation::insert_delta_in_full +
             * local_insert_in_delta, balanced_hash_relation.cpp:1120-1148, 1183-1231 */
            for (int ri : s.rels) {
                relation_state& r = rels[ri];
                for (const tuple& t : r.delta) r.full.insert(t);
                r.delta.clear();
                r.delta.swap(r.newt);
            }
            batch_size--;
            if (!s.fixpoint) break;
        }
        /* RAM::check_for_fixed_point, src/RAM/RA_tasks.cpp:1072-1085 (int sums) */
        uint32_t d = 0, f = 0;
        for (int ri : s.rels) {
            d += (uint32_t)rels[ri].delta.size();
            f += (uint32_t)rels[ri].full.size();
        }
        hist.push_back(d);
        hist.push_back(f);
    }

    /* LIE::execute, src/lie/lie.cpp:197-448 (no restart / checkpoint) */
    int execute(int batch_size)
    {
        auto t0 = std::chrono::steady_clock::now();
        for (;;) {
            /* LIE::one_runnable_tasks, src/lie/lie.cpp:27-60 */
            int next = -1;
            for (size_t i = 0; i < sccs.size() && next < 0; i++) {
                if (sccs[i].done) continue;
                bool blocked = false;
                for (auto& d : deps)
                    if (d.second == (int)i && !sccs[d.first].done) blocked = true;
                if (!blocked) next = (int)i;
            }
            if (next < 0) break;
            scc_state& s = sccs[next];
            for (size_t i = 0; i < s.rels.size(); i++) {
                if (!s.init_status[i]) continue;
                /* relation::insert_full_in_delta, balanced_hash_relation.cpp:1152-1179 */
                relation_state& r = rels[s.rels[i]];
                for (const tuple& t : r.full) r.delta.insert(t);
                r.full.clear();
            }
            std::vector<uint64_t> hist;
            if (!s.fixpoint) {
                execute_in_batches(s, batch_size, hist);
            } else {
                do {
                    execute_in_batches(s, batch_size, hist);
                } while (hist[hist.size() - 2] != 0);
            }
            /* RAM::insert_delta_in_full, src/RAM/RA_tasks.cpp:1062-1068 */
            for (int ri : s.rels) {
                relation_state& r = rels[ri];
                for (const tuple& t : r.delta) r.full.insert(t);
                r.delta.clear();
            }
            history.push_back((uint64_t)s.id);
            history.push_back(hist.size() / 2);
            history.insert(history.end(), hist.begin(), hist.end());
            s.done = true;
        }
        fixpoint_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        return 0;
    }
};

extern "C" {

oracle_prog* oracle_create(void) { return new oracle_prog(); }
void oracle_destroy(oracle_prog* p) { delete p; }

int oracle_relation(oracle_prog* p, uint32_t jcc, uint32_t arity, uint32_t tag, const char* name, int version)
{
    (void)version;
    if (arity + 1 > (uint32_t)kMaxCols || jcc > arity) return -1;
    relation_state r;
    r.jcc = jcc;
    r.arity = arity;
    r.tag = tag;
    r.name = name ? name : "";
    p->rels.push_back(std::move(r));
    return (int)p->rels.size() - 1;
}

/* relation::populate_full / populate_delta, balanced_hash_relation.cpp:773-810:
 * rows of arity+1 columns inserted with set semantics on all columns. */
int oracle_load_rows(oracle_prog* p, int rel, const uint64_t* rows, uint64_t nrows)
{
    if (rel < 0 || rel >= (int)p->rels.size()) return -1;
    relation_state& r = p->rels[rel];
    int w = (int)r.arity + 1;
    for (uint64_t i = 0; i < nrows; i++) {
        tuple t{};
        for (int c = 0; c < w; c++) t[c] = rows[i * w + c];
        r.full.insert(t);
    }
    return 0;
}

int oracle_scc(oracle_prog* p, int fixpoint, int id)
{
    scc_state s;
    s.fixpoint = fixpoint != 0;
    s.id = id;
    p->sccs.push_back(std::move(s));
    return (int)p->sccs.size() - 1;
}

int oracle_scc_add_relation(oracle_prog* p, int scc, int rel, int init_status)
{
    p->sccs[scc].rels.push_back(rel);
    p->sccs[scc].init_status.push_back(init_status != 0);
    return 0;
}

int oracle_scc_add_join(oracle_prog* p, int scc, int out, int in0, int ver0, int in1, int ver1,
                        const int* proj, int nproj)
{
    rule r{K_JOIN, out, in0, ver0, in1, ver1, std::vector<int>(proj, proj + nproj), 0};
    p->sccs[scc].rules.push_back(r);
    return 0;
}

int oracle_scc_add_copy(oracle_prog* p, int scc, int kind, int out, int in, int ver,
                        const int* proj, int nproj, int pred)
{
    rule_kind k = kind == ORACLE_ACOPY ? K_ACOPY : kind == ORACLE_COPY_FILTER ? K_FILTER : K_COPY;
    rule r{k, out, in, ver, -1, -1, std::vector<int>(proj, proj + nproj), pred};
    p->sccs[scc].rules.push_back(r);
    return 0;
}

int oracle_depend(oracle_prog* p, int src_scc, int dst_scc)
{
    p->deps.push_back({src_scc, dst_scc});
    return 0;
}

int oracle_execute(oracle_prog* p, int batch_size) { return p->execute(batch_size); }

uint64_t oracle_history_len(oracle_prog* p) { return p->history.size(); }

uint64_t oracle_history(oracle_prog* p, uint64_t* out, uint64_t cap)
{
    uint64_t n = p->history.size() < cap ? p->history.size() : cap;
    std::memcpy(out, p->history.data(), n * sizeof(uint64_t));
    return n;
}

uint64_t oracle_full_count(oracle_prog* p, int rel) { return p->rels[rel].full.size(); }

uint64_t oracle_dump_full(oracle_prog* p, int rel, uint64_t* out, uint64_t cap_rows)
{
    relation_state& r = p->rels[rel];
    int w = (int)r.arity + 1;
    uint64_t n = 0;
    for (const tuple& t : r.full) {
        if (n >= cap_rows) break;
        for (int c = 0; c < w; c++) out[n * w + c] = t[c];
        n++;
    }
    return n;
}

double oracle_fixpoint_seconds(oracle_prog* p) { return p->fixpoint_s; }

// Independent check of transitive closure (not a restatement of the reference):
// semi-naive TC over the rule T(z, x) :- T_delta(y, x), G(y, z) adds, at
// iteration k, exactly the pairs (x, z) whose shortest path from x to z has
// length k + 2 counted in edges (k + 1 for the copy SCC's base T = G), the
// shortest cycle through x for z == x.  hist[d] += number of pairs at shortest
// distance d, over every source, by one breadth-first search per source
// (`threads` threads, sources split in blocks).  Returns the largest distance
// seen, or ~0 when a distance reaches `cap`.
uint64_t oracle_tc_distance_histogram(const uint64_t* src, const uint64_t* dst, uint64_t m, uint64_t n,
                                      uint64_t* hist, uint64_t cap, int threads)
{
    std::vector<uint64_t> off(n + 1, 0);
    for (uint64_t e = 0; e < m; e++) off[src[e] + 1]++;
    for (uint64_t v = 0; v < n; v++) off[v + 1] += off[v];
    std::vector<uint32_t> adj(m);
    {
        std::vector<uint64_t> cur(off.begin(), off.end() - 1);
        for (uint64_t e = 0; e < m; e++) adj[cur[src[e]]++] = (uint32_t)dst[e];
    }
    if (threads < 1) threads = 1;
    std::vector<std::vector<uint64_t>> part(threads, std::vector<uint64_t>(cap, 0));
    std::vector<uint64_t> deepest(threads, 0);
    std::atomic<uint64_t> next{0};
    auto work = [&](int t) {
        std::vector<uint32_t> seen(n, 0);   // stamp of the search that reached the value
        std::vector<uint32_t> frontier, nxt;
        uint32_t stamp = 0;
        for (;;) {
            const uint64_t s0 = next.fetch_add(4096);
            if (s0 >= n) break;
            const uint64_t s1 = std::min<uint64_t>(n, s0 + 4096);
            for (uint64_t s = s0; s < s1; s++) {
                ++stamp;
                frontier.assign(1, (uint32_t)s);
                bool self = false;
                for (uint64_t d = 1; !frontier.empty(); d++) {
                    nxt.clear();
                    uint64_t found = 0;
                    for (uint32_t u : frontier)
                        for (uint64_t e = off[u]; e < off[u + 1]; e++) {
                            const uint32_t v = adj[e];
                            if (v == s) {
                                if (!self) {   // the shortest cycle through s
                                    self = true;
                                    found++;
                                }
                                continue;
                            }
                            if (seen[v] == stamp) continue;
                            seen[v] = stamp;
                            nxt.push_back(v);
                            found++;
                        }
                    if (found) {
                        if (d >= cap) {
                            deepest[t] = ~0ull;
                            return;
                        }
                        part[t][d] += found;
                        if (deepest[t] != ~0ull) deepest[t] = std::max(deepest[t], d);
                    }
                    frontier.swap(nxt);
                }
            }
        }
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; t++) pool.emplace_back(work, t);
    for (auto& th : pool) th.join();
    uint64_t deep = 0;
    for (int t = 0; t < threads; t++) {
        if (deepest[t] == ~0ull) return ~0ull;
        deep = std::max(deep, deepest[t]);
        for (uint64_t d = 0; d < cap; d++) hist[d] += part[t][d];
    }
    return deep;
}

}  // extern "C"
