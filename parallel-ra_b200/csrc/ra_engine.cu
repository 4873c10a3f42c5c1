// parallel-RA on B200: device engine behind the C ABI in include/ra_engine.h.
//
// One ra_program = the relations, SCCs and rules of one Datalog program on one
// GPU.  Replaces, on one device and without MPI:
//   * the hash partitioning + all_to_all tuple exchange (src/hash, src/comm):
//     every relation lives in one HBM address space, so a rule's outputs go
//     straight into the output relation's dedup set;
//   * the per-bucket B-tree tries (src/btree, src/shmap): a relation is an
//     append-only log of packed u64 keys + u64 ids, [ full | delta | newt ],
//     whose delta region is sorted (trie order), plus an open-addressing
//     "seen" set over its data columns and a CSR index on its join columns;
//   * RAM::local_compute / local_insert_in_newt / local_insert_in_full
//     (src/RAM/RA_tasks.cpp:305-555, 824-905, 1044-1058): join/copy expansion,
//     first-occurrence dedup with reference-order intern ids, radix sort of
//     the new delta, region bump instead of copying delta into full;
//   * RAM::check_for_fixed_point's MPI_Allreduce (RA_tasks.cpp:1072-1085):
//     device counters.
#include "../../include/ra_engine.h"
#include "ra_kernels.cuh"

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <functional>
#include <string>
#include <vector>

using namespace ra;

namespace {

constexpr int kSms = 148;
constexpr int kMaxGrid = kSms * 8;

int grid_for(u64 n)
{
    u64 g = (n + kThreads - 1) / kThreads;
    if (g < 1) g = 1;
    if (g > (u64)kMaxGrid) g = kMaxGrid;
    return (int)g;
}

struct ra_error {
    int status;
};

struct Rule {
    int kind;            // 3 = join, else RA_COPY / RA_ACOPY / RA_COPY_FILTER
    int out, in0, ver0, in1, ver1;
    std::vector<int> proj;
    int pred;
};
constexpr int kJoin = 3;

struct Scc {
    bool fixpoint;
    int id;
    std::vector<int> rels;
    std::vector<bool> init;
    std::vector<Rule> rules;
    bool done = false;
};

struct Relation {
    uint32_t jcc, arity, tag;
    std::string name;
    int version;
    // loaded rows (arity + 1 u64 each), kept on the device for reset
    u64* raw = nullptr;
    u64 raw_n = 0;
    // packed, sorted, distinct loaded tuples (restored by reset without repacking)
    u64* lkeys = nullptr;
    u64* lids = nullptr;
    u64 l_n = 0, l_cap = 0;
    bool l_keys_unique = true;
    // log [ full | delta | newt ]
    u64* keys = nullptr;
    u64* ids = nullptr;
    u64 cap = 0;
    u64 full_n = 0, delta_n = 0;
    int full_runs = 0;          // sorted runs making up the full region
    bool keys_unique = true;    // no two stored tuples share data columns
    u64 full_version = 0, delta_version = 0;
    // seen set over data columns
    Slot* seen = nullptr;
    u64 seen_cap = 0, seen_n = 0;
    // sorted view of full (used when full_runs > 1)
    u64* vkeys = nullptr;
    u64* vids = nullptr;
    u64 v_cap = 0, v_version = ~0ull;
    // CSR index on the join key, for full (version-stamped) and delta
    u64* csr_full = nullptr;
    u64 csr_full_version = ~0ull;
    u64* csr_delta = nullptr;
    u64 csr_delta_version = ~0ull;
    // newt staging for the running iteration
    u64 newt_n = 0;
};

}  // namespace

struct ra_program {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    uint32_t batch_size = 1;
    std::vector<Relation> rels;
    std::vector<Scc> sccs;
    std::vector<std::pair<int, int>> deps;
    std::vector<uint64_t> history;
    std::vector<std::pair<uint32_t, u64>> intern;   // (tag, next counter) -- LIE::intern_map
    int bits = 0;                 // packed bits per column for this run
    bool packed = false;          // loaded relations packed with `bits` (cleared by a new load)
    bool executed = false;
    bool running = false;         // between the first and the last SCC of a run
    double fixpoint_ms_acc = 0;
    u64 epoch = 0;
    std::string err;
    ra_stats stats{};
    // scratch
    u64* cand = nullptr;
    u64 cand_cap = 0;
    u32* flag = nullptr;
    u64* rank = nullptr;
    u64 rank_cap = 0;
    u64* cnt = nullptr;
    u64* off = nullptr;
    u64 cnt_cap = 0;
    u64* nkeys = nullptr;
    u64* nids = nullptr;
    u64 n_cap = 0;
    u64* tk = nullptr;
    u64* tv = nullptr;
    u64 t_cap = 0;
    u64* sums = nullptr;
    u64* dscalar = nullptr;       // device scalars: [0] total, [1] max, [2] flag
    u64* hscalar = nullptr;       // pinned host mirror
    u32* derr = nullptr;
    u32* hist_buf = nullptr;
    u64* hist_off = nullptr;
    u64 hist_cap = 0;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> dedup_events;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

namespace {

void fail(ra_program* p, int status, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (p) p->err = buf;
    throw ra_error{status};
}

void ck(ra_program* p, cudaError_t e, const char* what)
{
    if (e == cudaSuccess) return;
    if (e == cudaErrorMemoryAllocation) fail(p, RA_E_OOM, "%s: %s", what, cudaGetErrorString(e));
    fail(p, RA_E_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define CK(call) ck(p, (call), #call)
#define LAUNCHED() do { p->stats.kernel_launches++; ck(p, cudaGetLastError(), "kernel launch"); } while (0)

template <typename T>
void dev_alloc(ra_program* p, T** ptr, u64 count)
{
    void* q = nullptr;
    if (count == 0) count = 1;
    CK(cudaMallocAsync(&q, count * sizeof(T), p->stream));
    *ptr = (T*)q;
}

template <typename T>
void dev_free(ra_program* p, T** ptr)
{
    if (*ptr) cudaFreeAsync(*ptr, p->stream);
    *ptr = nullptr;
}

// grow a pair of u64 buffers to at least n elements (contents preserved when keep)
void grow2(ra_program* p, u64** a, u64** b, u64* cap, u64 n, bool keep, u64 keep_n)
{
    if (n <= *cap) return;
    u64 nc = std::max<u64>(n + n / 2, 1024);
    u64 *na, *nb;
    dev_alloc(p, &na, nc);
    dev_alloc(p, &nb, nc);
    if (keep && keep_n) {
        CK(cudaMemcpyAsync(na, *a, keep_n * 8, cudaMemcpyDeviceToDevice, p->stream));
        CK(cudaMemcpyAsync(nb, *b, keep_n * 8, cudaMemcpyDeviceToDevice, p->stream));
    }
    dev_free(p, a);
    dev_free(p, b);
    *a = na;
    *b = nb;
    *cap = nc;
}

void grow1(ra_program* p, u64** a, u64* cap, u64 n)
{
    if (n <= *cap) return;
    u64 nc = std::max<u64>(n + n / 2, 1024);
    dev_free(p, a);
    dev_alloc(p, a, nc);
    *cap = nc;
}

u64 read_scalar(ra_program* p, const u64* dptr)
{
    CK(cudaMemcpyAsync(p->hscalar, dptr, 8, cudaMemcpyDeviceToHost, p->stream));
    CK(cudaStreamSynchronize(p->stream));
    return p->hscalar[0];
}

// ---------------------------------------------------------------------------
// exclusive scan of n values into out (u64); returns the total (synchronises)
// ---------------------------------------------------------------------------
template <typename T>
u64 scan_exclusive(ra_program* p, const T* in, u64 n, u64* out, bool want_total = true)
{
    if (n == 0) return 0;
    int g = grid_for(n);
    if (g > 32 * kThreads) g = 32 * kThreads;
    u64 chunk = (n + g - 1) / g;
    g = (int)((n + chunk - 1) / chunk);
    scan_chunk_sums<T><<<g, kThreads, 0, p->stream>>>(in, n, chunk, p->sums);
    LAUNCHED();
    scan_sums_single<<<1, kThreads, 0, p->stream>>>(p->sums, g, p->dscalar);
    LAUNCHED();
    scan_chunk_apply<T><<<g, kThreads, 0, p->stream>>>(in, n, chunk, p->sums, out);
    LAUNCHED();
    return want_total ? read_scalar(p, p->dscalar) : 0;
}

// ---------------------------------------------------------------------------
// LSD radix sort of (k, v) by key bits [lo, hi); result back in (k, v).
// ---------------------------------------------------------------------------
void ensure_tmp(ra_program* p, u64 n)
{
    if (n > p->t_cap) {
        dev_free(p, &p->tk);
        dev_free(p, &p->tv);
        u64 nc = std::max<u64>(n + n / 2, 1024);
        dev_alloc(p, &p->tk, nc);
        dev_alloc(p, &p->tv, nc);
        p->t_cap = nc;
    }
}

void radix_sort(ra_program* p, u64* k, u64* v, u64 n, int lo, int hi)
{
    if (n <= 1 || hi <= lo) return;
    ensure_tmp(p, n);
    int g = grid_for(n);
    if (g > 4 * kSms) g = 4 * kSms;
    u64 chunk = (n + g - 1) / g;
    g = (int)((n + chunk - 1) / chunk);
    u64 hn = (u64)kRadix * g;
    if (hn > p->hist_cap) {
        dev_free(p, &p->hist_buf);
        dev_free(p, &p->hist_off);
        dev_alloc(p, &p->hist_buf, hn);
        dev_alloc(p, &p->hist_off, hn);
        p->hist_cap = hn;
    }
    u64 *sk = k, *sv = v, *dk = p->tk, *dv = p->tv;
    int passes = 0;
    for (int shift = lo; shift < hi; shift += kRadixBits) {
        radix_histogram<<<g, kThreads, 0, p->stream>>>(sk, n, chunk, shift, p->hist_buf, g);
        LAUNCHED();
        scan_exclusive<u32>(p, p->hist_buf, hn, p->hist_off, false);
        radix_scatter<<<g, kThreads, 0, p->stream>>>(sk, sv, dk, dv, n, chunk, shift, p->hist_off, g);
        LAUNCHED();
        std::swap(sk, dk);
        std::swap(sv, dv);
        passes++;
    }
    if (passes & 1) {
        CK(cudaMemcpyAsync(k, sk, n * 8, cudaMemcpyDeviceToDevice, p->stream));
        CK(cudaMemcpyAsync(v, sv, n * 8, cudaMemcpyDeviceToDevice, p->stream));
    }
}

int key_bits(ra_program* p, const Relation& r) { return (int)r.arity * p->bits; }

// sort rows lexicographically by (key, id): by id first when keys may repeat
void sort_rows(ra_program* p, const Relation& r, u64* k, u64* v, u64 n, bool keys_unique)
{
    if (!keys_unique) {
        // LSD order: id digits first, then key digits (ids become the values)
        radix_sort(p, v, k, n, 0, 64);
    }
    radix_sort(p, k, v, n, 0, key_bits(p, r));
}

Relation& rel_at(ra_program* p, int rel)
{
    if (rel < 0 || rel >= (int)p->rels.size()) fail(p, RA_E_BADARG, "bad relation handle %d", rel);
    return p->rels[rel];
}

void ensure_log(ra_program* p, Relation& r, u64 n)
{
    grow2(p, &r.keys, &r.ids, &r.cap, n, true, r.full_n + r.delta_n + r.newt_n);
}

// ---------------------------------------------------------------------------
// load: pack raw rows -> sorted, distinct (key, id) rows in the log's full region
// ---------------------------------------------------------------------------
void pack_relation(ra_program* p, Relation& r)
{
    r.full_n = r.delta_n = r.newt_n = 0;
    r.full_runs = 0;
    r.keys_unique = true;
    r.full_version++;
    r.delta_version++;
    if (r.raw_n == 0) return;
    ensure_log(p, r, r.raw_n);
    rows_pack<<<grid_for(r.raw_n), kThreads, 0, p->stream>>>(r.raw, r.raw_n, (int)r.arity, p->bits, r.keys, r.ids);
    LAUNCHED();
    radix_sort(p, r.keys, r.ids, r.raw_n, 0, key_bits(p, r));
    CK(cudaMemsetAsync(p->dscalar + 2, 0, 8, p->stream));
    any_equal_adjacent<<<grid_for(r.raw_n), kThreads, 0, p->stream>>>(r.keys, r.raw_n, (u32*)(p->dscalar + 2));
    LAUNCHED();
    bool dup_keys = read_scalar(p, p->dscalar + 2) != 0;
    u64 n = r.raw_n;
    if (dup_keys) {
        r.keys_unique = false;
        sort_rows(p, r, r.keys, r.ids, n, false);
        // drop exact duplicate rows
        grow1(p, &p->rank, &p->rank_cap, n);
        if (n > p->cand_cap) grow1(p, &p->cand, &p->cand_cap, n);
        dev_free(p, &p->flag);
        dev_alloc(p, &p->flag, std::max(n, p->rank_cap));
        flag_distinct_rows<<<grid_for(n), kThreads, 0, p->stream>>>(r.keys, r.ids, n, p->flag);
        LAUNCHED();
        u64 m = scan_exclusive<u32>(p, p->flag, n, p->rank);
        ensure_tmp(p, n);
        compact_flagged<<<grid_for(n), kThreads, 0, p->stream>>>(r.keys, r.ids, p->flag, p->rank, n, p->tk, p->tv);
        LAUNCHED();
        CK(cudaMemcpyAsync(r.keys, p->tk, m * 8, cudaMemcpyDeviceToDevice, p->stream));
        CK(cudaMemcpyAsync(r.ids, p->tv, m * 8, cudaMemcpyDeviceToDevice, p->stream));
        n = m;
    }
    if (r.version == RA_DELTA) {
        r.delta_n = n;
    } else {
        r.full_n = n;
        r.full_runs = 1;
    }
    grow2(p, &r.lkeys, &r.lids, &r.l_cap, n, false, 0);
    if (n) {
        CK(cudaMemcpyAsync(r.lkeys, r.keys, n * 8, cudaMemcpyDeviceToDevice, p->stream));
        CK(cudaMemcpyAsync(r.lids, r.ids, n * 8, cudaMemcpyDeviceToDevice, p->stream));
    }
    r.l_n = n;
    r.l_keys_unique = r.keys_unique;
}

// back to the loaded tuples packed by pack_relation (same column width)
void restore_loaded(ra_program* p, Relation& r)
{
    r.full_n = r.delta_n = r.newt_n = 0;
    r.full_runs = 0;
    r.keys_unique = r.l_keys_unique;
    r.full_version++;
    r.delta_version++;
    if (!r.l_n) return;
    ensure_log(p, r, r.l_n);
    CK(cudaMemcpyAsync(r.keys, r.lkeys, r.l_n * 8, cudaMemcpyDeviceToDevice, p->stream));
    CK(cudaMemcpyAsync(r.ids, r.lids, r.l_n * 8, cudaMemcpyDeviceToDevice, p->stream));
    if (r.version == RA_DELTA) {
        r.delta_n = r.l_n;
    } else {
        r.full_n = r.l_n;
        r.full_runs = 1;
    }
}

// sorted (key, id) rows of a relation version; FULL may need a sorted copy
void version_rows(ra_program* p, Relation& r, int ver, const u64** k, const u64** v, u64* n)
{
    if (ver == RA_DELTA) {
        *k = r.keys + r.full_n;
        *v = r.ids + r.full_n;
        *n = r.delta_n;
        return;
    }
    if (r.full_runs <= 1) {
        *k = r.keys;
        *v = r.ids;
        *n = r.full_n;
        return;
    }
    if (r.v_version != r.full_version) {
        grow2(p, &r.vkeys, &r.vids, &r.v_cap, r.full_n, false, 0);
        CK(cudaMemcpyAsync(r.vkeys, r.keys, r.full_n * 8, cudaMemcpyDeviceToDevice, p->stream));
        CK(cudaMemcpyAsync(r.vids, r.ids, r.full_n * 8, cudaMemcpyDeviceToDevice, p->stream));
        sort_rows(p, r, r.vkeys, r.vids, r.full_n, r.keys_unique);
        r.v_version = r.full_version;
    }
    *k = r.vkeys;
    *v = r.vids;
    *n = r.full_n;
}

// CSR offsets (2^(jcc*W) + 1 entries) over the join key of a version's rows
const u64* version_csr(ra_program* p, Relation& r, int ver)
{
    const int jbits = (int)r.jcc * p->bits;
    if (jbits > 30)
        fail(p, RA_E_UNSUPPORTED, "relation %s: join key of %d bits exceeds the CSR index limit (30)",
             r.name.c_str(), jbits);
    u64** slot = (ver == RA_DELTA) ? &r.csr_delta : &r.csr_full;
    u64* stamp = (ver == RA_DELTA) ? &r.csr_delta_version : &r.csr_full_version;
    u64 want = (ver == RA_DELTA) ? r.delta_version : r.full_version;
    if (*slot && *stamp == want) return *slot;
    const u64 nk = (1ull << jbits) + 1;
    if (!*slot) dev_alloc(p, slot, nk);
    const u64 *k, *v;
    u64 n;
    version_rows(p, r, ver, &k, &v, &n);
    u32* counts;
    dev_alloc(p, &counts, nk);
    CK(cudaMemsetAsync(counts, 0, nk * 4, p->stream));
    if (n) {
        csr_count<<<grid_for(n), kThreads, 0, p->stream>>>(k, n, (int)(r.arity - r.jcc) * p->bits, counts);
        LAUNCHED();
    }
    scan_exclusive<u32>(p, counts, nk, *slot, false);
    dev_free(p, &counts);
    *stamp = want;
    return *slot;
}

void build_seen(ra_program* p, Relation& r, u64 need)
{
    u64 want = 1024;
    while (want < 2 * need) want <<= 1;
    if (r.seen && r.seen_cap >= want) return;
    dev_free(p, &r.seen);
    dev_alloc(p, &r.seen, want);
    CK(cudaMemsetAsync(r.seen, 0xff, want * sizeof(Slot), p->stream));
    r.seen_cap = want;
    u64 n = r.full_n + r.delta_n;   // every stored tuple; newt is empty between iterations
    CK(cudaMemsetAsync(p->derr, 0, 4, p->stream));
    if (n) {
        seen_insert_existing<<<grid_for(n), kThreads, 0, p->stream>>>(r.seen, want - 1, r.keys, n, p->derr);
        LAUNCHED();
    }
    r.seen_n = n;   // upper bound (duplicate keys of loaded rows count once in the table)
}

u64& intern_counter(ra_program* p, uint32_t tag)
{
    for (auto& e : p->intern)
        if (e.first == tag) return e.second;
    p->intern.push_back({tag, 0});
    return p->intern.back().second;
}

// ---------------------------------------------------------------------------
// rule geometry: which side is outer, and the projection in packed columns
// ---------------------------------------------------------------------------
struct JoinPlan {
    int outer_rel, outer_ver, inner_rel, inner_ver;
    Projection pj;
};

Projection make_copy_proj(ra_program* p, const Rule& ru, const Relation& in, const Relation& out)
{
    Projection pj{};
    pj.n = (int)ru.proj.size();
    pj.outer_arity = (int)in.arity;
    pj.inner_arity = 1;
    if ((uint32_t)pj.n != out.arity)
        fail(p, RA_E_BADARG, "copy into %s: reorder list has %d entries, relation arity is %u", out.name.c_str(),
             pj.n, out.arity);
    for (int j = 0; j < pj.n; j++) {
        int x = ru.proj[j];
        if (x < 0 || x > (int)in.arity) fail(p, RA_E_BADARG, "copy: reorder index %d out of range", x);
        if (x == (int)in.arity)
            fail(p, RA_E_UNSUPPORTED, "copy into %s: moving the intern id into a data column is not supported",
                 out.name.c_str());
        pj.side[j] = 0;
        pj.col[j] = (signed char)x;
    }
    return pj;
}

JoinPlan make_join_plan(ra_program* p, const Rule& ru)
{
    JoinPlan jp{};
    const Relation& in0 = p->rels[ru.in0];
    const Relation& in1 = p->rels[ru.in1];
    const Relation& out = p->rels[ru.out];
    const int jcc = (int)in0.jcc;
    if (in1.jcc != in0.jcc)
        fail(p, RA_E_UNSUPPORTED, "join %s x %s: inputs hash on different column counts", in0.name.c_str(),
             in1.name.c_str());
    // dispatch of src/RAM/RA_tasks.cpp:452-520
    const bool left = (ru.ver0 == RA_DELTA);
    if (left) {
        jp.outer_rel = ru.in0;
        jp.outer_ver = RA_DELTA;
        jp.inner_rel = ru.in1;
        jp.inner_ver = ru.ver1;
    } else {
        jp.outer_rel = ru.in1;
        jp.outer_ver = ru.ver1;
        jp.inner_rel = ru.in0;
        jp.inner_ver = RA_FULL;
    }
    const int a0 = (int)in0.arity, a1 = (int)in1.arity;
    Projection& pj = jp.pj;
    pj.n = (int)ru.proj.size();
    if ((uint32_t)pj.n != out.arity)
        fail(p, RA_E_BADARG, "join into %s: projection has %d entries, relation arity is %u", out.name.c_str(),
             pj.n, out.arity);
    pj.outer_arity = left ? a0 : a1;
    pj.inner_arity = left ? a1 : a0;
    // reordered tuple = input0 row (a0 + id) ++ input1 row minus its join columns (a1 - jcc + id)
    for (int j = 0; j < pj.n; j++) {
        int x = ru.proj[j];
        int side_in1, col;
        if (x >= 0 && x < a0) {
            side_in1 = 0;
            col = x;
        } else if (x > a0 && x < a0 + 1 + (a1 - jcc)) {
            side_in1 = 1;
            col = jcc + (x - a0 - 1);
        } else if (x == a0 || x == a0 + 1 + (a1 - jcc)) {
            fail(p, RA_E_UNSUPPORTED, "join into %s: projecting an intern id column is not supported",
                 out.name.c_str());
        } else {
            fail(p, RA_E_BADARG, "join: projection index %d out of range", x);
        }
        // input0 is the outer side for LEFT order, the inner side for RIGHT order
        pj.side[j] = (signed char)(left ? side_in1 : !side_in1);
        pj.col[j] = (signed char)col;
    }
    return jp;
}

// ---------------------------------------------------------------------------
// semi-naive swaps on the log
// ---------------------------------------------------------------------------
// relation::insert_full_in_delta (balanced_hash_relation.cpp:1152-1179)
void full_to_delta(ra_program* p, Relation& r)
{
    u64 n = r.full_n + r.delta_n;
    bool sorted = (r.delta_n == 0 && r.full_runs <= 1) || (r.full_n == 0);
    if (!sorted && n) sort_rows(p, r, r.keys, r.ids, n, r.keys_unique);
    r.full_n = 0;
    r.full_runs = 0;
    r.delta_n = n;
    r.full_version++;
    r.delta_version++;
}

// relation::insert_delta_in_full (balanced_hash_relation.cpp:1120-1148)
void delta_to_full(Relation& r)
{
    if (r.delta_n) {
        r.full_runs += 1;
        r.full_n += r.delta_n;
        r.delta_n = 0;
        r.full_version++;
        r.delta_version++;
    }
}

// ---------------------------------------------------------------------------
// one iteration of RAM::execute_in_batches' body for SCC s
// ---------------------------------------------------------------------------
void iterate(ra_program* p, Scc& s)
{
    p->epoch++;
    const size_t R = s.rules.size();
    std::vector<u64> c(R, 0), base(R, 0);
    std::vector<JoinPlan> plans(R);
    std::vector<Projection> cps(R);
    std::vector<const u64*> in_keys(R, nullptr);
    std::vector<u64> in_n(R, 0);
    std::vector<const u64*> csr(R, nullptr);

    // 1. candidate counts per rule
    u64 total = 0;
    for (size_t r = 0; r < R; r++) {
        const Rule& ru = s.rules[r];
        if (ru.kind == RA_ACOPY)
            fail(p, RA_E_UNSUPPORTED, "parallel_acopy into %s is not supported by this engine",
                 p->rels[ru.out].name.c_str());
        if (ru.kind == kJoin) {
            plans[r] = make_join_plan(p, ru);
            Relation& o = p->rels[plans[r].outer_rel];
            Relation& in = p->rels[plans[r].inner_rel];
            const u64 *ok, *ov, *ik, *iv;
            u64 on, inn;
            version_rows(p, o, plans[r].outer_ver, &ok, &ov, &on);
            version_rows(p, in, plans[r].inner_ver, &ik, &iv, &inn);
            in_keys[r] = ok;
            in_n[r] = on;
            if (on == 0 || inn == 0) continue;
            csr[r] = version_csr(p, in, plans[r].inner_ver);
            if (on > p->cnt_cap) {
                dev_free(p, &p->cnt);
                dev_free(p, &p->off);
                p->cnt_cap = on + on / 2;
                dev_alloc(p, &p->cnt, p->cnt_cap);
                dev_alloc(p, &p->off, p->cnt_cap);
            }
            join_count<<<grid_for(on), kThreads, 0, p->stream>>>(ok, on, (int)(o.arity - o.jcc) * p->bits, csr[r],
                                                                  p->cnt);
            LAUNCHED();
            c[r] = scan_exclusive<u64>(p, p->cnt, on, p->off);
            // keep this rule's offsets: expand right away into the candidate buffer
            if (total + c[r] > p->cand_cap) {
                u64 nc = (total + c[r]) * 3 / 2 + 1024;
                u64* nb;
                dev_alloc(p, &nb, nc);
                if (total) CK(cudaMemcpyAsync(nb, p->cand, total * 8, cudaMemcpyDeviceToDevice, p->stream));
                dev_free(p, &p->cand);
                p->cand = nb;
                p->cand_cap = nc;
            }
            base[r] = total;
            if (c[r]) {
                join_expand<<<grid_for(on), kThreads, 0, p->stream>>>(
                    ok, on, (int)(o.arity - o.jcc) * p->bits, csr[r], ik, p->off, plans[r].pj, p->bits,
                    p->cand + total);
                LAUNCHED();
            }
            total += c[r];
        } else {
            Relation& in = p->rels[ru.in0];
            cps[r] = make_copy_proj(p, ru, in, p->rels[ru.out]);
            if (ru.kind == RA_COPY_FILTER && ru.pred >= 2 && in.arity < 2)
                fail(p, RA_E_UNSUPPORTED, "copy_filter on %s: predicate needs two data columns", in.name.c_str());
            const u64 *k, *v;
            u64 n;
            version_rows(p, in, ru.ver0, &k, &v, &n);
            c[r] = n;
            if (total + n > p->cand_cap) {
                u64 nc = (total + n) * 3 / 2 + 1024;
                u64* nb;
                dev_alloc(p, &nb, nc);
                if (total) CK(cudaMemcpyAsync(nb, p->cand, total * 8, cudaMemcpyDeviceToDevice, p->stream));
                dev_free(p, &p->cand);
                p->cand = nb;
                p->cand_cap = nc;
            }
            base[r] = total;
            if (n) {
                copy_expand<<<grid_for(n), kThreads, 0, p->stream>>>(
                    k, n, cps[r], p->bits, ru.kind == RA_COPY_FILTER ? ru.pred : 0, p->cand + total);
                LAUNCHED();
            }
            total += n;
        }
    }
    p->stats.join_candidates += total;

    // 2. make room in every output relation's seen set
    for (size_t r = 0; r < R; r++) {
        Relation& out = p->rels[s.rules[r].out];
        u64 incoming = 0;
        for (size_t q = 0; q < R; q++)
            if (s.rules[q].out == s.rules[r].out) incoming += c[q];
        build_seen(p, out, out.seen_n + incoming);
    }

    // 3. first-occurrence dedup: insert all, then flag winners
    if (total > p->rank_cap) {
        grow1(p, &p->rank, &p->rank_cap, total);
        dev_free(p, &p->flag);
        dev_alloc(p, &p->flag, p->rank_cap);
    }
    CK(cudaMemsetAsync(p->derr, 0, 4, p->stream));
    const u64 tag0 = p->epoch << 40;
    for (size_t r = 0; r < R; r++) {
        if (!c[r]) continue;
        Relation& out = p->rels[s.rules[r].out];
        cudaEvent_t a = nullptr, b = nullptr;
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        cudaEventRecord(a, p->stream);
        dedup_insert<<<grid_for(c[r]), kThreads, 0, p->stream>>>(out.seen, out.seen_cap - 1, p->cand + base[r], c[r],
                                                                  tag0 + base[r], p->derr);
        LAUNCHED();
        cudaEventRecord(b, p->stream);
        p->dedup_events.push_back({a, b});
        p->stats.dedup_launches++;
        p->stats.dedup_bytes += c[r] * (8 + 2 * sizeof(Slot));
    }
    for (size_t r = 0; r < R; r++) {
        if (!c[r]) continue;
        Relation& out = p->rels[s.rules[r].out];
        dedup_flag<<<grid_for(c[r]), kThreads, 0, p->stream>>>(out.seen, out.seen_cap - 1, p->cand + base[r], c[r],
                                                                tag0 + base[r], p->flag + base[r]);
        LAUNCHED();
    }
    // 4. winners -> newt staging, in rule order (RAM::local_insert_in_newt order)
    for (size_t r = 0; r < R; r++) {
        if (!c[r]) continue;
        Relation& out = p->rels[s.rules[r].out];
        u64 w = scan_exclusive<u32>(p, p->flag + base[r], c[r], p->rank + base[r]);
        if (!w) continue;
        u64 need = out.full_n + out.delta_n + out.newt_n + w;
        ensure_log(p, out, need);
        grow2(p, &p->nkeys, &p->nids, &p->n_cap, need, false, 0);
        u64& ctr = intern_counter(p, out.tag);
        const u64 id_base = ((u64)out.tag << 46) | ctr;
        u64* dst_k = out.keys + out.full_n + out.delta_n + out.newt_n;
        u64* dst_v = out.ids + out.full_n + out.delta_n + out.newt_n;
        dedup_compact<<<grid_for(c[r]), kThreads, 0, p->stream>>>(p->cand + base[r], p->flag + base[r],
                                                                   p->rank + base[r], c[r], id_base, dst_k, dst_v);
        LAUNCHED();
        ctr += w;
        out.newt_n += w;
        out.seen_n += w;
    }
    if (read_scalar(p, (const u64*)p->derr) & 0xffffffffull)
        fail(p, RA_E_STATE, "seen-set overflow (internal sizing error)");

    // 5. sort each relation's newt into trie order; then the semi-naive swap
    //    (RAM::local_insert_in_full -> insert_delta_in_full + local_insert_in_delta)
    for (int ri : s.rels) {
        Relation& r = p->rels[ri];
        if (r.newt_n > 1) {
            u64* nk = r.keys + r.full_n + r.delta_n;
            u64* nv = r.ids + r.full_n + r.delta_n;
            radix_sort(p, nk, nv, r.newt_n, 0, key_bits(p, r));
        }
        p->stats.new_tuples += r.newt_n;
    }
    for (int ri : s.rels) {
        Relation& r = p->rels[ri];
        delta_to_full(r);
        r.delta_n = r.newt_n;
        r.newt_n = 0;
        r.delta_version++;
    }
    p->stats.iterations++;
}

void run_scc(ra_program* p, Scc& s)
{
    for (const Rule& ru : s.rules)
        if (std::find(s.rels.begin(), s.rels.end(), ru.out) == s.rels.end())
            fail(p, RA_E_UNSUPPORTED, "SCC %d: rule output %s is not one of the SCC's relations", s.id,
                 p->rels[ru.out].name.c_str());
    for (size_t i = 0; i < s.rels.size(); i++)
        if (s.init[i]) full_to_delta(p, p->rels[s.rels[i]]);
    std::vector<uint64_t> hist;
    for (;;) {
        uint32_t b = p->batch_size;
        while (b != 0) {
            iterate(p, s);
            b--;
            if (!s.fixpoint) break;
        }
        uint32_t d = 0, f = 0;
        for (int ri : s.rels) {
            d += (uint32_t)p->rels[ri].delta_n;
            f += (uint32_t)p->rels[ri].full_n;
        }
        hist.push_back(d);
        hist.push_back(f);
        if (!s.fixpoint || d == 0) break;
    }
    for (int ri : s.rels) delta_to_full(p->rels[ri]);
    p->history.push_back((uint64_t)s.id);
    p->history.push_back(hist.size() / 2);
    p->history.insert(p->history.end(), hist.begin(), hist.end());
}

void choose_bits(ra_program* p)
{
    CK(cudaMemsetAsync(p->dscalar + 1, 0, 8, p->stream));
    for (Relation& r : p->rels)
        if (r.raw_n) {
            rows_max_value<<<grid_for(r.raw_n), kThreads, 0, p->stream>>>(r.raw, r.raw_n, (int)r.arity,
                                                                           p->dscalar + 1);
            LAUNCHED();
        }
    u64 mx = read_scalar(p, p->dscalar + 1);
    int bits = 1;
    while (bits < 64 && (mx >> bits)) bits++;
    for (Relation& r : p->rels)
        if ((int)r.arity * bits > 63)
            fail(p, RA_E_UNSUPPORTED,
                 "relation %s: %u columns of %d bits do not pack into one 63-bit key (largest value %llu)",
                 r.name.c_str(), r.arity, bits, (unsigned long long)mx);
    p->bits = bits;
}

void free_relation_state(ra_program* p, Relation& r)
{
    dev_free(p, &r.keys);
    dev_free(p, &r.ids);
    dev_free(p, &r.seen);
    dev_free(p, &r.vkeys);
    dev_free(p, &r.vids);
    dev_free(p, &r.csr_full);
    dev_free(p, &r.csr_delta);
    r.cap = r.seen_cap = r.seen_n = r.v_cap = 0;
    r.v_version = r.csr_full_version = r.csr_delta_version = ~0ull;
    r.full_n = r.delta_n = r.newt_n = 0;
}

void reset_state(ra_program* p)
{
    for (Relation& r : p->rels) free_relation_state(p, r);
    for (Scc& s : p->sccs) s.done = false;
    p->history.clear();
    p->intern.clear();
    p->executed = false;
    p->running = false;
    p->epoch = 0;
}

void begin_run(ra_program* p)
{
    if (p->executed || p->running) reset_state(p);
    p->stats = ra_stats{};
    for (auto& e : p->dedup_events) {
        cudaEventDestroy(e.first);
        cudaEventDestroy(e.second);
    }
    p->dedup_events.clear();
    if (!p->packed) {
        choose_bits(p);
        for (Relation& r : p->rels) pack_relation(p, r);
        p->packed = true;
    } else {
        for (Relation& r : p->rels) restore_loaded(p, r);
    }
    p->running = true;
    p->fixpoint_ms_acc = 0;
}

// LIE::one_runnable_tasks (src/lie/lie.cpp:27-60): first SCC, in add order, that
// is not the destination of a dependency edge whose source has not run.
int next_runnable(ra_program* p)
{
    for (size_t i = 0; i < p->sccs.size(); i++) {
        if (p->sccs[i].done) continue;
        bool blocked = false;
        for (auto& d : p->deps)
            if (d.second == (int)i && !p->sccs[d.first].done) blocked = true;
        if (!blocked) return (int)i;
    }
    return -1;
}

void finish_run(ra_program* p)
{
    CK(cudaStreamSynchronize(p->stream));
    double dms = 0;
    for (auto& e : p->dedup_events) {
        float m = 0;
        cudaEventElapsedTime(&m, e.first, e.second);
        dms += m;
    }
    p->stats.dedup_ms = dms;
    p->stats.fixpoint_ms = p->fixpoint_ms_acc;
    p->stats.value_bits = (uint32_t)p->bits;
    p->executed = true;
    p->running = false;
}

// returns the SCC id that ran, or -1 when none is left (finishing the run)
int step(ra_program* p)
{
    if (!p->running) begin_run(p);
    int next = next_runnable(p);
    if (next < 0) {
        finish_run(p);
        return -1;
    }
    CK(cudaEventRecord(p->ev0, p->stream));
    run_scc(p, p->sccs[next]);
    p->sccs[next].done = true;
    CK(cudaEventRecord(p->ev1, p->stream));
    CK(cudaEventSynchronize(p->ev1));
    float ms = 0;
    cudaEventElapsedTime(&ms, p->ev0, p->ev1);
    p->fixpoint_ms_acc += ms;
    if (next_runnable(p) < 0) finish_run(p);
    return p->sccs[next].id;
}

void execute(ra_program* p)
{
    if (p->executed || p->running) reset_state(p);
    while (step(p) != -1 && p->running) {}
    if (p->running) finish_run(p);
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================

namespace {
int guard(ra_program* p, const std::function<void()>& f)
{
    if (!p) return RA_E_BADARG;
    try {
        if (p->device >= 0) cudaSetDevice(p->device);
        p->err.clear();
        f();
        return RA_OK;
    } catch (const ra_error& e) {
        return e.status;
    } catch (const std::bad_alloc&) {
        p->err = "host allocation failed";
        return RA_E_OOM;
    }
}
}  // namespace

extern "C" {

int ra_program_create(int device, ra_program** out)
{
    if (!out) return RA_E_BADARG;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) return RA_E_CUDA;
    ra_program* p = new ra_program();
    p->device = device;
    int st = guard(p, [&] {
        CK(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
        p->own_stream = true;
        cudaMemPool_t pool;
        CK(cudaDeviceGetDefaultMemPool(&pool, device));
        uint64_t thresh = ~0ull;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thresh);
        dev_alloc(p, &p->sums, 32 * kThreads);
        dev_alloc(p, &p->dscalar, 8);
        dev_alloc(p, &p->derr, 4);
        CK(cudaMallocHost(&p->hscalar, 64));
        CK(cudaEventCreate(&p->ev0));
        CK(cudaEventCreate(&p->ev1));
    });
    if (st != RA_OK) {
        delete p;
        return st;
    }
    *out = p;
    return RA_OK;
}

int ra_program_destroy(ra_program* p)
{
    if (!p) return RA_E_BADARG;
    cudaSetDevice(p->device);
    if (p->stream) cudaStreamSynchronize(p->stream);
    for (Relation& r : p->rels) {
        free_relation_state(p, r);
        dev_free(p, &r.raw);
        dev_free(p, &r.lkeys);
        dev_free(p, &r.lids);
    }
    dev_free(p, &p->cand);
    dev_free(p, &p->flag);
    dev_free(p, &p->rank);
    dev_free(p, &p->cnt);
    dev_free(p, &p->off);
    dev_free(p, &p->nkeys);
    dev_free(p, &p->nids);
    dev_free(p, &p->tk);
    dev_free(p, &p->tv);
    dev_free(p, &p->sums);
    dev_free(p, &p->dscalar);
    dev_free(p, &p->derr);
    dev_free(p, &p->hist_buf);
    dev_free(p, &p->hist_off);
    for (auto& e : p->dedup_events) {
        cudaEventDestroy(e.first);
        cudaEventDestroy(e.second);
    }
    if (p->stream) cudaStreamSynchronize(p->stream);
    if (p->hscalar) cudaFreeHost(p->hscalar);
    if (p->ev0) cudaEventDestroy(p->ev0);
    if (p->ev1) cudaEventDestroy(p->ev1);
    if (p->own_stream && p->stream) cudaStreamDestroy(p->stream);
    delete p;
    return RA_OK;
}

int ra_program_set_stream(ra_program* p, void* stream)
{
    return guard(p, [&] {
        CK(cudaStreamSynchronize(p->stream));
        if (p->own_stream) cudaStreamDestroy(p->stream);
        if (stream) {
            p->stream = (cudaStream_t)stream;
            p->own_stream = false;
        } else {
            CK(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
            p->own_stream = true;
        }
    });
}

int ra_program_set_batch_size(ra_program* p, uint32_t batch_size)
{
    return guard(p, [&] {
        if (batch_size == 0) fail(p, RA_E_BADARG, "batch size must be positive");
        p->batch_size = batch_size;
    });
}

int ra_relation_create(ra_program* p, uint32_t jcc, uint32_t arity, uint32_t tag, const char* name, int version,
                       int* rel_out)
{
    return guard(p, [&] {
        if (!rel_out || arity == 0 || arity > (uint32_t)kMaxArity || jcc == 0 || jcc > arity)
            fail(p, RA_E_BADARG, "relation: need 1 <= jcc <= arity <= %d", kMaxArity);
        if (version != RA_DELTA && version != RA_FULL) fail(p, RA_E_BADARG, "relation: version must be DELTA or FULL");
        if (tag >= (1u << 18)) fail(p, RA_E_BADARG, "relation: intern tag must be below 2^18");
        Relation r;
        r.jcc = jcc;
        r.arity = arity;
        r.tag = tag;
        r.name = name ? name : "";
        r.version = version;
        p->rels.push_back(r);
        *rel_out = (int)p->rels.size() - 1;
    });
}

static void set_raw(ra_program* p, Relation& r, const uint64_t* rows, uint64_t nrows, cudaMemcpyKind kind)
{
    p->packed = false;
    dev_free(p, &r.raw);
    r.raw_n = nrows;
    dev_alloc(p, &r.raw, nrows * (r.arity + 1));
    if (nrows) CK(cudaMemcpyAsync(r.raw, rows, nrows * (r.arity + 1) * 8, kind, p->stream));
    CK(cudaStreamSynchronize(p->stream));
}

int ra_relation_load_rows(ra_program* p, int rel, const uint64_t* host_rows, uint64_t nrows)
{
    return guard(p, [&] {
        Relation& r = rel_at(p, rel);
        if (nrows && !host_rows) fail(p, RA_E_BADARG, "null rows");
        set_raw(p, r, host_rows, nrows, cudaMemcpyHostToDevice);
    });
}

int ra_relation_load_rows_device(ra_program* p, int rel, const uint64_t* dev_rows, uint64_t nrows)
{
    return guard(p, [&] {
        Relation& r = rel_at(p, rel);
        if (nrows && !dev_rows) fail(p, RA_E_BADARG, "null rows");
        set_raw(p, r, dev_rows, nrows, cudaMemcpyDeviceToDevice);
    });
}

int ra_relation_load_file(ra_program* p, int rel, const char* path)
{
    return guard(p, [&] {
        Relation& r = rel_at(p, rel);
        if (!path) fail(p, RA_E_BADARG, "null path");
        std::string meta = std::string(path) + ".size";
        FILE* f = fopen(meta.c_str(), "r");
        if (!f) fail(p, RA_E_IO, "cannot open %s", meta.c_str());
        unsigned long long rows = 0, cols = 0;
        int got = fscanf(f, "%llu %llu", &rows, &cols);
        fclose(f);
        if (got != 2) fail(p, RA_E_IO, "%s: expected \"<rows>\\n<cols>\"", meta.c_str());
        // parallel_io.cpp:180 asserts arity + 1 == col_count
        if (cols != r.arity + 1)
            fail(p, RA_E_IO, "%s: %llu columns, relation %s needs %u", meta.c_str(), cols, r.name.c_str(), r.arity + 1);
        std::vector<uint64_t> buf((size_t)(rows * cols));
        if (rows) {
            FILE* d = fopen(path, "rb");
            if (!d) fail(p, RA_E_IO, "cannot open %s", path);
            size_t n = fread(buf.data(), 8, buf.size(), d);
            fclose(d);
            if (n != buf.size()) fail(p, RA_E_IO, "%s: short read (%zu of %zu u64)", path, n, buf.size());
        }
        set_raw(p, r, buf.data(), rows, cudaMemcpyHostToDevice);
    });
}

int ra_scc_create(ra_program* p, int fixpoint, int scc_id, int* scc_out)
{
    return guard(p, [&] {
        if (!scc_out) fail(p, RA_E_BADARG, "null output");
        Scc s;
        s.fixpoint = fixpoint != 0;
        s.id = scc_id;
        p->sccs.push_back(s);
        *scc_out = (int)p->sccs.size() - 1;
    });
}

static Scc& scc_at(ra_program* p, int scc)
{
    if (scc < 0 || scc >= (int)p->sccs.size()) fail(p, RA_E_BADARG, "bad SCC handle %d", scc);
    return p->sccs[scc];
}

int ra_scc_add_relation(ra_program* p, int scc, int rel, int init_status)
{
    return guard(p, [&] {
        Scc& s = scc_at(p, scc);
        rel_at(p, rel);
        s.rels.push_back(rel);
        s.init.push_back(init_status != 0);
    });
}

int ra_scc_add_join(ra_program* p, int scc, int out, int in0, int ver0, int in1, int ver1, const int* proj, int nproj)
{
    return guard(p, [&] {
        Scc& s = scc_at(p, scc);
        rel_at(p, out);
        rel_at(p, in0);
        rel_at(p, in1);
        if ((ver0 != RA_DELTA && ver0 != RA_FULL) || (ver1 != RA_DELTA && ver1 != RA_FULL))
            fail(p, RA_E_BADARG, "join versions must be DELTA or FULL");
        if (nproj <= 0 || nproj > kMaxArity || !proj) fail(p, RA_E_BADARG, "join projection size");
        Rule r{kJoin, out, in0, ver0, in1, ver1, std::vector<int>(proj, proj + nproj), 0};
        s.rules.push_back(r);
    });
}

int ra_scc_add_copy(ra_program* p, int scc, int kind, int out, int in, int ver, const int* proj, int nproj, int pred)
{
    return guard(p, [&] {
        Scc& s = scc_at(p, scc);
        rel_at(p, out);
        rel_at(p, in);
        if (kind != RA_COPY && kind != RA_ACOPY && kind != RA_COPY_FILTER) fail(p, RA_E_BADARG, "copy kind");
        if (ver != RA_DELTA && ver != RA_FULL) fail(p, RA_E_BADARG, "copy version must be DELTA or FULL");
        if (nproj <= 0 || nproj > kMaxArity + 1 || !proj) fail(p, RA_E_BADARG, "copy reorder size");
        if (kind == RA_COPY_FILTER && (pred < RA_PRED_TRUE || pred > RA_PRED_GE)) fail(p, RA_E_BADARG, "predicate");
        Rule r{kind, out, in, ver, -1, -1, std::vector<int>(proj, proj + nproj), kind == RA_COPY_FILTER ? pred : 0};
        s.rules.push_back(r);
    });
}

int ra_scc_depend(ra_program* p, int src_scc, int dst_scc)
{
    return guard(p, [&] {
        scc_at(p, src_scc);
        scc_at(p, dst_scc);
        p->deps.push_back({src_scc, dst_scc});
    });
}

int ra_program_execute(ra_program* p)
{
    return guard(p, [&] { execute(p); });
}

int ra_program_run_next_scc(ra_program* p, int* scc_id)
{
    return guard(p, [&] {
        int id = -1;
        if (!(p->executed && !p->running)) id = step(p);
        if (scc_id) *scc_id = id;
    });
}

int ra_program_reset(ra_program* p)
{
    return guard(p, [&] {
        reset_state(p);
        CK(cudaStreamSynchronize(p->stream));
    });
}

int ra_program_history(ra_program* p, uint64_t* out, uint64_t cap, uint64_t* len)
{
    return guard(p, [&] {
        if (len) *len = p->history.size();
        if (out) std::memcpy(out, p->history.data(), std::min<u64>(cap, p->history.size()) * 8);
    });
}

int ra_program_stats(ra_program* p, ra_stats* out)
{
    return guard(p, [&] {
        if (!out) fail(p, RA_E_BADARG, "null stats");
        *out = p->stats;
    });
}

int ra_relation_counts(ra_program* p, int rel, uint64_t* full, uint64_t* delta)
{
    return guard(p, [&] {
        Relation& r = rel_at(p, rel);
        if (full) *full = r.full_n;
        if (delta) *delta = r.delta_n;
    });
}

int ra_relation_dump_full(ra_program* p, int rel, uint64_t* host_rows, uint64_t cap_rows, uint64_t* rows_out)
{
    return guard(p, [&] {
        Relation& r = rel_at(p, rel);
        if (!p->executed) fail(p, RA_E_STATE, "dump before execute");
        const u64 *k, *v;
        u64 n;
        version_rows(p, r, RA_FULL, &k, &v, &n);
        u64 m = std::min<u64>(n, cap_rows);
        if (rows_out) *rows_out = m;
        if (!m || !host_rows) return;
        u64* rows;
        dev_alloc(p, &rows, m * (r.arity + 1));
        rows_unpack<<<grid_for(m), kThreads, 0, p->stream>>>(k, v, m, (int)r.arity, p->bits, rows);
        LAUNCHED();
        CK(cudaMemcpyAsync(host_rows, rows, m * (r.arity + 1) * 8, cudaMemcpyDeviceToHost, p->stream));
        dev_free(p, &rows);
        CK(cudaStreamSynchronize(p->stream));
    });
}

const char* ra_status_string(int status)
{
    switch (status) {
    case RA_OK: return "ok";
    case RA_E_BADARG: return "bad argument";
    case RA_E_IO: return "I/O error";
    case RA_E_OOM: return "out of device memory";
    case RA_E_CUDA: return "CUDA error";
    case RA_E_UNSUPPORTED: return "unsupported program shape";
    case RA_E_TIMEOUT: return "device wait timed out";
    case RA_E_STATE: return "invalid state";
    }
    return "unknown status";
}

const char* ra_last_error(ra_program* p) { return p ? p->err.c_str() : "null program"; }

}  // extern "C"
