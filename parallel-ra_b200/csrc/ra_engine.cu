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
#include "ra_dense.cuh"
#include "ra_persist.cuh"
#include "ra_reach.cuh"
#include "ra_tail.cuh"
#include "ra_wide.cuh"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <functional>
#include <fstream>
#include <string>
#include <sys/stat.h>
#include <unistd.h>
#include <unordered_map>
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

// process-wide unique version stamps (caches are keyed by them)
std::atomic<unsigned long long> g_stamp{0};
u64 fresh_stamp() { return ++g_stamp; }

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
    // instantiated fixed-point graph, reused while everything it captured is unchanged
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<unsigned char> graph_sig;
    int graph_kernels = 0;
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
    u64 l_full_stamp = 0, l_delta_stamp = 0;   // stamps of the packed loaded state
    bool seen_dirty = false;                    // seen set holds a previous run's keys
    // log [ full | delta | newt ]
    u64* keys = nullptr;
    u64* ids = nullptr;
    u64 cap = 0;
    u64 full_n = 0, delta_n = 0;
    bool full_sorted = true;    // full region in trie order (lexicographic on (key, id))
    bool delta_sorted = true;   // delta region in trie order
    bool keys_unique = true;    // no two stored tuples share data columns
    u64 full_version = 0, delta_version = 0;
    // seen set over data columns
    Slot* seen = nullptr;
    u64 seen_cap = 0, seen_n = 0;
    // sorted view of full (used when the full region is not sorted)
    u64* vkeys = nullptr;
    u64* vids = nullptr;
    u64 v_cap = 0, v_version = ~0ull;
    // CSR index on the join key, for full (version-stamped) and delta
    u64* csr_full = nullptr;
    u64 csr_full_version = ~0ull;
    u64 csr_full_cap = 0;          // entries (2^join-key-bits + 1 of the run that built it)
    u64* csr_delta = nullptr;
    u64 csr_delta_version = ~0ull;
    u64 csr_delta_cap = 0;
    u64 csr_full_longest = 0;      // most rows sharing one join key, per CSR
    u64 csr_delta_longest = 0;
    // bitmap seen set (binary relations over small domains), kept between runs
    u32* bm_seen = nullptr;
    u32* bm_fresh = nullptr;
    u8* bm_dirty = nullptr;
    u64 bm_words = 0;             // capacity of bm_seen / bm_fresh (u32 words)
    u64 bm_rows = 0;              // capacity of bm_dirty (rows)
    // newt staging for the running iteration
    u64 newt_n = 0;
    // wide programs: versions as rows of arity + 1 u64 in trie order (counts above)
    u64* wfull = nullptr;
    u64* wdelta = nullptr;
    u64* wnewt = nullptr;
    u64* wspare = nullptr;   // merge target, swapped with full / delta
    u64* wcand = nullptr;    // the running iteration's candidates into this relation
    u32* wflag = nullptr;    // their winner flags
    u64* wpos = nullptr;     // and the winners' positions
    u64 wfull_cap = 0, wdelta_cap = 0, wnewt_cap = 0, wspare_cap = 0, wcand_cap = 0, wflag_cap = 0, wpos_cap = 0;
    int wcand_w = 0;         // columns per candidate row of wcand
};

}  // namespace

struct ra_program {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    uint32_t batch_size = 1;
    int id_order = RA_IDS_EMISSION;
    ra_tuning tune = {0.45, 4.0, 1.5, 8, 4, 8e9};   // the B200 choice (tuning.json)
    std::vector<Relation> rels;
    std::vector<Scc> sccs;
    std::vector<std::pair<int, int>> deps;
    std::vector<uint64_t> history;
    std::vector<double> iter_us;  // device time of each device-driven iteration of the last run
    std::vector<std::pair<uint32_t, u64>> intern;   // (tag, next counter) -- LIE::intern_map
    int bits = 0;                 // packed bits per column for this run
    u64 max_value = 0;            // largest data value loaded (sets `bits`)
    bool packed = false;          // loaded relations packed with `bits` (cleared by a new load)
    bool wide = false;            // this run keeps tuples as rows of u64 columns (ra_wide.cu)
    u64* wbuf[12] = {};           // scratch of the wide path
    u64 wbuf_cap[12] = {};
    bool executed = false;
    bool running = false;         // between the first and the last SCC of a run
    double fixpoint_ms_acc = 0;
    u64 epoch = 0;
    std::string err;
    ra_stats stats{};
    std::unordered_map<void*, u64> alloc_bytes;   // live device allocations
    u64 live_bytes = 0;
    u64 alloc_cap = 0;            // most device bytes the program may hold (0: no cap)
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
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> phase_events;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // device-driven SCC runs (graph mode)
    IterCtl* ctl = nullptr;
    IterCtl* hctl = nullptr;      // pinned mirror (header part)
    u64* dcand = nullptr;
    u32* dloser = nullptr;        // per stream position: epoch in which it lost (not a first occurrence)
    u64 dcand_cap = 0;
    u64* doff[kMaxSccRules] = {};
    u64* dstart[kMaxSccRules] = {};
    u64 doff_cap = 0;
    u64* stage_k[kMaxSccRels] = {};
    u64* stage_v[kMaxSccRels] = {};
    u64 stage_cap = 0;
    u64* sort_k[2] = {};
    u64* sort_v[2] = {};
    u64* status = nullptr;
    u64 status_cap = 0;
    HeavyItem* dheavy = nullptr;  // heavy-row work items of the join launches
    u64 heavy_cap = 0;
    u64 heavy_cands = 0;          // candidates of an iteration the heavy list must cover (bitmap rules write none)
    // instances (batched programs): instance i owns values [inst_base_h[i], inst_base_h[i + 1])
    std::vector<u64> inst_base_h;  // n_inst + 1 entries, the last ~0
    u64* dinst_base = nullptr;
    u32 n_inst = 0;
    u64* dinst_new = nullptr;      // [iteration][instance] new tuples of the running SCC
    u64 inst_rows_cap = 0;
    std::vector<u64> inst_hist;    // per iteration of the run: n_inst new-tuple counts
    bool inst_hist_ok = true;      // false once an SCC ran without instance accounting
    u64* dhist = nullptr;
    u64 dhist_cap = 0;
    // checkpoint dumps (LIE::write_checkpoint_dump) and restart (LIE::execute's restart path)
    std::string cp_dir;
    uint32_t cp_every = 0;        // dump after every cp_every-th batch of an SCC; 0: no dumps
    bool cp_separate = false;     // per-rank file names (LIE::enable_separate_io)
    std::string rs_dir;           // restart from this dump directory ("" : no restart)
    bool rs_separate = false;
    std::vector<int> executed_ids;   // SCC ids completed (the dump's scc_metadata)
    std::vector<int> rs_skip;        // SCC ids a restart does not run again
    int loop_counter = 0;         // batches of the running SCC (LIE::execute's loop_counter)
    std::vector<int> pending_merge;  // relations of the last SCC whose delta still awaits full
    // per-row tables of the instances' bit matrices (bitmap seen sets of batched runs)
    u64* bmt_word = nullptr;
    u32* bmt_base = nullptr;
    u32* bmt_words = nullptr;
    u32* bmt_inst = nullptr;
    u64 bmt_rows = 0, bmt_total = 0;
    std::vector<u64> bmt_bases;      // the instance bases the tables were built for
    bool use_graphs = true;       // RA_NO_GRAPH=1: replay the iteration from the host instead
    bool use_persist = false;     // RA_PERSIST=1: the persistent SCC kernel instead of CUDA-graph iterations
    bool use_reach = false;       // RA_REACH=1: closure-shaped SCCs by composing reachable sets
    u64 reach_arena_hint = 0;     // arena entries the last reachability evaluation used
    bool use_tail = true;         // RA_NO_TAIL=1: no tail kernel in the iteration body
    int tail_ctas = -1;           // CTAs of the tail kernel's cluster (0: none fits; -1: not yet asked)
    bool kernel_events = false;   // RA_KERNEL_EVENTS=1: per-launch events on the claim kernels (no graph)
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
    if (p->alloc_cap && p->live_bytes + count * sizeof(T) > p->alloc_cap)
        fail(p, RA_E_OOM, "device-memory cap of %llu bytes reached (%llu held, %llu more asked)",
             (unsigned long long)p->alloc_cap, (unsigned long long)p->live_bytes,
             (unsigned long long)(count * sizeof(T)));
    CK(cudaMallocAsync(&q, count * sizeof(T), p->stream));
    *ptr = (T*)q;
    p->alloc_bytes[q] = count * sizeof(T);
    p->live_bytes += count * sizeof(T);
    p->stats.device_bytes = p->live_bytes;
    p->stats.device_bytes_peak = std::max<uint64_t>(p->stats.device_bytes_peak, p->live_bytes);
}

template <typename T>
void dev_free(ra_program* p, T** ptr)
{
    if (*ptr) {
        cudaFreeAsync(*ptr, p->stream);
        auto it = p->alloc_bytes.find((void*)*ptr);
        if (it != p->alloc_bytes.end()) {
            p->live_bytes -= it->second;
            p->alloc_bytes.erase(it);
        }
        p->stats.device_bytes = p->live_bytes;
    }
    *ptr = nullptr;
}

// grow a pair of u64 buffers to at least n elements, capacity growth x n
// (contents preserved when keep)
void grow2(ra_program* p, u64** a, u64** b, u64* cap, u64 n, bool keep, u64 keep_n, double growth = 1.5)
{
    if (n <= *cap) return;
    u64 nc = std::max<u64>((u64)((double)n * growth), 1024);
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
    *cap = 0;   // a failed allocation leaves no stale capacity behind
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
    grow2(p, &r.keys, &r.ids, &r.cap, n, true, r.full_n + r.delta_n + r.newt_n, p->tune.log_growth);
}

// ---------------------------------------------------------------------------
// load: pack raw rows -> sorted, distinct (key, id) rows in the log's full region
// ---------------------------------------------------------------------------
void pack_relation(ra_program* p, Relation& r)
{
    r.full_n = r.delta_n = r.newt_n = 0;
    r.full_sorted = r.delta_sorted = true;
    r.keys_unique = true;
    r.full_version = fresh_stamp();
    r.delta_version = fresh_stamp();
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
    if (r.version == RA_DELTA) r.delta_n = n;
    else r.full_n = n;
    grow2(p, &r.lkeys, &r.lids, &r.l_cap, n, false, 0);
    if (n) {
        CK(cudaMemcpyAsync(r.lkeys, r.keys, n * 8, cudaMemcpyDeviceToDevice, p->stream));
        CK(cudaMemcpyAsync(r.lids, r.ids, n * 8, cudaMemcpyDeviceToDevice, p->stream));
    }
    r.l_n = n;
    r.l_keys_unique = r.keys_unique;
    r.l_full_stamp = r.full_version;
    r.l_delta_stamp = r.delta_version;
}

// back to the loaded tuples packed by pack_relation (same column width)
void restore_loaded(ra_program* p, Relation& r)
{
    r.full_n = r.delta_n = r.newt_n = 0;
    r.full_sorted = r.delta_sorted = true;
    r.keys_unique = r.l_keys_unique;
    // same content as when packed: caches built on the loaded state stay valid
    r.full_version = r.l_full_stamp;
    r.delta_version = r.l_delta_stamp;
    if (!r.l_n) return;
    ensure_log(p, r, r.l_n);
    CK(cudaMemcpyAsync(r.keys, r.lkeys, r.l_n * 8, cudaMemcpyDeviceToDevice, p->stream));
    CK(cudaMemcpyAsync(r.ids, r.lids, r.l_n * 8, cudaMemcpyDeviceToDevice, p->stream));
    if (r.version == RA_DELTA) r.delta_n = r.l_n;
    else r.full_n = r.l_n;
}

// (key, id) rows of a relation version.  FULL rows are always returned in trie
// order (a sorted copy when the region is not sorted); DELTA rows are sorted in
// place when `sorted` is requested.
void version_rows(ra_program* p, Relation& r, int ver, const u64** k, const u64** v, u64* n, bool sorted = true)
{
    if (ver == RA_DELTA) {
        if (sorted && !r.delta_sorted && r.delta_n > 1) {
            sort_rows(p, r, r.keys + r.full_n, r.ids + r.full_n, r.delta_n, r.keys_unique);
            r.delta_version = fresh_stamp();
        }
        if (sorted) r.delta_sorted = true;
        *k = r.keys + r.full_n;
        *v = r.ids + r.full_n;
        *n = r.delta_n;
        return;
    }
    if (r.full_sorted) {
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

// CSR offsets (2^(jcc*W) + 1 entries) over the join key of a version's rows;
// its longest row (most rows sharing one key) goes to csr_{full,delta}_longest
const u64* version_csr(ra_program* p, Relation& r, int ver)
{
    const int jbits = (int)r.jcc * p->bits;
    if (jbits > 30)
        fail(p, RA_E_UNSUPPORTED, "relation %s: join key of %d bits exceeds the CSR index limit (30)",
             r.name.c_str(), jbits);
    u64** slot = (ver == RA_DELTA) ? &r.csr_delta : &r.csr_full;
    u64* stamp = (ver == RA_DELTA) ? &r.csr_delta_version : &r.csr_full_version;
    u64* cap = (ver == RA_DELTA) ? &r.csr_delta_cap : &r.csr_full_cap;
    u64 want = (ver == RA_DELTA) ? r.delta_version : r.full_version;
    if (*slot && *stamp == want) return *slot;
    // the key width changes with the values loaded: a reloaded program may need a larger index
    const u64 nk = (1ull << jbits) + 1;
    if (*cap < nk + 1) {
        dev_free(p, slot);
        dev_alloc(p, slot, nk + 1);
        *cap = nk + 1;
    }
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
    CK(cudaMemsetAsync(*slot + nk, 0, 8, p->stream));
    csr_row_max<<<grid_for(nk), kThreads, 0, p->stream>>>(counts, nk, (unsigned long long*)(*slot + nk));
    LAUNCHED();
    (ver == RA_DELTA ? r.csr_delta_longest : r.csr_full_longest) = read_scalar(p, *slot + nk);
    dev_free(p, &counts);
    *stamp = want;
    return *slot;
}

// seen set with room for `need` keys at the tuned maximum load (slot count
// rounded up to whole 128-byte lines)
void build_seen(ra_program* p, Relation& r, u64 need)
{
    u64 want = std::max<u64>((u64)std::ceil((double)need / p->tune.seen_load_max), 1024);
    want = (want + 7) & ~7ull;
    if (r.seen && r.seen_cap >= want && !r.seen_dirty) return;
    if (!r.seen || r.seen_cap < want) {
        dev_free(p, &r.seen);
        dev_alloc(p, &r.seen, want);
        r.seen_cap = want;
    }
    want = r.seen_cap;
    r.seen_dirty = false;
    CK(cudaMemsetAsync(r.seen, 0xff, want * sizeof(Slot), p->stream));
    u64 n = r.full_n + r.delta_n;   // every stored tuple; newt is empty between iterations
    CK(cudaMemsetAsync(p->derr, 0, 4, p->stream));
    if (n) {
        seen_insert_existing<<<grid_for(n), kThreads, 0, p->stream>>>(r.seen, want, r.keys, n, p->derr);
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
    bool sorted = (r.delta_n == 0 && r.full_sorted) || (r.full_n == 0 && r.delta_sorted);
    if (!sorted && n && p->id_order == RA_IDS_REFERENCE) {
        sort_rows(p, r, r.keys, r.ids, n, r.keys_unique);
        sorted = true;
    }
    r.full_n = 0;
    r.full_sorted = true;
    r.delta_sorted = sorted || n <= 1;
    r.delta_n = n;
    r.full_version = fresh_stamp();
    r.delta_version = fresh_stamp();
}

// relation::insert_delta_in_full (balanced_hash_relation.cpp:1120-1148)
void delta_to_full(Relation& r)
{
    if (r.delta_n) {
        r.full_sorted = (r.full_n == 0) ? r.delta_sorted : false;
        r.full_n += r.delta_n;
        r.delta_n = 0;
        r.full_version = fresh_stamp();
        r.delta_version = fresh_stamp();
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
            version_rows(p, o, plans[r].outer_ver, &ok, &ov, &on, p->id_order == RA_IDS_REFERENCE);
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
            version_rows(p, in, ru.ver0, &k, &v, &n, p->id_order == RA_IDS_REFERENCE);
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
        dedup_insert<<<grid_for(c[r]), kThreads, 0, p->stream>>>(out.seen, out.seen_cap, p->cand + base[r], c[r],
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
        dedup_flag<<<grid_for(c[r]), kThreads, 0, p->stream>>>(out.seen, out.seen_cap, p->cand + base[r], c[r],
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
        if (r.newt_n > 1 && p->id_order == RA_IDS_REFERENCE) {
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
        r.delta_sorted = p->id_order == RA_IDS_REFERENCE || r.delta_n <= 1;
        r.delta_version = fresh_stamp();
    }
    p->stats.iterations++;
}


// ===========================================================================
// Device-driven SCC execution (CUDA graph with a WHILE conditional node)
// ===========================================================================
struct DevRule {
    int kind;
    int out_slot;
    RowsRef in;            // join: outer rows; copy: input rows
    Projection pj;
    const u64* csr = nullptr;
    u64 longest = 0;                // join: the inner CSR's longest row (heavy-row split above kHeavyRow)
    const u64* inner = nullptr;
    int outer_shift = 0;
    int pred = 0;
};

struct DevScc {
    SccPlan plan;
    SccRelMap rm;
    std::vector<DevRule> rules;
    std::vector<int> rel_of_slot;   // slot -> program relation index
    std::vector<uint32_t> tags;     // tag slot -> tag
    int passes[kMaxSccRels];
    BitSeen bit[kMaxSccRels] = {};  // bitmap seen sets (bit[s].seen null: the hash set)
};

size_t ctl_header_bytes() { return offsetof(IterCtl, sort_hist); }

int grid_blocks(uint32_t per_sm) { return kSms * (int)per_sm; }

// Can SCC s run without host work between iterations?  Every rule must read
// rows that either are the DELTA of one of the SCC's relations (tracked on the
// device) or do not change while the SCC runs.
bool build_dev_scc(ra_program* p, Scc& s, DevScc& d)
{
    if (s.rels.size() > (size_t)kMaxSccRels || s.rules.size() > (size_t)kMaxSccRules) return false;
    auto slot_of = [&](int rel) {
        for (size_t i = 0; i < s.rels.size(); i++)
            if (s.rels[i] == rel) return (int)i;
        return -1;
    };
    auto written = [&](int rel) {
        for (const Rule& ru : s.rules)
            if (ru.out == rel) return true;
        return false;
    };
    auto static_full = [&](int rel) {
        return !written(rel) && (slot_of(rel) < 0 || p->rels[rel].delta_n == 0);
    };
    // fixed rows of (rel, ver), or slot-tracked delta
    auto rows_ref = [&](int rel, int ver, RowsRef& out) -> bool {
        Relation& r = p->rels[rel];
        if (ver == RA_DELTA) {
            int sl = slot_of(rel);
            if (sl >= 0) {
                out = RowsRef{r.keys, sl, 0};
                return true;
            }
            out = RowsRef{r.keys + r.full_n, -1, r.delta_n};
            return true;
        }
        if (!static_full(rel)) return false;
        const u64 *k, *v;
        u64 n;
        version_rows(p, r, RA_FULL, &k, &v, &n);
        out = RowsRef{k, -1, n};
        return true;
    };
    d = DevScc{};
    SccPlan& pl = d.plan;
    pl.n_rels = (int)s.rels.size();
    pl.n_rules = (int)s.rules.size();
    pl.fixpoint = s.fixpoint ? 1 : 0;
    pl.batch_size = p->batch_size;
    pl.iter_limit = 1ull << 40;
    for (int ri : s.rels) d.rel_of_slot.push_back(ri);
    for (size_t i = 0; i < s.rels.size(); i++) {
        Relation& r = p->rels[s.rels[i]];
        pl.rel_tag_word[i] = (u64)r.tag << 46;
        d.passes[i] = std::max(1, (key_bits(p, r) + kRadixBits - 1) / kRadixBits);
        if (d.passes[i] > kMaxPasses) return false;
    }
    for (size_t q = 0; q < s.rules.size(); q++) {
        const Rule& ru = s.rules[q];
        DevRule dr;
        dr.kind = ru.kind;
        dr.out_slot = slot_of(ru.out);
        if (dr.out_slot < 0) return false;
        uint32_t tag = p->rels[ru.out].tag;
        int ts = -1;
        for (size_t t = 0; t < d.tags.size(); t++)
            if (d.tags[t] == tag) ts = (int)t;
        if (ts < 0) {
            if (d.tags.size() >= (size_t)kMaxTagSlots) return false;
            d.tags.push_back(tag);
            ts = (int)d.tags.size() - 1;
        }
        pl.rule_out[q] = dr.out_slot;
        pl.rule_tag[q] = ts;
        if (ru.kind == kJoin) {
            JoinPlan jp = make_join_plan(p, ru);
            // the inner side must not change while the SCC runs
            if (jp.inner_ver == RA_FULL ? !static_full(jp.inner_rel) : slot_of(jp.inner_rel) >= 0) return false;
            if (!rows_ref(jp.outer_rel, jp.outer_ver, dr.in)) return false;
            Relation& in = p->rels[jp.inner_rel];
            const u64 *ik, *iv;
            u64 inn;
            version_rows(p, in, jp.inner_ver, &ik, &iv, &inn);
            dr.inner = ik;
            dr.csr = version_csr(p, in, jp.inner_ver);
            dr.longest = jp.inner_ver == RA_DELTA ? in.csr_delta_longest : in.csr_full_longest;
            dr.pj = jp.pj;
            const Relation& o = p->rels[jp.outer_rel];
            dr.outer_shift = (int)(o.arity - o.jcc) * p->bits;
            pl.rule_is_join[q] = 1;
            pl.rule_in_slot[q] = -1;
        } else {
            if (ru.kind == RA_ACOPY) return false;
            Relation& in = p->rels[ru.in0];
            dr.pj = make_copy_proj(p, ru, in, p->rels[ru.out]);
            if (ru.kind == RA_COPY_FILTER && ru.pred >= 2 && in.arity < 2)
                fail(p, RA_E_UNSUPPORTED, "copy_filter on %s: predicate needs two data columns", in.name.c_str());
            dr.pred = ru.kind == RA_COPY_FILTER ? ru.pred : 0;
            if (!rows_ref(ru.in0, ru.ver0, dr.in)) return false;
            pl.rule_is_join[q] = 0;
            pl.rule_in_slot[q] = dr.in.slot;
            pl.rule_in_static_n[q] = dr.in.static_n;
        }
        d.rules.push_back(dr);
    }
    for (int sl = 0; sl < pl.n_rels; sl++) {
        d.rm.n_rules_in[sl] = 0;
        for (int q = 0; q < pl.n_rules; q++)
            if (pl.rule_out[q] == sl) d.rm.rules_in[sl][d.rm.n_rules_in[sl]++] = q;
    }
    return true;
}

// rows read from an SCC relation's DELTA follow its log, which may have moved
void refresh_refs(ra_program* p, DevScc& d)
{
    for (DevRule& r : d.rules)
        if (r.in.slot >= 0) r.in.keys = p->rels[d.rel_of_slot[r.in.slot]].keys;
}

// (Re)size every buffer the iteration touches to the plan's capacities.
void dev_size_buffers(ra_program* p, DevScc& d, u64 cand_cap, u64 stage_cap, u64 hist_cap)
{
    if (cand_cap > p->dcand_cap) {
        dev_free(p, &p->dcand);
        dev_free(p, &p->dloser);
        p->dcand_cap = 0;   // a failed allocation leaves no capacity behind a freed buffer
        dev_alloc(p, &p->dcand, cand_cap);
        dev_alloc(p, &p->dloser, cand_cap);
        CK(cudaMemsetAsync(p->dloser, 0, cand_cap * 4, p->stream));   // epoch 0: no marks
        p->dcand_cap = cand_cap;
    }
    const bool ref = p->id_order == RA_IDS_REFERENCE;
    if (ref && stage_cap > p->stage_cap) {
        for (int sl = 0; sl < kMaxSccRels; sl++) {
            dev_free(p, &p->stage_k[sl]);
            dev_free(p, &p->stage_v[sl]);
        }
        for (int b = 0; b < 2; b++) {
            dev_free(p, &p->sort_k[b]);
            dev_free(p, &p->sort_v[b]);
            dev_alloc(p, &p->sort_k[b], stage_cap);
            dev_alloc(p, &p->sort_v[b], stage_cap);
        }
        p->stage_cap = stage_cap;
    }
    for (int sl = 0; sl < d.plan.n_rels && ref; sl++)
        if (d.rm.n_rules_in[sl] && !p->stage_k[sl]) {
            dev_alloc(p, &p->stage_k[sl], p->stage_cap);
            dev_alloc(p, &p->stage_v[sl], p->stage_cap);
        }
    // outer rows of a join: a static input's rows, or an SCC relation's delta -- at most its
    // log's capacity, and (hash-set outputs) at most the candidates of one iteration
    u64 max_outer = 0;
    for (const DevRule& r : d.rules)
        max_outer = std::max(max_outer, r.in.slot >= 0 ? std::max(p->dcand_cap, p->rels[d.rel_of_slot[r.in.slot]].cap)
                                                       : r.in.static_n);
    u64 bit_rows = 0;
    for (int sl = 0; sl < d.plan.n_rels; sl++)
        if (d.bit[sl].seen) bit_rows = std::max<u64>(bit_rows, d.bit[sl].n);
    u64 st_need = std::max<u64>({max_outer / kJRows + 2, p->dcand_cap / kSelTile + 2,
                                 (p->stage_cap / kSortTile + 2) * kRadix, bit_rows / kWarps + 2,
                                 max_outer / kPJChunk + 2, p->dcand_cap / kPSChunk + 2});
    if (st_need > p->status_cap) {
        dev_free(p, &p->status);
        p->status_cap = 0;
        dev_alloc(p, &p->status, st_need);
        p->status_cap = st_need;
    }
    // heavy-row slices: at most one per kHeavyPiece candidates plus one per heavy row
    const u64 heavy_cands = std::max(p->dcand_cap, p->heavy_cands);
    const u64 heavy_need = heavy_cands / kHeavyPiece + heavy_cands / kHeavyRow + 64;
    if (heavy_need > p->heavy_cap) {
        dev_free(p, &p->dheavy);
        p->heavy_cap = 0;
        dev_alloc(p, &p->dheavy, heavy_need);
        p->heavy_cap = heavy_need;
    }
    if (hist_cap > p->dhist_cap) {
        // layout: hist_cap (sum_delta, sum_full) pairs, then hist_cap iteration end times
        u64* nh;
        dev_alloc(p, &nh, 3 * hist_cap);
        if (p->dhist) {
            CK(cudaMemcpyAsync(nh, p->dhist, 2 * p->dhist_cap * 8, cudaMemcpyDeviceToDevice, p->stream));
            CK(cudaMemcpyAsync(nh + 2 * hist_cap, p->dhist + 2 * p->dhist_cap, p->dhist_cap * 8,
                               cudaMemcpyDeviceToDevice, p->stream));
        }
        dev_free(p, &p->dhist);
        p->dhist = nh;
        p->dhist_cap = hist_cap;
    }
    SccPlan& pl = d.plan;
    pl.cand_cap = p->dcand_cap;
    pl.stage_cap = ref ? p->stage_cap : ~0ull;
    pl.hist_cap = p->dhist_cap;
    p->hctl->time_cap = p->dhist_cap;
    for (int sl = 0; sl < pl.n_rels; sl++) {
        Relation& r = p->rels[d.rel_of_slot[sl]];
        pl.log_cap[sl] = r.cap;
        pl.seen_limit[sl] = d.bit[sl].seen ? ~0ull : r.seen ? (u64)(p->tune.seen_load_max * (double)r.seen_cap) : 0;
    }
}

// Instance matrix with room for `rows` iterations; keeps the rows already written.
void size_instance_rows(ra_program* p, u64 rows)
{
    if (!p->n_inst || rows <= p->inst_rows_cap) return;
    u64* nm;
    dev_alloc(p, &nm, rows * p->n_inst);
    CK(cudaMemsetAsync(nm, 0, rows * p->n_inst * 8, p->stream));
    if (p->dinst_new)
        CK(cudaMemcpyAsync(nm, p->dinst_new, p->inst_rows_cap * p->n_inst * 8, cudaMemcpyDeviceToDevice, p->stream));
    dev_free(p, &p->dinst_new);
    p->dinst_new = nm;
    p->inst_rows_cap = rows;
}

// The fused join of a rule: with the heavy-row list when its inner CSR has a
// row longer than kHeavyRow (a skewed key), else the plain tile loop.
decltype(&join_fused_kernel<false>) join_kernel(const DevRule& r)
{
    return r.longest > kHeavyRow ? join_fused_kernel<true> : join_fused_kernel<false>;
}

// per-launch events (diagnostic mode only; never inside a graph capture)
struct PhaseTimer {
    ra_program* p;
    int phase;
    bool on;
    PhaseTimer(ra_program* pp, int ph) : p(pp), phase(ph), on(pp->kernel_events)
    {
        if (!on) return;
        cudaEvent_t a = nullptr, b = nullptr;
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        cudaEventRecord(a, p->stream);
        p->phase_events.push_back({phase, {a, b}});
    }
    ~PhaseTimer()
    {
        if (on) cudaEventRecord(p->phase_events.back().second.second, p->stream);
    }
};

// The tail kernel's cluster: 16 CTAs where the GPU can place such a cluster,
// else 8 (portable), else none.  Asked once per program, outside any capture.
void tail_setup(ra_program* p)
{
    if (p->tail_ctas >= 0) return;
    p->tail_ctas = 0;
    if (cudaFuncSetAttribute(tail_cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTailSmem) !=
            cudaSuccess ||
        cudaFuncSetAttribute(tail_cluster_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    for (int nc : {kTailMaxCtas, 8}) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(nc);
        cfg.blockDim = dim3(kTailThreads);
        cfg.dynamicSmemBytes = kTailSmem;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = nc;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        int clusters = 0;
        if (cudaOccupancyMaxActiveClusters(&clusters, tail_cluster_kernel, &cfg) == cudaSuccess && clusters > 0) {
            p->tail_ctas = nc;
            return;
        }
        cudaGetLastError();
    }
}

// Does the iteration body of SCC d start with the tail kernel?  Join rules only
// (at most kTailMaxRules) into hash seen sets, written straight to the log in
// emission order, no instances.
bool tail_ok(ra_program* p, const DevScc& d)
{
    if (!p->use_tail || p->tail_ctas <= 0 || p->id_order != RA_IDS_EMISSION || p->n_inst || !d.plan.fixpoint ||
        d.plan.n_rules > kTailMaxRules)
        return false;
    for (const DevRule& r : d.rules)
        if (r.kind != kJoin || d.bit[r.out_slot].seen || r.in.slot < 0) return false;
    return true;
}

void launch_tail(ra_program* p, DevScc& d)
{
    TailArgs A{};
    A.ctl = p->ctl;
    A.plan = d.plan;
    A.rm = d.rm;
    A.n_rules = d.plan.n_rules;
    for (int q = 0; q < A.n_rules; q++) {
        const DevRule& r = d.rules[q];
        Relation& out = p->rels[d.rel_of_slot[r.out_slot]];
        A.rule[q] = TailRule{r.in, r.outer_shift, r.csr, r.inner, r.pj, out.seen, out.seen_cap, out.keys, out.ids};
    }
    A.bits = p->bits;
    A.cand = p->dcand;
    A.cand_cap = p->dcand_cap;
    A.loser = p->dloser;
    A.history = p->dhist;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(p->tail_ctas);
    cfg.blockDim = dim3(kTailThreads);
    cfg.dynamicSmemBytes = kTailSmem;
    cfg.stream = p->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = p->tail_ctas;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    CK(cudaLaunchKernelEx(&cfg, tail_cluster_kernel, A));
}

// launches of one iteration, in order; returns the number of kernels
int launch_iteration(ra_program* p, DevScc& d, cudaGraphConditionalHandle cond, int use_cond)
{
    const SccPlan& pl = d.plan;
    const int G = grid_blocks(p->tune.join_blocks_per_sm);
    const int GS = grid_blocks(p->tune.select_blocks_per_sm);
    const bool ref = p->id_order == RA_IDS_REFERENCE;
    int launches = 0;
    int slot = 0;
    // graph bodies of SCCs the tail kernel serves: the WHILE loop stops before an
    // iteration small enough for it (the tail kernel follows the loop in the graph)
    const bool tail = use_cond && tail_ok(p, d);
    for (int q = 0; q < pl.n_rules; q++) {
        const DevRule& r = d.rules[q];
        Relation& out = p->rels[d.rel_of_slot[r.out_slot]];
        PhaseTimer pt(p, 2);
        if (r.kind == kJoin)
            join_kernel(r)<<<G, kThreads, 0, p->stream>>>(p->ctl, q, r.in, r.outer_shift, r.csr, r.inner, r.pj,
                                                          p->bits, p->dcand, p->dcand_cap, out.seen, out.seen_cap,
                                                          p->dloser, p->status, p->status_cap, slot++,
                                                          d.bit[r.out_slot], JoinSlice{0, 0, 0, 0}, p->dheavy,
                                                          p->heavy_cap);
        else
            copy_claim_kernel<<<2 * G, kThreads, 0, p->stream>>>(p->ctl, pl, q, r.in, r.pj, p->bits, r.pred,
                                                                 p->dcand, p->dcand_cap, out.seen, out.seen_cap,
                                                                 p->dloser, d.bit[r.out_slot]);
        launches++;
    }
    // the selects: one per hash-set rule; one per bitmap relation (at its first rule)
    auto selects_rule = [&](int q) {
        const int sl = d.rules[q].out_slot;
        return !d.bit[sl].seen || d.rm.rules_in[sl][0] == q;
    };
    int last_select = -1;
    for (int q = 0; q < pl.n_rules; q++)
        if (selects_rule(q)) last_select = q;
    for (int q = 0; q < pl.n_rules; q++) {
        if (!selects_rule(q)) continue;
        const DevRule& r = d.rules[q];
        Relation& out = p->rels[d.rel_of_slot[r.out_slot]];
        PhaseTimer pt(p, 3);
        if (d.bit[r.out_slot].seen) {
            BitSelectArgs b{};
            b.rel = r.out_slot;
            b.first_rule = q;
            b.last = q == last_select ? 1 : 0;
            b.dst_keys = out.keys;
            b.dst_ids = out.ids;
            b.bs = d.bit[r.out_slot];
            b.bits = p->bits;
            if (p->n_inst) {
                b.inst_new = p->dinst_new;
                b.n_inst = p->n_inst;
                b.inst_iter_cap = p->inst_rows_cap;
            }
            // twice the select's CTAs per SM: its rows are independent warps (measured on
            // sg-tree15: 22.66 -> 22.09 ms per step; the hash-set select is faster at the tuned count)
            bitmap_select_kernel<<<grid_blocks(std::min<uint32_t>(16, 2 * p->tune.select_blocks_per_sm)), kThreads, 0,
                                   p->stream>>>(p->ctl, pl, d.rm, b, p->status, p->status_cap,
                                                                 slot++, p->dhist, cond, use_cond);
            launches++;
            continue;
        }
        SelectArgs a{};
        a.rule = q;
        a.last = (!ref && q == last_select) ? 1 : 0;
        a.to_log = ref ? 0 : 1;
        a.dst_keys = ref ? p->stage_k[r.out_slot] : out.keys;
        a.dst_ids = ref ? p->stage_v[r.out_slot] : out.ids;
        a.passes = ref ? d.passes[r.out_slot] : 0;
        a.stage_cap = p->stage_cap;
        if (tail) {
            a.tail_on = 1;
            a.tail_nslots = pl.n_rules;
            for (int t = 0; t < pl.n_rules; t++) a.tail_slot[t] = d.rules[t].in.slot;
            a.tail_rows = (u64)p->tail_ctas * kTailRowsGo;
        }
        if (p->n_inst) {
            a.inst_base = p->dinst_base;
            a.n_inst = p->n_inst;
            a.inst_shift = (int)(out.arity - 1) * p->bits;
            a.inst_new = p->dinst_new;
            a.inst_iter_cap = p->inst_rows_cap;
        }
        select_kernel<<<GS, kThreads, 0, p->stream>>>(p->ctl, pl, d.rm, a, p->dcand, p->dloser, p->status, slot++,
                                                     p->dhist, cond, use_cond);
        launches++;
    }
    if (ref) {
        for (int sl = 0; sl < pl.n_rels; sl++) {
            if (!d.rm.n_rules_in[sl]) continue;
            Relation& r = p->rels[d.rel_of_slot[sl]];
            const int P = d.passes[sl];
            for (int ps = 0; ps < P; ps++) {
                SortPassArgs a{};
                a.rel = sl;
                a.pass = ps;
                a.shift = ps * kRadixBits;
                a.src_k = ps == 0 ? p->stage_k[sl] : p->sort_k[(ps - 1) & 1];
                a.src_v = ps == 0 ? p->stage_v[sl] : p->sort_v[(ps - 1) & 1];
                a.dst_log = (ps == P - 1) ? 1 : 0;
                a.dst_k = a.dst_log ? r.keys : p->sort_k[ps & 1];
                a.dst_v = a.dst_log ? r.ids : p->sort_v[ps & 1];
                a.log_cap = r.cap;
                a.n_rules_in = d.rm.n_rules_in[sl];
                for (int q = 0; q < a.n_rules_in; q++) a.rules_in[q] = d.rm.rules_in[sl][q];
                PhaseTimer pt(p, 4);
                sort_pass_kernel<<<GS, kThreads, 0, p->stream>>>(p->ctl, a, p->status, slot++);
                launches++;
            }
        }
        PhaseTimer pt(p, 5);
        iter_end_kernel<<<64, kThreads, 0, p->stream>>>(p->ctl, pl, d.rm, p->dhist, cond, use_cond);
        launches++;
    }
    ck(p, cudaGetLastError(), "iteration launch");
    return launches;
}

// Every value an iteration's launches capture (pointers, capacities, plans).
std::vector<unsigned char> graph_signature(ra_program* p, const DevScc& d)
{
    std::vector<unsigned char> sig;
    auto put = [&](const void* a, size_t n) {
        const unsigned char* b = (const unsigned char*)a;
        sig.insert(sig.end(), b, b + n);
    };
    put(&d.plan, sizeof d.plan);
    put(&d.rm, sizeof d.rm);
    put(d.passes, sizeof d.passes);
    for (const DevRule& r : d.rules) put(&r, sizeof r);
    for (int sl = 0; sl < d.plan.n_rels; sl++) {
        const Relation& r = p->rels[d.rel_of_slot[sl]];
        const void* ptrs[4] = {r.keys, r.ids, r.seen, nullptr};
        put(ptrs, sizeof ptrs);
        put(&r.seen_cap, sizeof r.seen_cap);
        put(&r.cap, sizeof r.cap);
    }
    const void* scratch[9] = {p->ctl, p->dcand, p->status, p->dhist, p->sort_k[0], p->sort_k[1], p->sort_v[0],
                              p->sort_v[1], p->dloser};
    put(scratch, sizeof scratch);
    put(p->stage_k, sizeof p->stage_k);
    put(p->stage_v, sizeof p->stage_v);
    put(&p->bits, sizeof p->bits);
    put(&p->stream, sizeof p->stream);
    put(&p->id_order, sizeof p->id_order);
    put(&p->stage_cap, sizeof p->stage_cap);
    put(&p->dcand_cap, sizeof p->dcand_cap);
    const void* inst[2] = {p->dinst_base, p->dinst_new};
    put(inst, sizeof inst);
    put(&p->n_inst, sizeof p->n_inst);
    put(&p->tune, sizeof p->tune);
    put(d.bit, sizeof d.bit);
    put(&p->inst_rows_cap, sizeof p->inst_rows_cap);
    put(&p->status_cap, sizeof p->status_cap);
    return sig;
}

// ---------------------------------------------------------------------------
// checkpoint dumps and restart loading, in the reference's layout
// ---------------------------------------------------------------------------

// One region of a relation's log as a dump file: rows (arity + 1 u64) in trie
// order, plus its size metadata (relation::parallel_IO,
// src/relation/balanced_hash_relation.cpp:109-430): with per-rank files the rows
// file is written when not empty and the size file always ("<bytes/24>\n3");
// with shared files both only when not empty ("<rows>\n<arity+1>").
// One relation version's rows (arity + 1 u64, trie order) into a dump file and its
// .size, in the layout of relation::parallel_IO (balanced_hash_relation.cpp:109-430).
void write_rows_file(ra_program* p, const Relation& r, const std::vector<u64>& host, u64 n, const std::string& path)
{
    const u64 bytes = host.size() * 8;
    const std::string file = p->cp_separate ? path + "_0" : path;
    if (n) {
        FILE* f = fopen(file.c_str(), "wb");
        if (!f || fwrite(host.data(), 1, bytes, f) != bytes) {
            if (f) fclose(f);
            fail(p, RA_E_IO, "cannot write %s", file.c_str());
        }
        fclose(f);
    }
    if (p->cp_separate || n) {
        FILE* f = fopen((file + ".size").c_str(), "w");
        if (!f) fail(p, RA_E_IO, "cannot write %s.size", file.c_str());
        if (p->cp_separate) fprintf(f, "%d\n3", (int)(bytes / 24));
        else fprintf(f, "%d\n%d", (int)n, (int)r.arity + 1);
        fclose(f);
    }
}

void dump_region(ra_program* p, Relation& r, const u64* keys, const u64* ids, u64 n, const std::string& path)
{
    std::vector<u64> host(n * (r.arity + 1));
    if (n) {
        u64 *tk, *tv, *rows;
        dev_alloc(p, &tk, n);
        dev_alloc(p, &tv, n);
        dev_alloc(p, &rows, n * (r.arity + 1));
        CK(cudaMemcpyAsync(tk, keys, n * 8, cudaMemcpyDeviceToDevice, p->stream));
        CK(cudaMemcpyAsync(tv, ids, n * 8, cudaMemcpyDeviceToDevice, p->stream));
        sort_rows(p, r, tk, tv, n, r.keys_unique);
        rows_unpack<<<grid_for(n), kThreads, 0, p->stream>>>(tk, tv, n, (int)r.arity, p->bits, rows);
        LAUNCHED();
        CK(cudaMemcpyAsync(host.data(), rows, host.size() * 8, cudaMemcpyDeviceToHost, p->stream));
        CK(cudaStreamSynchronize(p->stream));
        dev_free(p, &tk);
        dev_free(p, &tv);
        dev_free(p, &rows);
    }
    write_rows_file(p, r, host, n, path);
}

// The same from a wide relation version (its rows are already in trie order).
void dump_wide_region(ra_program* p, Relation& r, const u64* rows, u64 n, const std::string& path)
{
    std::vector<u64> host(n * (r.arity + 1));
    if (n) {
        CK(cudaMemcpyAsync(host.data(), rows, host.size() * 8, cudaMemcpyDeviceToHost, p->stream));
        CK(cudaStreamSynchronize(p->stream));
    }
    write_rows_file(p, r, host, n, path);
}

// LIE::create_checkpoint_dump + write_checkpoint_dump (src/lie/lie.cpp:154-193):
// directory <output>/checkpoint-<scc>-<loop counter>, the executed SCC ids,
// every relation's full and delta.  `counts` gives (full, delta) per relation.
void write_checkpoint(ra_program* p, int scc_id, const std::vector<std::pair<u64, u64>>& counts)
{
    const std::string dir = p->cp_dir + "/checkpoint-" + std::to_string(scc_id) + "-" + std::to_string(p->loop_counter);
    mkdir(dir.c_str(), S_IRWXU | S_IRWXG | S_IROTH | S_IXOTH);
    FILE* f = fopen((dir + "/scc_metadata").c_str(), "w");
    if (!f) fail(p, RA_E_IO, "cannot write %s/scc_metadata", dir.c_str());
    for (int id : p->executed_ids) fprintf(f, "%d\n", id);
    fclose(f);
    for (size_t i = 0; i < p->rels.size(); i++) {
        Relation& r = p->rels[i];
        const u64 fn = counts[i].first, dn = counts[i].second;
        if (p->wide) {
            dump_wide_region(p, r, r.wfull, fn, dir + "/" + r.name + "_full");
            dump_wide_region(p, r, r.wdelta, dn, dir + "/" + r.name + "_delta");
            continue;
        }
        dump_region(p, r, r.keys, r.ids, fn, dir + "/" + r.name + "_full");
        dump_region(p, r, r.keys + fn, r.ids + fn, dn, dir + "/" + r.name + "_delta");
    }
}

// After each completed batch of SCC s (one execute_in_batches call of the reference):
// record completion and write the dump every cp_every batches.
void checkpoint_batch(ra_program* p, const Scc& s, bool finished, const std::vector<std::pair<u64, u64>>& counts)
{
    if (finished) p->executed_ids.push_back(s.id);
    if (p->cp_every && p->loop_counter % (int)p->cp_every == 0) write_checkpoint(p, s.id, counts);
    p->loop_counter++;
}

std::vector<std::pair<u64, u64>> host_counts(ra_program* p)
{
    std::vector<std::pair<u64, u64>> c;
    for (const Relation& r : p->rels) c.push_back({r.full_n, r.delta_n});
    return c;
}

// Restart: a relation's delta from <dir>/<name>_delta (LIE::execute, lie.cpp:300-330),
// appended after its full version; no file, no delta.
// The rows of a relation's delta dump (none when the file does not exist).
bool read_restart_rows(ra_program* p, const Relation& r, std::vector<u64>& host, std::string& path)
{
    path = p->rs_dir + "/" + r.name + "_delta";
    if (p->rs_separate) path += "_0";
    if (access(path.c_str(), F_OK) != 0) return false;
    FILE* f = fopen(path.c_str(), "rb");
    if (!f) fail(p, RA_E_IO, "cannot open %s", path.c_str());
    fseek(f, 0, SEEK_END);
    const long bytes = ftell(f);
    fseek(f, 0, SEEK_SET);
    const u64 w = (r.arity + 1) * 8, n = (u64)bytes / w;
    host.assign(n * (r.arity + 1), 0);
    if (n && fread(host.data(), 1, n * w, f) != n * w) {
        fclose(f);
        fail(p, RA_E_IO, "short read of %s", path.c_str());
    }
    fclose(f);
    return true;
}

void load_restart_delta(ra_program* p, Relation& r)
{
    std::vector<u64> host;
    std::string path;
    if (!read_restart_rows(p, r, host, path)) return;
    const u64 w = (r.arity + 1) * 8, n = host.size() / (r.arity + 1);
    for (u64 i = 0; i < n; i++)
        for (u32 c = 0; c < r.arity; c++)
            if (host[i * (r.arity + 1) + c] >> p->bits)
                fail(p, RA_E_UNSUPPORTED, "%s: a value wider than the %d-bit columns of the loaded relations",
                     path.c_str(), p->bits);
    r.full_n += r.delta_n;   // any delta present becomes full, as the reference's trie insert would keep it
    r.delta_n = 0;
    if (!n) return;
    ensure_log(p, r, r.full_n + n);
    u64* raw;
    dev_alloc(p, &raw, n * (r.arity + 1));
    CK(cudaMemcpyAsync(raw, host.data(), n * w, cudaMemcpyHostToDevice, p->stream));
    rows_pack<<<grid_for(n), kThreads, 0, p->stream>>>(raw, n, (int)r.arity, p->bits, r.keys + r.full_n,
                                                       r.ids + r.full_n);
    LAUNCHED();
    CK(cudaStreamSynchronize(p->stream));
    dev_free(p, &raw);
    r.delta_n = n;
    r.delta_sorted = false;
    r.full_sorted = false;
    r.full_version = fresh_stamp();
    r.delta_version = fresh_stamp();
}

// Words of the bit matrices a bitmap relation needs: one rows x rows matrix, or with
// instances one n_i x n_i matrix per instance (0 when an instance is too wide).
u64 bitmap_words(ra_program* p)
{
    const u64 rows = p->max_value + 1;
    if (!p->n_inst) return rows <= kDenseMaxN ? rows * ((rows + 31) / 32) : 0;
    u64 total = 0;
    for (u32 i = 0; i < p->n_inst; i++) {
        const u64 b = p->inst_base_h[i];
        if (b >= rows) break;
        const u64 e = std::min<u64>(p->inst_base_h[i + 1], rows), n = e - b;
        if (n > kDenseMaxN) return 0;
        total += n * ((n + 31) / 32);
    }
    return total;
}

// Does output relation r of a device-driven SCC take a bitmap seen set?  Binary,
// values (per instance) below 65,536, default id order, bit matrices within the
// tuned budget of the dense representations, and a fixpoint SCC: a bitmap costs
// clearing and scanning rows x rows bits, paid back only by the many iterations and
// tuples of a recursive SCC (one pass of a copy or join costs its candidates only).
bool bitmap_ok(ra_program* p, const Scc& s, const Relation& r)
{
    if (!s.fixpoint || r.arity != 2 || p->id_order != RA_IDS_EMISSION || p->tune.dense_max_bytes <= 0) return false;
    const u64 words = bitmap_words(p);
    return words && 8.0 * (double)words + (double)(p->max_value + 1) <= p->tune.dense_max_bytes;
}

// With instances: row v's word offset, base value, words per row and instance, for
// every value of the union (built on the device once per instance layout; the host
// computes only each instance's first word).
void bitmap_tables(ra_program* p)
{
    const u64 rows = p->max_value + 1;
    if (p->bmt_word && p->bmt_rows == rows && p->bmt_bases == p->inst_base_h) return;
    std::vector<u64> first(p->n_inst, 0);
    u64 off = 0;
    for (u32 i = 0; i < p->n_inst; i++) {
        first[i] = off;
        const u64 b = p->inst_base_h[i];
        if (b >= rows) continue;
        const u64 n = std::min<u64>(p->inst_base_h[i + 1], rows) - b;
        off += n * ((n + 31) / 32);
    }
    dev_free(p, &p->bmt_word);
    dev_free(p, &p->bmt_base);
    dev_free(p, &p->bmt_words);
    dev_free(p, &p->bmt_inst);
    p->bmt_rows = 0;
    p->bmt_bases.clear();
    dev_alloc(p, &p->bmt_word, rows);
    dev_alloc(p, &p->bmt_base, rows);
    dev_alloc(p, &p->bmt_words, rows);
    dev_alloc(p, &p->bmt_inst, rows);
    u64* dfirst;
    dev_alloc(p, &dfirst, p->n_inst);
    CK(cudaMemcpyAsync(dfirst, first.data(), p->n_inst * 8, cudaMemcpyHostToDevice, p->stream));
    bitmap_tables_kernel<<<grid_for(rows), kThreads, 0, p->stream>>>(p->dinst_base, p->n_inst, dfirst, rows,
                                                                     p->bmt_word, p->bmt_base, p->bmt_words,
                                                                     p->bmt_inst);
    LAUNCHED();
    dev_free(p, &dfirst);
    CK(cudaStreamSynchronize(p->stream));
    p->bmt_rows = rows;
    p->bmt_total = off;
    p->bmt_bases = p->inst_base_h;
}

// r's bitmap seen set holding its stored tuples, fresh bits and dirty rows cleared.
BitSeen prepare_bitmap(ra_program* p, Relation& r)
{
    const u64 rows = p->max_value + 1;
    if (p->n_inst) bitmap_tables(p);
    const u64 words = p->n_inst ? p->bmt_total : rows * ((rows + 31) / 32);
    if (r.bm_words < words) {
        dev_free(p, &r.bm_seen);
        dev_free(p, &r.bm_fresh);
        r.bm_words = 0;
        dev_alloc(p, &r.bm_seen, words);
        dev_alloc(p, &r.bm_fresh, words);
        r.bm_words = words;
    }
    if (r.bm_rows < rows) {
        dev_free(p, &r.bm_dirty);
        r.bm_rows = 0;
        dev_alloc(p, &r.bm_dirty, rows);
        r.bm_rows = rows;
    }
    CK(cudaMemsetAsync(r.bm_seen, 0, words * 4, p->stream));
    CK(cudaMemsetAsync(r.bm_fresh, 0, words * 4, p->stream));
    CK(cudaMemsetAsync(r.bm_dirty, 0, rows, p->stream));
    BitSeen b{};
    b.seen = r.bm_seen;
    b.fresh = r.bm_fresh;
    b.dirty = r.bm_dirty;
    b.words = (u32)((rows + 31) / 32);
    b.n = (u32)rows;
    if (p->n_inst) {
        b.row_word = p->bmt_word;
        b.row_base = p->bmt_base;
        b.row_words = p->bmt_words;
        b.row_inst = p->bmt_inst;
    }
    const u64 n = r.full_n + r.delta_n;
    if (n) {
        CK(cudaMemsetAsync(p->derr, 0, 4, p->stream));
        bitmap_build_kernel<<<grid_for(n), kThreads, 0, p->stream>>>(b, r.keys, n, p->bits, p->derr);
        LAUNCHED();
        if (p->n_inst && (read_scalar(p, (const u64*)p->derr) & 0xffffffffull))
            fail(p, RA_E_BADARG, "relation %s: a tuple's columns lie in different instances", r.name.c_str());
    }
    return b;
}

// A completed iteration of run_scc_device that closed a batch (a new history
// entry): counts of the SCC's relations from the control block.
void checkpoint_device_batch(ra_program* p, const Scc& s, const DevScc& d, u64& hist_seen)
{
    const IterCtl& h = *p->hctl;
    if (h.hist_n <= hist_seen) return;
    hist_seen = h.hist_n;
    auto counts = host_counts(p);
    for (int sl = 0; sl < d.plan.n_rels; sl++) counts[d.rel_of_slot[sl]] = {h.full_n[sl], h.delta_n[sl]};
    checkpoint_batch(p, s, h.done != 0, counts);
}

void drop_graph(Scc& s)
{
    if (s.exec) cudaGraphExecDestroy(s.exec);
    if (s.graph) cudaGraphDestroy(s.graph);
    s.exec = nullptr;
    s.graph = nullptr;
    s.graph_sig.clear();
}

void ctl_download(ra_program* p)
{
    CK(cudaMemcpyAsync(p->hctl, p->ctl, ctl_header_bytes(), cudaMemcpyDeviceToHost, p->stream));
    CK(cudaStreamSynchronize(p->stream));
}

// Can the running iteration of SCC s run in slices of outer rows?  Join rules
// only, into hash seen sets, with new tuples written straight to the log.
bool sliceable(ra_program* p, const DevScc& d)
{
    if (p->id_order != RA_IDS_EMISSION || p->n_inst) return false;
    for (const DevRule& r : d.rules)
        if (r.kind != kJoin || d.bit[r.out_slot].seen) return false;
    return true;
}

// One iteration of SCC s in slices of outer rows, when its candidates exceed the
// candidate buffer that the program's memory cap leaves room for (the
// reference bounds a join call's output in the same spirit and resumes from an
// offset, src/RAM/RA_tasks.cpp:312 and src/RA/parallel_join.cpp:196-201).  Per
// rule, per slice of whole tiles: the join claims with the slice's stream
// positions (so first occurrences and losers are the unsliced ones: a later
// slice never displaces an earlier one's tuple) and its select appends the
// slice's winners after the previous slices'.  Then the iteration end, as the
// loop's.  The log, ids included, and the history are those of an unsliced
// iteration.  Expects the control block downloaded in hctl.
void run_sliced_iteration(ra_program* p, Scc& s, DevScc& d)
{
    IterCtl& h = *p->hctl;
    // a sliced iteration appends as it goes and cannot be replayed: room for its history entry first
    if (h.hist_n + 1 >= p->dhist_cap) {
        dev_size_buffers(p, d, p->dcand_cap, p->stage_cap, 2 * p->dhist_cap);
        CK(cudaMemcpyAsync(&p->ctl->time_cap, &p->hctl->time_cap, 8, cudaMemcpyHostToDevice, p->stream));
    }
    const SccPlan& pl = d.plan;
    const int G = grid_blocks(p->tune.join_blocks_per_sm);
    const int GS = grid_blocks(p->tune.select_blocks_per_sm);
    std::vector<u64> appended(pl.n_rels, 0), id_app(kMaxTagSlots, 0), cand_tot(pl.n_rules, 0), win_tot(pl.n_rules, 0);
    u64 pos = 0;   // stream position of the next rule's first candidate
    u64* tile_cnt = nullptr;
    struct Free {
        ra_program* p;
        u64** q;
        ~Free() { dev_free(p, q); }
    } free_tiles{p, &tile_cnt};
    for (int q = 0; q < pl.n_rules; q++) {
        const DevRule& r = d.rules[q];
        Relation& out = p->rels[d.rel_of_slot[r.out_slot]];
        const u64 n = r.in.slot >= 0 ? h.delta_n[r.in.slot] : r.in.static_n;
        const u64 ntiles = (n + kJRows - 1) / kJRows;
        std::vector<u64> cnt(ntiles);
        if (ntiles) {
            dev_free(p, &tile_cnt);
            dev_alloc(p, &tile_cnt, ntiles);
            join_tile_counts_kernel<<<(int)std::min<u64>(ntiles, (u64)kMaxGrid), kThreads, 0, p->stream>>>(
                p->ctl, r.in, r.outer_shift, r.csr, tile_cnt);
            LAUNCHED();
            CK(cudaMemcpyAsync(cnt.data(), tile_cnt, ntiles * 8, cudaMemcpyDeviceToHost, p->stream));
            CK(cudaStreamSynchronize(p->stream));
        }
        u64 rule_pos = 0;
        for (u64 t = 0; t < ntiles || (t == 0 && ntiles == 0);) {
            u64 t1 = t, c = 0;
            while (t1 < ntiles && c + cnt[t1] <= p->dcand_cap) c += cnt[t1++];
            if (t1 == t && ntiles)
                fail(p, RA_E_OOM, "SCC %d: %llu outer rows have %llu candidates, more than the %llu the memory cap "
                                  "leaves room for", s.id, (unsigned long long)kJRows, (unsigned long long)cnt[t],
                     (unsigned long long)p->dcand_cap);
            const u64 lo = t * kJRows, rows = std::min(n, t1 * kJRows) - lo;
            // a fresh slice: no marks, no look-back statuses, tile counters at zero
            CK(cudaMemsetAsync(p->dloser, 0, std::max<u64>(c, 1) * 4, p->stream));
            CK(cudaMemsetAsync(p->status, 0, p->status_cap * 8, p->stream));
            CK(cudaMemsetAsync(p->ctl->tile_ctr, 0, sizeof(p->ctl->tile_ctr), p->stream));
            join_kernel(r)<<<G, kThreads, 0, p->stream>>>(p->ctl, q, r.in, r.outer_shift, r.csr, r.inner, r.pj,
                                                          p->bits, p->dcand, p->dcand_cap, out.seen, out.seen_cap,
                                                          p->dloser, p->status, p->status_cap, 0, d.bit[r.out_slot],
                                                          JoinSlice{lo, rows, pos + rule_pos, 1}, p->dheavy,
                                                          p->heavy_cap);
            LAUNCHED();
            SelectArgs a{};
            a.rule = q;
            a.last = 0;
            a.to_log = 1;
            a.dst_keys = out.keys;
            a.dst_ids = out.ids;
            a.sliced = 1;
            a.appended = appended[r.out_slot];
            a.id_appended = id_app[pl.rule_tag[q]];
            select_kernel<<<GS, kThreads, 0, p->stream>>>(p->ctl, pl, d.rm, a, p->dcand, p->dloser, p->status, 1,
                                                         p->dhist, 0, 0);
            LAUNCHED();
            ctl_download(p);
            if (h.flags & kFlagTimeout) fail(p, RA_E_TIMEOUT, "SCC %d: a device-side look-back wait gave up", s.id);
            if (h.flags)
                fail(p, RA_E_OOM, "SCC %d: a sliced iteration ran out of room (flags %u) under the memory cap", s.id,
                     h.flags);
            const u64 w = h.win_n[q];
            appended[r.out_slot] += w;
            id_app[pl.rule_tag[q]] += w;
            cand_tot[q] += h.cand_n[q];
            win_tot[q] += w;
            rule_pos += c;
            p->stats.sliced_passes++;
            if (ntiles == 0) break;
            t = t1;
        }
        pos += cand_tot[q];
    }
    // the iteration end with the iteration's totals, as the loop's last select runs it
    for (int q = 0; q < pl.n_rules; q++) {
        h.cand_n[q] = cand_tot[q];
        h.win_n[q] = win_tot[q];
    }
    for (int i = 0; i < 2 * kBankWords; i++) h.tile_ctr[i] = 0;
    CK(cudaMemcpyAsync(p->ctl, p->hctl, ctl_header_bytes(), cudaMemcpyHostToDevice, p->stream));
    CK(cudaMemsetAsync(p->status, 0, p->status_cap * 8, p->stream));
    iter_end_kernel<<<64, kThreads, 0, p->stream>>>(p->ctl, pl, d.rm, p->dhist, 0, 0);
    LAUNCHED();
    ctl_download(p);
    p->stats.sliced_iterations++;
}

// Kernel parameters of the persistent SCC kernel (ra_persist.cuh) for the plan's
// current buffers and capacities.
PersistArgs persist_args(ra_program* p, const DevScc& d)
{
    PersistArgs A{};
    A.ctl = p->ctl;
    A.plan = d.plan;
    A.rm = d.rm;
    A.bits = p->bits;
    A.cand = p->dcand;
    A.loser = p->dloser;
    A.status = p->status;
    A.status_cap = p->status_cap;
    A.heavy = p->dheavy;
    A.heavy_cap = p->heavy_cap;
    A.history = p->dhist;
    for (int q = 0; q < d.plan.n_rules; q++) {
        const DevRule& r = d.rules[q];
        Relation& out = p->rels[d.rel_of_slot[r.out_slot]];
        PRule& P = A.rule[q];
        P.kind = r.kind == kJoin ? kJoinRule : r.kind;
        P.out_slot = r.out_slot;
        P.in = r.in;
        P.pj = r.pj;
        P.csr = r.csr;
        P.inner = r.inner;
        P.outer_shift = r.outer_shift;
        P.pred = r.pred;
        P.seen = out.seen;
        P.seen_cap = out.seen_cap;
        P.dst_keys = out.keys;
        P.dst_ids = out.ids;
        P.inst_shift = (int)(out.arity - 1) * p->bits;
    }
    if (p->n_inst) {
        A.inst_base = p->dinst_base;
        A.n_inst = p->n_inst;
        A.inst_new = p->dinst_new;
        A.inst_iter_cap = p->inst_rows_cap;
    }
    return A;
}

// One cooperative launch of the persistent SCC kernel: every block resident at
// once (its grid barriers wait on all of them), as many as the device holds.
void launch_persistent(ra_program* p, const DevScc& d)
{
    static int occ = 0, sms = 0;
    if (!occ) {
        int dev = 0;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, scc_persistent_kernel, kThreads, 0));
        if (occ < 1) fail(p, RA_E_CUDA, "the persistent SCC kernel does not fit on an SM");
    }
    PersistArgs A = persist_args(p, d);
    void* args[] = {&A};
    CK(cudaLaunchCooperativeKernel((const void*)scc_persistent_kernel, dim3(sms * occ), dim3(kThreads), args, 0,
                                   p->stream));
    LAUNCHED();
}

void run_scc_device(ra_program* p, Scc& s, DevScc& d)
{
    const SccPlan& pl = d.plan;
    // control block: counters of the SCC's relations
    IterCtl& h = *p->hctl;
    std::memset(&h, 0, ctl_header_bytes());
    std::vector<u64> full0(pl.n_rels), delta0(pl.n_rels);
    std::vector<bool> dsorted0(pl.n_rels);
    for (int sl = 0; sl < pl.n_rels; sl++) {
        Relation& r = p->rels[d.rel_of_slot[sl]];
        h.full_n[sl] = r.full_n;
        h.delta_n[sl] = r.delta_n;
        full0[sl] = r.full_n;
        delta0[sl] = r.delta_n;
        dsorted0[sl] = r.delta_sorted;
    }
    for (size_t t = 0; t < d.tags.size(); t++) h.intern[t] = intern_counter(p, d.tags[t]);
    h.epoch = p->epoch + 1;
    // seen sets of the output relations (sized with room for growth)
    for (int sl = 0; sl < pl.n_rels; sl++) {
        if (!d.rm.n_rules_in[sl]) continue;
        Relation& r = p->rels[d.rel_of_slot[sl]];
        u64 base = r.full_n + r.delta_n;
        if (bitmap_ok(p, s, r)) {
            d.bit[sl] = prepare_bitmap(p, r);
            h.seen_n[sl] = base;
            p->stats.bitmap_relations++;
        } else {
            d.bit[sl] = BitSeen{};
            build_seen(p, r, std::max<u64>(2 * base, 1u << 20));
            h.seen_n[sl] = r.seen_n;
        }
        ensure_log(p, r, base + std::max<u64>(base, 1u << 20));
    }
    refresh_refs(p, d);
    CK(cudaMemcpyAsync(p->ctl, p->hctl, ctl_header_bytes(), cudaMemcpyHostToDevice, p->stream));
    CK(cudaMemsetAsync(&p->ctl->sort_hist[0][0][0], 0, sizeof(p->ctl->sort_hist), p->stream));
    u64 outer0 = 0;
    for (const DevRule& r : d.rules) outer0 = std::max(outer0, r.in.slot >= 0 ? p->rels[d.rel_of_slot[r.in.slot]].delta_n : r.in.static_n);
    for (u64 want = std::max<u64>({p->dcand_cap, 1u << 22, 2 * outer0});; want /= 2) {
        try {
            dev_size_buffers(p, d, want, std::max<u64>({p->stage_cap, 1u << 22, 2 * outer0}),
                             std::max<u64>(p->dhist_cap, 1u << 12));
            break;
        } catch (ra_error& e) {
            // under a memory cap a smaller candidate buffer will do: iterations that outgrow
            // it run in slices of outer rows (run_sliced_iteration)
            if (e.status != RA_E_OOM || !sliceable(p, d) || want <= (1u << 12)) throw;
            p->err.clear();
        }
    }
    CK(cudaMemsetAsync(p->status, 0, p->status_cap * 8, p->stream));
    CK(cudaMemcpyAsync(&p->ctl->time_cap, &p->hctl->time_cap, 8, cudaMemcpyHostToDevice, p->stream));
    if (p->n_inst) {
        size_instance_rows(p, 256);
        CK(cudaMemsetAsync(p->dinst_new, 0, p->inst_rows_cap * p->n_inst * 8, p->stream));
    }
    scc_start_kernel<<<1, 1, 0, p->stream>>>(p->ctl);
    LAUNCHED();

    int body_kernels = 0;
    u64 tail_launches = 0;   // graph launches whose graph ends with the tail kernel
    bool any_bitmap = false;
    for (int sl = 0; sl < pl.n_rels; sl++) any_bitmap = any_bitmap || d.bit[sl].seen;
    // the whole fixed point as one cooperative launch: default id order, hash seen sets
    const bool persist_mode = p->use_persist && p->use_graphs && !p->kernel_events && !p->cp_every &&
                              p->id_order == RA_IDS_EMISSION && !any_bitmap && pl.n_rules > 0;
    const bool graph_mode = !persist_mode && p->use_graphs && !p->kernel_events && s.fixpoint && !p->cp_every;
    u64 hist_seen = 0;   // history entries (completed batches) already checkpointed
    for (;;) {
        if (persist_mode) {
            h.bar_count = 0;
            CK(cudaMemcpyAsync(&p->ctl->bar_count, &h.bar_count, 4, cudaMemcpyHostToDevice, p->stream));
            launch_persistent(p, d);
            p->stats.persistent_launches++;
            ctl_download(p);
        } else if (graph_mode) {
            std::vector<unsigned char> sig = graph_signature(p, d);
            if (s.exec && sig != s.graph_sig) drop_graph(s);
            if (!s.exec) {
                auto gt0 = std::chrono::steady_clock::now();
                cudaGraph_t graph = nullptr;
                cudaGraphExec_t exec = nullptr;
                CK(cudaGraphCreate(&graph, 0));
                cudaGraphConditionalHandle cond;
                tail_setup(p);
                CK(cudaGraphConditionalHandleCreate(&cond, graph, 1, cudaGraphCondAssignDefault));
                cudaGraphNodeParams cp = {};
                cp.type = cudaGraphNodeTypeConditional;
                cp.conditional.handle = cond;
                cp.conditional.type = cudaGraphCondTypeWhile;
                cp.conditional.size = 1;
                cudaGraphNode_t node;
                CK(cudaGraphAddNode(&node, graph, nullptr, 0, &cp));
                cudaGraph_t body = cp.conditional.phGraph_out[0];
                CK(cudaStreamBeginCaptureToGraph(p->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
                const int body_kernels_captured = launch_iteration(p, d, cond, 1);
                CK(cudaStreamEndCapture(p->stream, &body));
                if (tail_ok(p, d)) {
                    // the tail kernel after the loop: the small iterations that end it
                    CK(cudaStreamBeginCaptureToGraph(p->stream, graph, &node, nullptr, 1,
                                                     cudaStreamCaptureModeRelaxed));
                    launch_tail(p, d);
                    CK(cudaStreamEndCapture(p->stream, &graph));
                }
                CK(cudaGraphInstantiate(&exec, graph, 0));
                s.graph = graph;
                s.exec = exec;
                s.graph_sig = sig;
                body_kernels = 0;
                p->stats.graph_builds++;
                p->stats.graph_build_ms +=
                    std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - gt0).count();
                s.graph_kernels = body_kernels_captured;
            }
            body_kernels = s.graph_kernels;
            if (tail_ok(p, d)) tail_launches++;
            CK(cudaGraphLaunch(s.exec, p->stream));
            ctl_download(p);
        } else {
            // one iteration per host round trip (non-fixpoint SCCs, or graphs disabled)
            body_kernels = launch_iteration(p, d, 0, 0);
            ctl_download(p);
        }
        if (h.flags & kFlagTimeout) fail(p, RA_E_TIMEOUT, "SCC %d: a device-side look-back wait gave up", s.id);
        if (h.flags & kFlagRange) fail(p, RA_E_BADARG, "SCC %d: a derived tuple's columns lie in different instances", s.id);
        if (h.flags & kFlagStatus)
            fail(p, RA_E_UNSUPPORTED, "SCC %d: a launch has more tiles than its look-back status array holds", s.id);
        if (h.flags & (kFlagOverflow | kFlagProbe | kFlagGrow)) {
            // Overflow / probe: the iteration stopped before select wrote anything and its
            // claims are idempotent, so grow and replay it.  Grow: the iteration finished;
            // make room in the seen sets before the next one.
            const bool replay = (h.flags & (kFlagOverflow | kFlagProbe)) != 0;
            p->stats.regrows++;
            u64 total = 0;
            u64 incoming[kMaxSccRels] = {0};
            for (int q = 0; q < pl.n_rules; q++) {
                if (!d.bit[pl.rule_out[q]].seen) total += h.cand_n[q];   // bitmap rules write no candidates
                incoming[pl.rule_out[q]] += h.cand_n[q];
            }
            u64 stage_need = 0;
            for (int sl = 0; sl < pl.n_rels; sl++) stage_need = std::max(stage_need, incoming[sl]);
            for (int sl = 0; sl < pl.n_rels; sl++) {
                if (!d.rm.n_rules_in[sl]) continue;
                Relation& r = p->rels[d.rel_of_slot[sl]];
                r.full_n = h.full_n[sl];
                r.delta_n = h.delta_n[sl];
                const u64 stored = r.full_n + r.delta_n;
                if (replay && stored + incoming[sl] > r.cap) ensure_log(p, r, stored + 2 * incoming[sl]);
                const bool tight = !d.bit[sl].seen &&
                    h.seen_n[sl] + 2 * incoming[sl] > (u64)(p->tune.seen_load_max * (double)r.seen_cap);
                if (!d.bit[sl].seen && ((h.flags & kFlagProbe) || tight)) {
                    // rebuild from the stored tuples: every key older than the next (or replayed) iteration;
                    // at least twice the slots (a probe overflow means long clusters)
                    const u64 want = std::max<u64>((u64)(p->tune.seen_grow * (double)(stored + incoming[sl])),
                                                   (u64)(2.0 * p->tune.seen_load_max * (double)r.seen_cap));
                    dev_free(p, &r.seen);
                    r.seen_cap = 0;
                    build_seen(p, r, want);
                    h.seen_n[sl] = r.seen_n;
                }
            }
            refresh_refs(p, d);
            const bool cand_short = replay && total > p->dcand_cap;
            if (replay) {   // the heavy-row list covers every rule's candidates, bitmap rules' included
                u64 all = 0;
                for (int q = 0; q < pl.n_rules; q++) all += h.cand_n[q];
                p->heavy_cands = std::max(p->heavy_cands, 2 * all);
            }
            try {
                dev_size_buffers(p, d, replay ? std::max(p->dcand_cap, 2 * total) : p->dcand_cap,
                                 replay ? std::max(p->stage_cap, 2 * stage_need) : p->stage_cap,
                                 h.hist_n >= p->dhist_cap ? 2 * p->dhist_cap : p->dhist_cap);
            } catch (ra_error& e) {
                // the memory cap leaves no room for the iteration's candidates: the largest
                // candidate buffer that fits, and the iteration in slices of outer rows
                if (e.status != RA_E_OOM || !cand_short || !sliceable(p, d)) throw;
                u64 cap = std::max<u64>(total / 2, 1u << 16);
                for (;;) {
                    try {
                        dev_size_buffers(p, d, cap, p->stage_cap, p->dhist_cap);
                        break;
                    } catch (ra_error& e2) {
                        if (e2.status != RA_E_OOM || cap <= (1u << 12)) throw;
                        cap /= 2;
                    }
                }
                p->err.clear();
                h.flags = 0;
                h.exit_ctr = 0;
                h.bar_count = 0;
                for (int i = 0; i < 2 * kBankWords; i++) h.tile_ctr[i] = 0;
                CK(cudaMemcpyAsync(p->ctl, p->hctl, ctl_header_bytes(), cudaMemcpyHostToDevice, p->stream));
                run_sliced_iteration(p, s, d);
                if (h.flags & kFlagGrow) continue;   // handled by the next pass through this block
                if (p->cp_every) checkpoint_device_batch(p, s, d, hist_seen);
                if (h.done) break;
                continue;
            }
            if (p->n_inst && h.iteration >= p->inst_rows_cap) size_instance_rows(p, 2 * p->inst_rows_cap);
            h.flags = 0;
            h.exit_ctr = 0;
            h.bar_count = 0;
            if (replay) {
                for (int i = 0; i < 2 * kBankWords; i++) h.tile_ctr[i] = 0;
                h.heavy_n = 0;
                h.heavy_ctr = 0;
            }
            CK(cudaMemcpyAsync(p->ctl, p->hctl, ctl_header_bytes(), cudaMemcpyHostToDevice, p->stream));
            if (replay) {
                CK(cudaMemsetAsync(&p->ctl->sort_hist[0][0][0], 0, sizeof(p->ctl->sort_hist), p->stream));
                CK(cudaMemsetAsync(p->status, 0, p->status_cap * 8, p->stream));
            }
            if (!replay && p->cp_every) checkpoint_device_batch(p, s, d, hist_seen);
            if (h.done) break;
            continue;
        }
        if (p->cp_every) checkpoint_device_batch(p, s, d, hist_seen);
        if (h.done) break;
    }
    // results back into the host-side relation records
    std::vector<u64> hist(2 * h.hist_n);
    const u64 nt = std::min<u64>(h.iteration, p->dhist_cap);
    std::vector<u64> ends(nt);
    if (h.hist_n) CK(cudaMemcpyAsync(hist.data(), p->dhist, 2 * h.hist_n * 8, cudaMemcpyDeviceToHost, p->stream));
    if (nt) CK(cudaMemcpyAsync(ends.data(), p->dhist + 2 * p->dhist_cap, nt * 8, cudaMemcpyDeviceToHost, p->stream));
    if (p->n_inst && h.iteration) {
        const size_t at = p->inst_hist.size();
        p->inst_hist.resize(at + (size_t)h.iteration * p->n_inst);
        CK(cudaMemcpyAsync(p->inst_hist.data() + at, p->dinst_new, (size_t)h.iteration * p->n_inst * 8,
                           cudaMemcpyDeviceToHost, p->stream));
    }
    CK(cudaStreamSynchronize(p->stream));
    {
        u64 prev = h.t_start;
        for (u64 i = 0; i < nt; i++) {
            p->iter_us.push_back(ends[i] >= prev ? (double)(ends[i] - prev) / 1e3 : 0.0);
            prev = ends[i];
        }
    }
    for (int sl = 0; sl < pl.n_rels; sl++) {
        Relation& r = p->rels[d.rel_of_slot[sl]];
        // compare with the counts at SCC start (a mid-SCC regrow refreshes r's counts)
        if (h.full_n[sl] != full0[sl] || h.delta_n[sl] != delta0[sl] || h.iteration) {
            // deltas come out sorted in reference id order and from a bitmap relation's select
            const bool ref = p->id_order == RA_IDS_REFERENCE || d.bit[sl].seen;
            if (h.runs[sl]) {
                // one run into an empty full keeps it sorted when that run was sorted: the SCC's
                // initial delta, or a new delta in reference id order
                const bool run_sorted = delta0[sl] ? dsorted0[sl] : ref;
                r.full_sorted = full0[sl] == 0 && h.runs[sl] == 1 && run_sorted;
            }
            if (h.iteration) r.delta_sorted = ref || h.delta_n[sl] <= 1;
            r.full_n = h.full_n[sl];
            r.delta_n = h.delta_n[sl];
            r.full_version = fresh_stamp();
            r.delta_version = fresh_stamp();
        }
        if (d.rm.n_rules_in[sl]) r.seen_n = h.seen_n[sl];
        if (d.bit[sl].seen && r.seen) r.seen_dirty = true;   // its hash set missed this SCC's tuples
    }
    for (size_t t = 0; t < d.tags.size(); t++) intern_counter(p, d.tags[t]) = h.intern[t];
    if (persist_mode) {   // the persistent kernel's own phase clocks (barrier to barrier)
        p->stats.phase_ms[2] += (double)(h.ns_claims + h.ns_heavy) / 1e6;
        p->stats.phase_ms[3] += (double)h.ns_select / 1e6;
    }
    p->epoch = h.epoch;
    p->stats.iterations += h.iteration;
    p->stats.join_candidates += h.candidates;
    p->stats.heavy_items += h.heavy_items;
    p->stats.tail_iterations += h.tail_iters;
    p->stats.new_tuples += h.new_tuples;
    // loop bodies for the iterations the loop ran, one tail kernel per graph launch that has it
    p->stats.kernel_launches += (u64)body_kernels * (h.iteration - h.tail_iters) + tail_launches;
    p->stats.dedup_launches += (u64)d.rules.size() * h.iteration;
    // algorithmic bytes: a hash seen set costs 48 B per candidate (inner key read, candidate
    // write, 16-byte slot read + write); a bitmap one 8 B (the inner key; the claim is a bit
    // test and an atomicOr on a mostly L2-resident word); 24 B per outer row either way
    bool bitmap_scc = false;
    for (int sl = 0; sl < d.plan.n_rels; sl++) bitmap_scc = bitmap_scc || d.bit[sl].seen;
    p->stats.dedup_bytes += (bitmap_scc ? 8 : 48) * h.candidates + 24 * h.outer_rows;
    p->history.push_back((uint64_t)s.id);
    p->history.push_back(h.hist_n);
    p->history.insert(p->history.end(), hist.begin(), hist.end());
}

// Device buffers of one dense evaluation, freed on every exit.
struct DenseBufs {
    ra_program* p;
    u32* known = nullptr;
    u32* delta0 = nullptr;
    u64* row_new = nullptr;
    u64* row_off = nullptr;
    u64* level_total = nullptr;
    u64* counters = nullptr;
    u32* flags = nullptr;
    u32* s_local = nullptr;
    DenseInst* inst = nullptr;
    DenseChunk* chunks = nullptr;
    u64* inst_init = nullptr;
    explicit DenseBufs(ra_program* pp) : p(pp) {}
    ~DenseBufs()
    {
        dev_free(p, &known);
        dev_free(p, &delta0);
        dev_free(p, &row_new);
        dev_free(p, &row_off);
        dev_free(p, &level_total);
        dev_free(p, &counters);
        dev_free(p, &flags);
        dev_free(p, &s_local);
        dev_free(p, &inst);
        dev_free(p, &chunks);
        dev_free(p, &inst_init);
    }
};

// The end of a closure-shaped SCC run by an evaluator that is not the iteration
// loop (dense rows, composed reachable sets): `total` new tuples already written
// after R's `n_stored` stored ones, lv[k] of them new in iteration k (k < L),
// `iterations` iterations in all (the last finds nothing).  Records the same
// per-iteration history as the semi-naive bookkeeping (end_of_iteration,
// RAM::check_for_fixed_point, src/RAM/RA_tasks.cpp:1072-1085) and leaves R as the
// loop would: every tuple in its full version.
void finish_closure_scc(ra_program* p, Scc& s, int out, Relation& R, u64 n_stored, u64 total,
                        const std::vector<u64>& lv, u64 L, u64 iterations)
{
    std::vector<u64> f(s.rels.size()), d(s.rels.size());
    for (size_t i = 0; i < s.rels.size(); i++) {
        f[i] = p->rels[s.rels[i]].full_n;
        d[i] = p->rels[s.rels[i]].delta_n;
    }
    std::vector<uint64_t> hist;
    for (u64 k = 0; k < iterations; k++) {
        u64 sd = 0, sf = 0;
        for (size_t i = 0; i < s.rels.size(); i++) {
            f[i] += d[i];
            d[i] = (s.rels[i] == out && k < L) ? lv[k] : 0;
            sd += d[i];
            sf += f[i];
        }
        hist.push_back(sd);
        hist.push_back(sf);
    }
    p->history.push_back((uint64_t)s.id);
    p->history.push_back(iterations);
    p->history.insert(p->history.end(), hist.begin(), hist.end());

    // the log is [old full | old delta | new]: sorted only when a single sorted region holds it all
    const bool sorted = total == 0 && ((R.delta_n == 0 && R.full_sorted) || (R.full_n == 0 && R.delta_sorted));
    intern_counter(p, R.tag) += total;
    R.full_n = n_stored + total;
    R.delta_n = 0;
    R.newt_n = 0;
    R.full_sorted = sorted;
    R.delta_sorted = true;
    R.full_version = fresh_stamp();
    R.delta_version = fresh_stamp();
    if (R.seen) R.seen_dirty = true;   // the hash set holds none of the new tuples
    p->stats.iterations += iterations;
    p->stats.new_tuples += total;
}

// Runs SCC s with the dense row-closure evaluator (ra_dense.cuh) when its one
// rule has the transitive-closure shape and the bit matrices fit the tuned
// budget; returns false (nothing done) otherwise.  Leaves the SCC's relations
// as the semi-naive loop would after its fixed point (new tuples appended to
// R's log, everything in R's full version after the caller's delta_to_full),
// and records the same per-iteration history (RAM::check_for_fixed_point,
// src/RAM/RA_tasks.cpp:1072-1085) and per-instance counts.
bool run_scc_dense(ra_program* p, Scc& s)
{
    if (!s.fixpoint || s.rules.size() != 1 || s.rules[0].kind != kJoin) return false;
    if (p->id_order != RA_IDS_EMISSION || p->batch_size != 1 || p->tune.dense_max_bytes <= 0) return false;
    if (p->cp_every) return false;   // checkpoints need the relations after every iteration
    const Rule& ru = s.rules[0];
    const JoinPlan jp = make_join_plan(p, ru);
    if (jp.outer_rel != ru.out || jp.outer_ver != RA_DELTA || jp.inner_ver != RA_FULL || jp.inner_rel == ru.out)
        return false;
    Relation& R = p->rels[ru.out];
    Relation& S = p->rels[jp.inner_rel];
    if (R.arity != 2 || S.arity != 2 || R.jcc != 1) return false;
    const Projection& pj = jp.pj;
    if (pj.n != 2 || pj.side[0] != 1 || pj.col[0] != 1 || pj.side[1] != 0 || pj.col[1] != 1) return false;
    if (std::find(s.rels.begin(), s.rels.end(), jp.inner_rel) != s.rels.end() && S.delta_n != 0) return false;

    // geometry: one bit matrix per instance, rows = its values
    const u64 rows = p->max_value + 1;
    const u32 ninst = std::max<u32>(p->n_inst, 1);
    std::vector<DenseInst> hi(ninst);
    u64 words = 0;
    for (u32 i = 0; i < ninst; i++) {
        const u64 b = p->n_inst ? p->inst_base_h[i] : 0;
        const u64 e = (p->n_inst && i + 1 < p->n_inst) ? p->inst_base_h[i + 1] : rows;
        const u64 n = e > b ? e - b : 1;
        if (n > kDenseMaxN) return false;
        hi[i] = DenseInst{b, n, (n + 31) / 32, words};
        words += n * hi[i].words;
    }
    if (2.0 * 4.0 * (double)words + 16.0 * (double)rows > p->tune.dense_max_bytes) return false;

    DenseBufs B(p);
    dev_alloc(p, &B.known, words);
    dev_alloc(p, &B.delta0, words);
    dev_alloc(p, &B.row_new, rows);
    dev_alloc(p, &B.row_off, rows);
    dev_alloc(p, &B.counters, 8);
    dev_alloc(p, &B.flags, 1);
    dev_alloc(p, &B.inst, ninst);
    dev_alloc(p, &B.inst_init, ninst);
    constexpr int kShapes = 4;   // search kernels: warp per row with 1, 4, 16 words per lane; CTA per row
    CK(cudaMemcpyAsync(B.inst, hi.data(), ninst * sizeof(DenseInst), cudaMemcpyHostToDevice, p->stream));
    const u64 *sk, *sv;
    u64 sn;
    version_rows(p, S, RA_FULL, &sk, &sv, &sn);
    const u64* scsr = version_csr(p, S, RA_FULL);
    dev_alloc(p, &B.s_local, sn);
    const u64 n_stored = R.full_n + R.delta_n;
    u64 level_cap = 256;
    std::vector<u64> hflags(2);
    for (;;) {
        dev_free(p, &B.level_total);
        dev_alloc(p, &B.level_total, level_cap);
        if (p->n_inst) {
            size_instance_rows(p, level_cap);
            CK(cudaMemsetAsync(p->dinst_new, 0, p->inst_rows_cap * p->n_inst * 8, p->stream));
        }
        CK(cudaMemsetAsync(B.known, 0, words * 4, p->stream));
        CK(cudaMemsetAsync(B.delta0, 0, words * 4, p->stream));
        CK(cudaMemsetAsync(B.row_new, 0, rows * 8, p->stream));
        CK(cudaMemsetAsync(B.level_total, 0, level_cap * 8, p->stream));
        CK(cudaMemsetAsync(B.counters, 0, 8 * 8, p->stream));
        CK(cudaMemsetAsync(B.flags, 0, 4, p->stream));
        CK(cudaMemsetAsync(B.inst_init, 0, ninst * 8, p->stream));
        DenseArgs a{};
        a.inst = B.inst;
        a.inst_base = p->n_inst ? p->dinst_base : nullptr;
        a.n_inst = ninst;
        a.rows = rows;
        a.known = B.known;
        a.delta0 = B.delta0;
        a.bits = p->bits;
        a.s_keys = sk;
        a.s_csr = scsr;
        a.s_local = B.s_local;
        a.row_new = B.row_new;
        a.level_total = B.level_total;
        a.inst_level = p->n_inst ? p->dinst_new : nullptr;
        a.level_cap = p->n_inst ? std::min(level_cap, p->inst_rows_cap) : level_cap;
        a.inst_init = B.inst_init;
        a.counters = B.counters;
        a.flags = B.flags;
        if (sn) {
            dense_local_kernel<<<grid_for(sn), kThreads, 0, p->stream>>>(a, sn);
            LAUNCHED();
        }
        if (n_stored) {
            dense_load_kernel<<<grid_for(n_stored), kThreads, 0, p->stream>>>(a, R.keys, R.full_n, n_stored);
            LAUNCHED();
        }
        // work: chunks of rows of one instance.  A row's search reaches about s * n values when the
        // initial delta averages d > 1 tuples per row (s = 1 - exp(-d s), the giant component of a
        // random graph), a handful otherwise.  Instances whose rows reach at most 1024 values (and
        // of at most 16384 values) run one warp per row (words per lane 1, 4 or 16: three kernel
        // shapes), with no block barriers; wider searches run one CTA per row.
        std::vector<u64> init(ninst);
        CK(cudaMemcpyAsync(init.data(), B.inst_init, ninst * 8, cudaMemcpyDeviceToHost, p->stream));
        CK(cudaStreamSynchronize(p->stream));
        auto shape_of = [&](u32 i) {
            const u64 w = hi[i].words;
            const double n = (double)hi[i].n, deg = (double)init[i] / n;
            double sfrac = 0.0;
            if (deg > 1.0) {
                sfrac = 0.5;
                for (int it = 0; it < 60; it++) sfrac = 1.0 - std::exp(-deg * sfrac);
            }
            if (w > 512 || (w > 32 && sfrac * n > 1024.0)) return 3;
            return w <= 32 ? 0 : w <= 128 ? 1 : 2;
        };
        std::vector<DenseChunk> chunks;
        u64 first[kShapes + 1] = {0};
        u64 cta_wmax = 1;
        for (int sh = 0; sh < kShapes; sh++) {
            first[sh] = chunks.size();
            for (u32 i = 0; i < ninst; i++) {
                const DenseInst& di = hi[i];
                if (shape_of(i) != sh || di.base >= rows) continue;
                if (sh == 3) cta_wmax = std::max(cta_wmax, di.words);
                const u64 cnt = std::min(di.n, rows - di.base), per = sh == 3 ? 4 : 8;
                for (u64 r0 = 0; r0 < cnt; r0 += per)
                    chunks.push_back(DenseChunk{di.base + r0, i, (u32)std::min(per, cnt - r0)});
            }
        }
        first[kShapes] = chunks.size();
        dev_free(p, &B.chunks);
        dev_alloc(p, &B.chunks, std::max<size_t>(chunks.size(), 1));
        if (!chunks.empty())
            CK(cudaMemcpyAsync(B.chunks, chunks.data(), chunks.size() * sizeof(DenseChunk), cudaMemcpyHostToDevice,
                               p->stream));
        const size_t smem = 3 * cta_wmax * sizeof(u32);
        // grids: resident CTAs of each kernel, at most one warp (CTA) per chunk
        auto resident = [&](const void* fn, size_t dyn) {
            int per_sm = 0;
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kThreads, dyn));
            return (u64)kSms * (u64)std::max(per_sm, 1);
        };
        const void* fns[kShapes] = {(const void*)dense_closure_warp_kernel<1>, (const void*)dense_closure_warp_kernel<4>,
                                    (const void*)dense_closure_warp_kernel<16>, (const void*)dense_closure_kernel};
        int grids[kShapes];
        for (int sh = 0; sh < kShapes; sh++) {
            const u64 n = first[sh + 1] - first[sh];
            const u64 want = sh == 3 ? n : (n + kWarps - 1) / kWarps;
            grids[sh] = (int)std::max<u64>(1, std::min(resident(fns[sh], sh == 3 ? smem : 0), want));
        }
        cudaEvent_t ev[2] = {nullptr, nullptr};
        if (p->kernel_events) {
            CK(cudaEventCreate(&ev[0]));
            CK(cudaEventCreate(&ev[1]));
            CK(cudaEventRecord(ev[0], p->stream));
        }
        // one chunk counter per shape: counters[0] and [2] .. [4]
        u64* ctr[kShapes] = {B.counters + 2, B.counters + 3, B.counters + 4, B.counters};
        const u64 nc[kShapes] = {first[1] - first[0], first[2] - first[1], first[3] - first[2], first[4] - first[3]};
        if (nc[0])
            dense_closure_warp_kernel<1><<<grids[0], kThreads, 0, p->stream>>>(a, B.chunks + first[0], nc[0], ctr[0]);
        if (nc[1])
            dense_closure_warp_kernel<4><<<grids[1], kThreads, 0, p->stream>>>(a, B.chunks + first[1], nc[1], ctr[1]);
        if (nc[2])
            dense_closure_warp_kernel<16><<<grids[2], kThreads, 0, p->stream>>>(a, B.chunks + first[2], nc[2], ctr[2]);
        if (nc[3])
            dense_closure_kernel<<<grids[3], kThreads, smem, p->stream>>>(a, (u32)cta_wmax, B.chunks + first[3], nc[3],
                                                                          ctr[3]);
        for (int sh = 0; sh < kShapes; sh++)
            if (nc[sh]) LAUNCHED();
        if (p->kernel_events) {
            CK(cudaEventRecord(ev[1], p->stream));
            CK(cudaEventSynchronize(ev[1]));
            float ms = 0;
            CK(cudaEventElapsedTime(&ms, ev[0], ev[1]));
            p->stats.dense_search_ms += ms;
            cudaEventDestroy(ev[0]);
            cudaEventDestroy(ev[1]);
        }
        u32 fl = 0;
        CK(cudaMemcpyAsync(&fl, B.flags, 4, cudaMemcpyDeviceToHost, p->stream));
        CK(cudaStreamSynchronize(p->stream));
        if (fl & kDenseFlagRange) {
            u64 bad[2] = {0, 0};
            CK(cudaMemcpyAsync(bad, B.counters + 5, 16, cudaMemcpyDeviceToHost, p->stream));
            CK(cudaStreamSynchronize(p->stream));
            const u64 key = bad[0] - 1, mask = (1ull << p->bits) - 1;
            const u64 c0 = (key >> p->bits) & mask, c1 = key & mask;
            // R's rows are keyed by column 1's instance, S's by column 0's
            const u64 at = bad[1] == 1 ? c1 : c0;
            u32 inst = 0;
            while (p->n_inst && inst + 1 < p->n_inst && p->inst_base_h[inst + 1] <= at) inst++;
            fail(p, RA_E_BADARG,
                 "SCC %d: tuple (%llu, %llu) of %s has a value outside its instance %u (values %llu .. %llu)",
                 s.id, (unsigned long long)c0, (unsigned long long)c1, bad[1] == 1 ? R.name.c_str() : S.name.c_str(),
                 inst, (unsigned long long)hi[inst].base, (unsigned long long)(hi[inst].base + hi[inst].n - 1));
        }
        if (!(fl & kDenseFlagLevels)) {
            level_cap = a.level_cap;
            break;
        }
        level_cap *= 4;   // a deeper search than the level arrays held: again with room
        p->stats.regrows++;
    }

    // new tuples, row by row, after R's stored ones
    const u64 total = scan_exclusive<u64>(p, B.row_new, rows, B.row_off);
    u64& ctr = intern_counter(p, R.tag);
    if (total) {
        ensure_log(p, R, n_stored + total);
        cudaEvent_t ev[2] = {nullptr, nullptr};
        if (p->kernel_events) {
            CK(cudaEventCreate(&ev[0]));
            CK(cudaEventCreate(&ev[1]));
            CK(cudaEventRecord(ev[0], p->stream));
        }
        dense_emit_kernel<<<std::min<u64>((rows + kWarps - 1) / kWarps, (u64)kSms * 16), kThreads, 0, p->stream>>>(
            DenseArgs{B.inst, p->n_inst ? p->dinst_base : nullptr, ninst, rows, B.known, B.delta0, p->bits, sk, scsr,
                      B.s_local, B.row_new, B.level_total, nullptr, level_cap, B.inst_init, B.counters, B.flags},
            B.row_off, R.keys + n_stored, R.ids + n_stored, (u64)R.tag << 46, ctr);
        LAUNCHED();
        if (p->kernel_events) {
            CK(cudaEventRecord(ev[1], p->stream));
            CK(cudaEventSynchronize(ev[1]));
            float ms = 0;
            CK(cudaEventElapsedTime(&ms, ev[0], ev[1]));
            p->stats.dense_emit_ms += ms;
            cudaEventDestroy(ev[0]);
            cudaEventDestroy(ev[1]);
        }
    }
    std::vector<u64> lv(level_cap), cnt(4);
    CK(cudaMemcpyAsync(lv.data(), B.level_total, level_cap * 8, cudaMemcpyDeviceToHost, p->stream));
    CK(cudaMemcpyAsync(cnt.data(), B.counters, 4 * 8, cudaMemcpyDeviceToHost, p->stream));
    CK(cudaStreamSynchronize(p->stream));
    u64 L = 0;
    while (L < level_cap && lv[L]) L++;
    const u64 iterations = L + 1;   // the last one finds nothing new
    if (p->n_inst) {
        const size_t at = p->inst_hist.size();
        p->inst_hist.resize(at + (size_t)iterations * p->n_inst);
        CK(cudaMemcpyAsync(p->inst_hist.data() + at, p->dinst_new, (size_t)iterations * p->n_inst * 8,
                           cudaMemcpyDeviceToHost, p->stream));
        CK(cudaStreamSynchronize(p->stream));
    }

    finish_closure_scc(p, s, ru.out, R, n_stored, total, lv, L, iterations);
    p->stats.join_candidates += cnt[1];
    p->stats.dense_sccs++;
    return true;
}

// Device buffers of one reachability evaluation, freed on every exit.
struct ReachBufs {
    ra_program* p;
    u32 *sval = nullptr, *indeg = nullptr, *rpar = nullptr, *rem = nullptr, *seg_len = nullptr;
    u32 *front0 = nullptr, *front1 = nullptr, *hlist = nullptr;
    u32* flags = nullptr;
    u64 *rcsr = nullptr, *ctr = nullptr, *seg_off = nullptr, *row_new = nullptr, *row_off = nullptr;
    u64 *level_total = nullptr, *arena = nullptr;
    u32* cyc = nullptr;
    u64* cyc_n = nullptr;
    u64 *c_soff = nullptr, *c_singles = nullptr, *c_xoff = nullptr;
    u32 *c_node = nullptr, *c_xnode = nullptr, *c_xdist = nullptr;
    explicit ReachBufs(ra_program* pp) : p(pp) {}
    ~ReachBufs()
    {
        for (u32** q : {&sval, &indeg, &rpar, &rem, &front0, &front1, &hlist, &seg_len, &flags, &cyc, &c_node,
                        &c_xnode, &c_xdist})
            dev_free(p, q);
        for (u64** q : {&rcsr, &ctr, &seg_off, &row_new, &row_off, &level_total, &arena, &cyc_n, &c_soff, &c_singles,
                        &c_xoff})
            dev_free(p, q);
    }
};

constexpr u64 kReachLevels = 1ull << kDistBits;   // distances fit 16 bits

// A failed index check of the reachability kernels (none was dereferenced).
void reach_check_corrupt(ra_program* p, u32 fl, const std::vector<u64>& hc)
{
    if (fl & kReachCorrupt)
        fail(p, RA_E_CUDA, "reachability evaluator: index check %llu failed (value %llu, bound %llu)",
             (unsigned long long)(hc[kCCheck] - 1), (unsigned long long)hc[kCCheck + 1],
             (unsigned long long)hc[kCCheck + 2]);
}

// Runs SCC s with the reachability evaluator (ra_reach.cuh) when its one rule has
// the transitive-closure shape and R's stored tuples are exactly S reversed;
// returns false (nothing done) otherwise, or when the graph is mostly cyclic or
// too deep for 16-bit distances (the semi-naive loop runs it instead).  Leaves
// the relations and the per-iteration history as the semi-naive loop would.
bool run_scc_reach(ra_program* p, Scc& s)
{
    if (!p->use_reach || !s.fixpoint || s.rules.size() != 1 || s.rules[0].kind != kJoin) return false;
    if (p->id_order != RA_IDS_EMISSION || p->batch_size != 1 || p->cp_every || p->n_inst) return false;
    const Rule& ru = s.rules[0];
    const JoinPlan jp = make_join_plan(p, ru);
    if (jp.outer_rel != ru.out || jp.outer_ver != RA_DELTA || jp.inner_ver != RA_FULL || jp.inner_rel == ru.out)
        return false;
    Relation& R = p->rels[ru.out];
    Relation& S = p->rels[jp.inner_rel];
    if (R.arity != 2 || S.arity != 2 || R.jcc != 1) return false;
    const Projection& pj = jp.pj;
    if (pj.n != 2 || pj.side[0] != 1 || pj.col[0] != 1 || pj.side[1] != 0 || pj.col[1] != 1) return false;
    if (std::find(s.rels.begin(), s.rels.end(), jp.inner_rel) != s.rels.end() && S.delta_n != 0) return false;
    if (R.full_n != 0 || !R.keys_unique || !S.keys_unique || p->bits > 31) return false;
    const u64 *sk, *sv;
    u64 sn;
    version_rows(p, S, RA_FULL, &sk, &sv, &sn);
    if (R.delta_n != sn || sn == 0) return false;
    const u64 n = p->max_value + 1;
    if (n > 16 * sn + (1u << 16)) return false;   // a sparse value domain: per-value arrays would dwarf the input
    const u64* scsr = version_csr(p, S, RA_FULL);

    const auto t_setup = std::chrono::steady_clock::now();
    ReachBufs B(p);
    dev_alloc(p, &B.sval, sn);
    dev_alloc(p, &B.indeg, n + 1);
    dev_alloc(p, &B.rcsr, n + 1);
    dev_alloc(p, &B.rpar, sn);
    dev_alloc(p, &B.rem, n);
    dev_alloc(p, &B.front0, n);
    dev_alloc(p, &B.front1, n);
    dev_alloc(p, &B.hlist, n);
    dev_alloc(p, &B.seg_len, n);
    dev_alloc(p, &B.seg_off, n);
    dev_alloc(p, &B.ctr, kCtrWords);
    dev_alloc(p, &B.flags, 1);
    // predecessor lists (a counting sort of S by column 1)
    CK(cudaMemsetAsync(B.indeg, 0, (n + 1) * 4, p->stream));
    reach_sval_kernel<<<grid_for(sn), kThreads, 0, p->stream>>>(sk, sn, p->bits, B.sval, B.indeg);
    LAUNCHED();
    scan_exclusive<u32>(p, B.indeg, n + 1, B.rcsr, false);
    CK(cudaMemsetAsync(B.indeg, 0, (n + 1) * 4, p->stream));
    reach_parents_kernel<<<grid_for(sn), kThreads, 0, p->stream>>>(sk, sn, p->bits, B.rcsr, B.indeg, B.rpar);
    LAUNCHED();
    ReachArgs a{};
    a.n = n;
    a.scsr = scsr;
    a.sval = B.sval;
    a.rcsr = B.rcsr;
    a.rpar = B.rpar;
    a.rem = B.rem;
    a.ctr = B.ctr;
    a.seg_off = B.seg_off;
    a.seg_len = B.seg_len;
    a.flags = B.flags;
    // R's stored tuples must be exactly S reversed (equal counts, distinct, each one found)
    CK(cudaMemsetAsync(B.flags, 0, 4, p->stream));
    reach_check_kernel<<<grid_for(R.delta_n), kThreads, 0, p->stream>>>(a, R.keys, R.delta_n, p->bits);
    LAUNCHED();
    u32 fl = 0;
    CK(cudaMemcpyAsync(&fl, B.flags, 4, cudaMemcpyDeviceToHost, p->stream));
    CK(cudaStreamSynchronize(p->stream));
    if (fl & kReachMismatch) return false;

    static int occ = 0, sms = 0;
    if (!occ) {
        int dev = 0;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, reach_levels_kernel, kThreads, 0));
        if (occ < 1) fail(p, RA_E_CUDA, "the reachability kernel does not fit on an SM");
    }
    auto tp = t_setup;
    auto phase_done = [&](int k) {   // host time since the last mark, after a synchronisation
        const auto now = std::chrono::steady_clock::now();
        p->stats.reach_phase_ms[k] += std::chrono::duration<double, std::milli>(now - tp).count();
        tp = now;
    };
    phase_done(0);
    u64 cap = std::max<u64>(p->reach_arena_hint, 24 * sn + (1u << 20));
    std::vector<u64> hc(kCtrWords);
    for (;;) {
        dev_free(p, &B.arena);
        dev_alloc(p, &B.arena, cap);
        a.arena = B.arena;
        a.arena_cap = cap;
        CK(cudaMemsetAsync(B.ctr, 0, kCtrWords * 8, p->stream));
        CK(cudaMemsetAsync(B.flags, 0, 4, p->stream));
        reach_init_kernel<<<grid_for(n), kThreads, 0, p->stream>>>(a, B.front0);
        LAUNCHED();
        void* args[] = {&a, &B.front0, &B.front1, &B.hlist};
        CK(cudaLaunchCooperativeKernel((const void*)reach_levels_kernel, dim3(sms * occ), dim3(kThreads), args, 0,
                                       p->stream));
        LAUNCHED();
        CK(cudaMemcpyAsync(&fl, B.flags, 4, cudaMemcpyDeviceToHost, p->stream));
        CK(cudaMemcpyAsync(hc.data(), B.ctr, kCtrWords * 8, cudaMemcpyDeviceToHost, p->stream));
        CK(cudaStreamSynchronize(p->stream));
        reach_check_corrupt(p, fl, hc);
        if (fl & kReachTimeout) fail(p, RA_E_TIMEOUT, "SCC %d: a bounded wait of the reachability evaluator gave up", s.id);
        if (fl & kReachArena) {   // room for what it asked, and some
            cap = std::max<u64>(2 * cap, hc[kCArena] + hc[kCArena] / 4);
            p->stats.regrows++;
            continue;
        }
        break;
    }
    phase_done(1);
    if (fl & kReachDepth) return false;
    // nodes that reach a cycle: searched on the host over that part of the graph
    const u64 finished = hc[kCDone];
    p->stats.reach_levels += hc[kCLevels];
    if (finished < n) {
        const u64 U = n - finished;
        if (U > std::max<u64>(1u << 16, n / 64)) return false;   // mostly cyclic: the semi-naive loop
        dev_alloc(p, &B.cyc, U);
        dev_alloc(p, &B.cyc_n, 1);
        CK(cudaMemsetAsync(B.cyc_n, 0, 8, p->stream));
        reach_cyclic_list_kernel<<<grid_for(n), kThreads, 0, p->stream>>>(a, B.cyc, B.cyc_n, U);
        LAUNCHED();
        std::vector<u32> cyc(U);
        CK(cudaMemcpyAsync(cyc.data(), B.cyc, U * 4, cudaMemcpyDeviceToHost, p->stream));
        CK(cudaStreamSynchronize(p->stream));
        std::sort(cyc.begin(), cyc.end());
        // successors of those nodes (S's rows are the CSR ranges), gathered on the device
        CK(cudaMemcpyAsync(B.cyc, cyc.data(), U * 4, cudaMemcpyHostToDevice, p->stream));
        dev_alloc(p, &B.c_soff, 2 * U);
        reach_gather_ranges_kernel<<<grid_for(U), kThreads, 0, p->stream>>>(scsr, B.cyc, U, n, B.c_soff);
        LAUNCHED();
        std::vector<u64> lohi(2 * U), off(U + 1);
        CK(cudaMemcpyAsync(lohi.data(), B.c_soff, 2 * U * 8, cudaMemcpyDeviceToHost, p->stream));
        CK(cudaStreamSynchronize(p->stream));
        off[0] = 0;
        for (u64 i = 0; i < U; i++) off[i + 1] = off[i] + (lohi[2 * i + 1] - lohi[2 * i]);
        std::vector<u32> succ(off[U]);
        if (off[U]) {
            dev_alloc(p, &B.c_xoff, U + 1);
            dev_alloc(p, &B.c_xnode, off[U]);
            CK(cudaMemcpyAsync(B.c_xoff, off.data(), (U + 1) * 8, cudaMemcpyHostToDevice, p->stream));
            reach_gather_succ_kernel<<<std::max<u64>(1, std::min<u64>((U + kWarps - 1) / kWarps, (u64)kSms * 8)),
                                       kThreads, 0, p->stream>>>(B.sval, B.c_soff, B.c_xoff, U, B.c_xnode);
            LAUNCHED();
            CK(cudaMemcpyAsync(succ.data(), B.c_xnode, off[U] * 4, cudaMemcpyDeviceToHost, p->stream));
            CK(cudaStreamSynchronize(p->stream));
            dev_free(p, &B.c_xoff);
            dev_free(p, &B.c_xnode);
        }
        dev_free(p, &B.c_soff);
        auto index_of = [&](u32 v) -> long {
            auto it = std::lower_bound(cyc.begin(), cyc.end(), v);
            return (it != cyc.end() && *it == v) ? (long)(it - cyc.begin()) : -1;
        };
        // per node: a breadth-first search over the nodes that reach a cycle, recording the
        // cycle-free nodes met first (their own sets are complete) with their distances
        std::vector<u64> soff(1, 0), singles, xoff(1, 0);
        std::vector<u32> xnode, xdist;
        std::vector<u32> dist(U, 0), seen(U, 0);
        std::vector<u32> frontier, next;
        std::unordered_map<u32, u32> exits;
        u32 stamp = 0;
        for (u64 i = 0; i < U; i++) {
            ++stamp;
            exits.clear();
            frontier.assign(1, (u32)i);
            std::vector<std::pair<u32, u32>> found;   // (value, distance)
            for (u32 d = 1; !frontier.empty(); d++) {
                if (d >= kReachLevels) return false;
                next.clear();
                for (u32 ui : frontier)
                    for (u64 e = off[ui]; e < off[ui + 1]; e++) {
                        const u32 w = succ[e];
                        const long wi = index_of(w);
                        if (wi < 0) {
                            auto it = exits.find(w);
                            if (it == exits.end()) exits.emplace(w, d);
                            continue;
                        }
                        if (seen[wi] == stamp) continue;
                        seen[wi] = stamp;
                        dist[wi] = d;
                        found.push_back({w, d});
                        if ((u64)wi != i) next.push_back((u32)wi);
                    }
                frontier.swap(next);
            }
            std::vector<std::pair<u32, u32>> ex(exits.begin(), exits.end());
            std::sort(ex.begin(), ex.end());
            for (auto& e : ex) found.push_back(e);
            std::sort(found.begin(), found.end());
            for (auto& f : found) singles.push_back(((u64)f.first << kDistBits) | f.second);
            soff.push_back(singles.size());
            for (auto& e : ex) {
                xnode.push_back(e.first);
                xdist.push_back(e.second);
            }
            xoff.push_back(xnode.size());
        }
        dev_alloc(p, &B.c_node, U);
        dev_alloc(p, &B.c_soff, U + 1);   // (freed above after the gather)
        dev_alloc(p, &B.c_singles, std::max<size_t>(singles.size(), 1));
        dev_alloc(p, &B.c_xoff, U + 1);
        dev_alloc(p, &B.c_xnode, std::max<size_t>(xnode.size(), 1));
        dev_alloc(p, &B.c_xdist, std::max<size_t>(xdist.size(), 1));
        CK(cudaMemcpyAsync(B.c_node, cyc.data(), U * 4, cudaMemcpyHostToDevice, p->stream));
        CK(cudaMemcpyAsync(B.c_soff, soff.data(), (U + 1) * 8, cudaMemcpyHostToDevice, p->stream));
        if (!singles.empty())
            CK(cudaMemcpyAsync(B.c_singles, singles.data(), singles.size() * 8, cudaMemcpyHostToDevice, p->stream));
        CK(cudaMemcpyAsync(B.c_xoff, xoff.data(), (U + 1) * 8, cudaMemcpyHostToDevice, p->stream));
        if (!xnode.empty()) {
            CK(cudaMemcpyAsync(B.c_xnode, xnode.data(), xnode.size() * 4, cudaMemcpyHostToDevice, p->stream));
            CK(cudaMemcpyAsync(B.c_xdist, xdist.data(), xdist.size() * 4, cudaMemcpyHostToDevice, p->stream));
        }
        ReachCyclic c{B.c_node, B.c_soff, B.c_singles, B.c_xoff, B.c_xnode, B.c_xdist, U};
        for (;;) {
            CK(cudaMemsetAsync(B.flags, 0, 4, p->stream));
            reach_cyclic_kernel<<<std::max<u64>(1, std::min<u64>((U + kWarps - 1) / kWarps, (u64)kSms * 4)), kThreads, 0,
                                  p->stream>>>(a, c);
            LAUNCHED();
            CK(cudaMemcpyAsync(&fl, B.flags, 4, cudaMemcpyDeviceToHost, p->stream));
            CK(cudaMemcpyAsync(hc.data(), B.ctr, kCtrWords * 8, cudaMemcpyDeviceToHost, p->stream));
            CK(cudaStreamSynchronize(p->stream));
            reach_check_corrupt(p, fl, hc);
            if (fl & kReachDepth) return false;
            if (!(fl & kReachArena)) break;
            // a larger arena, keeping what the cycle-free nodes wrote
            const u64 ncap = std::max<u64>(2 * cap, hc[kCArena] + hc[kCArena] / 4);
            u64* na;
            dev_alloc(p, &na, ncap);
            CK(cudaMemcpyAsync(na, B.arena, cap * 8, cudaMemcpyDeviceToDevice, p->stream));
            dev_free(p, &B.arena);
            B.arena = na;
            a.arena = na;
            a.arena_cap = cap = ncap;
            p->stats.regrows++;
            // the failed launch's allocations are past the old end: nothing it wrote is kept
            CK(cudaMemcpyAsync(B.ctr + kCArena, &hc[kCArena], 8, cudaMemcpyHostToDevice, p->stream));
        }
    }
    p->reach_arena_hint = std::max<u64>(p->reach_arena_hint, hc[kCArena] + hc[kCArena] / 8);
    phase_done(2);

    // new tuples, row by row, after R's stored ones
    dev_alloc(p, &B.row_new, n);
    dev_alloc(p, &B.row_off, n);
    reach_count_kernel<<<grid_for(n), kThreads, 0, p->stream>>>(a, B.row_new);
    LAUNCHED();
    const u64 total = scan_exclusive<u64>(p, B.row_new, n, B.row_off);
    const u64 n_stored = R.full_n + R.delta_n;
    ensure_log(p, R, n_stored + total);
    dev_alloc(p, &B.level_total, kReachLevels + 1);
    CK(cudaMemsetAsync(B.level_total, 0, (kReachLevels + 1) * 8, p->stream));
    reach_emit_kernel<<<std::min<u64>((n + kWarps - 1) / kWarps, (u64)kSms * 16), kThreads, 0, p->stream>>>(
        a, B.row_off, p->bits, R.keys + n_stored, R.ids + n_stored, (u64)R.tag << 46, intern_counter(p, R.tag),
        B.level_total, kReachLevels, B.level_total + kReachLevels, total);
    LAUNCHED();
    std::vector<u64> lv(kReachLevels + 1);
    CK(cudaMemcpyAsync(lv.data(), B.level_total, (kReachLevels + 1) * 8, cudaMemcpyDeviceToHost, p->stream));
    CK(cudaMemcpyAsync(&fl, B.flags, 4, cudaMemcpyDeviceToHost, p->stream));
    CK(cudaMemcpyAsync(hc.data(), B.ctr, kCtrWords * 8, cudaMemcpyDeviceToHost, p->stream));
    CK(cudaStreamSynchronize(p->stream));
    reach_check_corrupt(p, fl, hc);
    phase_done(3);
    p->stats.reach_ms = p->stats.reach_phase_ms[0] + p->stats.reach_phase_ms[1] + p->stats.reach_phase_ms[2] +
                         p->stats.reach_phase_ms[3];
    u64 L = 0;
    while (L < kReachLevels && lv[L]) L++;
    p->stats.join_candidates += lv[kReachLevels];   // what the semi-naive loop's joins would have produced
    finish_closure_scc(p, s, ru.out, R, n_stored, total, lv, L, L + 1);
    p->stats.reach_sccs++;
    return true;
}

// RAM::insert_delta_in_full of the previous SCC (lie.cpp:436): done when the next SCC
// starts or the run ends, so that counts read between SCCs are the ones the
// reference prints there (its size print precedes the merge).
#include "ra_wide.cu"

void merge_pending(ra_program* p)
{
    for (int ri : p->pending_merge) {
        if (p->wide) wide_delta_to_full(p, p->rels[ri]);
        else delta_to_full(p->rels[ri]);
    }
    p->pending_merge.clear();
}

void run_scc(ra_program* p, Scc& s)
{
    merge_pending(p);
    for (const Rule& ru : s.rules)
        if (std::find(s.rels.begin(), s.rels.end(), ru.out) == s.rels.end())
            fail(p, RA_E_UNSUPPORTED, "SCC %d: rule output %s is not one of the SCC's relations", s.id,
                 p->rels[ru.out].name.c_str());
    p->loop_counter = 0;
    if (p->wide) {
        run_scc_wide(p, s);
        return;
    }
    if (!p->rs_dir.empty()) {
        // restart (lie.cpp:300-330): deltas from the dump instead of full -> delta
        for (int ri : s.rels) load_restart_delta(p, p->rels[ri]);
    } else {
        for (size_t i = 0; i < s.rels.size(); i++)
            if (s.init[i]) full_to_delta(p, p->rels[s.rels[i]]);
    }
    if (run_scc_dense(p, s) || run_scc_reach(p, s)) {
        p->pending_merge = s.rels;
        return;
    }
    {
        DevScc d;
        if (build_dev_scc(p, s, d)) {
            run_scc_device(p, s, d);
            p->pending_merge = s.rels;
            return;
        }
    }
    p->inst_hist_ok = false;   // the host path keeps no per-instance counts
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
        checkpoint_batch(p, s, !s.fixpoint || d == 0, host_counts(p));
        if (!s.fixpoint || d == 0) break;
    }
    p->pending_merge = s.rels;
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
    // tuples that do not pack into one 63-bit key (or joins the CSR index cannot
    // hold) run on the wide path
    p->wide = program_needs_wide(p, bits);
    p->bits = bits;
    p->max_value = mx;
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
    dev_free(p, &r.bm_seen);
    dev_free(p, &r.bm_fresh);
    dev_free(p, &r.bm_dirty);
    r.bm_rows = r.bm_words = 0;
    wide_free_relation(p, r);
    r.cap = r.seen_cap = r.seen_n = r.v_cap = r.csr_full_cap = r.csr_delta_cap = 0;
    r.v_version = r.csr_full_version = r.csr_delta_version = ~0ull;
    r.full_n = r.delta_n = r.newt_n = 0;
}

// Back to the pre-run state.  Device buffers are kept (capacities carry over to
// the next run); only counters, caches of derived data and seen sets are reset.
void reset_state(ra_program* p)
{
    for (Relation& r : p->rels) {
        r.full_n = r.delta_n = r.newt_n = 0;
        r.full_sorted = r.delta_sorted = true;
        r.seen_n = 0;
        if (r.seen) r.seen_dirty = true;
        r.full_version = fresh_stamp();
        r.delta_version = fresh_stamp();
    }
    for (Scc& s : p->sccs) s.done = false;
    p->history.clear();
    p->pending_merge.clear();
    p->iter_us.clear();
    p->inst_hist.clear();
    p->inst_hist_ok = true;
    p->intern.clear();
    p->executed = false;
    p->running = false;
    // p->epoch keeps counting across runs: loser marks and seen-set tags are epoch-stamped
}

// Free every device buffer a run sizes (relation logs, seen sets, indexes,
// iteration scratch) and the captured graphs; loaded rows and the packed
// loaded state stay, so the next run re-allocates only what it needs.
void release_buffers(ra_program* p)
{
    for (Relation& r : p->rels) free_relation_state(p, r);
    dev_free(p, &p->cand);
    dev_free(p, &p->flag);
    dev_free(p, &p->rank);
    dev_free(p, &p->cnt);
    dev_free(p, &p->off);
    dev_free(p, &p->nkeys);
    dev_free(p, &p->nids);
    dev_free(p, &p->tk);
    dev_free(p, &p->tv);
    dev_free(p, &p->hist_buf);
    dev_free(p, &p->hist_off);
    p->cand_cap = p->rank_cap = p->cnt_cap = p->n_cap = p->t_cap = p->hist_cap = 0;
    dev_free(p, &p->dcand);
    dev_free(p, &p->dloser);
    p->dcand_cap = 0;
    for (int q = 0; q < kMaxSccRules; q++) {
        dev_free(p, &p->doff[q]);
        dev_free(p, &p->dstart[q]);
    }
    p->doff_cap = 0;
    for (int sl = 0; sl < kMaxSccRels; sl++) {
        dev_free(p, &p->stage_k[sl]);
        dev_free(p, &p->stage_v[sl]);
    }
    for (int b = 0; b < 2; b++) {
        dev_free(p, &p->sort_k[b]);
        dev_free(p, &p->sort_v[b]);
    }
    p->stage_cap = 0;
    dev_free(p, &p->status);
    p->status_cap = 0;
    dev_free(p, &p->dheavy);
    p->heavy_cap = 0;
    dev_free(p, &p->dinst_new);
    p->inst_rows_cap = 0;
    dev_free(p, &p->dhist);
    p->dhist_cap = 0;
    dev_free(p, &p->bmt_word);
    dev_free(p, &p->bmt_base);
    dev_free(p, &p->bmt_words);
    dev_free(p, &p->bmt_inst);
    p->bmt_rows = 0;
    p->bmt_bases.clear();
    for (int i = 0; i < 12; i++) {
        dev_free(p, &p->wbuf[i]);
        p->wbuf_cap[i] = 0;
    }
    for (Scc& sc : p->sccs) drop_graph(sc);
    CK(cudaStreamSynchronize(p->stream));
}

void begin_run(ra_program* p)
{
    if (p->executed || p->running) reset_state(p);
    p->stats = ra_stats{};
    p->stats.device_bytes = p->stats.device_bytes_peak = p->live_bytes;
    for (auto& e : p->dedup_events) {
        cudaEventDestroy(e.first);
        cudaEventDestroy(e.second);
    }
    p->dedup_events.clear();
    if (!p->packed) {
        choose_bits(p);
        if (!p->wide)
            for (Relation& r : p->rels) pack_relation(p, r);
        p->packed = true;
    } else if (!p->wide) {
        for (Relation& r : p->rels) restore_loaded(p, r);
    }
    if (p->wide) {
        if (p->n_inst) fail(p, RA_E_UNSUPPORTED, "batched instances of a wide-tuple program");
        for (Relation& r : p->rels) wide_load(p, r);
    }
    p->running = true;
    p->fixpoint_ms_acc = 0;
    p->executed_ids = p->rs_skip;
    if (p->cp_every) mkdir(p->cp_dir.c_str(), S_IRWXU | S_IRWXG | S_IROTH | S_IXOTH);
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
    merge_pending(p);
    CK(cudaStreamSynchronize(p->stream));
    double dms = 0;
    for (auto& e : p->dedup_events) {
        float m = 0;
        cudaEventElapsedTime(&m, e.first, e.second);
        dms += m;
    }
    for (auto& e : p->phase_events) {
        float m = 0;
        cudaEventElapsedTime(&m, e.second.first, e.second.second);
        p->stats.phase_ms[e.first] += m;
        if (e.first == 2) {
            dms += m;
        }
        cudaEventDestroy(e.second.first);
        cudaEventDestroy(e.second.second);
    }
    p->phase_events.clear();
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
    // a restart does not run the SCCs its dump lists as executed (lie.cpp:276-287)
    while (next >= 0 && std::find(p->rs_skip.begin(), p->rs_skip.end(), p->sccs[next].id) != p->rs_skip.end()) {
        p->sccs[next].done = true;
        next = next_runnable(p);
    }
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
    // the run ends at the next step, so that counts read after the last SCC are, as
    // the reference prints them there, from before its final delta -> full merge
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
        dev_alloc(p, &p->ctl, 1);
        CK(cudaMallocHost(&p->hctl, sizeof(IterCtl)));
        if (const char* e = getenv("RA_NO_GRAPH")) p->use_graphs = atoi(e) == 0;
        if (const char* e = getenv("RA_NO_TAIL")) p->use_tail = atoi(e) == 0;
        if (const char* e = getenv("RA_PERSIST")) p->use_persist = atoi(e) != 0;
        if (const char* e = getenv("RA_REACH")) p->use_reach = atoi(e) != 0;
        if (const char* e = getenv("RA_KERNEL_EVENTS")) p->kernel_events = atoi(e) != 0;
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
    dev_free(p, &p->ctl);
    dev_free(p, &p->dcand);
    dev_free(p, &p->dloser);
    for (int q = 0; q < kMaxSccRules; q++) {
        dev_free(p, &p->doff[q]);
        dev_free(p, &p->dstart[q]);
    }
    for (int sl = 0; sl < kMaxSccRels; sl++) {
        dev_free(p, &p->stage_k[sl]);
        dev_free(p, &p->stage_v[sl]);
    }
    for (int b = 0; b < 2; b++) {
        dev_free(p, &p->sort_k[b]);
        dev_free(p, &p->sort_v[b]);
    }
    dev_free(p, &p->status);
    dev_free(p, &p->dheavy);
    dev_free(p, &p->dhist);
    dev_free(p, &p->dinst_base);
    dev_free(p, &p->dinst_new);
    dev_free(p, &p->bmt_word);
    dev_free(p, &p->bmt_base);
    dev_free(p, &p->bmt_words);
    dev_free(p, &p->bmt_inst);
    for (Scc& sc : p->sccs) drop_graph(sc);
    for (auto& e : p->dedup_events) {
        cudaEventDestroy(e.first);
        cudaEventDestroy(e.second);
    }
    if (p->stream) cudaStreamSynchronize(p->stream);
    if (p->hscalar) cudaFreeHost(p->hscalar);
    if (p->hctl) cudaFreeHost(p->hctl);
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

int ra_program_set_id_order(ra_program* p, int mode)
{
    return guard(p, [&] {
        if (mode != RA_IDS_REFERENCE && mode != RA_IDS_EMISSION) fail(p, RA_E_BADARG, "id order mode");
        if (p->running) fail(p, RA_E_STATE, "id order cannot change during a run");
        p->id_order = mode;
    });
}

int ra_program_set_launch_timing(ra_program* p, int on)
{
    return guard(p, [&] {
        if (p->running) fail(p, RA_E_STATE, "launch timing cannot change during a run");
        p->kernel_events = on != 0;
    });
}

int ra_program_set_evaluators(ra_program* p, int reach, int persistent)
{
    return guard(p, [&] {
        if (p->running) fail(p, RA_E_STATE, "evaluators cannot change during a run");
        p->use_reach = reach != 0;
        p->use_persist = persistent != 0;
    });
}

int ra_relation_create(ra_program* p, uint32_t jcc, uint32_t arity, uint32_t tag, const char* name, int version,
                       int* rel_out)
{
    return guard(p, [&] {
        if (!rel_out || arity == 0 || arity >= (uint32_t)kWideMaxCols || jcc > arity)
            fail(p, RA_E_BADARG, "relation: need 0 <= jcc <= arity <= %d", kWideMaxCols - 1);
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
        if (rows) {
            struct stat st {};
            if (stat(path, &st) != 0) fail(p, RA_E_IO, "cannot open %s", path);
            if (rows > (unsigned long long)st.st_size / (8 * cols))
                fail(p, RA_E_IO, "%s: %llu rows of %llu columns announced, the file holds %lld bytes", meta.c_str(),
                     rows, cols, (long long)st.st_size);
        }
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
        if (nproj <= 0 || nproj >= kWideMaxCols || !proj) fail(p, RA_E_BADARG, "join projection size");
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
        if (nproj <= 0 || nproj > kWideMaxCols || !proj) fail(p, RA_E_BADARG, "copy reorder size");
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

// A run that failed (out of device memory, a device wait that timed out, ...)
// leaves the program reusable: an open stream capture is closed, queued work
// drains, every device buffer of the run is freed (a failure may have struck
// between a buffer's release and its regrowth), and the run ends -- the next
// execute starts from the loaded state.
static int end_failed_run(ra_program* p, int st)
{
    if (st == RA_OK || !p) return st;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (p->stream && cudaStreamIsCapturing(p->stream, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(p->stream, &g);
        if (g) cudaGraphDestroy(g);
    }
    if (p->stream) cudaStreamSynchronize(p->stream);
    cudaGetLastError();   // clear a non-sticky error (allocation failure) left by the run
    const std::string msg = p->err;
    try {
        release_buffers(p);   // also drops every SCC's graph
    } catch (...) {
    }
    p->err = msg;
    reset_state(p);       // every SCC runs again next time; counters, history and seen sets start over
    return st;
}

int ra_program_execute(ra_program* p)
{
    return end_failed_run(p, guard(p, [&] { execute(p); }));
}

int ra_program_run_next_scc(ra_program* p, int* scc_id)
{
    return end_failed_run(p, guard(p, [&] {
        int id = -1;
        if (!(p->executed && !p->running)) id = step(p);
        if (scc_id) *scc_id = id;
    }));
}

int ra_program_release(ra_program* p)
{
    return guard(p, [&] {
        if (p->running) fail(p, RA_E_STATE, "release during a run");
        release_buffers(p);
        reset_state(p);   // the last run's results lived in the freed logs
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

int ra_program_iteration_times(ra_program* p, double* out_us, uint64_t cap, uint64_t* len)
{
    return guard(p, [&] {
        if (len) *len = p->iter_us.size();
        if (out_us) std::memcpy(out_us, p->iter_us.data(), std::min<u64>(cap, p->iter_us.size()) * 8);
    });
}

int ra_program_set_memory_cap(ra_program* p, uint64_t bytes)
{
    return guard(p, [&] { p->alloc_cap = bytes; });
}

int ra_selftest_bounded_wait(int device, uint64_t max_polls)
{
    if (cudaSetDevice(device) != cudaSuccess) return RA_E_CUDA;
    if (max_polls == 0 || max_polls > kSpinLimit) return RA_E_BADARG;
    void* mem = nullptr;
    if (cudaMalloc(&mem, 4 * sizeof(u64)) != cudaSuccess) return RA_E_OOM;
    u64* status = (u64*)mem;
    u32* flags = (u32*)(status + 2);
    int st = RA_OK;
    if (cudaMemset(mem, 0, 4 * sizeof(u64)) != cudaSuccess) st = RA_E_CUDA;
    if (st == RA_OK) {
        lookback_selftest_kernel<<<1, 32>>>(status, flags, max_polls);
        u32 hf = 0;
        if (cudaGetLastError() != cudaSuccess || cudaMemcpy(&hf, flags, 4, cudaMemcpyDeviceToHost) != cudaSuccess)
            st = RA_E_CUDA;
        else if (hf & kFlagTimeout)
            st = RA_E_TIMEOUT;
    }
    cudaFree(mem);
    return st;
}

namespace {
// kind 0: empty -> key CAS on 16-byte slots; kind 1: 8-byte loads.  Four independent
// accesses per thread in flight, slots from the claims' own hash of the operation index.
__global__ void __launch_bounds__(kThreads) calibrate_kernel(Slot* __restrict__ t, u64 cap, u64 ops, u64 salt, int kind,
                                                             u64* __restrict__ sink)
{
    u64 acc = 0;
    const u64 stride = (u64)gridDim.x * kThreads * 4;
    for (u64 i0 = ((u64)blockIdx.x * kThreads + threadIdx.x) * 4; i0 < ops; i0 += stride) {
        u64 h[4];
#pragma unroll
        for (int b = 0; b < 4; b++) h[b] = slot_start(i0 + b + salt, cap);
#pragma unroll
        for (int b = 0; b < 4; b++) {
            if (i0 + b >= ops) continue;
            if (kind == 0) {
                const Slot r = atomicCAS(&t[h[b]], Slot{kEmpty, ~0ull}, Slot{i0 + b, salt});
                acc += r.key;
            } else {
                acc += __ldcg(&t[h[b]].key);
            }
        }
    }
    if (acc == 0x5eed) *sink = acc;   // keeps the accesses
}
}  // namespace

int ra_calibrate_random_access(int device, uint64_t slots, uint64_t ops, double* out_rates)
{
    if (!out_rates || slots < 1024 || ops == 0) return RA_E_BADARG;
    if (cudaSetDevice(device) != cudaSuccess) return RA_E_CUDA;
    Slot* t = nullptr;
    u64* sink = nullptr;
    if (cudaMalloc(&t, slots * sizeof(Slot)) != cudaSuccess) return RA_E_OOM;
    if (cudaMalloc(&sink, 8) != cudaSuccess) {
        cudaFree(t);
        return RA_E_OOM;
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int st = RA_OK;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) st = RA_E_CUDA;
    for (int kind = 0; kind < 2 && st == RA_OK; kind++) {
        float best = 0;
        for (int rep = 0; rep < 3 && st == RA_OK; rep++) {
            if (cudaMemset(t, 0xff, slots * sizeof(Slot)) != cudaSuccess) st = RA_E_CUDA;
            cudaEventRecord(e0);
            calibrate_kernel<<<kSms * 8, kThreads>>>(t, slots, ops, 1000003ull * (rep + 1), kind, sink);
            cudaEventRecord(e1);
            if (cudaEventSynchronize(e1) != cudaSuccess || cudaGetLastError() != cudaSuccess) st = RA_E_CUDA;
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            if (rep == 0 || ms < best) best = ms;
        }
        out_rates[kind] = best > 0 ? (double)ops / (best / 1e3) : 0.0;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(sink);
    cudaFree(t);
    return st;
}

int ra_program_set_checkpoint(ra_program* p, const char* output_dir, uint32_t every_batches, int separate_files)
{
    return guard(p, [&] {
        if (p->running) fail(p, RA_E_STATE, "set_checkpoint during a run");
        if (every_batches && (!output_dir || !*output_dir)) fail(p, RA_E_BADARG, "checkpoint directory missing");
        p->cp_every = every_batches;
        p->cp_dir = every_batches ? std::string(output_dir) : std::string();
        p->cp_separate = separate_files != 0;
    });
}

int ra_program_set_restart(ra_program* p, const char* dump_dir, int separate_files)
{
    return guard(p, [&] {
        if (p->running) fail(p, RA_E_STATE, "set_restart during a run");
        p->rs_skip.clear();
        p->rs_dir.clear();
        if (!dump_dir || !*dump_dir) return;   // restart off
        std::string dir(dump_dir);
        while (dir.size() > 1 && dir.back() == '/') dir.pop_back();
        p->rs_dir = dir;
        p->rs_separate = separate_files != 0;
        std::ifstream meta(dir + "/scc_metadata");
        int id;
        while (meta >> id) p->rs_skip.push_back(id);
    });
}

int ra_program_get_tuning(ra_program* p, ra_tuning* out)
{
    return guard(p, [&] {
        if (!out) fail(p, RA_E_BADARG, "null tuning");
        *out = p->tune;
    });
}

int ra_program_set_tuning(ra_program* p, const ra_tuning* t)
{
    return guard(p, [&] {
        if (!t) fail(p, RA_E_BADARG, "null tuning");
        if (p->running) fail(p, RA_E_STATE, "set_tuning during a run");
        if (!(t->seen_load_max >= 0.1 && t->seen_load_max <= 0.9)) fail(p, RA_E_BADARG, "seen_load_max outside [0.1, 0.9]");
        if (!(t->seen_grow >= 1.1 && t->seen_grow <= 8.0)) fail(p, RA_E_BADARG, "seen_grow outside [1.1, 8]");
        if (!(t->log_growth >= 1.1 && t->log_growth <= 4.0)) fail(p, RA_E_BADARG, "log_growth outside [1.1, 4]");
        if (t->join_blocks_per_sm < 1 || t->join_blocks_per_sm > 16 || t->select_blocks_per_sm < 1 ||
            t->select_blocks_per_sm > 16)
            fail(p, RA_E_BADARG, "blocks per SM outside [1, 16]");
        if (!(t->dense_max_bytes >= 0.0 && t->dense_max_bytes <= 1e12)) fail(p, RA_E_BADARG, "dense_max_bytes outside [0, 1e12]");
        p->tune = *t;
    });
}

int ra_program_set_instances(ra_program* p, const uint64_t* value_base, uint32_t n_instances)
{
    return guard(p, [&] {
        if (p->running) fail(p, RA_E_STATE, "set_instances during a run");
        if (n_instances && !value_base) fail(p, RA_E_BADARG, "null value_base");
        for (uint32_t i = 1; i < n_instances; i++)
            if (value_base[i] <= value_base[i - 1]) fail(p, RA_E_BADARG, "value_base must increase strictly");
        dev_free(p, &p->dinst_base);
        dev_free(p, &p->dinst_new);
        p->inst_rows_cap = 0;
        p->inst_base_h.clear();
        p->n_inst = n_instances;
        p->inst_hist.clear();
        if (!n_instances) return;
        p->inst_base_h.assign(value_base, value_base + n_instances);
        p->inst_base_h.push_back(~0ull);
        dev_alloc(p, &p->dinst_base, n_instances + 1);
        CK(cudaMemcpyAsync(p->dinst_base, p->inst_base_h.data(), (n_instances + 1) * 8, cudaMemcpyHostToDevice,
                           p->stream));
        CK(cudaStreamSynchronize(p->stream));
    });
}

int ra_program_instance_history(ra_program* p, uint64_t* out, uint64_t cap_rows, uint64_t* rows)
{
    return guard(p, [&] {
        if (!p->n_inst) fail(p, RA_E_STATE, "no instances set");
        if (!p->inst_hist_ok) fail(p, RA_E_UNSUPPORTED, "an SCC of the run kept no per-instance counts");
        const u64 n = p->inst_hist.size() / p->n_inst;
        if (rows) *rows = n;
        if (out) std::memcpy(out, p->inst_hist.data(), std::min<u64>(cap_rows, n) * p->n_inst * 8);
    });
}

int ra_relation_instance_summary(ra_program* p, int rel, uint64_t* counts, uint64_t* digests)
{
    return guard(p, [&] {
        Relation& r = rel_at(p, rel);
        if (!p->executed) fail(p, RA_E_STATE, "summary before execute");
        if (!counts || !digests) fail(p, RA_E_BADARG, "null output");
        const u64 m = std::max<u32>(p->n_inst, 1);
        u64* acc;
        dev_alloc(p, &acc, 2 * m);
        CK(cudaMemsetAsync(acc, 0, 2 * m * 8, p->stream));
        if (p->wide) {   // one instance (a wide program declares none)
            CK(cudaMemcpyAsync(acc, &r.full_n, 8, cudaMemcpyHostToDevice, p->stream));
            if (r.full_n) {
                wide_summary_kernel<<<wide_grid(r.full_n), kThreads, 0, p->stream>>>(r.wfull, (int)r.arity + 1,
                                                                                      r.full_n, acc);
                LAUNCHED();
            }
        } else if (r.full_n) {
            const int g = grid_for((r.full_n + kSummaryRowsPerLane - 1) / kSummaryRowsPerLane);
            const u64* bs = p->n_inst ? p->dinst_base : nullptr;
            if (r.arity == 2)
                instance_summary_kernel<2><<<g, kThreads, 0, p->stream>>>(r.keys, r.full_n, 2, p->bits, bs, p->n_inst,
                                                                           acc, acc + m);
            else
                instance_summary_kernel<0><<<g, kThreads, 0, p->stream>>>(r.keys, r.full_n, (int)r.arity, p->bits, bs,
                                                                           p->n_inst, acc, acc + m);
            LAUNCHED();
        }
        CK(cudaMemcpyAsync(counts, acc, m * 8, cudaMemcpyDeviceToHost, p->stream));
        CK(cudaMemcpyAsync(digests, acc + m, m * 8, cudaMemcpyDeviceToHost, p->stream));
        CK(cudaStreamSynchronize(p->stream));
        dev_free(p, &acc);
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
        if (p->wide) {   // rows already in trie order
            const u64 m = std::min<u64>(r.full_n, cap_rows);
            if (rows_out) *rows_out = m;
            if (m && host_rows)
                CK(cudaMemcpyAsync(host_rows, r.wfull, m * (r.arity + 1) * 8, cudaMemcpyDeviceToHost, p->stream));
            CK(cudaStreamSynchronize(p->stream));
            return;
        }
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

// The scratch-free load-path entry point shares this translation unit (and its
// header-defined kernels); its static scratch array is defined in that file.
#include "ra_noalloc.cu"
