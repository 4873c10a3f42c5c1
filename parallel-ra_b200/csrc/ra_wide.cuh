// Wide tuples: programs whose tuples do not pack into one 63-bit key (arity x
// value bits > 63, e.g. the slog-generated analyses whose columns hold intern
// ids) or whose join keys exceed the CSR index.  A relation version is an array
// of rows of arity + 1 u64 (data columns, then the id) in trie order --
// lexicographic over all columns, the order in which the reference's tries
// enumerate tuples (src/relation/shmap_relation_exp.cpp:77-112).
//
// Operations are index sorts with a row comparator (bitonic networks in shared
// memory with the first key columns, or a row hash, cached beside each index;
// merge passes by binary-searched ranks for larger inputs), prefix binary
// searches (join ranges on the first jcc columns; membership on the data
// columns), and rank merges of sorted arrays.  All integer; with the small deltas
// of the generated analyses, latency-bound.
#pragma once

#include "ra_iter.cuh"

namespace ra {

constexpr int kWideMaxCols = 64;     // arity + 1 columns at most
constexpr int kWideSortTile = 1024;  // indices sorted per block before the merge passes
constexpr int kWideMaxSegs = 32;     // rules writing one relation within an SCC

// Lexicographic compare of two rows over their first `ncmp` columns: -1, 0, 1.
__device__ __forceinline__ int wide_cmp(const u64* __restrict__ a, const u64* __restrict__ b, int ncmp)
{
    for (int c = 0; c < ncmp; c++) {
        const u64 x = a[c], y = b[c];
        if (x != y) return x < y ? -1 : 1;
    }
    return 0;
}

// Strict total order on row indices: the first `ncmp` columns, then the index.
__device__ __forceinline__ bool wide_before(const u64* __restrict__ rows, int W, int ncmp, u64 i, u64 j)
{
    const int c = wide_cmp(rows + i * W, rows + j * W, ncmp);
    return c < 0 || (c == 0 && i < j);
}

// Bitonic sort of s[0..P) (P a power of two; padding holds the sentinel ~0) by
// (key[i], key2[i] when given, first ncmp columns of rows[s[i]], s[i]), by one
// block.  The keys ride along in shared memory, so a comparison reads global
// memory only when they tie: key (and key2) must be consistent with the row
// order -- the first (and second) column, or a hash for a grouping sort.
__device__ __forceinline__ void wide_block_sort(u64* s, u64* key, u64* key2, u32 P, const u64* __restrict__ rows,
                                                int W, int ncmp)
{
    for (u32 k = 2; k <= P; k <<= 1) {
        for (u32 j = k >> 1; j > 0; j >>= 1) {
            for (u32 t = threadIdx.x; t < P; t += blockDim.x) {
                const u32 partner = t ^ j;
                if (partner <= t) continue;
                const u64 a = s[t], b = s[partner];
                const u64 ka = key[t], kb = key[partner];
                const u64 ka2 = key2 ? key2[t] : 0, kb2 = key2 ? key2[partner] : 0;
                bool a_after_b;
                if (a == ~0ull) a_after_b = b != ~0ull;
                else if (b == ~0ull) a_after_b = false;
                else if (ka != kb) a_after_b = ka > kb;
                else if (ka2 != kb2) a_after_b = ka2 > kb2;
                else a_after_b = wide_before(rows, W, ncmp, b, a);
                if (a_after_b == ((t & k) == 0)) {
                    s[t] = b;
                    s[partner] = a;
                    key[t] = kb;
                    key[partner] = ka;
                    if (key2) {
                        key2[t] = kb2;
                        key2[partner] = ka2;
                    }
                }
            }
            __syncthreads();
        }
    }
}

// Tile sort: indices [tile * TILE, ...) of `n` rows, bitonic network in shared
// memory (missing entries are a sentinel that orders last).  Small inputs take
// a small tile: the network's depth grows with log^2 of the tile.
template <int TILE>
__global__ void __launch_bounds__(kThreads) wide_tile_sort_kernel(const u64* __restrict__ rows, int W, int ncmp,
                                                                  u64 n, u64* __restrict__ idx)
{
    __shared__ u64 s[TILE];
    __shared__ u64 key[TILE];
    __shared__ u64 key2[TILE];
    const u64 base = (u64)blockIdx.x * TILE;
    for (int t = threadIdx.x; t < TILE; t += kThreads) {
        const u64 g = base + t;
        s[t] = g < n ? g : ~0ull;
        key[t] = g < n ? rows[g * (u64)W] : ~0ull;
        key2[t] = (g < n && ncmp > 1) ? rows[g * (u64)W + 1] : 0;
    }
    __syncthreads();
    wide_block_sort(s, key, key2, TILE, rows, W, ncmp);
    for (int t = threadIdx.x; t < TILE; t += kThreads) {
        const u64 g = base + t;
        if (g < n) idx[g] = s[t];
    }
}

// Exclusive scan of at most kThreads * kWideScanPer values by one block; the
// total into *total (device memory: no host round trip).
constexpr int kWideScanPer = 16;
template <typename T>
__global__ void __launch_bounds__(kThreads) wide_scan_small_kernel(const T* __restrict__ in, u64 n,
                                                                   u64* __restrict__ out, u64* __restrict__ total)
{
    __shared__ u64 sm[kWarps + 1];
    const u64 base = (u64)threadIdx.x * kWideScanPer;
    u64 loc = 0;
    for (int k = 0; k < kWideScanPer; k++)
        if (base + k < n) loc += (u64)in[base + k];
    u64 agg;
    u64 ex = block_exclusive_scan(loc, sm, &agg);
    for (int k = 0; k < kWideScanPer; k++)
        if (base + k < n) {
            out[base + k] = ex;
            ex += (u64)in[base + k];
        }
    if (threadIdx.x == 0) *total = agg;
}

// One merge pass: sorted runs of length L in `in`, pairs merged into `out`.  An
// element's output position is its offset in its run plus its rank in the
// partner run (the order is strict, so the ranks of both runs interleave exactly).
__global__ void __launch_bounds__(kThreads) wide_merge_pass_kernel(const u64* __restrict__ rows, int W, int ncmp,
                                                                   u64 n, u64 L, const u64* __restrict__ in,
                                                                   u64* __restrict__ out)
{
    for (u64 p = (u64)blockIdx.x * kThreads + threadIdx.x; p < n; p += (u64)gridDim.x * kThreads) {
        const u64 start = (p / (2 * L)) * 2 * L;
        const u64 mid = min(start + L, n), end = min(start + 2 * L, n);
        const u64 v = in[p];
        const bool left = p < mid;
        u64 a = left ? mid : start, b = left ? end : mid;
        const u64 lo = a;
        while (a < b) {
            const u64 m = (a + b) >> 1;
            if (wide_before(rows, W, ncmp, in[m], v)) a = m + 1;
            else b = m;
        }
        out[start + (p - (left ? start : mid)) + (a - lo)] = v;
    }
}

// out row k = rows[idx[k]] (W columns), one thread per column value.
__global__ void __launch_bounds__(kThreads) wide_gather_kernel(const u64* __restrict__ rows, int W,
                                                               const u64* __restrict__ idx, u64 n,
                                                               u64* __restrict__ out)
{
    const u64 total = n * (u64)W;
    for (u64 e = (u64)blockIdx.x * kThreads + threadIdx.x; e < total; e += (u64)gridDim.x * kThreads) {
        const u64 k = e / (u64)W, c = e - k * (u64)W;
        out[e] = rows[idx[k] * (u64)W + c];
    }
}

// First row of `sorted` (n rows of Ws columns) whose first `ncmp` columns are not
// below `key`'s.
__device__ __forceinline__ u64 wide_lower_bound(const u64* __restrict__ sorted, int Ws, u64 n,
                                                const u64* __restrict__ key, int ncmp)
{
    u64 a = 0, b = n;
    while (a < b) {
        const u64 m = (a + b) >> 1;
        if (wide_cmp(sorted + m * (u64)Ws, key, ncmp) < 0) a = m + 1;
        else b = m;
    }
    return a;
}

__device__ __forceinline__ u64 wide_upper_bound(const u64* __restrict__ sorted, int Ws, u64 n,
                                                const u64* __restrict__ key, int ncmp)
{
    u64 a = 0, b = n;
    while (a < b) {
        const u64 m = (a + b) >> 1;
        if (wide_cmp(sorted + m * (u64)Ws, key, ncmp) <= 0) a = m + 1;
        else b = m;
    }
    return a;
}

// Does `sorted` hold a row whose first `ncmp` columns equal `key`'s
// (relation::find_in_full / find_in_delta, balanced_hash_relation.cpp:1015-1035)?
__device__ __forceinline__ bool wide_has_prefix(const u64* __restrict__ sorted, int Ws, u64 n,
                                                const u64* __restrict__ key, int ncmp)
{
    if (!n) return false;
    const u64 i = wide_lower_bound(sorted, Ws, n, key, ncmp);
    return i < n && wide_cmp(sorted + i * (u64)Ws, key, ncmp) == 0;
}

// Join ranges: per outer row, the inner rows (trie order) sharing its first jcc
// columns -- all of them when jcc is 0 (parallel_join::local_join,
// src/RA/parallel_join.cpp:157-230).
__global__ void __launch_bounds__(kThreads) wide_join_count_kernel(const u64* __restrict__ outer, int Wo, u64 no,
                                                                   const u64* __restrict__ inner, int Wi, u64 ni,
                                                                   int jcc, u64* __restrict__ lo, u64* __restrict__ cnt)
{
    for (u64 o = (u64)blockIdx.x * kThreads + threadIdx.x; o < no; o += (u64)gridDim.x * kThreads) {
        const u64* key = outer + o * (u64)Wo;
        const u64 a = jcc ? wide_lower_bound(inner, Wi, ni, key, jcc) : 0;
        const u64 b = jcc ? wide_upper_bound(inner, Wi, ni, key, jcc) : ni;
        lo[o] = a;
        cnt[o] = b - a;
    }
}

// Output column j of a rule = column src[j] of the concatenation
// (in0 row ++ in1 row[jcc..]) for a join (as_all_to_allv_{left,right}_join_buffer_helper,
// shmap_relation_exp.cpp:335-349, 403-417), or of the input row for a copy.
struct WideProj {
    int n;        // output columns
    int left;     // join: the outer rows are in0's (LEFT) or in1's (RIGHT)
    int W0, W1;   // join: in0 and in1 row widths (arity + 1)
    int jcc;
    int src[kWideMaxCols];
};

// copy_filter's predicate on columns 0 and 1 of each input row.
__global__ void __launch_bounds__(kThreads) wide_filter_kernel(const u64* __restrict__ in, int Wi, u64 n, int pred,
                                                               u32* __restrict__ keep)
{
    for (u64 r = (u64)blockIdx.x * kThreads + threadIdx.x; r < n; r += (u64)gridDim.x * kThreads) {
        const u64* row = in + r * (u64)Wi;
        keep[r] = eval_pred(pred, row[0], Wi > 1 ? row[1] : 0) ? 1u : 0u;
    }
}

// Up to kWideMaxSegs segments of a relation's candidate buffer, one per rule
// writing it, with the id base of each (the tag's intern counter when the rule runs).
struct WideSegs {
    int n;
    u64 start[kWideMaxSegs + 1];   // candidate positions; start[n] = total
    u64 win_base[kWideMaxSegs];    // winners before the segment
    u64 id_base[kWideMaxSegs];     // (tag << 46) | counter of the segment's first winner
};

// New tuples into newt rows (arity + 1 columns) in position order; a join or
// copy winner gets the next id of its rule's segment, an acopy candidate
// carries its own last column.
__global__ void __launch_bounds__(kThreads) wide_newt_kernel(const u64* __restrict__ cand, int cw, u64 n,
                                                             const u32* __restrict__ win, const u64* __restrict__ wpos,
                                                             WideSegs sg, int W, u64* __restrict__ newt)
{
    for (u64 c = (u64)blockIdx.x * kThreads + threadIdx.x; c < n; c += (u64)gridDim.x * kThreads) {
        if (!win[c]) continue;
        int q = 0;
        while (q + 1 < sg.n && c >= sg.start[q + 1]) q++;
        const u64 at = wpos[c];
        const u64* src = cand + c * (u64)cw;
        u64* dst = newt + at * (u64)W;
        for (int j = 0; j < cw; j++) dst[j] = src[j];
        if (cw < W) dst[W - 1] = sg.id_base[q] + (at - sg.win_base[q]);
    }
}

// Rank merge of two sorted arrays of W-column rows: a row of A goes before equal
// rows of B, so duplicates land next to each other.
__global__ void __launch_bounds__(kThreads) wide_merge_rows_kernel(const u64* __restrict__ A, u64 na,
                                                                   const u64* __restrict__ B, u64 nb, int W,
                                                                   u64* __restrict__ out)
{
    const u64 n = na + nb;
    for (u64 p = (u64)blockIdx.x * kThreads + threadIdx.x; p < n; p += (u64)gridDim.x * kThreads) {
        const bool fromA = p < na;
        const u64 i = fromA ? p : p - na;
        const u64* row = fromA ? A + i * (u64)W : B + i * (u64)W;
        const u64 r = fromA ? wide_lower_bound(B, W, nb, row, W) : wide_upper_bound(A, W, na, row, W);
        u64* dst = out + (i + r) * (u64)W;
        for (int j = 0; j < W; j++) dst[j] = row[j];
    }
}

// Rows equal (all columns) to their predecessor, in a sorted array.
__global__ void __launch_bounds__(kThreads) wide_dup_kernel(const u64* __restrict__ rows, int W, u64 n,
                                                            u32* __restrict__ keep, u32* __restrict__ any_dup)
{
    for (u64 k = (u64)blockIdx.x * kThreads + threadIdx.x; k < n; k += (u64)gridDim.x * kThreads) {
        const bool dup = k > 0 && wide_cmp(rows + (k - 1) * (u64)W, rows + k * (u64)W, W) == 0;
        keep[k] = dup ? 0u : 1u;
        if (dup) atomicOr(any_dup, 1u);
    }
}

// Kept rows to their scanned positions.
__global__ void __launch_bounds__(kThreads) wide_compact_kernel(const u64* __restrict__ rows, int W, u64 n,
                                                                const u32* __restrict__ keep,
                                                                const u64* __restrict__ pos, u64* __restrict__ out)
{
    for (u64 k = (u64)blockIdx.x * kThreads + threadIdx.x; k < n; k += (u64)gridDim.x * kThreads) {
        if (!keep[k]) continue;
        const u64* src = rows + k * (u64)W;
        u64* dst = out + pos[k] * (u64)W;
        for (int j = 0; j < W; j++) dst[j] = src[j];
    }
}

// Exclusive-scanned winner counts at each segment's start (the total past the
// end), i.e. the winners before each rule's candidates.
__global__ void wide_pick_kernel(const u64* __restrict__ scanned, u64 n, const u64* __restrict__ total,
                                 WideSegs sg, u64* __restrict__ out)
{
    const int q = threadIdx.x;
    if (q <= sg.n) out[q] = sg.start[q] < n ? scanned[sg.start[q]] : *total;
}

// ---------------------------------------------------------------------------
// Batched launches: one kernel per phase of an iteration for all of its small
// rules or relations (one block each, or one flattened index space), with the
// work list passed as a kernel parameter (no host-to-device copy).  Most
// iterations of a generated analysis move a few hundred tuples, so launches,
// not bytes, set their cost.
// ---------------------------------------------------------------------------
constexpr int kWideJobs = 64;          // work items per batched launch
constexpr u32 kWideBlockSort = 1024;   // rows a block sorts in shared memory
constexpr u32 kWideBlockScan = kThreads * kWideScanPer;   // rows a block counts and scans
constexpr int kWideWideBlock = 1024;   // threads of the per-relation sort kernels (no block scan)

// 64-bit hash of a row's first n columns (grouping key of the winner sorts).
__device__ __forceinline__ u64 wide_row_hash(const u64* __restrict__ row, int n)
{
    u64 h = 0x243f6a8885a308d3ull;
    for (int c = 0; c < n; c++) h = mix64(h ^ (row[c] + 0x9e3779b97f4a7c15ull * (u64)(c + 1)));
    return h;
}

__device__ __forceinline__ u32 wide_pow2(u64 n)
{
    u32 P = 2;
    while (P < n) P <<= 1;
    return P;
}

// Phase 1: per job, a join's range counts and their exclusive scan, or a
// copy_filter's pass flags and their scan; the total into *total.
struct WideCountJob {
    const u64* outer;
    const u64* inner;
    u64 no, ni;
    u64* lo;       // join: first match per outer row
    u64* cnt;      // join: matches per outer row
    u64* off;      // join: scanned counts; filter: scanned flags
    u32* keep;     // filter: pass flags
    u64* total;
    int Wo, Wi, jcc, pred;   // pred < 0: a join
};
struct WideCountBatch {
    int n;
    WideCountJob job[kWideJobs];
};

__global__ void __launch_bounds__(kThreads) wide_count_batch_kernel(const __grid_constant__ WideCountBatch b)
{
    __shared__ u64 sm[kWarps + 1];
    const WideCountJob& j = b.job[blockIdx.x];
    // the searches, one row per thread (their latencies overlap)
    for (u64 o = threadIdx.x; o < j.no; o += blockDim.x) {
        const u64* row = j.outer + o * (u64)j.Wo;
        if (j.pred < 0) {
            const u64 a = j.jcc ? wide_lower_bound(j.inner, j.Wi, j.ni, row, j.jcc) : 0;
            const u64 e = j.jcc ? wide_upper_bound(j.inner, j.Wi, j.ni, row, j.jcc) : j.ni;
            j.lo[o] = a;
            j.cnt[o] = e - a;
        } else {
            j.keep[o] = eval_pred(j.pred, row[0], j.Wo > 1 ? row[1] : 0) ? 1u : 0u;
        }
    }
    __syncthreads();
    // the scan, contiguous rows per thread
    const u64 base = (u64)threadIdx.x * kWideScanPer;
    u64 loc = 0;
    for (int k = 0; k < kWideScanPer; k++) {
        const u64 o = base + k;
        if (o >= j.no) break;
        loc += j.pred < 0 ? j.cnt[o] : (u64)j.keep[o];
    }
    u64 agg;
    u64 ex = block_exclusive_scan(loc, sm, &agg);
    for (int k = 0; k < kWideScanPer; k++) {
        const u64 o = base + k;
        if (o >= j.no) break;
        j.off[o] = ex;
        ex += j.pred < 0 ? j.cnt[o] : (u64)j.keep[o];
    }
    if (threadIdx.x == 0) *j.total = agg;
}

// Phase 2: every rule's candidates in one flattened index space.
struct WideExpandJob {
    const u64* outer;   // join: outer rows; copy: input rows
    const u64* inner;
    const u64* lo;
    const u64* off;     // join: scanned counts; filter: scanned pass flags (null for a plain copy)
    u64* dst;
    u64 no;
    u64 first;          // first flattened index of this job
    int Wi;             // copy: input width
    int n, left, W0, W1, jcc, kind;   // kind 0: join, 1: copy
    unsigned char src[kWideMaxCols];
};
struct WideExpandBatch {
    int n;
    u64 total;
    WideExpandJob job[kWideJobs];
};

__global__ void __launch_bounds__(kThreads) wide_expand_batch_kernel(const __grid_constant__ WideExpandBatch b)
{
    for (u64 g = (u64)blockIdx.x * kThreads + threadIdx.x; g < b.total; g += (u64)gridDim.x * kThreads) {
        int r = 0, hi = b.n;   // last job whose first index is <= g
        while (hi - r > 1) {
            const int m = (r + hi) >> 1;
            if (b.job[m].first <= g) r = m;
            else hi = m;
        }
        const WideExpandJob& j = b.job[r];
        const u64 c = g - j.first;
        u64* dst = j.dst + c * (u64)j.n;
        if (j.kind == 0) {
            u64 a = 0, e = j.no;
            while (a < e) {
                const u64 m = (a + e) >> 1;
                if (j.off[m] <= c) a = m + 1;
                else e = m;
            }
            const u64 o = a - 1, u = j.lo[o] + (c - j.off[o]);
            const int Wo = j.left ? j.W0 : j.W1, Wi = j.left ? j.W1 : j.W0;
            const u64* ro = j.outer + o * (u64)Wo;
            const u64* ri = j.inner + u * (u64)Wi;
            const u64* r0 = j.left ? ro : ri;
            const u64* r1 = j.left ? ri : ro;
            for (int k = 0; k < j.n; k++) {
                const int x = j.src[k];
                dst[k] = x < j.W0 ? r0[x] : r1[j.jcc + (x - j.W0)];
            }
        } else {
            u64 rin = c;
            if (j.off) {   // the c-th kept row: the last row whose scanned flag is <= c
                u64 a = 0, e = j.no;
                while (a < e) {
                    const u64 m = (a + e) >> 1;
                    if (j.off[m] <= c) a = m + 1;
                    else e = m;
                }
                rin = a - 1;
            }
            const u64* row = j.outer + rin * (u64)j.Wi;
            for (int k = 0; k < j.n; k++) dst[k] = row[j.src[k]];
        }
    }
}

// Phase 3a: per relation of at most kWideBlockSort candidates, one block sorts
// them by (row hash, row, position) and flags the first candidate of each group
// of equal ones (the group's first occurrence).
struct WideHeadJob {
    const u64* cand;
    u32* flag;
    u64 n;
    int cw;
};
struct WideHeadBatch {
    int n;
    WideHeadJob job[kWideJobs];
};

__global__ void __launch_bounds__(kWideWideBlock) wide_heads_batch_kernel(const __grid_constant__ WideHeadBatch b)
{
    __shared__ u64 s[kWideBlockSort];
    __shared__ u64 key[kWideBlockSort];
    const WideHeadJob& j = b.job[blockIdx.x];
    const u32 P = wide_pow2(j.n);
    // grouping needs equal candidates adjacent (first occurrence first), not trie
    // order: rows tie on the hash only when equal, but for a 64-bit hash collision,
    // which the row comparison then orders
    for (u32 t = threadIdx.x; t < P; t += blockDim.x) {
        s[t] = t < j.n ? t : ~0ull;
        key[t] = t < j.n ? wide_row_hash(j.cand + t * (u64)j.cw, j.cw) : ~0ull;
    }
    __syncthreads();
    wide_block_sort(s, key, nullptr, P, j.cand, j.cw, j.cw);
    for (u32 k = threadIdx.x; k < j.n; k += blockDim.x) {
        const u64 c = s[k];
        const bool h = k == 0 || key[k - 1] != key[k] ||
                       wide_cmp(j.cand + s[k - 1] * (u64)j.cw, j.cand + c * (u64)j.cw, j.cw) != 0;
        j.flag[c] = h ? 1u : 0u;
    }
}

// Heads of a larger relation, from its index sort (trie order).
__global__ void __launch_bounds__(kThreads) wide_head_flags_kernel(const u64* __restrict__ cand, int cw,
                                                                   const u64* __restrict__ idx, u64 n,
                                                                   u32* __restrict__ flag)
{
    for (u64 k = (u64)blockIdx.x * kThreads + threadIdx.x; k < n; k += (u64)gridDim.x * kThreads) {
        const u64 c = idx[k];
        flag[c] = (k == 0 || wide_cmp(cand + idx[k - 1] * (u64)cw, cand + c * (u64)cw, cw) != 0) ? 1u : 0u;
    }
}

// Phase 3b: a head loses when full or delta holds its data columns (all columns
// for acopy targets); one thread per candidate of every relation.
struct WideMemberJob {
    const u64* cand;
    const u64* full;
    const u64* delta;
    u32* flag;
    u64 n, nf, nd, first;
    int cw, W;
};
struct WideMemberBatch {
    int n;
    u64 total;
    WideMemberJob job[kWideJobs];
};

__global__ void __launch_bounds__(kThreads) wide_member_batch_kernel(const __grid_constant__ WideMemberBatch b)
{
    for (u64 g = (u64)blockIdx.x * kThreads + threadIdx.x; g < b.total; g += (u64)gridDim.x * kThreads) {
        int r = 0, hi = b.n;
        while (hi - r > 1) {
            const int m = (r + hi) >> 1;
            if (b.job[m].first <= g) r = m;
            else hi = m;
        }
        const WideMemberJob& j = b.job[r];
        const u64 c = g - j.first;
        if (!j.flag[c]) continue;
        const u64* row = j.cand + c * (u64)j.cw;
        if (wide_has_prefix(j.full, j.W, j.nf, row, j.cw) || wide_has_prefix(j.delta, j.W, j.nd, row, j.cw))
            j.flag[c] = 0u;
    }
}

// Phase 3c: per relation of at most kWideBlockScan candidates, one block scans
// the winner flags into positions and picks each rule segment's winners-before
// count (and the total at picks[kWideMaxSegs + 1]).
struct WideScanJob {
    const u32* flag;
    u64* pos;
    u64* picks;
    u64 n;
    int seg0, nseg;
};
struct WideScanBatch {
    int n;
    WideScanJob job[kWideJobs];
    u64 seg_start[2 * kWideJobs];
};

__global__ void __launch_bounds__(kThreads) wide_scan_pick_batch_kernel(const __grid_constant__ WideScanBatch b)
{
    __shared__ u64 sm[kWarps + 1];
    const WideScanJob& j = b.job[blockIdx.x];
    const u64 base = (u64)threadIdx.x * kWideScanPer;
    u64 loc = 0;
    for (int k = 0; k < kWideScanPer; k++)
        if (base + k < j.n) loc += j.flag[base + k];
    u64 agg;
    u64 ex = block_exclusive_scan(loc, sm, &agg);
    for (int k = 0; k < kWideScanPer; k++)
        if (base + k < j.n) {
            j.pos[base + k] = ex;
            ex += j.flag[base + k];
        }
    __syncthreads();   // positions visible to the picking threads
    if ((int)threadIdx.x <= j.nseg) {
        const u64 st = threadIdx.x < (u32)j.nseg ? b.seg_start[j.seg0 + threadIdx.x] : j.n;
        j.picks[threadIdx.x] = st < j.n ? j.pos[st] : agg;
    }
    if (threadIdx.x == 0) j.picks[kWideMaxSegs + 1] = agg;
}

// Phase 5: per relation of at most kWideBlockSort new tuples, one block writes
// the newt rows (ids per rule segment) into `rows`, sorts them into trie order
// and gathers them into the relation's newt.
struct WideNewtJob {
    const u64* cand;
    const u32* flag;
    const u64* pos;
    u64* rows;       // scratch: winners x W
    u64* newt;
    u64 n, winners;
    int cw, W, seg0, nseg;
};
struct WideNewtBatch {
    int n;
    WideNewtJob job[kWideJobs];
    u64 seg_start[2 * kWideJobs];
    u64 win_base[2 * kWideJobs];
    u64 id_base[2 * kWideJobs];
};

__global__ void __launch_bounds__(kWideWideBlock) wide_newt_batch_kernel(const __grid_constant__ WideNewtBatch b)
{
    __shared__ u64 s[kWideBlockSort];
    __shared__ u64 key[kWideBlockSort];
    __shared__ u64 key2[kWideBlockSort];
    const WideNewtJob& j = b.job[blockIdx.x];
    for (u64 c = threadIdx.x; c < j.n; c += blockDim.x) {
        if (!j.flag[c]) continue;
        int q = 0;
        while (q + 1 < j.nseg && c >= b.seg_start[j.seg0 + q + 1]) q++;
        const u64 at = j.pos[c];
        const u64* src = j.cand + c * (u64)j.cw;
        u64* dst = j.rows + at * (u64)j.W;
        for (int k = 0; k < j.cw; k++) dst[k] = src[k];
        if (j.cw < j.W) dst[j.W - 1] = b.id_base[j.seg0 + q] + (at - b.win_base[j.seg0 + q]);
    }
    __syncthreads();
    const u32 P = wide_pow2(j.winners);
    for (u32 t = threadIdx.x; t < P; t += blockDim.x) {
        s[t] = t < j.winners ? t : ~0ull;
        key[t] = t < j.winners ? j.rows[t * (u64)j.W] : ~0ull;
        key2[t] = t < j.winners ? j.rows[t * (u64)j.W + 1] : 0;
    }
    __syncthreads();
    wide_block_sort(s, key, key2, P, j.rows, j.W, j.W);
    const u64 total = j.winners * (u64)j.W;
    for (u64 e = threadIdx.x; e < total; e += blockDim.x) {
        const u64 k = e / (u64)j.W, c = e - k * (u64)j.W;
        j.newt[e] = j.rows[s[k] * (u64)j.W + c];
    }
}

// Phase 6: full + delta of every relation of the SCC, one flattened index space.
struct WideMergeJob {
    const u64* full;
    const u64* delta;
    u64* out;
    u64 nf, nd, first;
    int W;
};
struct WideMergeBatch {
    int n;
    u64 total;
    WideMergeJob job[kWideJobs];
};

__global__ void __launch_bounds__(kThreads) wide_merge_batch_kernel(const __grid_constant__ WideMergeBatch b)
{
    for (u64 g = (u64)blockIdx.x * kThreads + threadIdx.x; g < b.total; g += (u64)gridDim.x * kThreads) {
        int r = 0, hi = b.n;
        while (hi - r > 1) {
            const int m = (r + hi) >> 1;
            if (b.job[m].first <= g) r = m;
            else hi = m;
        }
        const WideMergeJob& j = b.job[r];
        const u64 p = g - j.first;
        const bool fromA = p < j.nf;
        const u64 i = fromA ? p : p - j.nf;
        const u64* row = fromA ? j.full + i * (u64)j.W : j.delta + i * (u64)j.W;
        const u64 rk = fromA ? wide_lower_bound(j.delta, j.W, j.nd, row, j.W) : wide_upper_bound(j.full, j.W, j.nf, row, j.W);
        u64* dst = j.out + (i + rk) * (u64)j.W;
        for (int k = 0; k < j.W; k++) dst[k] = row[k];
    }
}

// Count and digest of a relation's rows, data columns only (no instances).
__global__ void __launch_bounds__(kThreads) wide_summary_kernel(const u64* __restrict__ rows, int W, u64 n,
                                                                u64* __restrict__ acc)
{
    u64 d = 0;
    for (u64 k = (u64)blockIdx.x * kThreads + threadIdx.x; k < n; k += (u64)gridDim.x * kThreads)
        d += tuple_digest(rows + k * (u64)W, W - 1);
    for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
    if ((threadIdx.x & 31) == 0 && d) atomicAdd((unsigned long long*)&acc[1], (unsigned long long)d);
}

}  // namespace ra
