// Engine kernels: loading, inner-relation index, join / copy expansion and
// the hash-set dedup that replaces the reference's find_in_full/delta/newt +
// insert_in_newt (src/RAM/RA_tasks.cpp:824-905).
#pragma once
#include "ra_device.cuh"

namespace ra {

// ---------------------------------------------------------------------------
// Rule projection: output column j takes column `col[j]` of side `side[j]`
// (0 = the outer row, 1 = the inner row).  Built on the host from the
// reference's reorder/projection index lists (src/RA/parallel_join.h:34-51).
// ---------------------------------------------------------------------------
constexpr int kMaxArity = 8;
struct Projection {
    int n;                    // output arity
    int outer_arity, inner_arity;
    signed char side[kMaxArity];
    signed char col[kMaxArity];
};

__device__ __forceinline__ u64 project(const Projection& pj, u64 outer, u64 inner, int bits)
{
    u64 key = 0;
#pragma unroll
    for (int j = 0; j < kMaxArity; j++) {
        if (j >= pj.n) break;
        u64 v = pj.side[j] ? column_of(inner, pj.inner_arity, pj.col[j], bits)
                           : column_of(outer, pj.outer_arity, pj.col[j], bits);
        key = (bits >= 64) ? v : ((key << bits) | v);
    }
    return key;
}

// ---------------------------------------------------------------------------
// Loading: rows of (arity + 1) u64 -> max data value (for the column width),
// then packed keys + ids.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) rows_max_value(const u64* __restrict__ rows, u64 n, int arity,
                                                           u64* __restrict__ max_out)
{
    __shared__ u64 sm[kWarps + 1];
    u64 m = 0;
    const int w = arity + 1;
    for (u64 i = (u64)blockIdx.x * kThreads + threadIdx.x; i < n; i += (u64)gridDim.x * kThreads)
        for (int c = 0; c < arity; c++) m = max(m, rows[i * w + c]);
    // block max via warp shuffles
    for (int d = 16; d > 0; d >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, d));
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        u64 b = 0;
        for (int i = 0; i < kWarps; i++) b = max(b, sm[i]);
        atomicMax(max_out, b);
    }
}

__global__ void __launch_bounds__(kThreads) rows_pack(const u64* __restrict__ rows, u64 n, int arity, int bits,
                                                      u64* __restrict__ keys, u64* __restrict__ ids)
{
    const int w = arity + 1;
    for (u64 i = (u64)blockIdx.x * kThreads + threadIdx.x; i < n; i += (u64)gridDim.x * kThreads) {
        u64 k = 0;
        for (int c = 0; c < arity; c++) k = (k << bits) | rows[i * w + c];
        keys[i] = k;
        ids[i] = rows[i * w + arity];
    }
}

__global__ void __launch_bounds__(kThreads) rows_unpack(const u64* __restrict__ keys, const u64* __restrict__ ids,
                                                        u64 n, int arity, int bits, u64* __restrict__ rows)
{
    const int w = arity + 1;
    for (u64 i = (u64)blockIdx.x * kThreads + threadIdx.x; i < n; i += (u64)gridDim.x * kThreads) {
        u64 k = keys[i];
        for (int c = 0; c < arity; c++) rows[i * w + c] = column_of(k, arity, c, bits);
        rows[i * w + arity] = ids[i];
    }
}

// After sorting by (key, id): flag[i] = 1 unless row i repeats row i-1 exactly
// (relation::populate_full inserts all arity+1 columns into a set,
// src/relation/balanced_hash_relation.cpp:773-793).
__global__ void __launch_bounds__(kThreads) flag_distinct_rows(const u64* __restrict__ keys, const u64* __restrict__ ids,
                                                               u64 n, u32* __restrict__ flag)
{
    for (u64 i = (u64)blockIdx.x * kThreads + threadIdx.x; i < n; i += (u64)gridDim.x * kThreads)
        flag[i] = (i == 0 || keys[i] != keys[i - 1] || ids[i] != ids[i - 1]) ? 1u : 0u;
}

// 1 when some adjacent pair of sorted keys is equal (ids must then be ordered too).
__global__ void __launch_bounds__(kThreads) any_equal_adjacent(const u64* __restrict__ keys, u64 n, u32* __restrict__ out)
{
    for (u64 i = (u64)blockIdx.x * kThreads + threadIdx.x + 1; i < n; i += (u64)gridDim.x * kThreads)
        if (keys[i] == keys[i - 1]) *out = 1u;
}

__global__ void __launch_bounds__(kThreads) compact_flagged(const u64* __restrict__ kin, const u64* __restrict__ vin,
                                                            const u32* __restrict__ flag, const u64* __restrict__ pos,
                                                            u64 n, u64* __restrict__ kout, u64* __restrict__ vout)
{
    for (u64 i = (u64)blockIdx.x * kThreads + threadIdx.x; i < n; i += (u64)gridDim.x * kThreads)
        if (flag[i]) {
            kout[pos[i]] = kin[i];
            vout[pos[i]] = vin[i];
        }
}

// ---------------------------------------------------------------------------
// Inner index: CSR offsets over the join key (first jcc columns) of a relation
// sorted by key.  offsets has 2^(jcc*W) + 1 entries; rows with join key j are
// [offsets[j], offsets[j+1]).  Replaces descending the B-tree trie by the join
// prefix (src/relation/shmap_relation_exp.cpp:393-401).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) csr_count(const u64* __restrict__ keys, u64 n, int shift,
                                                      u32* __restrict__ counts)
{
    for (u64 i = (u64)blockIdx.x * kThreads + threadIdx.x; i < n; i += (u64)gridDim.x * kThreads)
        atomicAdd(&counts[keys[i] >> shift], 1u);
}

// The longest CSR row (most rows sharing one join key), stored after the offsets:
// the fused join reads it to skip its skewed-key machinery when no row can be heavy.
__global__ void __launch_bounds__(kThreads) csr_row_max(const u32* __restrict__ counts, u64 n,
                                                        unsigned long long* __restrict__ out)
{
    u32 m = 0;
    for (u64 i = (u64)blockIdx.x * kThreads + threadIdx.x; i < n; i += (u64)gridDim.x * kThreads)
        m = max(m, counts[i]);
    for (int d = 16; d > 0; d >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, d));
    if ((threadIdx.x & 31) == 0 && m) atomicMax(out, (unsigned long long)m);
}

// ---------------------------------------------------------------------------
// Join expansion.  Outer rows in trie order; for outer row i the matches are
// inner rows [start, start+cnt).  cnt[i] feeds an exclusive scan giving each
// row's first output slot, so candidate order = (outer row, inner row) order,
// the emission order of parallel_join::local_join (src/RA/parallel_join.cpp:157-230).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) join_count(const u64* __restrict__ outer, u64 n_outer, int outer_shift,
                                                       const u64* __restrict__ csr, u64* __restrict__ cnt)
{
    for (u64 i = (u64)blockIdx.x * kThreads + threadIdx.x; i < n_outer; i += (u64)gridDim.x * kThreads) {
        u64 j = outer[i] >> outer_shift;
        cnt[i] = csr[j + 1] - csr[j];
    }
}

__global__ void __launch_bounds__(kThreads) join_expand(const u64* __restrict__ outer, u64 n_outer, int outer_shift,
                                                        const u64* __restrict__ csr, const u64* __restrict__ inner,
                                                        const u64* __restrict__ off, Projection pj, int bits,
                                                        u64* __restrict__ cand)
{
    for (u64 i = (u64)blockIdx.x * kThreads + threadIdx.x; i < n_outer; i += (u64)gridDim.x * kThreads) {
        const u64 o = outer[i];
        const u64 j = o >> outer_shift;
        const u64 s = csr[j], e = csr[j + 1];
        u64 w = off[i];
        for (u64 r = s; r < e; r++) cand[w++] = project(pj, o, inner[r], bits);
    }
}

// ---------------------------------------------------------------------------
// Copy / copy_filter expansion: one candidate per input row (kEmpty when the
// predicate rejects it).  Predicates see input columns 0 and 1 only, as the
// reference's filter lambda does (src/relation/shmap_relation_exp.cpp:233-236).
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool eval_pred(int pred, u64 a, u64 b)
{
    switch (pred) {
    case 0: return true;
    case 1: return false;
    case 2: return a == b;
    case 3: return a != b;
    case 4: return a < b;
    case 5: return a > b;
    case 6: return a <= b;
    case 7: return a >= b;
    }
    return false;
}

__global__ void __launch_bounds__(kThreads) copy_expand(const u64* __restrict__ in, u64 n, Projection pj, int bits,
                                                        int pred, u64* __restrict__ cand)
{
    for (u64 i = (u64)blockIdx.x * kThreads + threadIdx.x; i < n; i += (u64)gridDim.x * kThreads) {
        const u64 k = in[i];
        bool keep = true;
        if (pred != 0) {
            u64 a = column_of(k, pj.outer_arity, 0, bits);
            u64 b = pj.outer_arity > 1 ? column_of(k, pj.outer_arity, 1, bits) : 0;
            keep = eval_pred(pred, a, b);
        }
        cand[i] = keep ? project(pj, k, 0, bits) : kEmpty;
    }
}

// ---------------------------------------------------------------------------
// Seen set: open-addressing table over the packed data columns of every tuple
// the relation has ever held (full u delta u newt -- relations only grow).
// A slot's tag is 0 for tuples older than the running iteration and
// (epoch << 40 | position) for tuples first produced in it; the minimum
// position among equal candidates marks the first occurrence, which is the
// tuple the reference inserts (and interns) first.
// ---------------------------------------------------------------------------
struct alignas(16) Slot {
    u64 key;
    u64 tag;
};
__device__ __forceinline__ bool slot_eq(const Slot& a, const Slot& b) { return a.key == b.key && a.tag == b.tag; }

// A seen set has `cap` slots, any count: a key's probe run starts at
// floor(mix64(k) * cap / 2^64) (multiplicative range reduction, so the table
// needs no power-of-two size and its load factor is exactly what the host
// sized it for) and steps linearly, wrapping at cap.
__device__ __forceinline__ u64 slot_start(u64 k, u64 cap) { return __umul64hi(mix64(k), cap); }
__device__ __forceinline__ u64 slot_next(u64 h, u64 cap) { return h + 1 == cap ? 0 : h + 1; }

// Returns the slot holding k (inserting it if absent), or ~0 if the table is full.
__device__ __forceinline__ u64 seen_find_or_insert(Slot* __restrict__ t, u64 cap, u64 k)
{
    u64 h = slot_start(k, cap);
    for (u64 probe = 0; probe < cap; probe++) {
        u64 cur = *((volatile u64*)&t[h].key);
        if (cur == k) return h;
        if (cur == kEmpty) {
            u64 prev = atomicCAS(&t[h].key, kEmpty, k);
            if (prev == kEmpty || prev == k) return h;
            continue;   // lost the slot to another key: re-examine nothing, move on
        }
        h = slot_next(h, cap);
    }
    return ~0ull;
}

__device__ __forceinline__ u64 seen_find(const Slot* __restrict__ t, u64 cap, u64 k)
{
    u64 h = slot_start(k, cap);
    for (u64 probe = 0; probe < cap; probe++) {
        u64 cur = t[h].key;
        if (cur == k) return h;
        if (cur == kEmpty) return ~0ull;
        h = slot_next(h, cap);
    }
    return ~0ull;
}

// Insert existing tuples with tag 0 (seen before any running iteration).
__global__ void __launch_bounds__(kThreads) seen_insert_existing(Slot* __restrict__ t, u64 cap,
                                                                 const u64* __restrict__ keys, u64 n,
                                                                 u32* __restrict__ err)
{
    for (u64 i = (u64)blockIdx.x * kThreads + threadIdx.x; i < n; i += (u64)gridDim.x * kThreads) {
        u64 h = seen_find_or_insert(t, cap, keys[i]);
        if (h == ~0ull) { *err = 1u; continue; }
        atomicMin(&t[h].tag, 0ull);
    }
}

// Candidate p (global stream position base + i) claims the first occurrence of its key.
__global__ void __launch_bounds__(kThreads) dedup_insert(Slot* __restrict__ t, u64 cap, const u64* __restrict__ cand,
                                                         u64 n, u64 tag_base, u32* __restrict__ err)
{
    for (u64 i = (u64)blockIdx.x * kThreads + threadIdx.x; i < n; i += (u64)gridDim.x * kThreads) {
        const u64 k = cand[i];
        if (k == kEmpty) continue;
        u64 h = seen_find_or_insert(t, cap, k);
        if (h == ~0ull) { *err = 1u; continue; }
        const u64 mine = tag_base + i;
        if (t[h].tag > mine) atomicMin(&t[h].tag, mine);
    }
}

// flag[i] = 1 when candidate i is the first occurrence of a tuple new to the relation.
__global__ void __launch_bounds__(kThreads) dedup_flag(const Slot* __restrict__ t, u64 cap, const u64* __restrict__ cand,
                                                       u64 n, u64 tag_base, u32* __restrict__ flag)
{
    for (u64 i = (u64)blockIdx.x * kThreads + threadIdx.x; i < n; i += (u64)gridDim.x * kThreads) {
        const u64 k = cand[i];
        u32 f = 0;
        if (k != kEmpty) {
            u64 h = seen_find(t, cap, k);
            f = (h != ~0ull && t[h].tag == tag_base + i) ? 1u : 0u;
        }
        flag[i] = f;
    }
}

// Winners -> newt rows with fresh intern ids (tag << 46 | counter), in
// candidate order (src/RAM/RA_tasks.cpp:861-875 at one bucket).
__global__ void __launch_bounds__(kThreads) dedup_compact(const u64* __restrict__ cand, const u32* __restrict__ flag,
                                                          const u64* __restrict__ rank, u64 n, u64 id_base,
                                                          u64* __restrict__ out_keys, u64* __restrict__ out_ids)
{
    for (u64 i = (u64)blockIdx.x * kThreads + threadIdx.x; i < n; i += (u64)gridDim.x * kThreads)
        if (flag[i]) {
            const u64 r = rank[i];
            out_keys[r] = cand[i];
            out_ids[r] = id_base + r;
        }
}

}  // namespace ra
