// Dense row-closure evaluation of a transitive-closure-shaped SCC.
//
// Shape: one recursive rule  R(z, x) :- R_delta(y, x), S_full(y, z)  with R and
// S binary, S fixed for the SCC, the join on column 0 of both, and the
// output keeping the outer row's column 1 -- the rule of
// tests/transitive_closure.cpp:60-68 of parallel-RA.  Row x of R (the tuples
// (., x)) then evolves on its own: iteration k adds to row x exactly
//     { z : y in delta_k(x), (y, z) in S } \ known(x),
// so every row's sequence of deltas is a breadth-first search over S from
// row x's initial delta, and iteration k of the semi-naive loop is level k of
// all rows' searches.  The evaluator keeps one bit matrix per instance (row x:
// one bit per value of x's instance) and runs each row's whole search in
// shared memory -- one CTA per row, bit sets for the known tuples, the
// frontier and the next level -- adding every level's new-tuple count to the
// per-iteration (and per-instance) totals.  The result is the same set of
// tuples, iteration by iteration, as the hash-set path produces; only the
// order in which the new tuples enter the log differs (row by row, values
// ascending).
#pragma once
#include "ra_iter.cuh"

namespace ra {

// One instance's bit matrix: `n` rows (its values, from `base`), each `words`
// u32 words long (bit c of row r: tuple (base + c, base + r) is known), rows
// contiguous from word `word_off`.
struct DenseInst {
    u64 base;
    u64 n;
    u64 words;
    u64 word_off;
};

constexpr u32 kDenseFlagLevels = 1;   // a row went deeper than the level arrays hold
constexpr u32 kDenseFlagRange = 2;    // a value outside its row's instance range
constexpr u64 kDenseMaxN = 65536;     // values per instance (3 rows of bits in shared memory)

struct DenseArgs {
    const DenseInst* inst;       // n_inst entries (1 without instances)
    const u64* inst_base;        // n_inst + 1 ascending bases for instance_of, or null (one instance)
    u32 n_inst;
    u64 rows;                    // rows 0 .. rows-1 are the values of the union
    u32* known;                  // known tuples; after the closure pass: the new ones
    u32* delta0;                 // the SCC's initial delta
    int bits;                    // packed column width
    const u64* s_keys;           // S full rows, sorted
    const u64* s_csr;            // S rows with column 0 == v: [s_csr[v], s_csr[v + 1])
    u64* row_new;                // per row: new tuples
    u64* level_total;            // per iteration: new tuples
    u64* inst_level;             // [iteration][instance] new tuples, or null
    u64 level_cap;
    u64* counters;               // [0] rows taken, [1] join candidates (S rows visited)
    u32* flags;
};

__device__ __forceinline__ u32 dense_instance(const DenseArgs& a, u64 v)
{
    return a.inst_base ? instance_of(a.inst_base, a.n_inst, v) : 0u;
}

// Bits of R's stored tuples: all of them into `known`, the delta region's also into `delta0`.
__global__ void __launch_bounds__(kThreads) dense_load_kernel(DenseArgs a, const u64* __restrict__ keys,
                                                              u64 n_full, u64 n_total)
{
    for (u64 i = (u64)blockIdx.x * kThreads + threadIdx.x; i < n_total; i += (u64)gridDim.x * kThreads) {
        const u64 k = keys[i];
        const u64 y = column_of(k, 2, 0, a.bits), x = column_of(k, 2, 1, a.bits);
        const DenseInst d = a.inst[dense_instance(a, x)];
        const u64 r = x - d.base, c = y - d.base;   // unsigned: values below the base wrap high
        if (r >= d.n || c >= d.n) {
            atomicOr(a.flags, kDenseFlagRange);
            continue;
        }
        const u64 w = d.word_off + r * d.words + (c >> 5);
        const u32 bit = 1u << (c & 31);
        atomicOr(&a.known[w], bit);
        if (i >= n_full) atomicOr(&a.delta0[w], bit);
    }
}

// One CTA per row (rows taken from a device counter): the row's whole search
// in shared memory.  Dynamic shared memory: 3 * wmax u32.
__global__ void __launch_bounds__(kThreads) dense_closure_kernel(DenseArgs a, u32 wmax)
{
    extern __shared__ u32 dsm[];
    u32* known = dsm;
    u32* frontier = dsm + wmax;
    u32* next = dsm + 2 * wmax;
    __shared__ u64 s_row;
    __shared__ u64 red[kWarps + 1];
    u64 relax = 0;
    for (;;) {
        if (threadIdx.x == 0) s_row = atomicAdd((unsigned long long*)&a.counters[0], 1ull);
        __syncthreads();
        const u64 row = s_row;
        if (row >= a.rows) break;
        const u32 inst = dense_instance(a, row);
        const DenseInst d = a.inst[inst];
        const u64 r = row - d.base;
        const u32 W = (u32)d.words;
        bool any = false;
        u32* krow = nullptr;
        if (r < d.n) {
            krow = a.known + d.word_off + r * d.words;
            const u32* drow = a.delta0 + d.word_off + r * d.words;
            for (u32 w = threadIdx.x; w < W; w += kThreads) {
                const u32 f = drow[w];
                frontier[w] = f;
                known[w] = krow[w];
                next[w] = 0;
                any |= f != 0;
            }
        }
        if (!__syncthreads_or(any)) continue;   // uniform: no initial delta in this row
        u64 level = 0, total = 0;
        for (;;) {
            for (u32 w = threadIdx.x; w < W; w += kThreads) {
                u32 f = frontier[w];
                if (!f) continue;
                frontier[w] = 0;
                while (f) {
                    const u32 b = __ffs(f) - 1;
                    f &= f - 1;
                    const u64 y = d.base + (u64)w * 32 + b;
                    const u64 s = a.s_csr[y], e = a.s_csr[y + 1];
                    relax += e - s;
                    for (u64 j = s; j < e; j++) {
                        const u64 z = column_of(a.s_keys[j], 2, 1, a.bits) - d.base;
                        if (z >= d.n) {
                            atomicOr(a.flags, kDenseFlagRange);
                            continue;
                        }
                        const u32 bit = 1u << (z & 31);
                        if (!(known[z >> 5] & bit)) atomicOr(&next[z >> 5], bit);
                    }
                }
            }
            __syncthreads();
            u64 cnt = 0;
            for (u32 w = threadIdx.x; w < W; w += kThreads) {
                const u32 nw = next[w] & ~known[w];
                next[w] = 0;
                known[w] |= nw;
                frontier[w] = nw;
                cnt += __popc(nw);
            }
            cnt = block_reduce_sum(cnt, red);   // synchronises the block
            if (cnt == 0) break;
            if (threadIdx.x == 0) {
                if (level < a.level_cap) {
                    atomicAdd((unsigned long long*)&a.level_total[level], (unsigned long long)cnt);
                    if (a.inst_level)
                        atomicAdd((unsigned long long*)&a.inst_level[level * a.n_inst + inst], (unsigned long long)cnt);
                } else {
                    atomicOr(a.flags, kDenseFlagLevels);
                }
            }
            total += cnt;
            level++;
        }
        // the row's new tuples replace its known bits in global memory
        for (u32 w = threadIdx.x; w < W; w += kThreads) krow[w] = known[w] & ~krow[w];
        if (threadIdx.x == 0) a.row_new[row] = total;
        __syncthreads();
    }
    relax = block_reduce_sum(relax, red);
    if (threadIdx.x == 0 && relax) atomicAdd((unsigned long long*)&a.counters[1], (unsigned long long)relax);
}

// New tuples of each row into the log: row by row (values ascending), within a
// row by column-0 value ascending; key (z, x), id tag_word | (id_base + position).
__global__ void __launch_bounds__(kThreads) dense_emit_kernel(DenseArgs a, const u64* __restrict__ row_off,
                                                              u64* __restrict__ keys_out, u64* __restrict__ ids_out,
                                                              u64 tag_word, u64 id_base)
{
    __shared__ u64 red[kWarps + 1];
    for (u64 row = blockIdx.x; row < a.rows; row += gridDim.x) {
        if (a.row_new[row] == 0) continue;   // uniform per block
        const DenseInst d = a.inst[dense_instance(a, row)];
        const u32* nrow = a.known + d.word_off + (row - d.base) * d.words;
        const u32 W = (u32)d.words;
        const u32 chunk = (W + kThreads - 1) / kThreads;
        const u32 w0 = min(W, threadIdx.x * chunk), w1 = min(W, w0 + chunk);
        u64 cnt = 0;
        for (u32 w = w0; w < w1; w++) cnt += __popc(nrow[w]);
        u64 tot;
        u64 pos = row_off[row] + block_exclusive_scan(cnt, red, &tot);
        for (u32 w = w0; w < w1; w++) {
            u32 f = nrow[w];
            while (f) {
                const u32 b = __ffs(f) - 1;
                f &= f - 1;
                const u64 z = d.base + (u64)w * 32 + b;
                keys_out[pos] = (z << a.bits) | row;
                ids_out[pos] = tag_word | (id_base + pos);
                pos++;
            }
        }
    }
}

}  // namespace ra
