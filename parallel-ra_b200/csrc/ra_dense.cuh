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
    u32* s_local;                // per S row: column 1 minus the instance base of its column 0
    u64* row_new;                // per row: new tuples
    u64* level_total;            // per iteration: new tuples
    u64* inst_level;             // [iteration][instance] new tuples, or null
    u64 level_cap;
    u64* inst_init;              // per instance: tuples of the initial delta
    u64* counters;               // [0], [2..4] chunks taken (per kernel shape), [1] join candidates (S rows visited),
                                 // [5] 1 + the first key found outside its instance, [6] its relation (1: R, 2: S)
    u32* flags;
};

__device__ __forceinline__ u32 dense_instance(const DenseArgs& a, u64 v)
{
    return a.inst_base ? instance_of(a.inst_base, a.n_inst, v) : 0u;
}

// A key with a value outside its row's instance: flag the run, keep the first such key.
__device__ __forceinline__ void dense_range_error(const DenseArgs& a, u64 key, u64 which)
{
    atomicOr(a.flags, kDenseFlagRange);
    if (atomicCAS((unsigned long long*)&a.counters[5], 0ull, (unsigned long long)(key + 1)) == 0ull)
        atomicExch((unsigned long long*)&a.counters[6], (unsigned long long)which);
}

// Bits of R's stored tuples: all of them into `known`, the delta region's also into `delta0`.
__global__ void __launch_bounds__(kThreads) dense_load_kernel(DenseArgs a, const u64* __restrict__ keys,
                                                              u64 n_full, u64 n_total)
{
    for (u64 i = (u64)blockIdx.x * kThreads + threadIdx.x; i < n_total; i += (u64)gridDim.x * kThreads) {
        const u64 k = keys[i];
        const u64 y = column_of(k, 2, 0, a.bits), x = column_of(k, 2, 1, a.bits);
        const u32 inst = dense_instance(a, x);
        const DenseInst d = a.inst[inst];
        const u64 r = x - d.base, c = y - d.base;   // unsigned: values below the base wrap high
        if (r >= d.n || c >= d.n) {
            dense_range_error(a, k, 1);
            continue;
        }
        const u64 w = d.word_off + r * d.words + (c >> 5);
        const u32 bit = 1u << (c & 31);
        atomicOr(&a.known[w], bit);
        if (i >= n_full) {
            atomicOr(&a.delta0[w], bit);
            atomicAdd((unsigned long long*)&a.inst_init[inst], 1ull);
        }
    }
}

// S's column 1 as instance-local values, once per SCC (the search's inner loop
// then reads 4 bytes per edge and compares once); a value outside its row's
// instance is stored as 0xffffffff, which the search rejects.
__global__ void __launch_bounds__(kThreads) dense_local_kernel(DenseArgs a, u64 n)
{
    for (u64 j = (u64)blockIdx.x * kThreads + threadIdx.x; j < n; j += (u64)gridDim.x * kThreads) {
        const u64 k = a.s_keys[j];
        const u64 y = column_of(k, 2, 0, a.bits), z = column_of(k, 2, 1, a.bits);
        const DenseInst d = a.inst[dense_instance(a, y)];
        const u64 zl = z - d.base;
        if (zl >= d.n || y - d.base >= d.n) {
            a.s_local[j] = 0xffffffffu;
            dense_range_error(a, k, 2);
        } else {
            a.s_local[j] = (u32)zl;
        }
    }
}

// Work unit of the searches: `count` consecutive rows of one instance.
struct DenseChunk {
    u64 first_row;
    u32 inst;
    u32 count;
};

constexpr u32 kDenseWarpWords = 512;  // instances of at most 16384 values: one warp per row
constexpr int kDenseLevels = 64;      // levels counted in shared memory per chunk (deeper ones directly)

// A level's new-tuple count of a row: into the chunk's shared counters, or
// (beyond kDenseLevels) straight into the per-iteration totals.
__device__ __forceinline__ void dense_count_level(const DenseArgs& a, u64* lvl, u64 level, u32 inst, u64 cnt)
{
    if (level < (u64)kDenseLevels) {
        lvl[level] += cnt;
    } else if (level < a.level_cap) {
        atomicAdd((unsigned long long*)&a.level_total[level], (unsigned long long)cnt);
        if (a.inst_level)
            atomicAdd((unsigned long long*)&a.inst_level[level * a.n_inst + inst], (unsigned long long)cnt);
    } else {
        atomicOr(a.flags, kDenseFlagLevels);
    }
}

__device__ __forceinline__ void dense_flush_levels(const DenseArgs& a, u64* lvl, u32 inst, int from, int step)
{
    for (int i = from; i < kDenseLevels; i += step) {
        const u64 v = lvl[i];
        if (!v) continue;
        lvl[i] = 0;
        if ((u64)i < a.level_cap) {
            atomicAdd((unsigned long long*)&a.level_total[i], (unsigned long long)v);
            if (a.inst_level) atomicAdd((unsigned long long*)&a.inst_level[(u64)i * a.n_inst + inst], (unsigned long long)v);
        } else {
            atomicOr(a.flags, kDenseFlagLevels);
        }
    }
}

// Rows of instances with more than kDenseWarpWords words: one CTA per row,
// chunks taken from a device counter; the row's whole search in shared
// memory.  Dynamic shared memory: 3 * wmax u32.
__global__ void __launch_bounds__(kThreads) dense_closure_kernel(DenseArgs a, u32 wmax, const DenseChunk* __restrict__ chunks,
                                                                 u64 n_chunks, u64* __restrict__ chunk_ctr)
{
    extern __shared__ u32 dsm[];
    u32* known = dsm;
    u32* frontier = dsm + wmax;
    u32* next = dsm + 2 * wmax;
    __shared__ u64 s_chunk;
    __shared__ u64 red[kWarps + 1];
    __shared__ u64 lvl[kDenseLevels];
    for (int i = threadIdx.x; i < kDenseLevels; i += kThreads) lvl[i] = 0;
    u64 relax = 0;
    for (;;) {
        if (threadIdx.x == 0) s_chunk = atomicAdd((unsigned long long*)chunk_ctr, 1ull);
        __syncthreads();
        const u64 c = s_chunk;
        if (c >= n_chunks) break;
        const DenseChunk ch = chunks[c];
        const DenseInst d = a.inst[ch.inst];
        const u32 W = (u32)d.words;
        for (u32 k = 0; k < ch.count; k++) {
            const u64 row = ch.first_row + k;
            u32* krow = a.known + d.word_off + (row - d.base) * d.words;
            const u32* drow = a.delta0 + d.word_off + (row - d.base) * d.words;
            bool any = false;
            for (u32 w = threadIdx.x; w < W; w += kThreads) {
                const u32 f = drow[w];
                frontier[w] = f;
                known[w] = krow[w];
                next[w] = 0;
                any |= f != 0;
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
                            const u32 z = a.s_local[j];
                            if (z >= (u32)d.n) continue;   // flagged by dense_local_kernel
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
                if (threadIdx.x == 0) dense_count_level(a, lvl, level, ch.inst, cnt);
                total += cnt;
                level++;
            }
            // the row's new tuples replace its known bits in global memory
            for (u32 w = threadIdx.x; w < W; w += kThreads) krow[w] = known[w] & ~krow[w];
            if (threadIdx.x == 0) a.row_new[row] = total;
            __syncthreads();
        }
        dense_flush_levels(a, lvl, ch.inst, threadIdx.x, kThreads);
        __syncthreads();
    }
    relax = block_reduce_sum(relax, red);
    if (threadIdx.x == 0 && relax) atomicAdd((unsigned long long*)&a.counters[1], (unsigned long long)relax);
}

// Rows of instances of at most 32 * MW words (MW * 1024 values): one warp per
// row, lane l owning words l, l + 32, ... (its frontier words in registers,
// the row's known and next-level bits in the warp's shared memory); no block
// barriers, so rows with small searches cost little.  Chunks are taken per
// warp from a device counter.
template <int MW>
__global__ void __launch_bounds__(kThreads) dense_closure_warp_kernel(DenseArgs a, const DenseChunk* __restrict__ chunks,
                                                                      u64 n_chunks, u64* __restrict__ chunk_ctr)
{
    constexpr int WW = 32 * MW;   // words a warp's row may have
    __shared__ u32 s_known[kWarps][WW];
    __shared__ u32 s_next[kWarps][WW];
    __shared__ u64 s_lvl[kWarps][kDenseLevels];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    u32* known = s_known[warp];
    u32* next = s_next[warp];
    u64* lvl = s_lvl[warp];
    for (int i = lane; i < kDenseLevels; i += 32) lvl[i] = 0;
    u64 relax = 0;
    for (;;) {
        u64 c = 0;
        if (lane == 0) c = atomicAdd((unsigned long long*)chunk_ctr, 1ull);
        c = __shfl_sync(0xffffffffu, c, 0);
        if (c >= n_chunks) break;
        const DenseChunk ch = chunks[c];
        const DenseInst d = a.inst[ch.inst];
        const u32 W = (u32)d.words;   // <= WW by the host's dispatch
        for (u32 k = 0; k < ch.count; k++) {
            const u64 row = ch.first_row + k;
            u32* krow = a.known + d.word_off + (row - d.base) * d.words;
            const u32* drow = a.delta0 + d.word_off + (row - d.base) * d.words;
            u32 fr[MW];
            bool any = false;
#pragma unroll
            for (int q = 0; q < MW; q++) {
                const u32 w = (u32)(q * 32 + lane);
                fr[q] = 0;
                if (w < W) {
                    known[w] = krow[w];
                    next[w] = 0;
                    fr[q] = drow[w];
                    any |= fr[q] != 0;
                }
            }
            __syncwarp();
            if (!__any_sync(0xffffffffu, any)) continue;
            u64 level = 0, total = 0;
            for (;;) {
#pragma unroll
                for (int q = 0; q < MW; q++) {
                    u32 f = fr[q];
                    const u64 w = (u64)(q * 32 + lane);
                    while (f) {
                        const u32 b = __ffs(f) - 1;
                        f &= f - 1;
                        const u64 y = d.base + w * 32 + b;
                        const u64 s = a.s_csr[y], e = a.s_csr[y + 1];
                        relax += e - s;
                        for (u64 j = s; j < e; j++) {
                            const u32 z = a.s_local[j];
                            if (z >= (u32)d.n) continue;   // flagged by dense_local_kernel
                            const u32 bit = 1u << (z & 31);
                            if (!(known[z >> 5] & bit)) atomicOr(&next[z >> 5], bit);
                        }
                    }
                }
                __syncwarp();
                u32 cnt = 0;
#pragma unroll
                for (int q = 0; q < MW; q++) {
                    const u32 w = (u32)(q * 32 + lane);
                    fr[q] = 0;
                    if (w < W) {
                        const u32 nw = next[w] & ~known[w];
                        next[w] = 0;
                        known[w] |= nw;
                        fr[q] = nw;
                        cnt += __popc(nw);
                    }
                }
                cnt = __reduce_add_sync(0xffffffffu, cnt);
                __syncwarp();
                if (cnt == 0) break;
                if (lane == 0) dense_count_level(a, lvl, level, ch.inst, cnt);
                total += cnt;
                level++;
            }
            // the row's new tuples replace its known bits in global memory
#pragma unroll
            for (int q = 0; q < MW; q++) {
                const u32 w = (u32)(q * 32 + lane);
                if (w < W) krow[w] = known[w] & ~krow[w];
            }
            if (lane == 0) a.row_new[row] = total;
            __syncwarp();
        }
        __syncwarp();
        dense_flush_levels(a, lvl, ch.inst, lane, 32);
        __syncwarp();
    }
    for (int o = 16; o > 0; o >>= 1) relax += __shfl_xor_sync(0xffffffffu, relax, o);
    if (lane == 0 && relax) atomicAdd((unsigned long long*)&a.counters[1], (unsigned long long)relax);
}

// New tuples of each row into the log: row by row (values ascending), within a
// row by column-0 value ascending; key (z, x), id tag_word | (id_base + position).
// One warp per row: it takes the row's words 32 at a time, scans their bit
// counts, and lane t writes output t, t + 32, ... of the group -- consecutive
// lanes write consecutive rows of the log (coalesced); a lane finds the word
// holding its output by a binary search over the lanes' inclusive counts and
// the bit by its rank within the word.
__global__ void __launch_bounds__(kThreads) dense_emit_kernel(DenseArgs a, const u64* __restrict__ row_off,
                                                              u64* __restrict__ keys_out, u64* __restrict__ ids_out,
                                                              u64 tag_word, u64 id_base)
{
    const int lane = threadIdx.x & 31;
    const u64 warps = (u64)gridDim.x * (kThreads / 32);
    for (u64 row = (u64)blockIdx.x * (kThreads / 32) + (threadIdx.x >> 5); row < a.rows; row += warps) {
        if (a.row_new[row] == 0) continue;   // uniform per warp
        const DenseInst d = a.inst[dense_instance(a, row)];
        const u32* nrow = a.known + d.word_off + (row - d.base) * d.words;
        const u32 W = (u32)d.words;
        u64 pos = row_off[row];
        for (u32 g = 0; g < W; g += 32) {
            const u32 word = (g + lane < W) ? nrow[g + lane] : 0u;
            const u32 c = __popc(word);
            u32 incl = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const u32 t = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += t;
            }
            const u32 group = __shfl_sync(0xffffffffu, incl, 31);
            for (u32 t0 = 0; t0 < group; t0 += 32) {
                const u32 t = t0 + lane;
                // first lane j with incl_j > t (every lane joins the shuffles)
                u32 lo = 0, hi = 31;
#pragma unroll
                for (int step = 0; step < 5; step++) {
                    const u32 mid = (lo + hi) >> 1;
                    const u32 im = __shfl_sync(0xffffffffu, incl, mid);
                    if (im > t) hi = mid;
                    else lo = mid + 1;
                }
                const u32 wj = __shfl_sync(0xffffffffu, word, lo);
                const u32 before = __shfl_sync(0xffffffffu, incl - c, lo);
                if (t < group) {
                    const u32 bit = __fns(wj, 0, (int)(t - before) + 1);
                    const u64 z = d.base + (u64)(g + lo) * 32 + bit;
                    const u64 at = pos + t;
                    keys_out[at] = (z << a.bits) | row;
                    ids_out[at] = tag_word | (id_base + at);
                }
            }
            pos += group;
        }
    }
}

}  // namespace ra
