// Device primitives of the B200 engine: packed-tuple helpers, hashing,
// block/warp scans, and the LSD radix sort used to keep deltas in trie order.
//
// Tuples are packed into one u64 key: with W bits per column, column c of an
// arity-a tuple sits at bits [(a-1-c)W, (a-c)W), so numeric key order equals
// the lexicographic column order in which the reference's tries enumerate
// tuples (src/relation/shmap_relation_exp.cpp:77-112).  The intern id column
// travels beside the key as a separate u64.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace ra {

typedef unsigned long long u64;
typedef unsigned char u8;
typedef unsigned int u32;

constexpr u64 kEmpty = ~0ull;          // empty hash slot / filtered candidate
constexpr int kThreads = 256;          // block size of every engine kernel
constexpr int kWarps = kThreads / 32;

// murmur3 64-bit finaliser: spreads packed keys over the hash table.
__device__ __forceinline__ u64 mix64(u64 k)
{
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ull;
    k ^= k >> 33;
    return k;
}

__device__ __forceinline__ u64 column_of(u64 key, int arity, int col, int bits)
{
    const u64 mask = (bits >= 64) ? ~0ull : ((1ull << bits) - 1);
    return (key >> ((arity - 1 - col) * bits)) & mask;
}

__device__ __forceinline__ u32 lanemask_lt()
{
    u32 m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Inclusive warp scan of u64.
__device__ __forceinline__ u64 warp_inclusive_scan(u64 v)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        u64 t = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= d) v += t;
    }
    return v;
}

// Exclusive block scan of one u64 per thread; returns the block total in *total.
// `smem` must hold kWarps + 1 u64.
__device__ __forceinline__ u64 block_exclusive_scan(u64 v, u64* smem, u64* total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    u64 inc = warp_inclusive_scan(v);
    if (lane == 31) smem[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        u64 w = (lane < kWarps) ? smem[lane] : 0;
        u64 wi = warp_inclusive_scan(w);
        if (lane < kWarps) smem[lane] = wi - w;
        if (lane == kWarps - 1) smem[kWarps] = wi;
    }
    __syncthreads();
    u64 out = inc - v + smem[warp];
    *total = smem[kWarps];
    __syncthreads();
    return out;
}

__device__ __forceinline__ u64 block_reduce_sum(u64 v, u64* smem)
{
    u64 t;
    block_exclusive_scan(v, smem, &t);
    return t;
}

// ---------------------------------------------------------------------------
// Exclusive scan over n u64 values (three launches: chunk sums, scan of the
// sums by one block, chunk scans).  Each of the G blocks owns one contiguous
// chunk of ceil(n/G) elements.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(kThreads) scan_chunk_sums(const T* __restrict__ in, u64 n, u64 chunk,
                                                            u64* __restrict__ sums)
{
    __shared__ u64 sm[kWarps + 1];
    u64 b = (u64)blockIdx.x * chunk, e = min(n, b + chunk);
    u64 acc = 0;
    for (u64 i = b + threadIdx.x; i < e; i += kThreads) acc += (u64)in[i];
    u64 tot = block_reduce_sum(acc, sm);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

// Exclusive scan of g <= 32 * kThreads chunk sums in place; total to *total_out.
__global__ void __launch_bounds__(kThreads) scan_sums_single(u64* sums, int g, u64* total_out)
{
    __shared__ u64 sm[kWarps + 1];
    constexpr int kPer = 32;
    u64 loc[kPer];
    u64 acc = 0;
    const int base = threadIdx.x * kPer;
#pragma unroll
    for (int i = 0; i < kPer; i++) {
        loc[i] = (base + i < g) ? sums[base + i] : 0;
        acc += loc[i];
    }
    u64 tot;
    u64 ex = block_exclusive_scan(acc, sm, &tot);
#pragma unroll
    for (int i = 0; i < kPer; i++) {
        if (base + i < g) sums[base + i] = ex;
        ex += loc[i];
    }
    if (threadIdx.x == 0 && total_out) *total_out = tot;
}

template <typename T>
__global__ void __launch_bounds__(kThreads) scan_chunk_apply(const T* __restrict__ in, u64 n, u64 chunk,
                                                             const u64* __restrict__ sums, u64* __restrict__ out)
{
    __shared__ u64 sm[kWarps + 1];
    u64 b = (u64)blockIdx.x * chunk, e = min(n, b + chunk);
    u64 carry = sums[blockIdx.x];
    for (u64 t = b; t < e; t += kThreads) {
        u64 i = t + threadIdx.x;
        u64 v = (i < e) ? (u64)in[i] : 0;
        u64 tot;
        u64 ex = block_exclusive_scan(v, sm, &tot);
        if (i < e) out[i] = carry + ex;
        carry += tot;
    }
}

// ---------------------------------------------------------------------------
// LSD radix sort of (key, value) pairs by key bits [lo, hi), 8 bits per pass.
// Pass = per-block digit histograms -> exclusive scan (digit-major) ->
// stable scatter.  Within a block, elements are ranked in index order with
// warp match + per-warp digit counts, so every pass is stable.
// ---------------------------------------------------------------------------
constexpr int kRadixBits = 8;
constexpr int kRadix = 1 << kRadixBits;

__global__ void __launch_bounds__(kThreads) radix_histogram(const u64* __restrict__ keys, u64 n, u64 chunk,
                                                            int shift, u32* __restrict__ hist, int g)
{
    __shared__ u32 h[kRadix];
    for (int i = threadIdx.x; i < kRadix; i += kThreads) h[i] = 0;
    __syncthreads();
    u64 b = (u64)blockIdx.x * chunk, e = min(n, b + chunk);
    for (u64 i = b + threadIdx.x; i < e; i += kThreads)
        atomicAdd(&h[(keys[i] >> shift) & (kRadix - 1)], 1u);
    __syncthreads();
    for (int d = threadIdx.x; d < kRadix; d += kThreads) hist[(u64)d * g + blockIdx.x] = h[d];
}

__global__ void __launch_bounds__(kThreads) radix_scatter(const u64* __restrict__ kin, const u64* __restrict__ vin,
                                                          u64* __restrict__ kout, u64* __restrict__ vout, u64 n,
                                                          u64 chunk, int shift, const u64* __restrict__ offs, int g)
{
    __shared__ u64 base[kRadix];              // next output position per digit for this block
    __shared__ u32 wcount[kWarps][kRadix];    // per-warp digit counts of the current tile
    __shared__ u64 wbase[kWarps][kRadix];     // per-warp output base per digit of the current tile
    for (int d = threadIdx.x; d < kRadix; d += kThreads) base[d] = offs[(u64)d * g + blockIdx.x];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const u64 b = (u64)blockIdx.x * chunk, e = min(n, b + chunk);
    for (u64 t = b; t < e; t += kThreads) {
        for (int i = threadIdx.x; i < kWarps * kRadix; i += kThreads) (&wcount[0][0])[i] = 0;
        __syncthreads();
        const u64 i = t + threadIdx.x;
        const bool valid = i < e;
        const u64 k = valid ? kin[i] : 0, v = valid ? vin[i] : 0;
        const int d = valid ? (int)((k >> shift) & (kRadix - 1)) : (kRadix + lane);
        const u32 peers = __match_any_sync(0xffffffffu, d);
        const u32 rank = __popc(peers & lanemask_lt());
        if (valid && rank == 0) wcount[warp][d] = __popc(peers);
        __syncthreads();
        for (int dd = threadIdx.x; dd < kRadix; dd += kThreads) {
            u64 run = base[dd];
#pragma unroll
            for (int w = 0; w < kWarps; w++) {
                wbase[w][dd] = run;
                run += wcount[w][dd];
            }
            base[dd] = run;
        }
        __syncthreads();
        if (valid) {
            const u64 pos = wbase[warp][d] + rank;
            kout[pos] = k;
            vout[pos] = v;
        }
        __syncthreads();
    }
}

}  // namespace ra
