// ra_rows_distinct_noalloc: the load-time "sort rows, drop exact duplicates"
// step of relation loading (what ra_relation_load_rows + ra_program_execute +
// ra_relation_dump_full produce for a relation's full version), for callers
// that must not allocate device memory.
//
// Who cannot allocate: code that runs while an application owns all device
// memory up front (serving runtimes that reserve the GPU in a fixed arena and
// treat any further cudaMalloc as a fault), code on latency-critical threads
// where cudaMalloc/cudaFree's implicit device synchronisation is not
// acceptable, and plug-ins whose host forbids the CUDA allocator outright.
//
// Compiled as part of ra_engine.cu's translation unit (included at its end).
// All scratch lives in one file-scope __device__ array of fixed size
// (kNoallocBytes below); every GPU that loads this library keeps that much
// memory reserved until the process exits.  The entry point launches kernels,
// memsets, copies and one stream synchronisation (to read the largest value,
// which sets the packing width) -- nothing that allocates.
#include "../../include/ra_engine.h"
#include "ra_kernels.cuh"

#include <utility>

using namespace ra;

namespace {

constexpr u64 kMaxRows = RA_NOALLOC_MAX_ROWS;
constexpr int kMaxBlocks = 128;                 // grid of the chunked sort / scan kernels

// scratch layout (u64 words)
constexpr u64 kOffKA = 0;                       // keys, ping
constexpr u64 kOffVA = kOffKA + kMaxRows;       // ids, ping
constexpr u64 kOffKB = kOffVA + kMaxRows;       // keys, pong
constexpr u64 kOffVB = kOffKB + kMaxRows;       // ids, pong
constexpr u64 kOffRank = kOffVB + kMaxRows;     // output slot of each distinct row
constexpr u64 kOffFlag = kOffRank + kMaxRows;   // u32 flags (kMaxRows / 2 words)
constexpr u64 kOffHist = kOffFlag + kMaxRows / 2;             // u32 digit counts (kRadix * kMaxBlocks / 2 words)
constexpr u64 kOffHistOff = kOffHist + kRadix * kMaxBlocks / 2;   // u64 digit offsets
constexpr u64 kOffSums = kOffHistOff + (u64)kRadix * kMaxBlocks;  // scan block sums (32 * kThreads)
constexpr u64 kOffScalar = kOffSums + 32 * kThreads;              // [0] scan total, [1] max value, [2] any-equal
constexpr u64 kWords = kOffScalar + 8;
constexpr u64 kNoallocBytes = kWords * 8;   // about 6 MB
static_assert(kNoallocBytes < (7u << 20), "no-alloc scratch stays modest");

// The scratch.  Host code must not use this name as an address: its device
// address comes from cudaGetSymbolAddress (see scratch_for).
static __device__ __align__(256) u64 g_noalloc_scratch[kWords];

// Device address of the scratch in the calling thread's current context.  Looked
// up on every call (the lookup allocates nothing), so an address never outlives
// the context it belongs to -- a device reset or another context on the same
// device gets its own.
int scratch_for(u64** out)
{
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return RA_E_CUDA;
    *out = (u64*)p;
    return RA_OK;
}

// rows_unpack for a row count that stays on the device
__global__ void __launch_bounds__(kThreads) unpack_counted_kernel(const u64* __restrict__ keys,
                                                                  const u64* __restrict__ ids,
                                                                  const u64* __restrict__ count, int arity, int bits,
                                                                  u64* __restrict__ rows)
{
    const u64 n = *count;
    const int w = arity + 1;
    for (u64 i = (u64)blockIdx.x * kThreads + threadIdx.x; i < n; i += (u64)gridDim.x * kThreads) {
        const u64 k = keys[i];
        for (int c = 0; c < arity; c++) rows[i * w + c] = column_of(k, arity, c, bits);
        rows[i * w + arity] = ids[i];
    }
}

int blocks_for(u64 n)
{
    u64 g = (n + kThreads - 1) / kThreads;
    if (g < 1) g = 1;
    if (g > (u64)kMaxBlocks) g = kMaxBlocks;
    return (int)g;
}

__global__ void copy_count_kernel(const u64* __restrict__ total, u64* __restrict__ out) { *out = *total; }

struct Ctx {
    cudaStream_t st;
    u64* s;
    cudaError_t err = cudaSuccess;
    void ck(cudaError_t e)
    {
        if (err == cudaSuccess && e != cudaSuccess) err = e;
    }
};

// exclusive scan of n (u32 or u64) values into out; total left in scratch[kOffScalar]
template <typename T>
void scan(Ctx& c, const T* in, u64 n, u64* out)
{
    if (n == 0) return;
    int g = blocks_for(n);
    u64 chunk = (n + g - 1) / g;
    g = (int)((n + chunk - 1) / chunk);
    scan_chunk_sums<T><<<g, kThreads, 0, c.st>>>(in, n, chunk, c.s + kOffSums);
    scan_sums_single<<<1, kThreads, 0, c.st>>>(c.s + kOffSums, g, c.s + kOffScalar);
    scan_chunk_apply<T><<<g, kThreads, 0, c.st>>>(in, n, chunk, c.s + kOffSums, out);
    c.ck(cudaGetLastError());
}

// LSD radix sort of (k, v) by k's bits [0, bits); the result ends in (ka, va)
void sort(Ctx& c, u64* ka, u64* va, u64* kb, u64* vb, u64 n, int bits)
{
    int g = blocks_for(n);
    u64 chunk = (n + g - 1) / g;
    g = (int)((n + chunk - 1) / chunk);
    u32* hist = (u32*)(c.s + kOffHist);
    u64* hoff = c.s + kOffHistOff;
    u64 *sk = ka, *sv = va, *dk = kb, *dv = vb;
    int passes = 0;
    for (int shift = 0; shift < bits; shift += kRadixBits) {
        radix_histogram<<<g, kThreads, 0, c.st>>>(sk, n, chunk, shift, hist, g);
        scan<u32>(c, hist, (u64)kRadix * g, hoff);
        radix_scatter<<<g, kThreads, 0, c.st>>>(sk, sv, dk, dv, n, chunk, shift, hoff, g);
        c.ck(cudaGetLastError());
        std::swap(sk, dk);
        std::swap(sv, dv);
        passes++;
    }
    if (passes & 1) {
        c.ck(cudaMemcpyAsync(ka, sk, n * 8, cudaMemcpyDeviceToDevice, c.st));
        c.ck(cudaMemcpyAsync(va, sv, n * 8, cudaMemcpyDeviceToDevice, c.st));
    }
}

}  // namespace

extern "C" int ra_rows_distinct_noalloc(const uint64_t* dev_rows_in, uint64_t nrows, uint32_t arity,
                                        uint64_t* dev_out_rows_in, uint64_t* dev_out_nrows_in, void* stream)
{
    const u64* dev_rows = (const u64*)dev_rows_in;
    u64* dev_out_rows = (u64*)dev_out_rows_in;
    u64* dev_out_nrows = (u64*)dev_out_nrows_in;
    if (nrows > kMaxRows || arity == 0 || arity > 8) return RA_E_BADARG;
    if ((nrows && (!dev_rows || !dev_out_rows)) || !dev_out_nrows) return RA_E_BADARG;
    Ctx c;
    c.st = (cudaStream_t)stream;
    int st = scratch_for(&c.s);
    if (st != RA_OK) return st;
    if (nrows == 0) {
        c.ck(cudaMemsetAsync(dev_out_nrows, 0, 8, c.st));
        return c.err == cudaSuccess ? RA_OK : RA_E_CUDA;
    }
    u64 hostv[3] = {0, 0, 0};
    // column width from the largest data value (as the engine packs relations)
    c.ck(cudaMemsetAsync(c.s + kOffScalar, 0, 3 * 8, c.st));
    rows_max_value<<<blocks_for(nrows), kThreads, 0, c.st>>>(dev_rows, nrows, (int)arity, c.s + kOffScalar + 1);
    c.ck(cudaGetLastError());
    c.ck(cudaMemcpyAsync(hostv, c.s + kOffScalar, 3 * 8, cudaMemcpyDeviceToHost, c.st));
    c.ck(cudaStreamSynchronize(c.st));
    if (c.err != cudaSuccess) return RA_E_CUDA;
    int bits = 1;
    while (bits < 64 && (hostv[1] >> bits)) bits++;
    if ((int)arity * bits > 63) return RA_E_UNSUPPORTED;
    const int kbits = (int)arity * bits;

    u64 *ka = c.s + kOffKA, *va = c.s + kOffVA, *kb = c.s + kOffKB, *vb = c.s + kOffVB;
    rows_pack<<<blocks_for(nrows), kThreads, 0, c.st>>>(dev_rows, nrows, (int)arity, bits, ka, va);
    c.ck(cudaGetLastError());
    // lexicographic (key, id): ids first, then keys (each pass is stable)
    sort(c, va, ka, vb, kb, nrows, 64);
    sort(c, ka, va, kb, vb, nrows, kbits);
    u32* flag = (u32*)(c.s + kOffFlag);
    u64* rank = c.s + kOffRank;
    flag_distinct_rows<<<blocks_for(nrows), kThreads, 0, c.st>>>(ka, va, nrows, flag);
    c.ck(cudaGetLastError());
    scan<u32>(c, flag, nrows, rank);
    compact_flagged<<<blocks_for(nrows), kThreads, 0, c.st>>>(ka, va, flag, rank, nrows, kb, vb);
    copy_count_kernel<<<1, 1, 0, c.st>>>(c.s + kOffScalar, dev_out_nrows);
    // the distinct rows stay stream-ordered: the count is read on the device
    unpack_counted_kernel<<<blocks_for(nrows), kThreads, 0, c.st>>>(kb, vb, c.s + kOffScalar, (int)arity, bits,
                                                                     dev_out_rows);
    c.ck(cudaGetLastError());
    return c.err == cudaSuccess ? RA_OK : RA_E_CUDA;
}
