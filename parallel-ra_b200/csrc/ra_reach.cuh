// Transitive closure by composing reachable sets (the reachability evaluator).
//
// Shape: the single recursive rule  R(z, x) :- R_delta(y, x), S_full(y, z)
// of tests/transitive_closure.cpp:60-68, with R's stored tuples exactly S
// reversed (R(y, x) for every S(x, y): what the program's copy SCC leaves
// before the recursive SCC, lie.cpp:295-301 moving it to delta).  Row x of R
// then runs a breadth-first search over S from x's successors, so when the
// fixed point is reached row x holds exactly
//     reach(x) = { (z, d) : z reachable from x in S, d = shortest path length },
// and iteration k of the semi-naive loop adds exactly the pairs with d = k + 2
// (its delta sizes are the histogram of d).  For a node v that reaches no
// cycle, reach(v) composes from its successors' sets:
//     reach(v) = min-merge over successors y of  {(y, 1)} u {(z, d + 1) : (z, d) in reach(y)}
// so the sets are computed children first: every node's set is a sorted run of
// (z << 16 | d) entries in an arena, merged from its successors' runs, level by
// level (level 0: the sinks; a node joins the next level when the counter of
// its unfinished successors reaches zero) in one cooperative launch -- a lane
// per cheap node, the whole warp for a long run or several successors.  Nodes
// that reach a cycle never join a level; the host finds the (few) of them, runs
// their searches over that small part of the graph, and the device merges in
// the sets of the cycle-free successors they lead to.  Every entry is read and written in
// order (merge paths), so the evaluator does no random read-modify-write of
// a multi-gigabyte table, which bounds the semi-naive hash-set path.
//
// The new tuples of row x are the entries with d >= 2 (d == 1: x's successors,
// R's stored tuples), emitted row by row, values ascending -- the dense
// evaluator's order, so both number intern ids alike.
#pragma once
#include "ra_iter.cuh"

namespace ra {

constexpr u32 kReachArena = 1;      // the arena is too small: grow it, run again
constexpr u32 kReachDepth = 2;      // a distance does not fit 16 bits
constexpr u32 kReachTimeout = 4;    // a bounded wait gave up
constexpr u32 kReachMismatch = 8;   // R's stored tuples are not S reversed
constexpr u32 kReachCorrupt = 16;   // an index outside its array (recorded at kCCheck, never dereferenced)
constexpr int kDistBits = 16;
constexpr u64 kDistMask = (1ull << kDistBits) - 1;
constexpr u64 kReachWaitNs = 4000000000ull;
// counters (u64 words of ReachArgs::ctr)
constexpr int kCFront0 = 0;     // nodes in frontier buffer 0 / 1
constexpr int kCFront1 = 16;
constexpr int kCArena = 32;     // arena entries handed out
constexpr int kCBarCount = 40;  // grid barrier: blocks arrived, generation
constexpr int kCBarGen = 44;
constexpr int kCCheck = 48;     // 1 + the first index check that failed, its value, its bound
constexpr int kCRound = 52;     // rounds of 32 frontier nodes taken in the running level
constexpr int kCHeavy = 24;     // nodes of the running level left to whole warps, and how many were taken
constexpr int kCHeavyTaken = 28;
constexpr int kCRoundHeavy = 56;
constexpr int kCLevels = 60;    // levels swept
constexpr int kCDone = 62;      // nodes whose set is finished
constexpr int kCtrWords = 64;

struct ReachArgs {
    u64 n;                 // nodes: the values 0 .. n - 1
    const u64* scsr;       // S rows with column 0 == v: [scsr[v], scsr[v + 1]), column 1 ascending
    const u32* sval;       // S's column 1 of every row
    const u64* rcsr;       // predecessors of v: rpar[rcsr[v] .. rcsr[v + 1])
    const u32* rpar;
    u32* rem;              // successors of v whose set is not finished
    u64* ctr;              // kCtrWords counters, each hot one on its own 128-byte line (see kC*)
    u64* seg_off;          // reach(v) = arena[seg_off[v], + seg_len[v]), ascending
    u32* seg_len;
    u64* arena;
    u64 arena_cap;
    u32* flags;
};

__device__ __forceinline__ u64 r_ld(const u64* p) { return __ldcg((const unsigned long long*)p); }
__device__ __forceinline__ u32 r_ld32(const u32* p) { return __ldcg(p); }

// Is v < bound?  Otherwise record (site, v, bound) once and report false: the
// caller skips the access, so a broken invariant ends the run with an error
// status instead of an out-of-range access.
__device__ __noinline__ bool r_ok(const ReachArgs& a, u32 site, u64 v, u64 bound)
{
    if (v < bound) return true;
    atomicOr(a.flags, kReachCorrupt);
    if (atomicCAS((unsigned long long*)&a.ctr[kCCheck], 0ull, (unsigned long long)site + 1) == 0ull) {
        a.ctr[kCCheck + 1] = v;
        a.ctr[kCCheck + 2] = bound;
    }
    return false;
}

// a node's run must lie inside the arena
__device__ __forceinline__ bool r_run_ok(const ReachArgs& a, u32 site, u64 off, u64 len)
{
    return r_ok(a, site, off + len, a.arena_cap + 1);
}

// S's column 1 as u32 (the values fit 31 bits when the evaluator runs)
__global__ void __launch_bounds__(kThreads) reach_sval_kernel(const u64* __restrict__ skeys, u64 m, int bits,
                                                              u32* __restrict__ sval, u32* __restrict__ indeg)
{
    const u64 mask = (1ull << bits) - 1;
    for (u64 j = (u64)blockIdx.x * kThreads + threadIdx.x; j < m; j += (u64)gridDim.x * kThreads) {
        const u32 z = (u32)(skeys[j] & mask);
        sval[j] = z;
        atomicAdd(&indeg[z], 1u);
    }
}

// predecessor lists (order within a list does not matter)
__global__ void __launch_bounds__(kThreads) reach_parents_kernel(const u64* __restrict__ skeys, u64 m, int bits,
                                                                 const u64* __restrict__ rcsr, u32* __restrict__ cursor,
                                                                 u32* __restrict__ rpar)
{
    const u64 mask = (1ull << bits) - 1;
    for (u64 j = (u64)blockIdx.x * kThreads + threadIdx.x; j < m; j += (u64)gridDim.x * kThreads) {
        const u64 k = skeys[j];
        const u32 y = (u32)(k >> bits), z = (u32)(k & mask);
        rpar[rcsr[z] + atomicAdd(&cursor[z], 1u)] = y;
    }
}

// Is every stored tuple (y, x) of R an S tuple (x, y)?  (With equal counts and
// distinct tuples on both sides, R is then exactly S reversed.)
__global__ void __launch_bounds__(kThreads) reach_check_kernel(ReachArgs a, const u64* __restrict__ rkeys, u64 nr,
                                                               int bits)
{
    const u64 mask = (1ull << bits) - 1;
    for (u64 i = (u64)blockIdx.x * kThreads + threadIdx.x; i < nr; i += (u64)gridDim.x * kThreads) {
        const u64 k = rkeys[i];
        const u64 y = (k >> bits) & mask, x = k & mask;
        bool found = false;
        if (x < a.n) {
            u64 lo = a.scsr[x], hi = a.scsr[x + 1];
            while (lo < hi) {
                const u64 mid = (lo + hi) >> 1;
                if ((u64)a.sval[mid] < y) lo = mid + 1;
                else hi = mid;
            }
            found = lo < a.scsr[x + 1] && (u64)a.sval[lo] == y;
        }
        if (!found) atomicOr(a.flags, kReachMismatch);
    }
}

// counters of unfinished successors; the sinks are the first frontier
// (warp-aggregated appends: one atomic per warp and round)
__global__ void __launch_bounds__(kThreads) reach_init_kernel(ReachArgs a, u32* __restrict__ front)
{
    const int lane = threadIdx.x & 31;
    for (u64 b = ((u64)blockIdx.x * kThreads + threadIdx.x) & ~31ull; b < a.n; b += (u64)gridDim.x * kThreads) {
        const u64 v = b + lane;
        bool sink = false;
        if (v < a.n) {
            const u32 deg = (u32)(a.scsr[v + 1] - a.scsr[v]);
            a.rem[v] = deg;
            a.seg_len[v] = 0;
            a.seg_off[v] = 0;
            sink = deg == 0;
        }
        const u32 bal = __ballot_sync(0xffffffffu, sink);
        u64 at = 0;
        if (lane == 0 && bal) at = atomicAdd((unsigned long long*)&a.ctr[kCFront0], (unsigned long long)__popc(bal));
        at = __shfl_sync(0xffffffffu, at, 0);
        if (sink) front[at + __popc(bal & lanemask_lt())] = (u32)v;
    }
}

// ---------------------------------------------------------------------------
// warp-level merge of two ascending runs (entries + a distance shift), and
// dropping of repeated values (keeping the first: the least distance)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void r_check_shift(const ReachArgs& a, u64 e, u64 sh)
{
    if ((e & kDistMask) + sh > kDistMask) atomicOr(a.flags, kReachDepth);
}

// Shared-memory windows of one warp's merges: kMTile entries of each run.
constexpr int kMTile = 256;
constexpr int kMPer = kMTile / 32;   // outputs per lane and tile
constexpr int kWarpSmemWords = 2 * kMTile;

// C = merge(A + sa, B + sb), ascending, ties A first.  Tiles of kMTile outputs:
// both runs' next kMTile entries into shared memory (coalesced), each lane
// merges kMPer outputs from a merge-path split found in shared memory, and the
// next tile starts where this one ended -- no search in global memory.  A shift
// that would carry a distance out of its 16 bits sets kReachDepth.
__device__ void r_merge(const ReachArgs& a, const u64* A, u64 la, u64 sa, const u64* B, u64 lb, u64 sb, u64* C,
                        u64* sm)
{
    const int lane = threadIdx.x & 31;
    u64* sA = sm;
    u64* sB = sm + kMTile;
    const u64 total = la + lb;
    u64 a0 = 0, b0 = 0;
    for (u64 t0 = 0; t0 < total; t0 += kMTile) {
        __syncwarp();
#pragma unroll
        for (int q = 0; q < kMPer; q++) {
            const int j = q * 32 + lane;
            u64 x = ~0ull, y = ~0ull;
            if (a0 + j < la) {
                x = A[a0 + j];
                if ((x & kDistMask) + sa > kDistMask) atomicOr(a.flags, kReachDepth);
                x += sa;
            }
            if (b0 + j < lb) {
                y = B[b0 + j];
                if ((y & kDistMask) + sb > kDistMask) atomicOr(a.flags, kReachDepth);
                y += sb;
            }
            sA[j] = x;
            sB[j] = y;
        }
        __syncwarp();
        const u32 n_out = (u32)min((u64)kMTile, total - t0);
        // merge-path split of the window at diagonal d: first i with sA[i] > sB[d - 1 - i]
        auto split = [&](u32 d) {
            u32 lo = 0, hi = d;
            while (lo < hi) {
                const u32 mid = (lo + hi) >> 1;
                if (sA[mid] <= sB[d - 1 - mid]) lo = mid + 1;
                else hi = mid;
            }
            return lo;
        };
        const u32 d0 = min(n_out, (u32)lane * kMPer), d1 = min(n_out, d0 + kMPer);
        u32 i = split(d0), j = d0 - i;
        for (u32 p = d0; p < d1; p++) {
            const u64 x = sA[i], y = sB[j];
            if (x <= y) {
                C[t0 + p] = x;
                i++;
            } else {
                C[t0 + p] = y;
                j++;
            }
        }
        const u32 ie = split(n_out);
        a0 += ie;
        b0 += n_out - ie;
    }
    __syncwarp();
}

// dst = src without repeated values (first of each value kept); returns the length.
// Each lane takes kMPer consecutive entries per round; dst may equal src (a
// round writes only positions below the end of what it has read).
__device__ u64 r_unique(const u64* src, u64 len, u64* dst)
{
    const int lane = threadIdx.x & 31;
    u64 out = 0, carry = ~0ull;   // last value of the previous round
    for (u64 b = 0; b < len; b += 32 * kMPer) {
        u64 v[kMPer];
        const u64 p0 = b + (u64)lane * kMPer;
#pragma unroll
        for (int q = 0; q < kMPer; q++) v[q] = p0 + q < len ? src[p0 + q] : ~0ull;
        u64 prev = __shfl_up_sync(0xffffffffu, v[kMPer - 1], 1);
        if (lane == 0) prev = carry;
        u32 keep = 0;
#pragma unroll
        for (int q = 0; q < kMPer; q++) {
            const u64 pv = q ? v[q - 1] : prev;
            if (p0 + q < len && (pv == ~0ull || (pv >> kDistBits) != (v[q] >> kDistBits))) keep |= 1u << q;
        }
        const u64 cnt = __popc(keep);
        u64 inc = cnt;
        for (int d = 1; d < 32; d <<= 1) {
            const u64 t = __shfl_up_sync(0xffffffffu, inc, d);
            if (lane >= d) inc += t;
        }
        const u64 rtot = __shfl_sync(0xffffffffu, inc, 31);
        carry = __shfl_sync(0xffffffffu, v[kMPer - 1], 31);
        if (len - b < 32 * kMPer) {   // a partial last round: the last real entry
            const u64 last = len - 1 - b;
            carry = __shfl_sync(0xffffffffu, v[last % kMPer], (int)(last / kMPer));
        }
        __syncwarp();
        u64 at = out + inc - cnt;
#pragma unroll
        for (int q = 0; q < kMPer; q++)
            if (keep >> q & 1) dst[at++] = v[q];
        out += rtot;
        __syncwarp();
    }
    return out;
}

// arena room for `count` entries (warp-uniform); ~0 when the arena is full
__device__ u64 r_alloc(const ReachArgs& a, u64 count)
{
    u64 off = 0;
    if ((threadIdx.x & 31) == 0) {
        off = atomicAdd((unsigned long long*)&a.ctr[kCArena], (unsigned long long)count);
        if (off + count > a.arena_cap) {
            atomicOr(a.flags, kReachArena);
            off = ~0ull;
        }
    }
    return __shfl_sync(0xffffffffu, off, 0);
}

// The set of a node from `ns` ascending single entries (final distances) and the
// sets of `nc` successors, successor c's set shifted by shift_of(c).  Runs: the
// singles, then every non-empty successor set; a balanced tree of pairwise
// merges (level 0 reads the successors' sets in place, later levels alternate
// between two halves of the node's arena room), then repeated values dropped --
// O(T log runs) for T entries in all, whatever the number of successors.
// Returns (offset, length) in *off / *len.  Warp-uniform.
template <typename ChildOf, typename ShiftOf, typename SingleOf>
__device__ void r_compose(const ReachArgs& a, u64 ns, SingleOf single_of, u64 nc, ChildOf child_of, ShiftOf shift_of,
                          u64* off, u32* len, u64* sm)
{
    const int lane = threadIdx.x & 31;
    // runs and their total (warp-uniform: each lane sums its children, then the warp sum)
    u64 T = ns, R = 1;
    for (u64 c0 = 0; c0 < nc; c0 += 32) {
        const u64 c = c0 + lane;
        u64 l = 0;
        if (c < nc) {
            const u32 y = child_of(c);
            if (r_ok(a, 1, y, a.n)) {
                l = r_ld32(&a.seg_len[y]);
                if (!r_run_ok(a, 2, r_ld(&a.seg_off[y]), l)) l = 0;
            }
        }
        const u32 bal = __ballot_sync(0xffffffffu, l != 0);
        u64 sum = l;
        for (int d = 16; d > 0; d >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, d);
        T += sum;   // the same on every lane
        R += __popc(bal);
    }
    // room: X and Y (T each), the singles (ns), run table (R successor ids, R + 1 offsets)
    const u64 base = r_alloc(a, 2 * T + ns + 2 * R + 1);
    if (base == ~0ull) {
        *off = 0;
        *len = 0;
        return;
    }
    u64* X = a.arena + base;
    u64* Y = X + T;
    u64* S = Y + T;
    u64* run_child = S + ns;        // run r >= 1: successor id
    u64* run_off = run_child + R;   // run r starts at run_off[r] of the merged order (run_off[R] = T)
    for (u64 i = lane; i < ns; i += 32) S[i] = single_of(i);
    if (lane == 0) run_off[0] = 0;
    u64 r = 1, acc = ns;
    for (u64 c0 = 0; c0 < nc; c0 += 32) {
        const u64 c = c0 + lane;
        const u32 y = c < nc ? child_of(c) : 0u;
        u64 l = 0;
        if (c < nc && y < a.n) {
            l = r_ld32(&a.seg_len[y]);
            if (r_ld(&a.seg_off[y]) + l > a.arena_cap) l = 0;   // recorded by the first pass
        }
        const u32 bal = __ballot_sync(0xffffffffu, l != 0);
        u64 inc = l;
        for (int d = 1; d < 32; d <<= 1) {
            const u64 t = __shfl_up_sync(0xffffffffu, inc, d);
            if (lane >= d) inc += t;
        }
        if (l) {
            const u64 at = r + __popc(bal & lanemask_lt());
            run_child[at] = c;
            run_off[at] = acc + inc - l;
        }
        r += __popc(bal);
        acc += __shfl_sync(0xffffffffu, inc, 31);
    }
    if (lane == 0) run_off[R] = T;
    __syncwarp();
    __threadfence_block();
    // run q of level 0: the singles or a successor's set (with its shift)
    auto run0 = [&](u64 q, const u64** ptr, u64* l, u64* sh) {
        if (q == 0) {
            *ptr = S;
            *l = ns;
            *sh = 0;
            return;
        }
        const u64 c = r_ld(&run_child[q]);
        if (!r_ok(a, 3, c, nc)) {
            *ptr = S;
            *l = 0;
            *sh = 0;
            return;
        }
        const u32 y = child_of(c);
        *ptr = a.arena + r_ld(&a.seg_off[y]);
        *l = r_ld32(&a.seg_len[y]);
        *sh = shift_of(c);
    };
    const u64* cur = S;   // the whole merged order so far (R == 1: the singles)
    u64* dst = X;
    for (u64 width = 1; width < R; width *= 2) {
        // merge runs [q, q + width) and [q + width, q + 2 width) of the previous level
        for (u64 q = 0; q < R; q += 2 * width) {
            const u64 m = min(q + width, R), e = min(q + 2 * width, R);
            u64 o0 = r_ld(&run_off[q]), o1 = r_ld(&run_off[m]), o2 = r_ld(&run_off[e]);
            if (!r_ok(a, 4, o2, T + 1) || !r_ok(a, 5, o1, o2 + 1) || !r_ok(a, 6, o0, o1 + 1)) o0 = o1 = o2 = 0;
            const u64 *A, *B;
            u64 la, lb, sa, sb;
            if (width == 1) {
                run0(q, &A, &la, &sa);
                if (m < e) run0(m, &B, &lb, &sb);
                else B = A, lb = 0, sb = 0;
                if (!r_ok(a, 7, la + lb, o2 - o0 + 1)) la = lb = 0;   // the runs fill exactly their slots
            } else {
                A = cur + o0;
                la = o1 - o0;
                sa = 0;
                B = cur + o1;
                lb = o2 - o1;
                sb = 0;
            }
            r_merge(a, A, la, sa, B, lb, sb, dst + o0, sm);
        }
        __syncwarp();
        __threadfence_block();
        cur = dst;
        dst = dst == X ? Y : X;
    }
    const u64 n = r_unique(cur, T, X);
    *off = base;
    *len = (u32)n;
}

// ---------------------------------------------------------------------------
// The sets, level by level: level 0 holds the sinks, level L + 1 the nodes whose
// last successor finished in level L.  One cooperative launch; the levels are
// separated by a bounded grid barrier, which also orders every set written in a
// level before the next level reads it.
// ---------------------------------------------------------------------------
// phase 0: after the lanes' pass of a level; phase 1: after the whole level
__device__ bool r_barrier(const ReachArgs& a, u64 level, int phase)
{
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long* cnt = (unsigned long long*)&a.ctr[kCBarCount];
        volatile u64* gen = &a.ctr[kCBarGen];
        const u64 g = *gen;
        __threadfence();
        s_ok = 1;
        if (atomicAdd(cnt, 1ull) == gridDim.x - 1) {
            if (phase == 0) {
                a.ctr[kCRound] = 0;
            } else {
                // the level is done: its frontier counter becomes the one after next
                u64* done_front = &a.ctr[(level & 1) ? kCFront1 : kCFront0];
                a.ctr[kCDone] += *((volatile u64*)done_front);
                *done_front = 0;
                a.ctr[kCHeavy] = 0;
                a.ctr[kCHeavyTaken] = 0;
                a.ctr[kCLevels] = level + 1;
            }
            *cnt = 0;
            __threadfence();
            atomicExch((unsigned long long*)gen, (unsigned long long)(g + 1));
        } else {
            const u64 t0 = global_ns();
            while (*gen == g) {
                if (global_ns() - t0 > kReachWaitNs) {
                    atomicOr(a.flags, kReachTimeout);
                    s_ok = 0;
                    break;
                }
                __nanosleep(32);
            }
            __threadfence();
        }
    }
    __syncthreads();
    return s_ok != 0;
}

// One node's set by the whole warp (a successor's long run, or several successors).
__device__ void r_node_warp(const ReachArgs& a, u32 v, u64* sm)
{
    const int lane = threadIdx.x & 31;
    const u64 e0 = a.scsr[v], e1 = a.scsr[v + 1];
    const u64 k = e1 - e0;
    u64 off = 0;
    u32 len = 0;
    if (k == 1) {
        // one successor: its set shifted by one with (y, 1) inserted -- no repeats possible
        const u32 y = a.sval[e0];
        u64 ly = 0, oy = 0;
        if (r_ok(a, 9, y, a.n)) {
            ly = r_ld32(&a.seg_len[y]);
            oy = r_ld(&a.seg_off[y]);
            if (!r_run_ok(a, 10, oy, ly)) ly = oy = 0;
        }
        const u64* B = a.arena + oy;
        off = r_alloc(a, ly + 1);
        if (off != ~0ull) {
            // entries below y keep their place, the others move up one; (y, 1) goes in between.
            // A run is written once, before the barrier its readers wait on: L1-cached loads are safe.
            u64* X = a.arena + off;
            u64 below = 0;   // the same on every lane: full-warp ballots over uniform rounds
#pragma unroll 4
            for (u64 p0 = 0; p0 < ly; p0 += 32) {
                const u64 p = p0 + lane;
                const bool in = p < ly;
                const u64 e = in ? B[p] : 0;
                const bool lt_y = in && (e >> kDistBits) < (u64)y;
                if (in) {
                    r_check_shift(a, e, 1);
                    X[p + (lt_y ? 0 : 1)] = e + 1;
                }
                below += __popc(__ballot_sync(0xffffffffu, lt_y));
            }
            if (lane == 0) X[below] = ((u64)y << kDistBits) | 1ull;
            len = (u32)(ly + 1);
        } else {
            off = 0;
        }
    } else if (k > 1) {
        r_compose(
            a, k, [&](u64 i) { return ((u64)a.sval[e0 + i] << kDistBits) | 1ull; }, k,
            [&](u64 c) { return a.sval[e0 + c]; }, [&](u64) { return 1ull; }, &off, &len, sm);
    }
    if (lane == 0) {
        a.seg_off[v] = off;
        a.seg_len[v] = len;
    }
    __syncwarp();
}

// A node whose successors and their sets hold at most this many entries in all
// is handled by one lane: gather, insertion sort, drop repeats.
constexpr int kLaneMax = 32;

// Node v's set is finished: predecessors whose last successor it was join the
// next level.  Lane-level (each lane its own v; invalid lanes pass np = 0).
__device__ __forceinline__ void r_release(const ReachArgs& a, u64 p0, u64 np, u32* __restrict__ nxt,
                                          unsigned long long* nnxt)
{
    const int lane = threadIdx.x & 31;
    u64 prounds = np;
    for (int d = 16; d > 0; d >>= 1) prounds = max(prounds, __shfl_xor_sync(0xffffffffu, prounds, d));
    for (u64 pr = 0; pr < prounds; pr++) {
        u32 par = 0;
        bool ready = false;
        if (pr < np) {
            par = a.rpar[p0 + pr];
            ready = atomicSub(&a.rem[par], 1u) == 1u;
        }
        const u32 bal = __ballot_sync(0xffffffffu, ready);
        if (!bal) continue;
        u64 at = 0;
        if (lane == 0) at = atomicAdd(nnxt, (unsigned long long)__popc(bal));
        at = __shfl_sync(0xffffffffu, at, 0);
        if (ready) nxt[at + __popc(bal & lanemask_lt())] = par;
    }
}

__global__ void __launch_bounds__(kThreads) reach_levels_kernel(ReachArgs a, u32* __restrict__ fa,
                                                                u32* __restrict__ fb, u32* __restrict__ hlist)
{
    __shared__ u64 s_merge[kWarps][kWarpSmemWords];
    u64* sm = s_merge[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const u32 lt = lanemask_lt();
    for (u64 level = 0;; level++) {
        const u32* __restrict__ cur = (level & 1) ? fb : fa;
        u32* __restrict__ nxt = (level & 1) ? fa : fb;
        const u64 ncur = r_ld(&a.ctr[(level & 1) ? kCFront1 : kCFront0]);
        unsigned long long* nnxt = (unsigned long long*)&a.ctr[(level & 1) ? kCFront0 : kCFront1];
        if (ncur == 0) break;   // the same value in every block: read after a barrier
        const bool stop = *((volatile u32*)a.flags) & (kReachArena | kReachTimeout | kReachCorrupt);
        const u64 nrounds = stop ? 0 : (ncur + 31) / 32;
        // phase 0: rounds of 32 nodes, a lane each; larger sets go to the heavy list
        for (;;) {
            u64 r = 0;
            if (lane == 0) r = atomicAdd((unsigned long long*)&a.ctr[kCRound], 1ull);
            r = __shfl_sync(0xffffffffu, r, 0);
            if (r >= nrounds) break;
            const u64 i = r * 32 + lane;
            const bool valid = i < ncur;
            u32 v = valid ? cur[i] : 0u;
            if (valid && !r_ok(a, 8, v, a.n)) v = 0;   // (never: frontiers hold node ids)
            const u64 e0 = valid ? a.scsr[v] : 0, k = valid ? a.scsr[v + 1] - e0 : 0;
            u64 T = k;
            bool small = valid && k <= (u64)kLaneMax;
            for (u64 c = 0; small && c < k; c++) {
                const u32 y = a.sval[e0 + c];
                if (!r_ok(a, 9, y, a.n)) continue;
                const u64 ly = r_ld32(&a.seg_len[y]);
                if (!r_run_ok(a, 10, r_ld(&a.seg_off[y]), ly)) continue;
                T += ly;
                if (T > (u64)kLaneMax) small = false;
            }
            u64 buf[kLaneMax];
            u32 m = 0;
            if (small && k) {
                for (u64 c = 0; c < k; c++) {
                    const u32 y = a.sval[e0 + c];
                    buf[m++] = ((u64)y << kDistBits) | 1ull;
                    if (y >= a.n) continue;
                    const u64 ly = r_ld32(&a.seg_len[y]);
                    const u64* B = a.arena + r_ld(&a.seg_off[y]);
                    for (u64 q = 0; q < ly && m < (u32)kLaneMax; q++) {
                        const u64 e = B[q];
                        r_check_shift(a, e, 1);
                        buf[m++] = e + 1;
                    }
                }
                // insertion sort by (value, distance), then the first of each value
                for (u32 x = 1; x < m; x++) {
                    const u64 t = buf[x];
                    u32 j = x;
                    while (j > 0 && buf[j - 1] > t) {
                        buf[j] = buf[j - 1];
                        j--;
                    }
                    buf[j] = t;
                }
                u32 w = 0;
                for (u32 x = 0; x < m; x++)
                    if (w == 0 || (buf[w - 1] >> kDistBits) != (buf[x] >> kDistBits)) buf[w++] = buf[x];
                m = w;
            }
            // warp-aggregated room for the lanes' sets
            u64 inc = m;
            for (int d = 1; d < 32; d <<= 1) {
                const u64 t = __shfl_up_sync(0xffffffffu, inc, d);
                if (lane >= d) inc += t;
            }
            const u64 tot = __shfl_sync(0xffffffffu, inc, 31);
            u64 base = 0;
            if (tot) base = r_alloc(a, tot);
            if (m && base != ~0ull) {
                u64* X = a.arena + base + inc - m;
                for (u32 x = 0; x < m; x++) X[x] = buf[x];
                a.seg_off[v] = base + inc - m;
                a.seg_len[v] = m;
            }
            // the larger sets: to whole warps in phase 1
            const u32 hb = __ballot_sync(0xffffffffu, valid && !small);
            if (hb) {
                u64 at = 0;
                if (lane == 0) at = atomicAdd((unsigned long long*)&a.ctr[kCHeavy], (unsigned long long)__popc(hb));
                at = __shfl_sync(0xffffffffu, at, 0);
                if (valid && !small) hlist[at + __popc(hb & lt)] = v;
            }
            // the finished small sets release their predecessors now
            const bool fin = valid && small;
            const u64 p0 = fin ? a.rcsr[v] : 0, np = fin ? a.rcsr[v + 1] - p0 : 0;
            r_release(a, p0, np, nxt, nnxt);
        }
        if (!r_barrier(a, level, 0)) break;
        // phase 1: the larger sets, one per warp of the whole grid
        const u64 nh = r_ld(&a.ctr[kCHeavy]);
        for (;;) {
            u64 h = 0;
            if (lane == 0) h = atomicAdd((unsigned long long*)&a.ctr[kCHeavyTaken], 1ull);
            h = __shfl_sync(0xffffffffu, h, 0);
            if (h >= nh) break;
            const u32 v = hlist[h];
            if (!r_ok(a, 11, v, a.n)) continue;
            r_node_warp(a, v, sm);
            const u64 p0 = a.rcsr[v], np = a.rcsr[v + 1] - p0;
            for (u64 q0 = 0; q0 < np; q0 += 32) {   // lanes split the predecessor list
                const bool has = q0 + lane < np;
                const u64 pp0 = has ? p0 + q0 + lane : 0;
                r_release(a, pp0, has ? 1 : 0, nxt, nnxt);
            }
        }
        if (!r_barrier(a, level, 1)) break;
    }
}

// Nodes that reach a cycle, after the host's searches: node u's set from its
// single entries (the part of the graph that reaches cycles, with the
// search's distances, and the first cycle-free nodes met, at theirs) and the
// cycle-free nodes' sets shifted by those distances.  One warp per node.
struct ReachCyclic {
    const u32* node;        // the nodes
    const u64* single_off;  // node i: singles [single_off[i], single_off[i + 1]) of `singles`
    const u64* singles;     // (value << 16 | distance), ascending per node
    const u64* exit_off;    // node i: exits [exit_off[i], exit_off[i + 1])
    const u32* exit_node;   // cycle-free node met first on a path
    const u32* exit_dist;   // its distance
    u64 count;
};

__global__ void __launch_bounds__(kThreads) reach_cyclic_kernel(ReachArgs a, ReachCyclic c)
{
    __shared__ u64 s_merge[kWarps][kWarpSmemWords];
    u64* sm = s_merge[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const u64 warps = (u64)gridDim.x * kWarps;
    for (u64 i = (u64)blockIdx.x * kWarps + (threadIdx.x >> 5); i < c.count; i += warps) {
        const u64 s0 = c.single_off[i], s1 = c.single_off[i + 1];
        const u64 x0 = c.exit_off[i], x1 = c.exit_off[i + 1];
        if (!r_ok(a, 11, c.node[i], a.n) || !r_ok(a, 12, s0, s1 + 1) || !r_ok(a, 13, x0, x1 + 1)) continue;
        u64 off;
        u32 len;
        r_compose(
            a, s1 - s0, [&](u64 j) { return c.singles[s0 + j]; }, x1 - x0, [&](u64 j) { return c.exit_node[x0 + j]; },
            [&](u64 j) { return (u64)c.exit_dist[x0 + j]; }, &off, &len, sm);
        if (lane == 0) {
            a.seg_off[c.node[i]] = off;
            a.seg_len[c.node[i]] = len;
        }
    }
}

// new tuples per row: the entries beyond the successors themselves
__global__ void __launch_bounds__(kThreads) reach_count_kernel(ReachArgs a, u64* __restrict__ row_new)
{
    for (u64 v = (u64)blockIdx.x * kThreads + threadIdx.x; v < a.n; v += (u64)gridDim.x * kThreads)
        row_new[v] = (u64)a.seg_len[v] - (a.scsr[v + 1] - a.scsr[v]);
}

// New tuples into R's log, row by row (values ascending): key (z, x), id
// tag_word | (id_base + position); per-distance counts (d - 2 = the iteration).
// One warp per row; ballot compaction of the entries with d >= 2.
// `cand_total` gets the semi-naive loop's join candidates: every pair (z, x) of the
// closure is once an outer row matching z's successors.
__global__ void __launch_bounds__(kThreads) reach_emit_kernel(ReachArgs a, const u64* __restrict__ row_off, int bits,
                                                              u64* __restrict__ keys_out, u64* __restrict__ ids_out,
                                                              u64 tag_word, u64 id_base, u64* __restrict__ level_total,
                                                              u64 level_cap, u64* __restrict__ cand_total, u64 total)
{
    u64 cands = 0;
    __shared__ u32 s_lvl[kWarps][64];   // counts of the first 64 levels per warp
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = lane; i < 64; i += 32) s_lvl[warp][i] = 0;
    __syncwarp();
    const u64 warps = (u64)gridDim.x * kWarps;
    for (u64 x = (u64)blockIdx.x * kWarps + warp; x < a.n; x += warps) {
        const u64 len = a.seg_len[x];
        if (len == 0 || !r_run_ok(a, 14, a.seg_off[x], len)) continue;
        const u64* E = a.arena + a.seg_off[x];
        u64 pos = row_off[x];
        for (u64 b = 0; b < len; b += 32) {
            const u64 p = b + lane;
            const u64 e = p < len ? E[p] : 0;
            const u64 d = e & kDistMask;
            const bool in = p < len && r_ok(a, 15, e >> kDistBits, a.n);
            const bool keep = in && d >= 2;
            if (in) {
                const u64 z = e >> kDistBits;
                cands += a.scsr[z + 1] - a.scsr[z];
            }
            const u32 bal = __ballot_sync(0xffffffffu, keep);
            if (keep && r_ok(a, 16, pos + __popc(bal & lanemask_lt()), total)) {
                const u64 at = pos + __popc(bal & lanemask_lt());
                keys_out[at] = ((e >> kDistBits) << bits) | x;
                ids_out[at] = tag_word | (id_base + at);
                const u64 lv = d - 2;
                if (lv < 64) atomicAdd(&s_lvl[warp][lv], 1u);
                else if (lv < level_cap) atomicAdd((unsigned long long*)&level_total[lv], 1ull);
            }
            pos += __popc(bal);
        }
    }
    __syncwarp();
    for (int i = lane; i < 64; i += 32)
        if (s_lvl[warp][i] && (u64)i < level_cap)
            atomicAdd((unsigned long long*)&level_total[i], (unsigned long long)s_lvl[warp][i]);
    for (int d = 16; d > 0; d >>= 1) cands += __shfl_xor_sync(0xffffffffu, cands, d);
    if (lane == 0 && cands) atomicAdd((unsigned long long*)cand_total, (unsigned long long)cands);
}

// CSR ranges of the nodes that reach a cycle, and their successors packed
__global__ void __launch_bounds__(kThreads) reach_gather_ranges_kernel(const u64* __restrict__ scsr,
                                                                       const u32* __restrict__ node, u64 count, u64 n,
                                                                       u64* __restrict__ lo_hi)
{
    for (u64 i = (u64)blockIdx.x * kThreads + threadIdx.x; i < count; i += (u64)gridDim.x * kThreads) {
        const u64 v = node[i] < n ? node[i] : 0;   // (never: the list holds node ids)
        lo_hi[2 * i] = scsr[v];
        lo_hi[2 * i + 1] = node[i] < n ? scsr[v + 1] : scsr[v];
    }
}
__global__ void __launch_bounds__(kThreads) reach_gather_succ_kernel(const u32* __restrict__ sval,
                                                                     const u64* __restrict__ lo_hi,
                                                                     const u64* __restrict__ off, u64 count,
                                                                     u32* __restrict__ out)
{
    const int lane = threadIdx.x & 31;
    const u64 warps = (u64)gridDim.x * kWarps;
    for (u64 i = (u64)blockIdx.x * kWarps + (threadIdx.x >> 5); i < count; i += warps)
        for (u64 e = lo_hi[2 * i] + lane; e < lo_hi[2 * i + 1]; e += 32) out[off[i] + e - lo_hi[2 * i]] = sval[e];
}

// nodes left with unfinished successors: they reach a cycle
__global__ void __launch_bounds__(kThreads) reach_cyclic_list_kernel(ReachArgs a, u32* __restrict__ out,
                                                                     u64* __restrict__ count, u64 cap)
{
    for (u64 v = (u64)blockIdx.x * kThreads + threadIdx.x; v < a.n; v += (u64)gridDim.x * kThreads)
        if (a.rem[v]) {
            const u64 at = atomicAdd((unsigned long long*)count, 1ull);
            if (at < cap) out[at] = (u32)v;
        }
}

}  // namespace ra
