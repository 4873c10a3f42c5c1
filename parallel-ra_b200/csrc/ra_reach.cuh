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
// (z << 16 | d) entries in an arena, merged from its successors' runs by one
// warp as soon as the last successor is done (a device work queue fed by
// per-node counters of unfinished successors).  Nodes that reach a cycle are
// never released; the host finds the (few) of them, runs their searches over
// that small part of the graph, and the device merges in the sets of the
// cycle-free successors they lead to.  Every entry is read and written in
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
constexpr u32 kQEmpty = 0xffffffffu;
constexpr int kDistBits = 16;
constexpr u64 kDistMask = (1ull << kDistBits) - 1;
constexpr u64 kReachWaitNs = 4000000000ull;

struct ReachArgs {
    u64 n;                 // nodes: the values 0 .. n - 1
    const u64* scsr;       // S rows with column 0 == v: [scsr[v], scsr[v + 1]), column 1 ascending
    const u32* sval;       // S's column 1 of every row
    const u64* rcsr;       // predecessors of v: rpar[rcsr[v] .. rcsr[v + 1])
    const u32* rpar;
    u32* rem;              // successors of v whose set is not finished
    u32* queue;            // nodes whose successors are all finished
    u64* ctr;              // [0] tickets taken, [1] nodes pushed, [2] nodes finished, [3] arena entries used
    u64* seg_off;          // reach(v) = arena[seg_off[v], + seg_len[v]), ascending
    u32* seg_len;
    u64* arena;
    u64 arena_cap;
    u32* flags;
};

__device__ __forceinline__ u64 r_ld(const u64* p) { return __ldcg((const unsigned long long*)p); }
__device__ __forceinline__ u32 r_ld32(const u32* p) { return __ldcg(p); }

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

// counters of unfinished successors; sinks go straight into the work queue
__global__ void __launch_bounds__(kThreads) reach_init_kernel(ReachArgs a)
{
    for (u64 v = (u64)blockIdx.x * kThreads + threadIdx.x; v < a.n; v += (u64)gridDim.x * kThreads) {
        const u32 deg = (u32)(a.scsr[v + 1] - a.scsr[v]);
        a.rem[v] = deg;
        a.seg_len[v] = 0;
        a.seg_off[v] = 0;
        a.queue[v] = kQEmpty;
    }
}
__global__ void __launch_bounds__(kThreads) reach_sinks_kernel(ReachArgs a)
{
    for (u64 v = (u64)blockIdx.x * kThreads + threadIdx.x; v < a.n; v += (u64)gridDim.x * kThreads)
        if (a.scsr[v + 1] == a.scsr[v]) {
            const u64 at = atomicAdd((unsigned long long*)&a.ctr[1], 1ull);
            a.queue[at] = (u32)v;
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

// C = merge(A + sa, B + sb), ascending, ties A first (merge path, one segment per
// lane).  A shift that would carry a distance out of its 16 bits sets kReachDepth.
__device__ void r_merge(const ReachArgs& a, const u64* A, u64 la, u64 sa, const u64* B, u64 lb, u64 sb, u64* C)
{
    const int lane = threadIdx.x & 31;
    const u64 total = la + lb;
    const u64 per = (total + 31) / 32;
    const u64 d0 = min(total, (u64)lane * per), d1 = min(total, d0 + per);
    if (d0 >= d1) return;
    u64 lo = d0 > lb ? d0 - lb : 0, hi = min(d0, la);
    while (lo < hi) {   // first i with A[i] + sa > B[d0 - 1 - i] + sb
        const u64 mid = (lo + hi) >> 1;
        if (r_ld(&A[mid]) + sa <= r_ld(&B[d0 - 1 - mid]) + sb) lo = mid + 1;
        else hi = mid;
    }
    u64 i = lo, j = d0 - lo;
    auto get = [&](const u64* X, u64 k, u64 sh) {
        const u64 e = r_ld(&X[k]);
        if ((e & kDistMask) + sh > kDistMask) atomicOr(a.flags, kReachDepth);
        return e + sh;
    };
    u64 av = i < la ? get(A, i, sa) : ~0ull, bv = j < lb ? get(B, j, sb) : ~0ull;
    for (u64 p = d0; p < d1; p++) {
        if (j >= lb || (i < la && av <= bv)) {
            C[p] = av;
            i++;
            av = i < la ? get(A, i, sa) : ~0ull;
        } else {
            C[p] = bv;
            j++;
            bv = j < lb ? get(B, j, sb) : ~0ull;
        }
    }
}

// dst = src without repeated values (first of each value kept); returns the length.
// dst may equal src: a round writes below its own start plus 32, and identical
// values where it writes in place, so no read of a later round is disturbed.
__device__ u64 r_unique(const u64* src, u64 len, u64* dst)
{
    const int lane = threadIdx.x & 31;
    u64 out = 0;
    for (u64 b = 0; b < len; b += 32) {
        const u64 p = b + lane;
        u64 v = 0;
        bool keep = false;
        if (p < len) {
            v = r_ld(&src[p]);
            keep = p == 0 || (r_ld(&src[p - 1]) >> kDistBits) != (v >> kDistBits);
        }
        const u32 bal = __ballot_sync(0xffffffffu, keep);
        __syncwarp();
        if (keep) dst[out + __popc(bal & lanemask_lt())] = v;
        out += __popc(bal);
        __syncwarp();
        __threadfence_block();
    }
    return out;
}

// arena room for `count` entries (warp-uniform); ~0 when the arena is full
__device__ u64 r_alloc(const ReachArgs& a, u64 count)
{
    u64 off = 0;
    if ((threadIdx.x & 31) == 0) {
        off = atomicAdd((unsigned long long*)&a.ctr[3], (unsigned long long)count);
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
                          u64* off, u32* len)
{
    const int lane = threadIdx.x & 31;
    // runs and their total
    u64 T = ns, R = 1;
    for (u64 c0 = 0; c0 < nc; c0 += 32) {
        const u64 c = c0 + lane;
        const u64 l = c < nc ? r_ld32(&a.seg_len[child_of(c)]) : 0;
        const u32 bal = __ballot_sync(0xffffffffu, l != 0);
        u64 sum = l;
        for (int d = 16; d > 0; d >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, d);
        T += sum;
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
        const u64 l = c < nc ? r_ld32(&a.seg_len[y]) : 0;
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
            const u64 o0 = r_ld(&run_off[q]), o1 = r_ld(&run_off[m]), o2 = r_ld(&run_off[e]);
            const u64 *A, *B;
            u64 la, lb, sa, sb;
            if (width == 1) {
                run0(q, &A, &la, &sa);
                if (m < e) run0(m, &B, &lb, &sb);
                else B = A, lb = 0, sb = 0;
            } else {
                A = cur + o0;
                la = o1 - o0;
                sa = 0;
                B = cur + o1;
                lb = o2 - o1;
                sb = 0;
            }
            r_merge(a, A, la, sa, B, lb, sb, dst + o0);
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
// the work queue: nodes whose successors are all finished, merged by whichever
// warp takes them; bounded waits; ends when every pushed node is finished
// ---------------------------------------------------------------------------
__device__ u32 r_pop(const ReachArgs& a)
{
    u32 v = kQEmpty;
    if ((threadIdx.x & 31) == 0) {
        const u64 h = atomicAdd((unsigned long long*)&a.ctr[0], 1ull);
        const u64 t0 = global_ns();
        for (;;) {
            if (h < a.n) {
                v = *((volatile u32*)&a.queue[h]);
                if (v != kQEmpty) break;
            }
            const u64 done = *((volatile u64*)&a.ctr[2]);
            const u64 tail = *((volatile u64*)&a.ctr[1]);
            if (done == tail && h >= tail) break;   // everything pushed is finished: no more work
            if (global_ns() - t0 > kReachWaitNs) {
                atomicOr(a.flags, kReachTimeout);
                break;
            }
            __nanosleep(64);
        }
    }
    v = __shfl_sync(0xffffffffu, v, 0);
    __threadfence();   // every lane: the successors' sets are read after this
    return v;
}

__device__ void r_finish(const ReachArgs& a, u32 v, bool wrote)
{
    const int lane = threadIdx.x & 31;
    __syncwarp();
    if (wrote) __threadfence();   // every lane's part of the node's set before a predecessor may read it
    __syncwarp();
    const u64 p0 = a.rcsr[v], p1 = a.rcsr[v + 1];
    for (u64 i = p0 + lane; i < p1; i += 32) {
        const u32 p = a.rpar[i];
        if (atomicSub(&a.rem[p], 1u) == 1u) {
            const u64 at = atomicAdd((unsigned long long*)&a.ctr[1], 1ull);
            atomicExch(&a.queue[at], p);
        }
    }
    __syncwarp();
    __threadfence();   // every lane's pushes before the completion count (the end test reads them in that order)
    __syncwarp();
    if (lane == 0) atomicAdd((unsigned long long*)&a.ctr[2], 1ull);
}

__global__ void __launch_bounds__(kThreads) reach_dataflow_kernel(ReachArgs a)
{
    const int lane = threadIdx.x & 31;
    for (;;) {
        const u32 v = r_pop(a);
        if (v == kQEmpty) break;
        if (*((volatile u32*)a.flags) & (kReachTimeout | kReachArena)) {
            r_finish(a, v, false);   // keep the protocol going; the host runs again
            continue;
        }
        const u64 e0 = a.scsr[v], e1 = a.scsr[v + 1];
        const u64 k = e1 - e0;
        if (k == 0) {   // a sink: empty set (seg_len is 0 from the init)
            r_finish(a, v, false);
            continue;
        }
        u64 off;
        u32 len;
        if (k == 1) {
            // one successor: its set shifted by one with (y, 1) inserted -- no repeats possible
            const u32 y = a.sval[e0];
            const u64 ly = r_ld32(&a.seg_len[y]);
            const u64* B = a.arena + r_ld(&a.seg_off[y]);
            off = r_alloc(a, ly + 1);
            len = 0;
            if (off != ~0ull) {
                u64 lo = 0, hi = ly;   // entries of B with a value below y
                while (lo < hi) {
                    const u64 mid = (lo + hi) >> 1;
                    if ((r_ld(&B[mid]) >> kDistBits) < (u64)y) lo = mid + 1;
                    else hi = mid;
                }
                u64* X = a.arena + off;
                for (u64 p = lane; p <= ly; p += 32) {
                    u64 e;
                    if (p < lo) e = r_ld(&B[p]);
                    else if (p == lo) e = ((u64)y << kDistBits);
                    else e = r_ld(&B[p - 1]);
                    r_check_shift(a, e, 1);
                    X[p] = e + 1;
                }
                len = (u32)(ly + 1);
            } else {
                off = 0;
            }
        } else {
            r_compose(
                a, k, [&](u64 i) { return ((u64)a.sval[e0 + i] << kDistBits) | 1ull; }, k,
                [&](u64 c) { return a.sval[e0 + c]; }, [&](u64) { return 1ull; }, &off, &len);
        }
        if (lane == 0) {
            a.seg_off[v] = off;
            a.seg_len[v] = len;
        }
        r_finish(a, v, true);
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
    const int lane = threadIdx.x & 31;
    const u64 warps = (u64)gridDim.x * kWarps;
    for (u64 i = (u64)blockIdx.x * kWarps + (threadIdx.x >> 5); i < c.count; i += warps) {
        const u64 s0 = c.single_off[i], s1 = c.single_off[i + 1];
        const u64 x0 = c.exit_off[i], x1 = c.exit_off[i + 1];
        u64 off;
        u32 len;
        r_compose(
            a, s1 - s0, [&](u64 j) { return c.singles[s0 + j]; }, x1 - x0, [&](u64 j) { return c.exit_node[x0 + j]; },
            [&](u64 j) { return (u64)c.exit_dist[x0 + j]; }, &off, &len);
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
                                                              u64 level_cap, u64* __restrict__ cand_total)
{
    u64 cands = 0;
    __shared__ u32 s_lvl[kWarps][64];   // counts of the first 64 levels per warp
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = lane; i < 64; i += 32) s_lvl[warp][i] = 0;
    __syncwarp();
    const u64 warps = (u64)gridDim.x * kWarps;
    for (u64 x = (u64)blockIdx.x * kWarps + warp; x < a.n; x += warps) {
        const u64 len = a.seg_len[x];
        if (len == 0) continue;
        const u64* E = a.arena + a.seg_off[x];
        u64 pos = row_off[x];
        for (u64 b = 0; b < len; b += 32) {
            const u64 p = b + lane;
            const u64 e = p < len ? E[p] : 0;
            const u64 d = e & kDistMask;
            const bool keep = p < len && d >= 2;
            if (p < len) {
                const u64 z = e >> kDistBits;
                cands += a.scsr[z + 1] - a.scsr[z];
            }
            const u32 bal = __ballot_sync(0xffffffffu, keep);
            if (keep) {
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
                                                                       const u32* __restrict__ node, u64 count,
                                                                       u64* __restrict__ lo_hi)
{
    for (u64 i = (u64)blockIdx.x * kThreads + threadIdx.x; i < count; i += (u64)gridDim.x * kThreads) {
        lo_hi[2 * i] = scsr[node[i]];
        lo_hi[2 * i + 1] = scsr[node[i] + 1];
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
