// Small iterations in one thread-block cluster (the tail kernel).
//
// A fixed point's last hundred-odd iterations move a few thousand tuples each;
// on the CUDA-graph path every one of them still costs a join launch and a
// select launch with their look-backs (about 20 us).  When every rule's outer
// delta is small (kTailRowsGo rows per CTA of a cluster), the first kernel of the
// iteration body runs iterations itself, back to back, until a delta outgrows
// it, the fixed point is reached or a buffer runs short:
//   * one cluster of CTAs (16 where the GPU can place them, else 8), each
//     owning an equal share of each rule's outer delta (contiguous rows);
//   * the control block lives in CTA 0's shared memory while the kernel runs
//     (every CTA reads it through distributed shared memory; CTA 0's thread 0
//     runs the iteration end on it, as the persistent kernel does), and goes
//     back to global memory when the kernel exits;
//   * per rule: match counts from the CSR, a block scan, a cluster scan of the
//     CTAs' totals (through distributed shared memory, hardware cluster
//     barriers), then the candidates expanded at their stream positions and
//     claimed in the seen set -- the join kernel's work, positions and claims;
//   * after a cluster barrier, the winners (mark not of this epoch) compacted
//     in stream order into the log with their intern ids -- select_kernel's
//     output, offsets and ids.
// Every stream position, claim, winner, id and history entry is the one the
// join + select launches produce, so the log is identical.  An iteration the
// kernel declines (a delta or a CTA's candidates too large, a flag, no room)
// is left to those launches, which follow in the same body: claims made before
// the decision are idempotent under the replay protocol (same epoch, same
// positions).  The join and select kernels return at once when the tail
// kernel has reached the fixed point (ctl->done).
#pragma once
#include <cooperative_groups.h>
#include "ra_persist.cuh"

namespace ra {

namespace cg = cooperative_groups;

constexpr int kTailThreads = 1024;
constexpr int kTailWarps = kTailThreads / 32;
constexpr int kTailRowsPerThread = 2;
constexpr int kTailRowsPerCta = kTailThreads * kTailRowsPerThread;   // capacity of a CTA's row arrays
// An iteration goes to the tail kernel when every rule's outer delta has at most
// kTailRowsGo rows per CTA of the cluster.  Claims are bound by each SM's rate of
// random 16-byte atomics (the device's ~21 G/s is ~0.15 G/s per SM), so the rows
// are spread evenly over the CTAs.  Measured on tc-er22 (ms per step, same box):
// 256 rows per CTA 12.15, 512 12.07, 1,024 11.97, 2,048 11.66; a variant with 4
// rows per thread and 4,096 rows per CTA 11.79.
constexpr int kTailRowsGo = kTailRowsPerCta;
constexpr u64 kTailCtaCands = 32768;   // a CTA's candidates per rule, above which the graph path is faster
constexpr int kTailMaxCtas = 16;
// dynamic shared memory: exclusive match prefix (rows + 1), first inner row and key per row
constexpr size_t kTailSmem = (size_t)(3 * kTailRowsPerCta + 1) * 8;

struct TailRule {
    RowsRef in;            // the outer rows (an SCC relation's delta)
    int outer_shift;
    const u64* csr;
    const u64* inner;
    Projection pj;
    Slot* seen;            // the output relation's seen set
    u64 seen_cap;
    u64* dst_keys;         // its log
    u64* dst_ids;
};

struct TailArgs {
    IterCtl* ctl;
    SccPlan plan;
    SccRelMap rm;
    int n_rules;
    TailRule rule[kTailMaxRules];
    int bits;
    u64* cand;
    u64 cand_cap;
    u32* loser;
    u64* history;
};

__device__ __forceinline__ u64 t_ld(const u64* p) { return __ldcg((const unsigned long long*)p); }
__device__ __forceinline__ u32 t_ld32(const u32* p) { return __ldcg(p); }

// exclusive scan over the CTA's 1024 threads
__device__ __forceinline__ u64 tail_block_scan(u64 v, u64* sm, u64* total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const u64 inc = warp_inclusive_scan(v);
    if (lane == 31) sm[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        const u64 w = sm[lane];
        const u64 wi = warp_inclusive_scan(w);
        sm[lane] = wi - w;
        if (lane == 31) sm[kTailWarps] = wi;
    }
    __syncthreads();
    const u64 out = inc - v + sm[warp];
    *total = sm[kTailWarps];
    __syncthreads();
    return out;
}

struct ClusterSum {
    u64 pre;    // sum over the CTAs ranked below this one
    u64 total;  // sum over the cluster
    u64 max;    // largest value of one CTA
};

// Cluster-wide exclusive sum of one value per CTA: each CTA posts its value in
// its own shared memory (slot alternates, so a slot is rewritten only after a
// later barrier), a cluster barrier, then warp 0 reads every CTA's value
// through distributed shared memory.  Every thread of every CTA calls it.
__device__ ClusterSum cluster_sum(cg::cluster_group& cl, u64* s_post, int slot, u64 v)
{
    __shared__ ClusterSum s_res;
    if (threadIdx.x == 0) s_post[slot] = v;
    cl.sync();
    if (threadIdx.x < 32) {
        const unsigned n = cl.num_blocks(), me = cl.block_rank(), r = threadIdx.x;
        const u64 x = r < n ? *cl.map_shared_rank(&s_post[slot], r) : 0;
        u64 pre = r < me ? x : 0, tot = x, mx = x;
        for (int d = 16; d > 0; d >>= 1) {
            pre += __shfl_xor_sync(0xffffffffu, pre, d);
            tot += __shfl_xor_sync(0xffffffffu, tot, d);
            mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, d));
        }
        if (threadIdx.x == 0) s_res = ClusterSum{pre, tot, mx};
    }
    __syncthreads();
    return s_res;
}

// What every CTA needs of the control block in one iteration.  CTA 0's
// thread 0 fills it from its copy after the iteration end (with the decision
// whether to take the iteration at all), and CTA 0's threads store it into
// every other CTA's shared memory before the barrier that starts the
// iteration: no CTA waits on a remote read of the control block.
struct TailIter {
    int go;                          // take this iteration
    u64 epoch;
    u64 n[kTailMaxRules];            // outer rows of each rule
    const u64* outer[kTailMaxRules];
    u64 dst[kTailMaxRules];          // full + delta rows of the rule's output: its winners go after them
    u64 id0[kTailMaxRules];          // intern counter of the rule's tag
    u64 stored[kMaxSccRels];         // full + delta rows of every relation (room check)
};

// CTA 0, thread 0: the next iteration's TailIter from CTA 0's copy of the
// control block and the flags the tail kernel's claims raised.
__device__ void tail_fill(const TailArgs& A, const IterCtl* L, u32 cflags, unsigned nctas, TailIter* t)
{
    bool go = L->flags == 0 && L->done == 0 && L->tail_off == 0 && cflags == 0;
    t->epoch = L->epoch;
    for (int q = 0; q < A.n_rules; q++) {
        const int out = A.plan.rule_out[q];
        t->n[q] = rows_n(L, A.rule[q].in);
        t->outer[q] = rows_ptr(L, A.rule[q].in);
        t->dst[q] = L->full_n[out] + L->delta_n[out];
        t->id0[q] = L->intern[A.plan.rule_tag[q]];
        go = go && t->n[q] <= (u64)nctas * kTailRowsGo;
    }
    for (int s = 0; s < A.plan.n_rels; s++) t->stored[s] = L->full_n[s] + L->delta_n[s];
    t->go = go ? 1 : 0;
}

constexpr int kTailSelIpt = 4;                                   // candidates per thread per select tile
constexpr int kTailSelTile = kTailThreads * kTailSelIpt;
constexpr int kTailSelTiles = (int)(kTailCtaCands / kTailSelTile);

// Memory ordering: the cluster barriers (barrier.cluster.arrive.release /
// wait.acquire) order each thread's earlier global and shared stores before
// the other CTAs' later loads; cross-CTA data (loser marks, candidates, the
// log rows of the previous iteration) is read with ld.global.cg.
//
// Per iteration: counts, cluster sum (barrier), claims, barrier, winner bits,
// cluster sum (barrier), then the winners' stores while CTA 0's thread 0 runs
// the iteration end and publishes the next TailIter (double-buffered, so no
// CTA still reading this iteration's copy is overwritten), barrier.
__global__ void __launch_bounds__(kTailThreads, 1) tail_cluster_kernel(TailArgs A)
{
    extern __shared__ u64 t_dyn[];
    u64* s_ex = t_dyn;                               // kTailRowsPerCta + 1
    u64* s_start = t_dyn + kTailRowsPerCta + 1;      // kTailRowsPerCta
    u64* s_key = s_start + kTailRowsPerCta;          // kTailRowsPerCta
    __shared__ u64 s_ctl[kCtlWords];                 // CTA 0's: the control block while the kernel runs
    __shared__ u64 s_scan[kTailWarps + 1];
    __shared__ u64 s_post[2];
    __shared__ TailIter s_it[2];                     // this iteration's and the next one's
    __shared__ unsigned char s_win[kTailSelTiles][kTailThreads];   // winner bits of a thread's select slice
    __shared__ u32 s_flags;                          // CTA 0's: flags raised by the claims of any CTA
    __shared__ int s_ok;
    cg::cluster_group cl = cg::this_cluster();
    const unsigned me = cl.block_rank(), nctas = cl.num_blocks();
    IterCtl* G = A.ctl;
    u64* gw = (u64*)G;
    IterCtl* L = (IterCtl*)s_ctl;   // CTA 0's own copy
    u32* cflags = cl.map_shared_rank(&s_flags, 0);
    // CTA 0, warp 0: fill buffer b of every CTA -- lane 0 its own, then the 32 lanes
    // store it word by word into the others' (distributed shared memory)
    static_assert(sizeof(TailIter) % 8 == 0, "TailIter is copied as words");
    constexpr int kItWords = (int)(sizeof(TailIter) / 8);
    auto publish = [&](int b) {
        if ((threadIdx.x & 31) == 0) tail_fill(A, L, s_flags, nctas, &s_it[b]);
        __syncwarp();
        const u64* src = (const u64*)&s_it[b];
        for (int i = threadIdx.x & 31; i < (int)(nctas - 1) * kItWords; i += 32) {
            const unsigned r = 1 + i / kItWords;
            cl.map_shared_rank((u64*)&s_it[b], r)[i % kItWords] = src[i % kItWords];
        }
    };
    if (me == 0) {
        for (int i = threadIdx.x; i < kCtlWords; i += kTailThreads) s_ctl[i] = t_ld(&gw[i]);
        if (threadIdx.x == 0) s_flags = 0;
        __syncthreads();
        if (threadIdx.x < 32) publish(0);
    }
    cl.sync();
    int post = 0;
    int ran = 0;
    int cur = 0;
    while (s_it[cur].go) {
        const TailIter& it = s_it[cur];
        const u64 epoch = it.epoch;
        const LoserMarks lm{A.loser, (u32)epoch, epoch << 40, 0};
        u64 cbase[kTailMaxRules], cpre[kTailMaxRules], cagg[kTailMaxRules], ctot[kTailMaxRules];
        u64 nrows = 0;
        bool ok = true;
        u64 pos0 = 0;   // stream position of the rule's first candidate
        for (int q = 0; q < A.n_rules; q++) {
            const TailRule& R = A.rule[q];
            const u64 n = it.n[q];
            const u64* outer = it.outer[q];
            nrows += n;
            // rows spread evenly: CTA c takes [c * per, (c + 1) * per), per <= kTailRowsGo
            const u64 per = (n + nctas - 1) / nctas;
            const u64 lo = (u64)me * per;
            const u64 nr = n > lo ? min(per, n - lo) : 0;
            u64 cnt[kTailRowsPerThread];
            u64 local = 0;
#pragma unroll
            for (int k = 0; k < kTailRowsPerThread; k++) {
                const int li = threadIdx.x * kTailRowsPerThread + k;
                cnt[k] = 0;
                if ((u64)li < nr) {
                    const u64 key = t_ld(&outer[lo + li]);
                    const u64 j = key >> R.outer_shift;
                    const u64 s = R.csr[j];
                    cnt[k] = R.csr[j + 1] - s;
                    s_start[li] = s;
                    s_key[li] = key;
                }
                local += cnt[k];
            }
            u64 agg;
            u64 ex = tail_block_scan(local, s_scan, &agg);
#pragma unroll
            for (int k = 0; k < kTailRowsPerThread; k++) {
                s_ex[threadIdx.x * kTailRowsPerThread + k] = ex;
                ex += cnt[k];
            }
            if (threadIdx.x == 0) s_ex[kTailRowsPerCta] = agg;
            const ClusterSum cs = cluster_sum(cl, s_post, post, agg);
            post ^= 1;
            if (pos0 + cs.total > A.cand_cap || cs.max > kTailCtaCands) {
                // every CTA sees the same sums: the same decision.  A CTA with too many
                // candidates (a skewed key) also turns the tail kernel off for the rest
                // of the SCC run: the loop's launches spread such rows over every SM.
                if (cs.max > kTailCtaCands && me == 0 && threadIdx.x == 0) {
                    L->tail_off = 1;
                    G->tail_off = 1;
                }
                ok = false;
                break;
            }
            cbase[q] = pos0;
            cpre[q] = cs.pre;
            cagg[q] = agg;
            ctot[q] = cs.total;
            // the CTA's candidates: stream position pos0 + cs.pre + j, j in [0, agg)
            const u64 tb = (epoch << 40) | (pos0 + cs.pre);
            for (u64 j0 = 0; j0 < agg; j0 += (u64)kTailThreads * kClaimBatch) {
                u64 key[kClaimBatch], mine[kClaimBatch], ik[kClaimBatch];
                bool valid[kClaimBatch];
                int rr[kClaimBatch];
#pragma unroll
                for (int k = 0; k < kClaimBatch; k++) {
                    const u64 j = j0 + threadIdx.x + (u64)k * kTailThreads;
                    valid[k] = j < agg;
                    rr[k] = 0;
                    ik[k] = 0;
                    if (valid[k]) {
                        rr[k] = (int)upper_bound_dev(s_ex, nr, j) - 1;
                        ik[k] = R.inner[s_start[rr[k]] + (j - s_ex[rr[k]])];
                    }
                }
#pragma unroll
                for (int k = 0; k < kClaimBatch; k++) {
                    const u64 j = j0 + threadIdx.x + (u64)k * kTailThreads;
                    key[k] = valid[k] ? project(R.pj, s_key[rr[k]], ik[k], A.bits) : 0;
                    mine[k] = tb + j;
                    if (valid[k]) A.cand[pos0 + cs.pre + j] = key[k];
                }
                claim_batch(R.seen, R.seen_cap, key, mine, valid, lm, cflags);
            }
            pos0 += cs.total;
            __syncthreads();   // s_ex / s_start / s_key are the next rule's
        }
        if (!ok) break;
        // ---- every claim of the iteration is in: winners in stream order
        cl.sync();
        if (threadIdx.x == 0) {
            // select_kernel's room check, and flags the claims raised (a probe that gave up);
            // the same inputs on every CTA
            bool go = *cflags == 0;
            for (int s = 0; s < A.plan.n_rels && go; s++) {
                u64 incoming = 0;
                for (int q = 0; q < A.rm.n_rules_in[s]; q++) incoming += ctot[A.rm.rules_in[s][q]];
                if (incoming && it.stored[s] + incoming > A.plan.log_cap[s]) go = false;
            }
            s_ok = go;
        }
        __syncthreads();
        if (!s_ok) break;   // the join + select launches redo it and raise the flag (nothing written here)
        u64 wtot[kTailMaxRules];
        for (int q = 0; q < A.n_rules; q++) {
            const TailRule& R = A.rule[q];
            const int out = A.plan.rule_out[q], tslot = A.plan.rule_tag[q];
            u64 dst_off = it.dst[q], id_ctr = it.id0[q];
            for (int r = 0; r < q; r++) {
                if (A.plan.rule_out[r] == out) dst_off += wtot[r];
                if (A.plan.rule_tag[r] == tslot) id_ctr += wtot[r];
            }
            const u64 tag_word = A.plan.rel_tag_word[out];
            const u64* in = A.cand + cbase[q] + cpre[q];
            const u32* mk = A.loser + cbase[q] + cpre[q];
            const u64 agg = cagg[q];
            const int ntile = (int)((agg + kTailSelTile - 1) / kTailSelTile);
            // pass 1: winner bits of this thread's kTailSelIpt consecutive candidates per tile
            u64 win = 0;
            u64 k0[kTailSelIpt];   // tile 0's keys, kept for pass 2
            for (int t = 0; t < ntile; t++) {
                const u64 base = (u64)t * kTailSelTile + (u64)threadIdx.x * kTailSelIpt;
                u64 kk[kTailSelIpt];
                u32 mm[kTailSelIpt];
#pragma unroll
                for (int k = 0; k < kTailSelIpt; k++) {
                    const bool v = base + k < agg;
                    kk[k] = v ? t_ld(&in[base + k]) : kEmpty;
                    mm[k] = v ? t_ld32(&mk[base + k]) : (u32)epoch;
                }
                unsigned mask = 0;
#pragma unroll
                for (int k = 0; k < kTailSelIpt; k++) {
                    if (kk[k] != kEmpty && mm[k] != (u32)epoch) mask |= 1u << k;
                    if (t == 0) k0[k] = kk[k];
                }
                s_win[t][threadIdx.x] = (unsigned char)mask;
                win += __popc(mask);
            }
            u64 wagg;
            tail_block_scan(win, s_scan, &wagg);
            const ClusterSum ws = cluster_sum(cl, s_post, post, wagg);
            post ^= 1;
            wtot[q] = ws.total;
            if (q == A.n_rules - 1 && me == 0 && threadIdx.x < 32) {
                // every total of the iteration is known: its end, on CTA 0's copy of the
                // control block, and the next TailIter, while the winners are stored
                if (threadIdx.x == 0) {
                    for (int r = 0; r < A.n_rules; r++) {
                        L->cand_n[r] = ctot[r];
                        L->win_n[r] = wtot[r];
                    }
                    L->outer_rows += nrows;
                    L->tail_iters++;
                    end_of_iteration(L, A.plan, A.rm, A.history, 0, 0);
                }
                __syncwarp();
                publish(cur ^ 1);
            }
            // pass 2: each tile's winners at their offsets in stream order
            u64 off = dst_off + ws.pre, idc = id_ctr + ws.pre;
            for (int t = 0; t < ntile; t++) {
                const u64 base = (u64)t * kTailSelTile + (u64)threadIdx.x * kTailSelIpt;
                const unsigned mask = s_win[t][threadIdx.x];
                u64 kk[kTailSelIpt];
#pragma unroll
                for (int k = 0; k < kTailSelIpt; k++)
                    kk[k] = t == 0 ? k0[k] : ((mask >> k) & 1 ? t_ld(&in[base + k]) : 0);
                u64 tt;
                const u64 ex = tail_block_scan((u64)__popc(mask), s_scan, &tt);
                u64 r = ex;
#pragma unroll
                for (int k = 0; k < kTailSelIpt; k++) {
                    if (!((mask >> k) & 1)) continue;
                    R.dst_keys[off + r] = kk[k];
                    R.dst_ids[off + r] = tag_word | (idc + r);
                    r++;
                }
                off += tt;
                idc += tt;
            }
        }
        ran++;
        cur ^= 1;
        cl.sync();
    }
    // leave: no CTA reads CTA 0's memory past this barrier; CTA 0 writes its copy
    // back (with the flags the claims raised) -- unchanged if no iteration ran
    cl.sync();
    if (me == 0 && (ran || s_flags)) {
        if (threadIdx.x == 0) L->flags |= s_flags;
        __syncthreads();
        for (int i = threadIdx.x; i < kCtlWords; i += kTailThreads) __stcg((unsigned long long*)&gw[i], s_ctl[i]);
    }
}

}  // namespace ra
