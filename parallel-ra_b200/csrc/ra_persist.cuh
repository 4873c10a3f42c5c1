// The whole fixed point of an SCC as one cooperative launch.
//
// RAM::execute_in_batches (src/RAM/RA_tasks.cpp:1121-1269) runs, per
// iteration, local_compute (join / copy) -> all_to_all -> local_insert_in_newt
// -> local_insert_in_full, then check_for_fixed_point's MPI_Allreduce
// (RA_tasks.cpp:1072-1085).  Here every block of one co-resident grid runs the
// iterations back to back, separated by bounded grid barriers; the barrier's
// last arriver does the single-threaded bookkeeping (capacity check, the
// iteration end of ra_iter.cuh) and publishes what every block needs to decide
// the next step, so all blocks take the same branches.  Per iteration:
//
//   claims   per rule, warps take chunks of 128 outer rows: match counts from
//            the inner CSR, warp scans, a warp-level decoupled look-back for the
//            chunk's first stream position, then the chunk's candidates are
//            expanded (smem row table, binary search per candidate) and claimed
//            in the output's seen set, kPClaim claims in flight per lane.  No
//            block barrier anywhere in the loop.  Rows with more than
//            kHeavyRow matches keep their stream positions but are expanded
//            after the chunks, as work items of kHeavyPiece candidates taken by
//            every warp of the grid (a hub row does not serialise on one warp).
//            Copy rules: one candidate per input row (position = row index).
//   barrier  (last arriver: does every relation have room for the iteration's
//            candidates? else the overflow flag)
//   heavy    the heavy-row items, when there are any; barrier
//   select   per rule, warps take chunks of 256 candidates: winner test (the
//            loser mark is not this epoch), ballot compaction, warp look-back,
//            winners written straight into the relation's log with intern ids
//   barrier  (last arriver of the last rule: end_of_iteration -- region bump,
//            history, intern counters; or the stop flag)
//
// Stream positions, claims, loser marks and winners are exactly those of the
// per-launch kernels of ra_iter.cuh (join_fused_kernel / select_kernel), so
// both paths produce the same log, ids included.  An iteration that finds a
// buffer too small stops at the next barrier with the overflow flag; its claims
// are idempotent, so the host grows the buffer and launches again, replaying it.
#pragma once
#include "ra_iter.cuh"

namespace ra {

#ifndef RA_PERSIST_MIN_BLOCKS
#define RA_PERSIST_MIN_BLOCKS 3
#endif
constexpr int kPRowsPerLane = 4;
constexpr int kPJChunk = 32 * kPRowsPerLane;   // outer rows per warp chunk
constexpr int kPSelPerLane = 8;
constexpr int kPSChunk = 32 * kPSelPerLane;    // candidates per warp chunk of the select
constexpr int kPClaim = 4;                     // claims in flight per lane
// a grid barrier gives up after this long (a legitimate phase of one iteration is
// far shorter; the limit only ends a wait that could otherwise never finish)
constexpr u64 kBarrierNs = 4000000000ull;

// Control-block fields written by other blocks are read from L2 (never a stale L1 line).
__device__ __forceinline__ u64 ldcg(const u64* p) { return __ldcg((const unsigned long long*)p); }
__device__ __forceinline__ u64 p_rows_n(const IterCtl* c, const RowsRef& r)
{
    return r.slot >= 0 ? ldcg(&c->delta_n[r.slot]) : r.static_n;
}
__device__ __forceinline__ const u64* p_rows_ptr(const IterCtl* c, const RowsRef& r)
{
    return r.slot >= 0 ? r.keys + ldcg(&c->full_n[r.slot]) : r.keys;
}
__device__ __forceinline__ u64 p_stream_base(const IterCtl* c, int rule)
{
    u64 b = 0;
    for (int q = 0; q < rule; q++) b += ldcg(&c->cand_n[q]);
    return b;
}
__device__ __forceinline__ u32 p_iter_tag(u64 iteration, int slot) { return (u32)(((iteration + 1) << 7) | (u64)slot); }

// Warp-cooperative decoupled look-back (lookback_warp's protocol) without
// fences: a status word is one atomic 64-bit store that carries everything a
// reader needs, so nothing else has to be ordered with it.
__device__ u64 p_lookback(u64* status, u32 tile, u64 agg, u32 tag, u32* flags)
{
    const int lane = threadIdx.x & 31;
    const u32 tg = tag & 0xffffffu;
    if (tile == 0) {
        if (lane == 0) atomicExch((unsigned long long*)&status[0], (unsigned long long)st_pack(tag, kStIncl, agg));
        return 0;
    }
    if (lane == 0) atomicExch((unsigned long long*)&status[tile], (unsigned long long)st_pack(tag, kStAgg, agg));
    u64 excl = 0;
    long base = (long)tile - 1;
    u64 spins = 0;
    for (;;) {
        const long t = base - lane;
        u64 s = 0;
        bool ready = true, incl = true;
        if (t >= 0) {
            s = st_read(&status[t]);
            ready = st_tag(s) == tg && st_flag(s) != 0;
            incl = ready && st_flag(s) == kStIncl;
        }
        const u32 inclmask = __ballot_sync(0xffffffffu, incl);
        const u32 notready = __ballot_sync(0xffffffffu, !ready);
        const int first = inclmask ? __ffs(inclmask) - 1 : 32;
        const u32 needed = first >= 31 ? 0xffffffffu : ((2u << first) - 1);
        if (notready & needed) {
            if (++spins > kSpinLimit) {
                if (lane == 0) atomicOr(flags, kFlagTimeout);
                break;
            }
            continue;
        }
        u64 v = (lane <= first && t >= 0) ? st_val(s) : 0;
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
        excl += v;
        if (first < 32) break;
        base -= 32;
    }
    if (lane == 0)
        atomicExch((unsigned long long*)&status[tile], (unsigned long long)st_pack(tag, kStIncl, excl + agg));
    return excl;
}

struct PRule {
    int kind;             // kJoinRule, or a copy kind
    int out_slot;
    RowsRef in;           // join: outer rows; copy: input rows
    Projection pj;
    const u64* csr;       // join: inner CSR over the join key
    const u64* inner;     // join: inner keys
    int outer_shift;
    int pred;             // copy_filter predicate
    Slot* seen;           // the output relation's seen set
    u64 seen_cap;
    u64* dst_keys;        // the output relation's log
    u64* dst_ids;
    int inst_shift;       // bit offset of column 0 in the output key (instance accounting)
};

constexpr int kJoinRule = 3;

struct PersistArgs {
    IterCtl* ctl;
    SccPlan plan;
    SccRelMap rm;
    PRule rule[kMaxSccRules];
    int bits;
    u64* cand;
    u32* loser;
    u64* status;
    u64 status_cap;
    HeavyItem* heavy;
    u64 heavy_cap;
    u64* history;
    const u64* inst_base;   // instances (batched programs), or null
    u32 n_inst;
    u64* inst_new;
    u64 inst_iter_cap;
};

// ---------------------------------------------------------------------------
// grid barrier (bounded)
// ---------------------------------------------------------------------------
struct BarSnap {
    u32 flags;
    u32 done;
    u64 heavy;
};

enum BarAct { kActClaims = 0, kActHeavy = 1, kActSelect = 2, kActClaimsDone = 3, kActIterEnd = 4 };

// Does every relation of the SCC have room in its log for all the candidates of
// the running iteration?  (select_kernel's check, made once per iteration.)
__device__ void p_check_room(const PersistArgs& A, IterCtl* c)
{
    bool over = A.inst_base && c->iteration >= A.inst_iter_cap;
    for (int s = 0; s < A.plan.n_rels; s++) {
        u64 incoming = 0;
        for (int q = 0; q < A.rm.n_rules_in[s]; q++) incoming += c->cand_n[A.rm.rules_in[s][q]];
        if (incoming && c->full_n[s] + c->delta_n[s] + incoming > A.plan.log_cap[s]) over = true;
    }
    if (over) c->flags |= kFlagOverflow;
}

// The last arriver's single-threaded part, on the shared-memory copy of the
// control block (kept out of line: it is rare and would only add register
// pressure to the phases).
__device__ __noinline__ BarSnap p_release_bookkeeping(const PersistArgs& A, IterCtl* sc, int act)
{
    const u64 now = global_ns();
    const u64 dt = now - sc->t_phase;
    sc->t_phase = now;
    if (act == kActHeavy) sc->ns_heavy += dt;
    else if (act == kActSelect || act == kActIterEnd) sc->ns_select += dt;
    else sc->ns_claims += dt;
    if (act == kActClaimsDone && sc->flags == 0) p_check_room(A, sc);
    if (act == kActIterEnd) end_of_iteration(sc, A.plan, A.rm, A.history, 0, 0);
    BarSnap b;
    b.flags = sc->flags;
    b.done = sc->done;
    b.heavy = sc->heavy_n;
    return b;
}

// the control block up to the barrier's own fields: what the last arriver updates
constexpr int kCtlWords = (int)(offsetof(IterCtl, bar_count) / 8);
static_assert(offsetof(IterCtl, bar_count) % 8 == 0, "control block copy is whole words");

// Every block of the grid arrives; the last block to arrive does the phase's
// bookkeeping on a shared-memory copy of the control block (loaded and written
// back by all its threads at once, so the single-threaded part touches no
// global memory), records the phase's device time, publishes flags / done /
// heavy items and releases the others.  Bounded: a wait gives up after
// kBarrierNs and sets the timeout flag.
__device__ BarSnap grid_barrier(const PersistArgs& A, int act)
{
    __shared__ BarSnap s_snap;
    __shared__ u32 s_gen;
    __shared__ int s_last;
    __shared__ u64 s_ctl[kCtlWords];
    IterCtl* c = A.ctl;
    __syncthreads();
    if (threadIdx.x == 0) {
        const u32 g = *((volatile u32*)&c->bar_gen);
        __threadfence();
        const u32 arrived = atomicAdd(&c->bar_count, 1u);
        s_gen = g;
        s_last = arrived == gridDim.x - 1;
        if (s_last) __threadfence();
    }
    __syncthreads();
    if (s_last) {
        u64* gc = (u64*)c;
        for (int i = threadIdx.x; i < kCtlWords; i += blockDim.x) s_ctl[i] = ldcg(&gc[i]);
        __syncthreads();
        if (threadIdx.x == 0) s_snap = p_release_bookkeeping(A, (IterCtl*)s_ctl, act);
        __syncthreads();
        for (int i = threadIdx.x; i < kCtlWords; i += blockDim.x) __stcg((unsigned long long*)&gc[i], s_ctl[i]);
        __syncthreads();
        if (threadIdx.x == 0) {
            c->bar_count = 0;
            c->bar_flags = s_snap.flags;
            c->bar_done = s_snap.done;
            c->bar_heavy = s_snap.heavy;
            __threadfence();
            atomicExch(&c->bar_gen, s_gen + 1);
        }
    } else if (threadIdx.x == 0) {
        volatile u32* genp = &c->bar_gen;
        const u64 t0 = global_ns();
        while (*genp == s_gen) {
            if (global_ns() - t0 > kBarrierNs) {
                atomicOr(&c->flags, kFlagTimeout);
                atomicOr(&c->bar_flags, kFlagTimeout);
                break;
            }
            __nanosleep(32);
        }
        __threadfence();
        s_snap.flags = *((volatile u32*)&c->bar_flags);
        s_snap.done = *((volatile u32*)&c->bar_done);
        s_snap.heavy = *((volatile u64*)&c->bar_heavy);
    }
    __syncthreads();
    return s_snap;
}

// ---------------------------------------------------------------------------
// claims of a join rule
// ---------------------------------------------------------------------------
struct PJoinSmem {
    u64 pos[kPJChunk];       // each row's first candidate, relative to the chunk (all matches)
    u64 start[kPJChunk];     // its first inner row
    u64 key[kPJChunk];       // the outer key
    u32 lex[kPJChunk + 1];   // exclusive offsets of the light rows' candidates
};

// last row r of the chunk with lex[r] <= t (lex[0] == 0): the row owning light candidate t
__device__ __forceinline__ int p_owner(const u32* lex, u32 t)
{
    int r = 0;
#pragma unroll
    for (int s = kPJChunk / 2; s > 0; s >>= 1)
        if (lex[r + s] <= t) r += s;
    return r;
}

__device__ void p_join(const PersistArgs& A, int q, PJoinSmem& sm, int tslot)
{
    IterCtl* c = A.ctl;
    const PRule& R = A.rule[q];
    const int lane = threadIdx.x & 31;
    const u64 n = p_rows_n(c, R.in);
    const u64* __restrict__ outer = p_rows_ptr(c, R.in);
    if (n == 0) {
        if (blockIdx.x == 0 && threadIdx.x == 0) c->cand_n[q] = 0;
        return;
    }
    const u64 nch = (n + kPJChunk - 1) / kPJChunk;
    if (nch > A.status_cap) {   // the host sizes status for the largest input: never taken
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(&c->flags, kFlagStatus);
        return;
    }
    const u64 cbase = p_stream_base(c, q);
    const u64 epoch = ldcg(&c->epoch);
    const u64 ep40 = epoch << 40;
    const u32 tag = p_iter_tag(ldcg(&c->iteration), tslot);
    const LoserMarks lm{A.loser, (u32)epoch, ep40, 0};
    const u64* __restrict__ csr = R.csr;
    const u64* __restrict__ inner = R.inner;
    // chunks dealt out statically (warp w: w, w + W, ...); every warp is resident, so a
    // chunk's look-back only ever waits on lower chunks, whose aggregates come first
    const u64 W = (u64)gridDim.x * kWarps;
    for (u64 ch = (u64)blockIdx.x * kWarps + (threadIdx.x >> 5); ch < nch; ch += W) {
        const u64 r0 = ch * kPJChunk;
        u64 cnt[kPRowsPerLane], st[kPRowsPerLane], ky[kPRowsPerLane];
#pragma unroll
        for (int k = 0; k < kPRowsPerLane; k++) {
            const u64 i = r0 + (u64)k * 32 + lane;
            cnt[k] = 0;
            st[k] = 0;
            ky[k] = 0;
            if (i < n) ky[k] = outer[i];
        }
#pragma unroll
        for (int k = 0; k < kPRowsPerLane; k++) {
            const u64 i = r0 + (u64)k * 32 + lane;
            if (i < n) {
                const u64 j = ky[k] >> R.outer_shift;
                st[k] = csr[j];
                cnt[k] = csr[j + 1] - st[k];
            }
        }
        // offsets in row order (row k * 32 + lane of the chunk)
        u64 run = 0;
        u32 lrun = 0;
#pragma unroll
        for (int k = 0; k < kPRowsPerLane; k++) {
            const u64 inc = warp_inclusive_scan(cnt[k]);
            const u32 lc = cnt[k] > kHeavyRow ? 0u : (u32)cnt[k];
            u32 linc = lc;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const u32 t = __shfl_up_sync(0xffffffffu, linc, d);
                if (lane >= d) linc += t;
            }
            const int li = k * 32 + lane;
            sm.pos[li] = run + inc - cnt[k];
            sm.start[li] = st[k];
            sm.key[li] = ky[k];
            sm.lex[li] = lrun + linc - lc;
            run += __shfl_sync(0xffffffffu, inc, 31);
            lrun += __shfl_sync(0xffffffffu, linc, 31);
        }
        if (lane == 0) sm.lex[kPJChunk] = lrun;
        const u64 agg = run;
        const u64 prefix = p_lookback(A.status, (u32)ch, agg, tag, &c->flags);
        if (ch == nch - 1 && lane == 0) {
            c->cand_n[q] = prefix + agg;
            c->outer_rows += n;
        }
        __syncwarp();
        if (cbase + prefix + agg > A.plan.cand_cap) {
            if (lane == 0) atomicOr(&c->flags, kFlagOverflow);
            __syncwarp();
            continue;
        }
        // heavy rows: slices of kHeavyPiece candidates for every warp of the grid
#pragma unroll
        for (int k = 0; k < kPRowsPerLane; k++) {
            if (cnt[k] <= kHeavyRow) continue;
            const u64 pieces = (cnt[k] + kHeavyPiece - 1) / kHeavyPiece;
            const u64 at = atomicAdd((unsigned long long*)&c->heavy_n, (unsigned long long)pieces);
            if (at + pieces > A.heavy_cap) {
                atomicOr(&c->flags, kFlagOverflow);
                continue;
            }
            const u64 p0 = cbase + prefix + sm.pos[k * 32 + lane];
            for (u64 pc = 0; pc < pieces; pc++) {
                const u64 off = pc * kHeavyPiece;
                A.heavy[at + pc] = HeavyItem{p0 + off, ky[k], st[k] + off, (u32)min(kHeavyPiece, cnt[k] - off), (u32)q};
            }
            atomicAdd((unsigned long long*)&c->heavy_items, (unsigned long long)pieces);
        }
        // light candidates: kPClaim per lane in flight
        for (u32 t0 = 0; t0 < lrun; t0 += 32 * kPClaim) {
            u64 key[kPClaim], mine[kPClaim], ik[kPClaim];
            bool valid[kPClaim];
            int rr[kPClaim];
            u32 rank[kPClaim];
#pragma unroll
            for (int b = 0; b < kPClaim; b++) {
                const u32 t = t0 + (u32)b * 32 + lane;
                valid[b] = t < lrun;
                rr[b] = 0;
                rank[b] = 0;
                ik[b] = 0;
                if (valid[b]) {
                    rr[b] = p_owner(sm.lex, t);
                    rank[b] = t - sm.lex[rr[b]];
                    ik[b] = inner[sm.start[rr[b]] + rank[b]];
                }
            }
#pragma unroll
            for (int b = 0; b < kPClaim; b++) {
                key[b] = 0;
                mine[b] = 0;
                if (valid[b]) {
                    const u64 sp = cbase + prefix + sm.pos[rr[b]] + rank[b];
                    key[b] = project(R.pj, sm.key[rr[b]], ik[b], A.bits);
                    A.cand[sp] = key[b];
                    mine[b] = ep40 + sp;
                }
            }
            claim_batch(R.seen, R.seen_cap, key, mine, valid, lm, &c->flags);
        }
        __syncwarp();
    }
}

// heavy-row work items of every join rule
__device__ void p_heavy(const PersistArgs& A, u64 items)
{
    IterCtl* c = A.ctl;
    const int lane = threadIdx.x & 31;
    const u64 epoch = ldcg(&c->epoch);
    const u64 ep40 = epoch << 40;
    const LoserMarks lm{A.loser, (u32)epoch, ep40, 0};
    for (;;) {
        u64 it = 0;
        if (lane == 0) it = atomicAdd(&c->heavy_ctr, 1u);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= items) break;
        const HeavyItem h = A.heavy[it];
        const PRule& R = A.rule[h.rule];
        for (u32 t0 = 0; t0 < h.count; t0 += 32 * kPClaim) {
            u64 key[kPClaim], mine[kPClaim], ik[kPClaim];
            bool valid[kPClaim];
#pragma unroll
            for (int b = 0; b < kPClaim; b++) {
                const u32 t = t0 + (u32)b * 32 + lane;
                valid[b] = t < h.count;
                ik[b] = valid[b] ? R.inner[h.start + t] : 0;
            }
#pragma unroll
            for (int b = 0; b < kPClaim; b++) {
                const u64 sp = h.pos + t0 + (u64)b * 32 + lane;
                key[b] = valid[b] ? project(R.pj, h.key, ik[b], A.bits) : 0;
                mine[b] = ep40 + sp;
                if (valid[b]) A.cand[sp] = key[b];
            }
            claim_batch(R.seen, R.seen_cap, key, mine, valid, lm, &c->flags);
        }
    }
}

// ---------------------------------------------------------------------------
// claims of a copy / copy_filter rule: one candidate per input row
// ---------------------------------------------------------------------------
__device__ void p_copy(const PersistArgs& A, int q)
{
    IterCtl* c = A.ctl;
    const PRule& R = A.rule[q];
    const u64 n = p_rows_n(c, R.in);
    if (blockIdx.x == 0 && threadIdx.x == 0) c->cand_n[q] = n;
    if (n == 0) return;
    const u64 cbase = p_stream_base(c, q);
    if (cbase + n > A.plan.cand_cap) {
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(&c->flags, kFlagOverflow);
        return;
    }
    const u64* __restrict__ in = p_rows_ptr(c, R.in);
    const u64 epoch = ldcg(&c->epoch);
    const u64 tag_base = (epoch << 40) | cbase;
    const LoserMarks lm{A.loser, (u32)epoch, epoch << 40, 0};
    u64* out = A.cand + cbase;
    const u64 stride = (u64)gridDim.x * kThreads * kPClaim;
    for (u64 p0 = (u64)blockIdx.x * kThreads * kPClaim; p0 < n; p0 += stride) {
        u64 key[kPClaim], mine[kPClaim];
        bool valid[kPClaim];
#pragma unroll
        for (int k = 0; k < kPClaim; k++) {
            const u64 p = p0 + threadIdx.x + (u64)k * kThreads;
            valid[k] = false;
            key[k] = 0;
            mine[k] = tag_base + p;
            if (p < n) {
                const u64 kk = in[p];
                bool keep = true;
                if (R.pred != 0) {
                    const u64 a = column_of(kk, R.pj.outer_arity, 0, A.bits);
                    const u64 b = R.pj.outer_arity > 1 ? column_of(kk, R.pj.outer_arity, 1, A.bits) : 0;
                    keep = eval_pred(R.pred, a, b);
                }
                key[k] = keep ? project(R.pj, kk, 0, A.bits) : kEmpty;
                out[p] = key[k];
                valid[k] = keep;
            }
        }
        claim_batch(R.seen, R.seen_cap, key, mine, valid, lm, &c->flags);
    }
}

// ---------------------------------------------------------------------------
// winner selection of rule q into its relation's log
// ---------------------------------------------------------------------------
__device__ void p_select(const PersistArgs& A, int q, int tslot)
{
    IterCtl* c = A.ctl;
    const PRule& R = A.rule[q];
    const int lane = threadIdx.x & 31;
    const u64 cnt = ldcg(&c->cand_n[q]);
    if (cnt == 0) {
        if (blockIdx.x == 0 && threadIdx.x == 0) c->win_n[q] = 0;
        return;
    }
    const u64 nch = (cnt + kPSChunk - 1) / kPSChunk;
    if (nch > A.status_cap) {
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(&c->flags, kFlagStatus);
        return;
    }
    const int out = A.plan.rule_out[q], ts = A.plan.rule_tag[q];
    u64 dst_off = ldcg(&c->full_n[out]) + ldcg(&c->delta_n[out]), id_ctr = ldcg(&c->intern[ts]);
    for (int p = 0; p < q; p++) {
        if (A.plan.rule_out[p] == out) dst_off += ldcg(&c->win_n[p]);
        if (A.plan.rule_tag[p] == ts) id_ctr += ldcg(&c->win_n[p]);
    }
    const u64 tag_word = A.plan.rel_tag_word[out];
    const u64 cbase = p_stream_base(c, q);
    const u64 iteration = ldcg(&c->iteration);
    const u32 ep = (u32)ldcg(&c->epoch);
    const u64* __restrict__ in = A.cand + cbase;
    const u32* __restrict__ mk = A.loser + cbase;
    const u32 tag = p_iter_tag(iteration, tslot);
    u64* __restrict__ dk = R.dst_keys + dst_off;
    u64* __restrict__ dv = R.dst_ids + dst_off;
    u64* inst_row = A.inst_base ? A.inst_new + iteration * A.n_inst : nullptr;
    const u64 W = (u64)gridDim.x * kWarps;
    for (u64 ch = (u64)blockIdx.x * kWarps + (threadIdx.x >> 5); ch < nch; ch += W) {
        const u64 p0 = ch * kPSChunk;
        u64 key[kPSelPerLane];
        u32 mark[kPSelPerLane];
#pragma unroll
        for (int k = 0; k < kPSelPerLane; k++) {
            const u64 p = p0 + (u64)k * 32 + lane;
            key[k] = kEmpty;
            mark[k] = ep;
            if (p < cnt) {
                key[k] = in[p];
                mark[k] = mk[p];
            }
        }
        u32 ball[kPSelPerLane];
        u64 agg = 0;
#pragma unroll
        for (int k = 0; k < kPSelPerLane; k++) {
            if (mark[k] == ep) key[k] = kEmpty;
            ball[k] = __ballot_sync(0xffffffffu, key[k] != kEmpty);
            agg += __popc(ball[k]);
        }
        const u64 prefix = p_lookback(A.status, (u32)ch, agg, tag, &c->flags);
        if (ch == nch - 1 && lane == 0) c->win_n[q] = prefix + agg;
        u64 r = prefix;
        const u32 lt = lanemask_lt();
#pragma unroll
        for (int k = 0; k < kPSelPerLane; k++) {
            if (key[k] != kEmpty) {
                const u64 at = r + __popc(ball[k] & lt);
                dk[at] = key[k];
                dv[at] = tag_word | (id_ctr + at);
            }
            r += __popc(ball[k]);
        }
        if (inst_row) {
#pragma unroll
            for (int k = 0; k < kPSelPerLane; k++) {
                const bool v = key[k] != kEmpty;
                const u32 inst = v ? instance_of(A.inst_base, A.n_inst, key[k] >> R.inst_shift)
                                   : (0x80000000u | (u32)lane);
                const u32 peers = __match_any_sync(0xffffffffu, inst);
                if (v && (peers & lt) == 0) atomicAdd((unsigned long long*)&inst_row[inst], (unsigned long long)__popc(peers));
            }
        }
    }
}

// ---------------------------------------------------------------------------
// the SCC's iterations until its fixed point, a full buffer or a stop flag
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads, RA_PERSIST_MIN_BLOCKS) scc_persistent_kernel(const __grid_constant__ PersistArgs A)
{
    __shared__ PJoinSmem s_join[kWarps];
    const int warp = threadIdx.x >> 5;
    const int nr = A.plan.n_rules;
    // uniform: nothing changes the flags before the first barrier (and the host runs
    // SCCs without rules elsewhere)
    if (nr == 0 || *((volatile u32*)&A.ctl->flags)) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) A.ctl->t_phase = global_ns();
    for (;;) {
        BarSnap b{};
        for (int q = 0; q < nr; q++) {
            if (A.rule[q].kind == kJoinRule) p_join(A, q, s_join[warp], q);
            else p_copy(A, q);
            b = grid_barrier(A, q == nr - 1 ? kActClaimsDone : kActClaims);
            if (b.flags) return;
        }
        if (b.heavy) {
            p_heavy(A, b.heavy);
            b = grid_barrier(A, kActHeavy);
            if (b.flags) return;
        }
        for (int q = 0; q < nr; q++) {
            p_select(A, q, nr + q);
            b = grid_barrier(A, q == nr - 1 ? kActIterEnd : kActSelect);
            if (b.flags) return;
        }
        if (b.done) return;
    }
}

}  // namespace ra
