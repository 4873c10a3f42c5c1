// Device-driven fixed-point iteration: every size lives in an IterCtl block in
// device memory, so one iteration is a fixed sequence of launches that can be
// captured once into a CUDA graph and replayed by a conditional WHILE node
// until the delta is empty (RAM::check_for_fixed_point's MPI_Allreduce,
// src/RAM/RA_tasks.cpp:1072-1085, becomes a device flag).
//
// Per iteration, for an SCC whose joins read the DELTA of one relation and the
// FULL of a relation no rule of the SCC writes:
//   join_scan      per outer (delta) row: match count from the inner CSR, single-
//                  pass decoupled look-back scan -> first output slot per row
//   iter_plan      stream position base per rule, capacity guard
//   join_insert    per candidate: merge-path row lookup, projection, candidate
//                  written, first-occurrence claim in the output's seen set
//   copy_insert    (copy / copy_filter rules) same for one candidate per row
//   select         per candidate: winner test, ordered compaction (look-back),
//                  intern ids, digit histograms for the sort
//   sort_pass x P  onesweep LSD radix passes (8-bit digits) into the log
//   iter_end       region bump, history, intern counters, graph condition
#pragma once
#include "ra_kernels.cuh"

namespace ra {

constexpr int kMaxSccRels = 8;
constexpr int kMaxSccRules = 8;
constexpr int kMaxTagSlots = 8;
constexpr int kMaxPasses = 8;
constexpr int kTileSlots = 128;

// flags
constexpr u32 kFlagOverflow = 1u;   // a buffer is too small for this iteration: nothing was mutated
constexpr u32 kFlagTimeout = 2u;    // a bounded look-back wait gave up
constexpr u32 kFlagProbe = 4u;      // a seen-set probe found no slot (table full)
constexpr u32 kFlagHistory = 8u;    // history buffer full

struct IterCtl {
    u64 full_n[kMaxSccRels], delta_n[kMaxSccRels], seen_n[kMaxSccRels];
    u64 cand_n[kMaxSccRules], cand_base[kMaxSccRules], win_n[kMaxSccRules];
    u64 intern[kMaxTagSlots];
    u64 iteration;          // iterations run in this SCC
    u64 epoch;              // seen-set epoch of the running iteration (>= 1)
    u64 batch_pos;
    u64 hist_n;             // (sum_delta, sum_full) pairs recorded
    u64 new_tuples, candidates, outer_rows;
    u64 runs[kMaxSccRels];  // non-empty deltas moved into full (sorted runs added)
    u32 tile_ctr[kTileSlots];
    u32 flags;
    u32 done;
    u64 sort_hist[kMaxSccRels][kMaxPasses][kRadix];
};

// static description of one SCC's iteration, passed by value to the kernels
struct SccPlan {
    int n_rels, n_rules;
    int rule_out[kMaxSccRules];          // output relation slot
    int rule_tag[kMaxSccRules];          // tag slot of the output relation
    int rule_is_join[kMaxSccRules];
    int rule_in_slot[kMaxSccRules];      // copy input: relation slot (DELTA region) or -1 for fixed rows
    u64 rule_in_static_n[kMaxSccRules];  // copy input: rows of a fixed input
    u64 rel_tag_word[kMaxSccRels];       // (tag << 46)
    u64 cand_cap;                        // candidate buffer capacity (all rules of one iteration)
    u64 stage_cap;                       // per-relation staging capacity
    u64 log_cap[kMaxSccRels];
    u64 seen_limit[kMaxSccRels];         // keys a seen set may hold
    u64 hist_cap;                        // history pairs
    u64 off_cap;                         // per-row scan buffers (outer rows of one join)
    u64 batch_size;
    u64 iter_limit;
    int fixpoint;
};

// Rows a rule reads: the DELTA region of an SCC relation (slot >= 0, sizes from
// the control block) or a fixed array (slot < 0: a FULL or DELTA no rule of the
// SCC changes).
struct RowsRef {
    const u64* keys;
    int slot;
    u64 static_n;
};

__device__ __forceinline__ u64 rows_n(const IterCtl* c, const RowsRef& r)
{
    return r.slot >= 0 ? c->delta_n[r.slot] : r.static_n;
}
__device__ __forceinline__ const u64* rows_ptr(const IterCtl* c, const RowsRef& r)
{
    return r.slot >= 0 ? r.keys + c->full_n[r.slot] : r.keys;
}

// ---------------------------------------------------------------------------
// decoupled look-back status words: [tag:24 | flag:2 | value:38]
// ---------------------------------------------------------------------------
constexpr u64 kStAgg = 1, kStIncl = 2;
constexpr int kValBits = 38;
constexpr u64 kValMask = (1ull << kValBits) - 1;
constexpr u64 kSpinLimit = 1ull << 24;

__device__ __forceinline__ u64 st_pack(u32 tag, u64 flag, u64 v)
{
    return ((u64)(tag & 0xffffffu) << 40) | (flag << kValBits) | (v & kValMask);
}
__device__ __forceinline__ u32 st_tag(u64 s) { return (u32)(s >> 40); }
__device__ __forceinline__ u64 st_flag(u64 s) { return (s >> kValBits) & 3; }
__device__ __forceinline__ u64 st_val(u64 s) { return s & kValMask; }

__device__ __forceinline__ void st_publish(u64* p, u64 w)
{
    __threadfence();
    atomicExch((unsigned long long*)p, (unsigned long long)w);
}

__device__ __forceinline__ u64 st_read(const u64* p) { return *((volatile const u64*)p); }

// Exclusive prefix of tile `tile`'s aggregate `agg` over all earlier tiles.
// Called by one thread.  Bounded: gives up after kSpinLimit polls (flag set).
__device__ u64 lookback_one(u64* status, u32 tile, u64 agg, u32 tag, u32* flags)
{
    if (tile == 0) {
        st_publish(&status[0], st_pack(tag, kStIncl, agg));
        return 0;
    }
    st_publish(&status[tile], st_pack(tag, kStAgg, agg));
    u64 excl = 0;
    long t = (long)tile - 1;
    u64 spins = 0;
    while (t >= 0) {
        u64 s = st_read(&status[t]);
        if (st_tag(s) != (tag & 0xffffffu) || st_flag(s) == 0) {
            if (++spins > kSpinLimit) {
                atomicOr(flags, kFlagTimeout);
                break;
            }
            continue;
        }
        excl += st_val(s);
        if (st_flag(s) == kStIncl) break;
        t--;
    }
    st_publish(&status[tile], st_pack(tag, kStIncl, excl + agg));
    return excl;
}

// Warp-cooperative look-back (all 32 lanes of one warp): each round reads the
// 32 nearest unresolved predecessors at once.  Returns the exclusive prefix on
// every lane.  Bounded like lookback_one.
__device__ u64 lookback_warp(u64* status, u32 tile, u64 agg, u32 tag, u32* flags)
{
    const int lane = threadIdx.x & 31;
    const u32 tg = tag & 0xffffffu;
    if (tile == 0) {
        if (lane == 0) st_publish(&status[0], st_pack(tag, kStIncl, agg));
        return 0;
    }
    if (lane == 0) st_publish(&status[tile], st_pack(tag, kStAgg, agg));
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
    if (lane == 0) st_publish(&status[tile], st_pack(tag, kStIncl, excl + agg));
    return excl;
}

__device__ __forceinline__ u32 iter_tag(const IterCtl* c, int slot)
{
    return (u32)(((c->iteration + 1) << 7) | (u64)slot);
}

// first index i in [0, n) with a[i] > x (n if none)
template <typename T>
__device__ __forceinline__ u64 upper_bound_dev(const T* a, u64 n, u64 x)
{
    u64 lo = 0, hi = n;
    while (lo < hi) {
        u64 mid = (lo + hi) >> 1;
        if ((u64)a[mid] <= x) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// ---------------------------------------------------------------------------
// join_scan: count + exclusive scan in one pass
// ---------------------------------------------------------------------------
constexpr int kScanIpt = 4;
constexpr int kScanTile = kThreads * kScanIpt;

__global__ void __launch_bounds__(kThreads) join_scan_kernel(IterCtl* __restrict__ ctl, int rule, RowsRef outer_ref,
                                                             int outer_shift, const u64* __restrict__ csr,
                                                             u64* __restrict__ off, u64* __restrict__ start,
                                                             u64 off_cap, u64* __restrict__ status, int tile_slot)
{
    __shared__ u64 sm[kWarps + 1];
    __shared__ u32 s_tile;
    __shared__ u64 s_prefix;
    if (ctl->flags) return;
    const u64 n = rows_n(ctl, outer_ref);
    const u64* outer = rows_ptr(ctl, outer_ref);
    const u64 ntiles = (n + kScanTile - 1) / kScanTile;
    if (n == 0 || n > off_cap) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            ctl->cand_n[rule] = 0;
            if (n > off_cap) atomicOr(&ctl->flags, kFlagOverflow);
        }
        return;
    }
    const u32 tag = iter_tag(ctl, tile_slot);
    if (blockIdx.x >= ntiles) return;
    for (;;) {
        if (threadIdx.x == 0) s_tile = atomicAdd(&ctl->tile_ctr[tile_slot], 1u);
        __syncthreads();
        const u64 tile = s_tile;
        __syncthreads();
        if (tile >= ntiles) break;
        const u64 base = tile * kScanTile + (u64)threadIdx.x * kScanIpt;
        u64 cnt[kScanIpt];
        u64 local = 0;
#pragma unroll
        for (int k = 0; k < kScanIpt; k++) {
            const u64 i = base + k;
            cnt[k] = 0;
            if (i < n) {
                const u64 j = outer[i] >> outer_shift;
                const u64 s = csr[j];
                cnt[k] = csr[j + 1] - s;
                start[i] = s;
            }
            local += cnt[k];
        }
        u64 agg;
        u64 ex = block_exclusive_scan(local, sm, &agg);
        if (threadIdx.x < 32) {
            const u64 pre = lookback_warp(status, (u32)tile, agg, tag, &ctl->flags);
            if (threadIdx.x == 0) s_prefix = pre;
        }
        __syncthreads();
        u64 run = s_prefix + ex;
#pragma unroll
        for (int k = 0; k < kScanIpt; k++) {
            const u64 i = base + k;
            if (i < n) off[i] = run;
            run += cnt[k];
        }
        if (tile == ntiles - 1 && threadIdx.x == 0) {
            ctl->cand_n[rule] = s_prefix + agg;
            ctl->outer_rows += n;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// iter_plan: stream bases + capacity guard (one warp)
// ---------------------------------------------------------------------------
__global__ void iter_plan_kernel(IterCtl* __restrict__ ctl, SccPlan plan)
{
    if (threadIdx.x != 0 || ctl->flags) return;
    u64 total = 0;
    u64 incoming[kMaxSccRels] = {0};
    for (int r = 0; r < plan.n_rules; r++) {
        if (!plan.rule_is_join[r]) {
            const int s = plan.rule_in_slot[r];
            ctl->cand_n[r] = (s >= 0) ? ctl->delta_n[s] : plan.rule_in_static_n[r];
        }
        ctl->cand_base[r] = total;
        total += ctl->cand_n[r];
        incoming[plan.rule_out[r]] += ctl->cand_n[r];
        ctl->win_n[r] = 0;
    }
    bool over = total > plan.cand_cap;
    // the history entry this iteration may record must fit before anything changes
    const bool records = !plan.fixpoint || ctl->batch_pos + 1 >= plan.batch_size;
    over = over || (records && ctl->hist_n >= plan.hist_cap);
    for (int s = 0; s < plan.n_rels; s++) {
        over = over || incoming[s] > plan.stage_cap;
        over = over || ctl->full_n[s] + ctl->delta_n[s] + incoming[s] > plan.log_cap[s];
        over = over || ctl->seen_n[s] + incoming[s] > plan.seen_limit[s];
    }
    if (over) atomicOr(&ctl->flags, kFlagOverflow);
    else ctl->candidates += total;
}

// ---------------------------------------------------------------------------
// candidate expansion + first-occurrence claim
// ---------------------------------------------------------------------------
constexpr int kInsTile = 1024;
constexpr int kLbsCap = 2048;

// First-occurrence claim of key k by stream position `mine` (tag word), one
// 16-byte CAS per probed slot: an empty slot becomes {k, mine}; a slot holding
// k keeps the smaller tag (older tuples carry tag 0).
__device__ __forceinline__ void claim(Slot* __restrict__ t, u64 mask, u64 k, u64 mine, u32* flags)
{
    const Slot empty{kEmpty, ~0ull};
    const Slot mineslot{k, mine};
    u64 h = mix64(k) & mask;
    for (u64 probe = 0; probe <= mask; probe++) {
        Slot cur = atomicCAS(&t[h], empty, mineslot);
        if (slot_eq(cur, empty)) return;
        if (cur.key == k) {
            while (cur.tag > mine) {
                const Slot prev = atomicCAS(&t[h], cur, mineslot);
                if (slot_eq(prev, cur)) return;
                cur = prev;
            }
            return;
        }
        h = (h + 1) & mask;
    }
    atomicOr(flags, kFlagProbe);
}

__global__ void __launch_bounds__(kThreads) join_insert_kernel(IterCtl* __restrict__ ctl, int rule, RowsRef outer_ref,
                                                               const u64* __restrict__ off,
                                                               const u64* __restrict__ start,
                                                               const u64* __restrict__ inner, Projection pj, int bits,
                                                               u64* __restrict__ cand, Slot* __restrict__ seen,
                                                               u64 seen_mask)
{
    __shared__ u64 s_off[kLbsCap];
    __shared__ u64 s_r0, s_r1;
    if (ctl->flags) return;
    const u64 c = ctl->cand_n[rule];
    if (c == 0) return;
    const u64 n = rows_n(ctl, outer_ref);
    const u64* outer = rows_ptr(ctl, outer_ref);
    const u64 cbase = ctl->cand_base[rule];
    const u64 tag_base = (ctl->epoch << 40) | cbase;
    u64* out = cand + cbase;
    for (u64 p0 = (u64)blockIdx.x * kInsTile; p0 < c; p0 += (u64)gridDim.x * kInsTile) {
        const u64 p1 = min(c, p0 + kInsTile);
        if (threadIdx.x == 0) {
            s_r0 = upper_bound_dev(off, n, p0) - 1;
            s_r1 = upper_bound_dev(off, n, p1 - 1) - 1;
        }
        __syncthreads();
        const u64 r0 = s_r0, span = s_r1 - s_r0 + 1;
        const bool staged = span <= (u64)kLbsCap;
        if (staged)
            for (u64 i = threadIdx.x; i < span; i += kThreads) s_off[i] = off[r0 + i];
        __syncthreads();
        constexpr int kPer = kInsTile / kThreads;
        u64 okey[kPer], ikey[kPer];
        u64 pp[kPer];
#pragma unroll
        for (int k = 0; k < kPer; k++) {
            const u64 p = p0 + threadIdx.x + (u64)k * kThreads;
            pp[k] = p;
            okey[k] = ikey[k] = 0;
            if (p < p1) {
                const u64 i = staged ? r0 + upper_bound_dev(s_off, span, p) - 1 : upper_bound_dev(off, n, p) - 1;
                const u64 j = p - (staged ? s_off[i - r0] : off[i]);
                okey[k] = outer[i];
                ikey[k] = inner[start[i] + j];
            }
        }
#pragma unroll
        for (int k = 0; k < kPer; k++) {
            if (pp[k] >= p1) continue;
            const u64 key = project(pj, okey[k], ikey[k], bits);
            out[pp[k]] = key;
            claim(seen, seen_mask, key, tag_base + pp[k], &ctl->flags);
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kThreads) copy_insert_kernel(IterCtl* __restrict__ ctl, int rule, RowsRef in_ref,
                                                               Projection pj,
                                                               int bits, int pred, u64* __restrict__ cand,
                                                               Slot* __restrict__ seen, u64 seen_mask)
{
    if (ctl->flags) return;
    const u64 c = ctl->cand_n[rule];
    if (c == 0) return;
    const u64* in = rows_ptr(ctl, in_ref);
    const u64 cbase = ctl->cand_base[rule];
    const u64 tag_base = (ctl->epoch << 40) | cbase;
    u64* out = cand + cbase;
    for (u64 p = (u64)blockIdx.x * kThreads + threadIdx.x; p < c; p += (u64)gridDim.x * kThreads) {
        const u64 k = in[p];
        bool keep = true;
        if (pred != 0) {
            u64 a = column_of(k, pj.outer_arity, 0, bits);
            u64 b = pj.outer_arity > 1 ? column_of(k, pj.outer_arity, 1, bits) : 0;
            keep = eval_pred(pred, a, b);
        }
        const u64 key = keep ? project(pj, k, 0, bits) : kEmpty;
        out[p] = key;
        if (keep) claim(seen, seen_mask, key, tag_base + p, &ctl->flags);
    }
}

// ---------------------------------------------------------------------------
// select: winners in candidate order -> staging rows with intern ids
// ---------------------------------------------------------------------------
constexpr int kSelIpt = 4;
constexpr int kSelTile = kThreads * kSelIpt;

// stage_* are the relation's staging rows (sorted afterwards) or, when
// `to_log` is set, the relation's log: winners then land directly in its newt
// region (emission id order, no sort).
__global__ void __launch_bounds__(kThreads) select_kernel(IterCtl* __restrict__ ctl, SccPlan plan, int rule,
                                                          const u64* __restrict__ cand, const Slot* __restrict__ seen,
                                                          u64 seen_mask, u64* __restrict__ stage_keys,
                                                          u64* __restrict__ stage_ids, u64* __restrict__ status,
                                                          int tile_slot, int passes, int to_log)
{
    __shared__ u64 sm[kWarps + 1];
    __shared__ u32 s_tile;
    __shared__ u64 s_prefix;
    __shared__ u32 s_hist[kMaxPasses][kRadix];
    if (ctl->flags) return;
    const u64 c = ctl->cand_n[rule];
    if (c == 0) return;
    const int out = plan.rule_out[rule], tslot = plan.rule_tag[rule];
    // staging offset and intern base: winners of earlier rules into the same relation / tag
    u64 stage_off = 0, id_ctr = ctl->intern[tslot];
    for (int q = 0; q < rule; q++) {
        if (plan.rule_out[q] == out) stage_off += ctl->win_n[q];
        if (plan.rule_tag[q] == tslot) id_ctr += ctl->win_n[q];
    }
    if (to_log) {
        const u64 o = ctl->full_n[out] + ctl->delta_n[out];
        stage_keys += o;
        stage_ids += o;
    }
    const u64 tag_word = plan.rel_tag_word[out];
    const u64 cbase = ctl->cand_base[rule];
    const u64 tag_base = (ctl->epoch << 40) | cbase;
    const u64* in = cand + cbase;
    const u64 ntiles = (c + kSelTile - 1) / kSelTile;
    const u32 tag = iter_tag(ctl, tile_slot);
    if (blockIdx.x >= ntiles) return;
    for (int i = threadIdx.x; i < kMaxPasses * kRadix; i += kThreads) (&s_hist[0][0])[i] = 0;
    for (;;) {
        if (threadIdx.x == 0) s_tile = atomicAdd(&ctl->tile_ctr[tile_slot], 1u);
        __syncthreads();
        const u64 tile = s_tile;
        __syncthreads();
        if (tile >= ntiles) break;
        const u64 base = tile * kSelTile + (u64)threadIdx.x * kSelIpt;
        u64 key[kSelIpt];
        u32 win = 0;
#pragma unroll
        for (int k = 0; k < kSelIpt; k++) {
            const u64 p = base + k;
            key[k] = kEmpty;
            if (p < c) {
                const u64 kk = in[p];
                if (kk != kEmpty) {
                    const u64 h = seen_find(seen, seen_mask, kk);
                    if (h != ~0ull && seen[h].tag == tag_base + p) {
                        key[k] = kk;
                        win++;
                    }
                }
            }
        }
        u64 agg;
        u64 ex = block_exclusive_scan((u64)win, sm, &agg);
        if (threadIdx.x < 32) {
            const u64 pre = lookback_warp(status, (u32)tile, agg, tag, &ctl->flags);
            if (threadIdx.x == 0) s_prefix = pre;
        }
        __syncthreads();
        u64 r = s_prefix + ex;
#pragma unroll
        for (int k = 0; k < kSelIpt; k++) {
            if (key[k] == kEmpty) continue;
            stage_keys[stage_off + r] = key[k];
            stage_ids[stage_off + r] = tag_word | (id_ctr + r);
            for (int ps = 0; ps < passes; ps++)
                atomicAdd(&s_hist[ps][(key[k] >> (ps * kRadixBits)) & (kRadix - 1)], 1u);
            r++;
        }
        if (tile == ntiles - 1 && threadIdx.x == 0) ctl->win_n[rule] = s_prefix + agg;
        __syncthreads();
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * kRadix; i += kThreads) {
        const u32 v = (&s_hist[0][0])[i];
        if (v) atomicAdd(&ctl->sort_hist[out][i / kRadix][i % kRadix], (u64)v);
    }
}

// ---------------------------------------------------------------------------
// onesweep LSD radix pass over a relation's staged rows
// ---------------------------------------------------------------------------
constexpr int kSortIpt = 8;
constexpr int kSortTile = kThreads * kSortIpt;

struct SortPassArgs {
    int rel;                  // relation slot
    int pass, shift;
    const u64* src_k;
    const u64* src_v;
    u64* dst_k;               // when dst_log: the log base (rows go to base + full_n + delta_n)
    u64* dst_v;
    int dst_log;
    int n_rules_in;           // rules writing this relation
    int rules_in[kMaxSccRules];
};

__global__ void __launch_bounds__(kThreads) sort_pass_kernel(IterCtl* __restrict__ ctl, SortPassArgs a,
                                                             u64* __restrict__ status, int tile_slot)
{
    __shared__ u64 s_gstart[kRadix];         // global start of each digit (exclusive scan of the histogram)
    __shared__ u64 s_out[kRadix];            // output position of each digit's run in this tile
    __shared__ u32 s_loc[kRadix];            // tile-local start of each digit's run
    __shared__ u32 s_wcnt[kWarps][kRadix];   // per-warp digit counts, then per-warp bases
    __shared__ u64 s_k[kSortTile];           // the tile, in digit order
    __shared__ u64 s_v[kSortTile];
    __shared__ u64 sm[kWarps + 1];
    __shared__ u32 s_tile;
    if (ctl->flags) return;
    u64 n = 0;
    for (int q = 0; q < a.n_rules_in; q++) n += ctl->win_n[a.rules_in[q]];
    if (n == 0) return;
    const u64 ntiles = (n + kSortTile - 1) / kSortTile;
    if (blockIdx.x >= ntiles) return;
    u64* dk = a.dst_k;
    u64* dv = a.dst_v;
    if (a.dst_log) {
        const u64 o = ctl->full_n[a.rel] + ctl->delta_n[a.rel];
        dk += o;
        dv += o;
    }
    const u32 tag = iter_tag(ctl, tile_slot);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    {
        u64 tot;
        s_gstart[threadIdx.x] = block_exclusive_scan(ctl->sort_hist[a.rel][a.pass][threadIdx.x], sm, &tot);
    }
    for (;;) {
        if (threadIdx.x == 0) s_tile = atomicAdd(&ctl->tile_ctr[tile_slot], 1u);
        for (int i = threadIdx.x; i < kWarps * kRadix; i += kThreads) (&s_wcnt[0][0])[i] = 0;
        __syncthreads();
        const u64 tile = s_tile;
        if (tile >= ntiles) break;
        const u64 t0 = tile * kSortTile;
        const u32 tn = (u32)min((u64)kSortTile, n - t0);
        // warp w owns items [w*32*IPT, (w+1)*32*IPT) of the tile, round-major = index order
        u64 kk[kSortIpt];
        u32 rk[kSortIpt];
#pragma unroll
        for (int r = 0; r < kSortIpt; r++) {
            const u32 li = (u32)(warp * 32 * kSortIpt + r * 32 + lane);
            const bool valid = li < tn;
            kk[r] = valid ? a.src_k[t0 + li] : 0;
            const int d = valid ? (int)((kk[r] >> a.shift) & (kRadix - 1)) : (kRadix + lane);
            const u32 peers = __match_any_sync(0xffffffffu, d);
            const u32 before = __popc(peers & lanemask_lt());
            const u32 prior = valid ? s_wcnt[warp][d] : 0;
            __syncwarp();
            if (valid && before == 0) s_wcnt[warp][d] = prior + __popc(peers);
            __syncwarp();
            rk[r] = prior + before;
        }
        __syncthreads();
        // digit totals of the tile -> tile-local run starts; per-warp bases inside each run
        const int d = threadIdx.x;   // kThreads == kRadix
        u32 run = 0;
#pragma unroll
        for (int w = 0; w < kWarps; w++) {
            const u32 c = s_wcnt[w][d];
            s_wcnt[w][d] = run;
            run += c;
        }
        {
            u64 tot;
            s_loc[d] = (u32)block_exclusive_scan((u64)run, sm, &tot);
        }
        // look-back for this digit across tiles (one thread per digit)
        u64* st = status + tile * kRadix + d;
        u64 excl = 0;
        if (tile == 0) {
            st_publish(st, st_pack(tag, kStIncl, run));
        } else {
            st_publish(st, st_pack(tag, kStAgg, run));
            long t = (long)tile - 1;
            u64 spins = 0;
            while (t >= 0) {
                const u64 sv = st_read(status + (u64)t * kRadix + d);
                if (st_tag(sv) != (tag & 0xffffffu) || st_flag(sv) == 0) {
                    if (++spins > kSpinLimit) {
                        atomicOr(&ctl->flags, kFlagTimeout);
                        break;
                    }
                    continue;
                }
                excl += st_val(sv);
                if (st_flag(sv) == kStIncl) break;
                t--;
            }
            st_publish(st, st_pack(tag, kStIncl, excl + run));
        }
        s_out[d] = s_gstart[d] + excl;
        __syncthreads();
        // place the tile in shared memory in digit order (stable)
#pragma unroll
        for (int r = 0; r < kSortIpt; r++) {
            const u32 li = (u32)(warp * 32 * kSortIpt + r * 32 + lane);
            if (li >= tn) continue;
            const int dd = (int)((kk[r] >> a.shift) & (kRadix - 1));
            const u32 pos = s_loc[dd] + s_wcnt[warp][dd] + rk[r];
            s_k[pos] = kk[r];
            s_v[pos] = a.src_v[t0 + li];
        }
        __syncthreads();
        // each digit's run is contiguous in the output: coalesced writes
        for (u32 q = threadIdx.x; q < tn; q += kThreads) {
            const u64 k = s_k[q];
            const int dd = (int)((k >> a.shift) & (kRadix - 1));
            const u64 pos = s_out[dd] + (q - s_loc[dd]);
            dk[pos] = k;
            dv[pos] = s_v[q];
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// iter_end: semi-naive swap on the counters, history, graph condition
// ---------------------------------------------------------------------------
struct SccRelMap {
    int n_rules_in[kMaxSccRels];
    int rules_in[kMaxSccRels][kMaxSccRules];
};

__global__ void iter_end_kernel(IterCtl* __restrict__ ctl, SccPlan plan, SccRelMap rm, u64* __restrict__ history,
                                cudaGraphConditionalHandle cond, int use_cond)
{
    // every block clears this iteration's sort histograms
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < (u64)kMaxSccRels * kMaxPasses * kRadix;
         i += (u64)gridDim.x * blockDim.x)
        (&ctl->sort_hist[0][0][0])[i] = 0;
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    bool cont = false;
    if (ctl->flags == 0) {
        u64 sum_delta = 0, sum_full = 0, added = 0;
        for (int s = 0; s < plan.n_rels; s++) {
            u64 nn = 0;
            for (int q = 0; q < rm.n_rules_in[s]; q++) nn += ctl->win_n[rm.rules_in[s][q]];
            // relation::insert_delta_in_full + local_insert_in_delta
            if (ctl->delta_n[s]) ctl->runs[s]++;
            ctl->full_n[s] += ctl->delta_n[s];
            ctl->delta_n[s] = nn;
            ctl->seen_n[s] += nn;
            added += nn;
            sum_delta += ctl->delta_n[s];
            sum_full += ctl->full_n[s];
        }
        u64 tag_add[kMaxTagSlots] = {0};
        for (int r = 0; r < plan.n_rules; r++) tag_add[plan.rule_tag[r]] += ctl->win_n[r];
        for (int t = 0; t < kMaxTagSlots; t++) ctl->intern[t] += tag_add[t];
        ctl->new_tuples += added;
        ctl->iteration++;
        ctl->epoch++;
        ctl->batch_pos++;
        cont = true;
        if (!plan.fixpoint) {
            // non-fixpoint SCC: one iteration, one history entry
            history[2 * ctl->hist_n] = sum_delta;
            history[2 * ctl->hist_n + 1] = sum_full;
            ctl->hist_n++;
            cont = false;
        } else if (ctl->batch_pos >= plan.batch_size) {
            ctl->batch_pos = 0;
            if (ctl->hist_n >= plan.hist_cap) {
                atomicOr(&ctl->flags, kFlagHistory);
                cont = false;
            } else {
                history[2 * ctl->hist_n] = sum_delta;
                history[2 * ctl->hist_n + 1] = sum_full;
                ctl->hist_n++;
                cont = sum_delta != 0;
            }
        }
        if (ctl->iteration >= plan.iter_limit) cont = false;
        ctl->done = cont ? 0u : 1u;
    }
    for (int i = 0; i < kTileSlots; i++) ctl->tile_ctr[i] = 0;
    if (use_cond) cudaGraphSetConditional(cond, cont ? 1u : 0u);
}

}  // namespace ra
