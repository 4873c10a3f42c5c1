// Device-driven fixed-point iteration: every size lives in an IterCtl block in
// device memory, so one iteration is a fixed sequence of launches that can be
// captured once into a CUDA graph and replayed by a conditional WHILE node
// until the delta is empty (RAM::check_for_fixed_point's MPI_Allreduce,
// src/RAM/RA_tasks.cpp:1072-1085, becomes a device flag).
//
// Per iteration, for an SCC whose rules read the DELTA of its relations and
// inputs that do not change while it runs (e.g. the FULL of a loaded relation):
//   join_fused     per tile of outer (delta) rows: match counts from the inner
//                  CSR, single-pass decoupled look-back scan of the counts, then
//                  the tile's candidates expanded in place (merge-path over the
//                  tile's rows, so a row is spread over all the block's warps;
//                  a row of more than kHeavyRow matches goes to every block of
//                  the launch as work items), written to the candidate stream and
//                  claimed in the output relation's seen set (first occurrence =
//                  least stream position) -- count, scan and write in one launch
//   copy_claim     (copy / copy_filter rules) one candidate per input row
//   select         per candidate: winner test, ordered compaction (look-back)
//                  straight into the relation's log, intern ids; the last tile
//                  of the last rule runs the iteration end: region bump,
//                  history, intern counters, graph condition
//   (reference id order only) digit histograms in select, onesweep LSD radix
//   passes over the new delta, then a separate iteration-end launch
// An iteration that finds a buffer too small stops before select writes
// anything; claims made so far are idempotent, so the host grows the buffer
// and replays the same iteration (same epoch, same stream positions).
#pragma once
#include "ra_kernels.cuh"

namespace ra {

constexpr int kMaxSccRels = 8;
constexpr int kMaxSccRules = 8;
constexpr int kMaxTagSlots = 8;
constexpr int kMaxPasses = 8;
constexpr int kTileSlots = 128;
constexpr int kTailMaxRules = 2;   // join rules of an SCC the tail kernel (ra_tail.cuh) runs
// a bank of launch counters: kTileSlots tile counters, then 3 heavy-row counters per rule
constexpr int kBankWords = kTileSlots + 3 * kMaxSccRules;

// flags
constexpr u32 kFlagOverflow = 1u;   // a buffer is too small: replay the iteration after growing it
constexpr u32 kFlagTimeout = 2u;    // a bounded look-back wait gave up (fatal)
constexpr u32 kFlagProbe = 4u;      // a seen-set probe gave up (table too full): grow, replay
constexpr u32 kFlagGrow = 8u;       // iteration done; the seen set needs room before the next one
constexpr u32 kFlagRange = 16u;     // a tuple whose columns lie in different instances (fatal)
constexpr u32 kFlagStatus = 32u;    // a launch has more tiles than the look-back status array (fatal)
constexpr u64 kMaxProbe = 4096;

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
    u64 t_start;                    // %globaltimer when the SCC started (ns)
    u64 time_cap;                   // entries of the per-iteration end-time buffer
    u32 tile_ctr[2 * kBankWords];   // two banks: iteration k uses bank k & 1
    u32 exit_ctr;                   // blocks of the running select launch that have finished
    u32 flags;
    u32 done;
    // persistent SCC kernel (ra_persist.cuh): heavy-row work items of the running
    // iteration, and the grid barrier with the values its last arriver publishes
    u32 heavy_ctr;                  // items taken
    u64 heavy_n;                    // items pushed
    u64 ns_claims, ns_heavy, ns_select;   // device time of the phases of the persistent kernel (ns)
    u64 t_phase;                    // %globaltimer at the last barrier release (or kernel start)
    u64 tail_iters;                 // iterations run by the tail kernel (ra_tail.cuh)
    u64 tail_off;                   // the tail kernel declined a skewed iteration: no more tail in this SCC run
    u32 bar_count;                  // blocks arrived at the running barrier
    u32 bar_gen;                    // barrier generation (bumped on release)
    u32 bar_flags;                  // flags / done / heavy_n as the last arriver saw them
    u32 bar_done;
    u64 bar_heavy;
    u64 heavy_items;                // heavy-row work items pushed in this SCC (both paths)
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
// polls before a look-back wait gives up (about a second of L2 round trips); a
// predecessor tile is always resident and running, so a legitimate wait is far shorter
constexpr u64 kSpinLimit = 1ull << 22;

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
__device__ u64 lookback_one(u64* status, u32 tile, u64 agg, u32 tag, u32* flags, u64 limit = kSpinLimit)
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
            if (++spins > limit) {
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

// Failure-path self-test: tile 1 of a look-back whose tile 0 never publishes.
// The wait must give up after `limit` polls and set kFlagTimeout.
__global__ void lookback_selftest_kernel(u64* status, u32* flags, u64 limit)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) lookback_one(status, 1, 1, 7, flags, limit);
}

__device__ __forceinline__ u32 iter_tag(const IterCtl* c, int slot)
{
    return (u32)(((c->iteration + 1) << 7) | (u64)slot);
}

__device__ __forceinline__ u32* tile_counter(IterCtl* c, int slot)
{
    return &c->tile_ctr[(c->iteration & 1) * kBankWords + slot];
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

// candidates of rules before `rule` in this iteration's stream
__device__ __forceinline__ u64 stream_base(const IterCtl* c, int rule)
{
    u64 b = 0;
    for (int q = 0; q < rule; q++) b += c->cand_n[q];
    return b;
}

// ---------------------------------------------------------------------------
// first-occurrence claims: one 16-byte CAS per probed slot.  An empty slot
// becomes {k, mine}; a slot holding k keeps the smaller tag (older tuples carry
// smaller tags: 0, or an earlier epoch).  Every candidate that is not the first
// occurrence of a new tuple ends up marked in `loser` (indexed by stream
// position, value = epoch): it marks itself when the key is older or holds a
// smaller position, and marks the position it displaces when it lowers the
// tag.  select then needs no access to the seen set.  kClaimBatch independent
// claims are issued back to back: two per thread, so that the join kernel fits
// 31 registers and a full SM of threads (measured on tc-er22: 12.03 ms per step
// against 12.55 with four per thread at 64 registers and 4 CTAs per SM).
// ---------------------------------------------------------------------------
constexpr int kClaimBatch = 2;
constexpr u64 kPosMask = (1ull << 40) - 1;

struct LoserMarks {
    u32* mark;      // per stream position (minus `base`)
    u32 epoch;      // marks of this iteration (older values mean "not a loser now")
    u64 epoch_tag;  // epoch << 40: tags below it belong to tuples from earlier iterations
    u64 base;       // stream position of mark[0] (a slice of outer rows starts there; else 0)
};

__device__ __forceinline__ void claim_rest(Slot* __restrict__ t, u64 cap, u64 k, u64 mine, u64 h, Slot cur,
                                           const LoserMarks& lm, u32* flags)
{
    const Slot empty{kEmpty, ~0ull};
    const Slot mineslot{k, mine};
    for (u64 probe = 0; probe < kMaxProbe; probe++) {
        if (slot_eq(cur, empty)) return;   // we inserted it
        if (cur.key == k) {
            for (;;) {
                if (cur.tag == mine) return;     // our own claim from an attempt being replayed
                if (cur.tag < mine) {            // older tuple, or an earlier position this iteration
                    lm.mark[(mine & kPosMask) - lm.base] = lm.epoch;
                    return;
                }
                const Slot prev = atomicCAS(&t[h], cur, mineslot);
                if (slot_eq(prev, cur)) {      // we took the slot from a later position
                    lm.mark[(cur.tag & kPosMask) - lm.base] = lm.epoch;   // a later position: same slice
                    return;
                }
                cur = prev;
            }
        }
        h = slot_next(h, cap);
        cur = atomicCAS(&t[h], empty, mineslot);
    }
    atomicOr(flags, kFlagProbe);
}

// N claims of one thread, issued back to back (N from the caller's arrays, so a
// caller's batch size and this loop cannot disagree)
template <int N>
__device__ __forceinline__ void claim_batch(Slot* __restrict__ t, u64 cap, const u64 (&key)[N], const u64 (&mine)[N],
                                            const bool (&valid)[N], const LoserMarks& lm, u32* flags)
{
    const Slot empty{kEmpty, ~0ull};
    Slot cur[N];
    u64 h[N];
#pragma unroll
    for (int k = 0; k < N; k++) {
        h[k] = slot_start(key[k], cap);
        if (valid[k]) cur[k] = atomicCAS(&t[h[k]], empty, Slot{key[k], mine[k]});
    }
#pragma unroll
    for (int k = 0; k < N; k++)
        if (valid[k]) claim_rest(t, cap, key[k], mine[k], h[k], cur[k], lm, flags);
}

__device__ __forceinline__ LoserMarks loser_marks(const IterCtl* c, u32* mark)
{
    return LoserMarks{mark, (u32)c->epoch, c->epoch << 40, 0};
}

// ---------------------------------------------------------------------------
// Bitmap seen set of a binary relation over a small value domain (at most
// 65,536 values): bit c1 of row c0 is set for every tuple (c0, c1) the relation
// holds.  A claim is a plain read and, for a new tuple, one atomicOr on a word of
// a table a fraction of the size of the hash set; `fresh` collects the
// iteration's new tuples and `dirty[c0]` marks rows holding some, from which
// bitmap_select_kernel emits them in key order.  No candidate stream and no
// loser marks: the set of new tuples is the same as the hash-set path's, and
// their order (sorted) does not depend on which duplicate claimed first.
// ---------------------------------------------------------------------------
struct BitSeen {
    u32* seen;      // null: the relation uses its hash seen set
    u32* fresh;
    u8* dirty;
    u32 words;      // u32 words per row (one matrix: no instances)
    u32 n;          // rows (values)
    // with instances, one matrix per instance: row v's first word, the base value and
    // the words of its instance's rows, the instance itself (null without instances)
    const u64* row_word;
    const u32* row_base;
    const u32* row_words;
    const u32* row_inst;
};

__device__ __forceinline__ u64 bit_word(const BitSeen& b, u64 c0, u64 c1)
{
    return b.row_word ? b.row_word[c0] + ((c1 - b.row_base[c0]) >> 5) : c0 * b.words + (c1 >> 5);
}
__device__ __forceinline__ u32 bit_of(const BitSeen& b, u64 c0, u64 c1)
{
    return 1u << ((b.row_word ? c1 - b.row_base[c0] : c1) & 31);
}

// With instances, is (c0, c1) inside c0's instance matrix?
__device__ __forceinline__ bool bit_in_range(const BitSeen& b, u64 c0, u64 c1)
{
    return !b.row_word || ((c1 - b.row_base[c0]) >> 5) < b.row_words[c0];
}

__device__ __forceinline__ void bit_claim(const BitSeen& b, u64 key, int bits, u32* flags)
{
    const u64 c0 = key >> bits, c1 = key & ((1ull << bits) - 1);
    if (!bit_in_range(b, c0, c1)) {
        atomicOr(flags, kFlagRange);
        return;
    }
    const u64 w = bit_word(b, c0, c1);
    const u32 bit = bit_of(b, c0, c1);
    if (*((volatile u32*)&b.seen[w]) & bit) return;   // known: no atomic
    if (atomicOr(&b.seen[w], bit) & bit) return;      // a duplicate claimed it first
    atomicOr(&b.fresh[w], bit);
    b.dirty[c0] = 1;
}

// Bits of a relation's stored tuples (its full and delta regions).
__global__ void __launch_bounds__(kThreads) bitmap_build_kernel(BitSeen b, const u64* __restrict__ keys, u64 n,
                                                                int bits, u32* __restrict__ err)
{
    for (u64 i = (u64)blockIdx.x * kThreads + threadIdx.x; i < n; i += (u64)gridDim.x * kThreads) {
        const u64 k = keys[i];
        const u64 c0 = k >> bits, c1 = k & ((1ull << bits) - 1);
        if (!bit_in_range(b, c0, c1)) {
            *err = 1u;
            continue;
        }
        atomicOr(&b.seen[bit_word(b, c0, c1)], bit_of(b, c0, c1));
    }
}

// ---------------------------------------------------------------------------
// join_fused: count + look-back scan + expansion + claim, one launch per rule
// ---------------------------------------------------------------------------
#ifndef RA_JOIN_ROWS_PER_THREAD
#define RA_JOIN_ROWS_PER_THREAD 2
#endif
#ifndef RA_JOIN_MIN_BLOCKS
#define RA_JOIN_MIN_BLOCKS 8   // 31 registers: 8 CTAs (2,048 threads) per SM hide the claims' latency
#endif
#ifndef RA_SELECT_IPT
#define RA_SELECT_IPT 4
#endif
#ifndef RA_SELECT_MIN_BLOCKS
#define RA_SELECT_MIN_BLOCKS 4
#endif
constexpr int kJRowsPerThread = RA_JOIN_ROWS_PER_THREAD;
constexpr int kJRows = kThreads * kJRowsPerThread;   // outer rows per tile

// One slice of a rule's outer rows (an iteration whose candidates exceed the
// candidate buffer runs in slices): rows [lo, lo + rows) of the rule's input,
// their candidates at buffer index 0.., stream positions from `pos`.
struct JoinSlice {
    u64 lo, rows, pos;
    int on;
};

// Skewed keys.  An outer row with more than kHeavyRow matches is not expanded
// by its tile's block: it keeps its stream positions, and the tile pushes it as
// work items of kHeavyPiece candidates that every warp of the grid takes from a
// shared list once all tiles have been scanned.
constexpr u64 kHeavyRow = 4096;
constexpr u64 kHeavyPiece = 2048;

// One heavy row's slice of candidates: stream positions [pos, pos + count).
struct __align__(16) HeavyItem {
    u64 pos;     // stream position of the first candidate (relative to the launch's first)
    u64 key;     // the outer row
    u64 start;   // its first inner row of the slice
    u32 count;
    u32 rule;
};
static_assert(sizeof(HeavyItem) == 32, "HeavyItem is read as two 16-byte words");

__device__ __forceinline__ u32 ldcg_u32(const u32* p) { return __ldcg(p); }
__device__ __forceinline__ HeavyItem ldcg_item(const HeavyItem* p)
{
    const ulonglong2 a = __ldcg((const ulonglong2*)p), b = __ldcg((const ulonglong2*)p + 1);
    HeavyItem h;
    h.pos = a.x;
    h.key = a.y;
    h.start = b.x;
    h.count = (u32)b.y;
    h.rule = (u32)(b.y >> 32);
    return h;
}

// Per-rule counters of the heavy-row list, banked with the tile counters.
enum HeavyWord { kHvItems = 0, kHvScanned = 1, kHvTaken = 2 };
__device__ __forceinline__ u32* heavy_counter(IterCtl* c, int rule, int w)
{
    return &c->tile_ctr[(c->iteration & 1) * kBankWords + kTileSlots + 3 * rule + w];
}

// Shared memory of one join block.
struct JoinSmem {
    u64 ex[kJRows + 1];   // exclusive prefix of match counts inside the tile
    u32 lx[kJRows + 1];   // the same over the rows this block expands (kSplit: heavy rows count 0)
    u64 start[kJRows];    // first inner row of each outer row
    u64 key[kJRows];      // outer keys
    u64 sm[kWarps + 1];
    u32 tile;
    u64 prefix, hbase, hn;
};

// The tiles of one join launch.  kSplit: the inner CSR has rows longer than
// kHeavyRow, so a tile's heavy rows go to the shared list and every block
// expands that list after the tiles; without it the code is the plain tile loop.
template <bool kSplit>
__device__ __forceinline__ void join_tiles(JoinSmem& S, IterCtl* __restrict__ ctl, int rule, const u64* __restrict__ outer,
                                           u64 n, int outer_shift, const u64* __restrict__ csr,
                                           const u64* __restrict__ inner, const Projection& pj, int bits,
                                           u64* __restrict__ cand, u64 cand_cap, Slot* __restrict__ seen,
                                           u64 seen_cap, u32* __restrict__ loser, u64* __restrict__ status,
                                           int tile_slot, const BitSeen& bs, const JoinSlice& sl,
                                           HeavyItem* __restrict__ heavy, u64 heavy_cap)
{
    const u64 ntiles = (n + kJRows - 1) / kJRows;
    if (!kSplit && blockIdx.x >= ntiles) return;
    const u64 cbase = sl.on ? 0 : stream_base(ctl, rule);   // buffer index of the first candidate
    const u64 tag_base = (ctl->epoch << 40) | (sl.on ? sl.pos : cbase);
    const u32 tag = iter_tag(ctl, tile_slot);
    u32* ctr = tile_counter(ctl, tile_slot);
    LoserMarks lm = loser_marks(ctl, loser);
    lm.base = sl.on ? sl.pos : 0;
    if (kSplit && threadIdx.x == 0) {   // heavy items of the earlier rules of this iteration come first
        u64 b = 0;
        for (int r = 0; r < rule; r++) b += *heavy_counter(ctl, r, kHvItems);
        S.hbase = b;
    }
    for (;;) {
        // (kSplit) a block beyond the tiles that sees every tile taken needs no atomic
        if (threadIdx.x == 0)
            S.tile = (kSplit && blockIdx.x >= ntiles && ldcg_u32(ctr) >= (u32)ntiles) ? (u32)ntiles
                                                                                     : atomicAdd(ctr, 1u);
        __syncthreads();
        const u64 tile = S.tile;
        __syncthreads();
        if (tile >= ntiles) break;
        const u64 r0 = tile * kJRows;
        u64 cnt[kJRowsPerThread];
        u64 local = 0;   // kSplit: (all matches << 24) | matches of the rows expanded here
#pragma unroll
        for (int k = 0; k < kJRowsPerThread; k++) {
            const int li = threadIdx.x * kJRowsPerThread + k;
            const u64 i = r0 + li;
            cnt[k] = 0;
            if (i < n) {
                const u64 key = outer[i];
                const u64 j = key >> outer_shift;
                const u64 s = csr[j];
                cnt[k] = csr[j + 1] - s;
                S.start[li] = s;
                S.key[li] = key;
            }
            local += kSplit ? ((cnt[k] << 24) | (cnt[k] > kHeavyRow ? 0 : cnt[k])) : cnt[k];
        }
        u64 aggp;
        u64 ex = block_exclusive_scan(local, S.sm, &aggp);
        bool mine_heavy = false;
#pragma unroll
        for (int k = 0; k < kJRowsPerThread; k++) {
            const int li = threadIdx.x * kJRowsPerThread + k;
            if (kSplit) {
                S.ex[li] = ex >> 24;
                S.lx[li] = (u32)(ex & 0xffffffu);
                ex += (cnt[k] << 24) | (cnt[k] > kHeavyRow ? 0 : cnt[k]);
                mine_heavy |= cnt[k] > kHeavyRow;
            } else {
                S.ex[li] = ex;
                ex += cnt[k];
            }
        }
        const u64 agg = kSplit ? aggp >> 24 : aggp, lagg = kSplit ? aggp & 0xffffffu : aggp;
        if (threadIdx.x == 0) {
            S.ex[kJRows] = agg;
            if (kSplit) S.lx[kJRows] = (u32)lagg;
        }
        if (threadIdx.x < 32) {
            const u64 pre = lookback_warp(status, (u32)tile, agg, tag, &ctl->flags);
            if (threadIdx.x == 0) S.prefix = pre;
        }
        __syncthreads();
        const u64 prefix = S.prefix;
        if (tile == ntiles - 1 && threadIdx.x == 0) {
            ctl->cand_n[rule] = prefix + agg;
            ctl->outer_rows += n;
        }
        const bool room = bs.seen || cbase + prefix + agg <= cand_cap;
        if (!room && threadIdx.x == 0) atomicOr(&ctl->flags, kFlagOverflow);
        if (kSplit) {
            if (room && mine_heavy) {
#pragma unroll
                for (int k = 0; k < kJRowsPerThread; k++) {
                    if (cnt[k] <= kHeavyRow) continue;
                    const int li = threadIdx.x * kJRowsPerThread + k;
                    const u64 pieces = (cnt[k] + kHeavyPiece - 1) / kHeavyPiece;
                    const u64 at = S.hbase + atomicAdd(heavy_counter(ctl, rule, kHvItems), (u32)pieces);
                    if (at + pieces > heavy_cap) {
                        atomicOr(&ctl->flags, kFlagOverflow);
                        continue;
                    }
                    const u64 p0 = prefix + S.ex[li];
                    for (u64 pc = 0; pc < pieces; pc++) {
                        const u64 off = pc * kHeavyPiece;
                        heavy[at + pc] = HeavyItem{p0 + off, S.key[li], S.start[li] + off,
                                                   (u32)min(kHeavyPiece, cnt[k] - off), (u32)rule};
                    }
                    atomicAdd((unsigned long long*)&ctl->heavy_items, (unsigned long long)pieces);
                }
                __threadfence();
            }
            __syncthreads();
            if (threadIdx.x == 0) atomicAdd(heavy_counter(ctl, rule, kHvScanned), 1u);
        }
        if (room) {
            // the tile's candidates expanded here: position prefix + ex[row] + rank
            const u64 nr = min((u64)kJRows, n - r0);
            for (u64 j0 = 0; j0 < lagg; j0 += (u64)kThreads * kClaimBatch) {
                u64 key[kClaimBatch], mine[kClaimBatch];
                bool valid[kClaimBatch];
                u64 ik[kClaimBatch];
                u64 at[kClaimBatch];
                int rr[kClaimBatch];
#pragma unroll
                for (int k = 0; k < kClaimBatch; k++) {
                    const u64 j = j0 + threadIdx.x + (u64)k * kThreads;
                    valid[k] = j < lagg;
                    rr[k] = 0;
                    at[k] = 0;
                    ik[k] = 0;
                    if (valid[k]) {
                        u64 rank;
                        if (!kSplit || lagg == agg) {   // no heavy row in the tile: j is the position
                            rr[k] = (int)upper_bound_dev(S.ex, nr, j) - 1;
                            rank = j - S.ex[rr[k]];
                            at[k] = prefix + j;
                        } else {
                            rr[k] = (int)upper_bound_dev(S.lx, nr, j) - 1;
                            rank = j - S.lx[rr[k]];
                            at[k] = prefix + S.ex[rr[k]] + rank;
                        }
                        ik[k] = inner[S.start[rr[k]] + rank];
                    }
                }
#pragma unroll
                for (int k = 0; k < kClaimBatch; k++) {
                    key[k] = valid[k] ? project(pj, S.key[rr[k]], ik[k], bits) : 0;
                    mine[k] = tag_base + at[k];
                    if (valid[k] && !bs.seen) cand[cbase + at[k]] = key[k];
                }
                if (bs.seen) {
#pragma unroll
                    for (int k = 0; k < kClaimBatch; k++)
                        if (valid[k]) bit_claim(bs, key[k], bits, &ctl->flags);
                } else {
                    claim_batch(seen, seen_cap, key, mine, valid, lm, &ctl->flags);
                }
            }
        }
        __syncthreads();
    }
    if (!kSplit) return;
    // Heavy rows.  This block saw every tile taken, each by a running block that
    // scans (and pushes) its tile before expanding it, so the wait ends once the
    // last tile's look-back has; bounded all the same.
    if (threadIdx.x == 0) {
        u64 spins = 0;
        const u32* scanned = heavy_counter(ctl, rule, kHvScanned);
        while (ldcg_u32(scanned) < (u32)ntiles) {
            if (++spins > kSpinLimit) {
                atomicOr(&ctl->flags, kFlagTimeout);
                break;
            }
            __nanosleep(64);
        }
        __threadfence();
        // a push that found the list full reserved items it never wrote: the
        // iteration is replayed with more room, so nothing is taken
        const u64 items = ldcg_u32(heavy_counter(ctl, rule, kHvItems));
        const bool bad = spins > kSpinLimit || (ldcg_u32(&ctl->flags) & (kFlagOverflow | kFlagTimeout)) ||
                         S.hbase + items > heavy_cap;
        S.hn = bad ? 0 : items;
    }
    __syncthreads();
    const u64 hn = S.hn;
    if (hn == 0) return;
    const int lane = threadIdx.x & 31;
    u32* taken = heavy_counter(ctl, rule, kHvTaken);
    for (;;) {
        u32 it = 0;
        if (lane == 0) it = atomicAdd(taken, 1u);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= hn) break;
        const HeavyItem h = ldcg_item(&heavy[S.hbase + it]);
        for (u32 t0 = 0; t0 < h.count; t0 += 32 * kClaimBatch) {
            u64 key[kClaimBatch], mine[kClaimBatch], ik[kClaimBatch];
            bool valid[kClaimBatch];
#pragma unroll
            for (int b = 0; b < kClaimBatch; b++) {
                const u32 t = t0 + (u32)b * 32 + lane;
                valid[b] = t < h.count;
                ik[b] = valid[b] ? inner[h.start + t] : 0;
            }
#pragma unroll
            for (int b = 0; b < kClaimBatch; b++) {
                const u64 at = h.pos + t0 + (u64)b * 32 + lane;
                key[b] = valid[b] ? project(pj, h.key, ik[b], bits) : 0;
                mine[b] = tag_base + at;
                if (valid[b] && !bs.seen) cand[cbase + at] = key[b];
            }
            if (bs.seen) {
#pragma unroll
                for (int b = 0; b < kClaimBatch; b++)
                    if (valid[b]) bit_claim(bs, key[b], bits, &ctl->flags);
            } else {
                claim_batch(seen, seen_cap, key, mine, valid, lm, &ctl->flags);
            }
        }
    }
}

// One join rule's launch.  kSplit (the host's choice: the inner CSR has a row
// longer than kHeavyRow) adds the heavy-row list; otherwise the plain tile loop.
template <bool kSplit>
__global__ void __launch_bounds__(kThreads, RA_JOIN_MIN_BLOCKS) join_fused_kernel(IterCtl* __restrict__ ctl, int rule, RowsRef outer_ref,
                                                              int outer_shift, const u64* __restrict__ csr,
                                                              const u64* __restrict__ inner, Projection pj, int bits,
                                                              u64* __restrict__ cand, u64 cand_cap,
                                                              Slot* __restrict__ seen, u64 seen_cap,
                                                              u32* __restrict__ loser, u64* __restrict__ status,
                                                              u64 status_cap, int tile_slot, BitSeen bs, JoinSlice sl,
                                                              HeavyItem* __restrict__ heavy, u64 heavy_cap)
{
    __shared__ JoinSmem S;
    if (ctl->flags || ctl->done) return;   // done: the tail kernel reached the fixed point
    const u64 n = sl.on ? sl.rows : rows_n(ctl, outer_ref);
    const u64* outer = rows_ptr(ctl, outer_ref) + (sl.on ? sl.lo : 0);
    if (n == 0) {
        if (blockIdx.x == 0 && threadIdx.x == 0) ctl->cand_n[rule] = 0;
        return;
    }
    const u64 ntiles = (n + kJRows - 1) / kJRows;
    if (ntiles > status_cap) {   // the host sizes status for the largest outer input: never taken
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(&ctl->flags, kFlagStatus);
        return;
    }
    join_tiles<kSplit>(S, ctl, rule, outer, n, outer_shift, csr, inner, pj, bits, cand, cand_cap, seen, seen_cap,
                       loser, status, tile_slot, bs, sl, heavy, heavy_cap);
}

// Candidates of every tile of kJRows outer rows (the host cuts an iteration
// whose candidates exceed the candidate buffer into slices of whole tiles).
__global__ void __launch_bounds__(kThreads) join_tile_counts_kernel(const IterCtl* __restrict__ ctl, RowsRef outer_ref,
                                                                    int outer_shift, const u64* __restrict__ csr,
                                                                    u64* __restrict__ tile_cnt)
{
    __shared__ u64 sm[kWarps + 1];
    const u64 n = rows_n(ctl, outer_ref);
    const u64* outer = rows_ptr(ctl, outer_ref);
    const u64 ntiles = (n + kJRows - 1) / kJRows;
    for (u64 t = blockIdx.x; t < ntiles; t += gridDim.x) {
        u64 c = 0;
        for (u64 i = t * kJRows + threadIdx.x; i < min(n, (t + 1) * kJRows); i += kThreads) {
            const u64 j = outer[i] >> outer_shift;
            c += csr[j + 1] - csr[j];
        }
        const u64 tot = block_reduce_sum(c, sm);
        if (threadIdx.x == 0) tile_cnt[t] = tot;
    }
}

// copy / copy_filter: one candidate per input row, stream position = row index
__global__ void __launch_bounds__(kThreads) copy_claim_kernel(IterCtl* __restrict__ ctl, SccPlan plan, int rule,
                                                              RowsRef in_ref, Projection pj, int bits, int pred,
                                                              u64* __restrict__ cand, u64 cand_cap,
                                                              Slot* __restrict__ seen, u64 seen_cap,
                                                              u32* __restrict__ loser, BitSeen bs)
{
    if (ctl->flags || ctl->done) return;
    const u64 c = rows_n(ctl, in_ref);
    if (blockIdx.x == 0 && threadIdx.x == 0) ctl->cand_n[rule] = c;
    if (c == 0) return;
    const u64 cbase = stream_base(ctl, rule);
    if (!bs.seen && cbase + c > cand_cap) {
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(&ctl->flags, kFlagOverflow);
        return;
    }
    const u64* in = rows_ptr(ctl, in_ref);
    const u64 tag_base = (ctl->epoch << 40) | cbase;
    const LoserMarks lm = loser_marks(ctl, loser);
    u64* out = cand + cbase;
    const u64 stride = (u64)gridDim.x * kThreads * kClaimBatch;
    for (u64 p0 = (u64)blockIdx.x * kThreads * kClaimBatch; p0 < c; p0 += stride) {
        u64 key[kClaimBatch], mine[kClaimBatch];
        bool valid[kClaimBatch];
#pragma unroll
        for (int k = 0; k < kClaimBatch; k++) {
            const u64 p = p0 + threadIdx.x + (u64)k * kThreads;
            valid[k] = false;
            key[k] = 0;
            mine[k] = tag_base + p;
            if (p < c) {
                const u64 kk = in[p];
                bool keep = true;
                if (pred != 0) {
                    u64 a = column_of(kk, pj.outer_arity, 0, bits);
                    u64 b = pj.outer_arity > 1 ? column_of(kk, pj.outer_arity, 1, bits) : 0;
                    keep = eval_pred(pred, a, b);
                }
                key[k] = keep ? project(pj, kk, 0, bits) : kEmpty;
                if (!bs.seen) out[p] = key[k];
                valid[k] = keep;
            }
        }
        if (bs.seen) {
#pragma unroll
            for (int k = 0; k < kClaimBatch; k++)
                if (valid[k]) bit_claim(bs, key[k], bits, &ctl->flags);
        } else {
            claim_batch(seen, seen_cap, key, mine, valid, lm, &ctl->flags);
        }
    }
    (void)plan;
}

// ---------------------------------------------------------------------------
// end of an iteration (one thread): semi-naive swap on the counters, history,
// intern counters, next bank of tile counters, graph condition.
// ---------------------------------------------------------------------------
struct SccRelMap {
    int n_rules_in[kMaxSccRels];
    int rules_in[kMaxSccRels][kMaxSccRules];
};

__device__ __forceinline__ u64 global_ns()
{
    u64 t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// history holds plan.hist_cap (sum_delta, sum_full) pairs, then time_cap
// per-iteration end times (%globaltimer, ns)
__device__ void end_of_iteration(IterCtl* __restrict__ ctl, const SccPlan& plan, const SccRelMap& rm,
                                 u64* __restrict__ history, cudaGraphConditionalHandle cond, int use_cond)
{
    bool cont = false;
    const bool records = !plan.fixpoint || ctl->batch_pos + 1 >= plan.batch_size;
    if (ctl->flags == 0 && records && ctl->hist_n >= plan.hist_cap) atomicOr(&ctl->flags, kFlagOverflow);
    if (ctl->flags == 0) {
        u64 sum_delta = 0, sum_full = 0, added = 0;
        bool grow = false;
        for (int s = 0; s < plan.n_rels; s++) {
            u64 nn = 0, in = 0;
            for (int q = 0; q < rm.n_rules_in[s]; q++) {
                nn += ctl->win_n[rm.rules_in[s][q]];
                in += ctl->cand_n[rm.rules_in[s][q]];
            }
            // relation::insert_delta_in_full + local_insert_in_delta
            if (ctl->delta_n[s]) ctl->runs[s]++;
            ctl->full_n[s] += ctl->delta_n[s];
            ctl->delta_n[s] = nn;
            ctl->seen_n[s] += nn;
            added += nn;
            sum_delta += ctl->delta_n[s];
            sum_full += ctl->full_n[s];
            if (rm.n_rules_in[s] && ctl->seen_n[s] + 2 * in > plan.seen_limit[s]) grow = true;
        }
        u64 tag_add[kMaxTagSlots] = {0};
        for (int r = 0; r < plan.n_rules; r++) tag_add[plan.rule_tag[r]] += ctl->win_n[r];
        for (int t = 0; t < kMaxTagSlots; t++) ctl->intern[t] += tag_add[t];
        u64 cands = 0;
        for (int r = 0; r < plan.n_rules; r++) cands += ctl->cand_n[r];
        ctl->candidates += cands;
        ctl->new_tuples += added;
        if (ctl->iteration < ctl->time_cap) history[2 * plan.hist_cap + ctl->iteration] = global_ns();
        ctl->iteration++;
        ctl->epoch++;
        ctl->batch_pos++;
        cont = true;
        if (records) {
            ctl->batch_pos = 0;
            history[2 * ctl->hist_n] = sum_delta;
            history[2 * ctl->hist_n + 1] = sum_full;
            ctl->hist_n++;
            cont = plan.fixpoint && sum_delta != 0;
        }
        if (ctl->iteration >= plan.iter_limit) cont = false;
        ctl->done = cont ? 0u : 1u;
        if (cont && grow) {
            atomicOr(&ctl->flags, kFlagGrow);
            cont = false;
        }
        // the next iteration's bank of tile counters (used last by the previous iteration)
        for (int i = 0; i < kBankWords; i++) ctl->tile_ctr[(ctl->iteration & 1) * kBankWords + i] = 0;
        ctl->heavy_n = 0;
        ctl->heavy_ctr = 0;
    }
    if (use_cond) cudaGraphSetConditional(cond, cont ? 1u : 0u);
}

// ---------------------------------------------------------------------------
// select: winners in candidate order -> the relation's log (emission ids) or
// its staging rows (reference ids, sorted afterwards)
// ---------------------------------------------------------------------------
constexpr int kSelIpt = RA_SELECT_IPT;
constexpr int kSelTile = kThreads * kSelIpt;

struct SelectArgs {
    int rule;
    int last;                 // last rule of the iteration: runs the iteration end
    u64* dst_keys;            // log (to_log) or staging rows
    u64* dst_ids;
    int to_log;
    int passes;               // digit histograms to accumulate (reference ids)
    u64 stage_cap;
    // a slice of the rule's outer rows: candidates at buffer index 0; `appended` winners of
    // this iteration already in the relation's log (earlier rules and slices), `id_appended`
    // already numbered under the rule's tag; the iteration end runs after the last slice
    int sliced;
    u64 appended, id_appended;
    // instance accounting (batched programs): instance i owns values [inst_base[i], inst_base[i+1])
    const u64* inst_base;     // n_inst + 1 entries, or null
    u32 n_inst;
    int inst_shift;           // bit offset of column 0 in the output relation's key
    u64* inst_new;            // [iteration][instance] counts of new tuples
    u64 inst_iter_cap;
    // the tail kernel (ra_tail.cuh) follows the graph's WHILE loop: the iteration end
    // stops the loop when every join rule's next outer delta has at most tail_rows rows
    int tail_on;
    int tail_nslots;
    int tail_slot[kTailMaxRules];
    u64 tail_rows;
};

// Does the next iteration go to the tail kernel?  (After the iteration end: not
// done, no flag, every join rule's next delta small.)
__device__ __forceinline__ bool tail_next(const IterCtl* c, const SelectArgs& a)
{
    bool small = c->flags == 0 && c->done == 0 && c->tail_off == 0;
    for (int i = 0; i < a.tail_nslots; i++) small = small && c->delta_n[a.tail_slot[i]] <= a.tail_rows;
    return small;
}

// instance owning value v (inst_base sorted, n + 1 entries)
__device__ __forceinline__ u32 instance_of(const u64* __restrict__ base, u32 n, u64 v)
{
    u32 lo = 0, hi = n;   // base[lo] <= v < base[hi]
    while (hi - lo > 1) {
        const u32 mid = (lo + hi) >> 1;
        if (__ldg(&base[mid]) <= v) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Per-row tables of the instances' bit matrices: row v of instance i (values
// base[i] .. min(base[i + 1], rows) - 1, words w_i = ceil(n_i / 32) per row) starts at
// word inst_word[i] + (v - base[i]) * w_i.  `base` holds n_inst + 1 entries (a sentinel last).
__global__ void __launch_bounds__(kThreads) bitmap_tables_kernel(const u64* __restrict__ base, u32 n_inst,
                                                                 const u64* __restrict__ inst_word, u64 rows,
                                                                 u64* __restrict__ row_word, u32* __restrict__ row_base,
                                                                 u32* __restrict__ row_words, u32* __restrict__ row_inst)
{
    for (u64 v = (u64)blockIdx.x * kThreads + threadIdx.x; v < rows; v += (u64)gridDim.x * kThreads) {
        const u32 i = instance_of(base, n_inst, v);
        const u64 b = base[i], e = min(base[i + 1], rows), w = v < b ? 0 : (e - b + 31) / 32;
        // a value below the first instance has no words: every tuple on its row is out of range
        row_word[v] = v < b ? 0 : inst_word[i] + (v - b) * w;
        row_base[v] = (u32)b;
        row_words[v] = (u32)w;
        row_inst[v] = i;
    }
}

__global__ void __launch_bounds__(kThreads, RA_SELECT_MIN_BLOCKS) select_kernel(IterCtl* __restrict__ ctl,
                                                          // read in place from the parameter space (indexed by rule / relation)
                                                          const __grid_constant__ SccPlan plan,
                                                          const __grid_constant__ SccRelMap rm,
                                                          const __grid_constant__ SelectArgs a, const u64* __restrict__ cand,
                                                          const u32* __restrict__ loser,
                                                          u64* __restrict__ status, int tile_slot,
                                                          u64* __restrict__ history, cudaGraphConditionalHandle cond,
                                                          int use_cond)
{
    static_assert(kSelIpt == 4, "select loads a thread's candidates as 2 x 16 bytes and its marks as 16 bytes");
    __shared__ u64 sm[kWarps + 1];
    __shared__ u32 s_tile;
    __shared__ u64 s_prefix;
    __shared__ u32 s_hist[kMaxPasses][kRadix];
    __shared__ u64 s_win[kSelTile];   // the tile's winners, compacted, for coalesced stores
    if (ctl->done) return;   // the tail kernel reached the fixed point in this body
    const int rule = a.rule;
    const u64 c = ctl->cand_n[rule];
    const int out = plan.rule_out[rule], tslot = plan.rule_tag[rule];
    bool active = ctl->flags == 0;
    if (active) {
        // Room for every candidate of every rule of the iteration, checked by every select
        // before any write, so that an iteration either writes all its winners or none
        // (a replay then never counts a winner twice).  The new delta lands in the log
        // either way (directly, or via staging + sort).
        bool over = a.inst_base && ctl->iteration >= a.inst_iter_cap;
        if (a.sliced) {
            const int s = plan.rule_out[rule];
            over = over || ctl->full_n[s] + ctl->delta_n[s] + a.appended + ctl->cand_n[rule] > plan.log_cap[s];
        } else {
            for (int s = 0; s < plan.n_rels; s++) {
                u64 incoming = 0;
                for (int q = 0; q < rm.n_rules_in[s]; q++) incoming += ctl->cand_n[rm.rules_in[s][q]];
                if (!incoming) continue;
                over = over || ctl->full_n[s] + ctl->delta_n[s] + incoming > plan.log_cap[s] ||
                       (!a.to_log && incoming > a.stage_cap);
            }
        }
        if (over) {
            if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(&ctl->flags, kFlagOverflow);
            active = false;
        }
    }
    if (c == 0 && blockIdx.x == 0 && threadIdx.x == 0) ctl->win_n[rule] = 0;
    const u64 ntiles = (c + kSelTile - 1) / kSelTile;
    if (active && c > 0 && blockIdx.x < ntiles) {
        // destination offset and intern base: winners of earlier rules into the same relation / tag
        u64 dst_off = 0, id_ctr = ctl->intern[tslot];
        if (a.sliced) {
            dst_off = a.appended;
            id_ctr += a.id_appended;
        } else {
            for (int q = 0; q < rule; q++) {
                if (plan.rule_out[q] == out) dst_off += ctl->win_n[q];
                if (plan.rule_tag[q] == tslot) id_ctr += ctl->win_n[q];
            }
        }
        u64* dk = a.dst_keys;
        u64* dv = a.dst_ids;
        if (a.to_log) dst_off += ctl->full_n[out] + ctl->delta_n[out];
        const u64 tag_word = plan.rel_tag_word[out];
        const u64 cbase = a.sliced ? 0 : stream_base(ctl, rule);
        const u32 ep = (u32)ctl->epoch;
        const u64* in = cand + cbase;
        const bool aligned = (cbase & 3) == 0;   // 16-byte vector loads of candidates and marks
        const u32 tag = iter_tag(ctl, tile_slot);
        u32* ctr = tile_counter(ctl, tile_slot);
        for (int i = threadIdx.x; i < a.passes * kRadix; i += kThreads) (&s_hist[0][0])[i] = 0;
        for (;;) {
            if (threadIdx.x == 0) s_tile = atomicAdd(ctr, 1u);
            __syncthreads();
            const u64 tile = s_tile;
            __syncthreads();
            if (tile >= ntiles) break;
            const u64 base = tile * kSelTile + (u64)threadIdx.x * kSelIpt;
            u64 key[kSelIpt];
            u32 mk[kSelIpt];
            if (aligned && base + kSelIpt <= c) {
                // a thread's 4 candidates and their marks in three 16-byte loads
                const ulonglong2 k01 = *(const ulonglong2*)(in + base), k23 = *(const ulonglong2*)(in + base + 2);
                const uint4 m = *(const uint4*)(loser + cbase + base);
                key[0] = k01.x; key[1] = k01.y; key[2] = k23.x; key[3] = k23.y;
                mk[0] = m.x; mk[1] = m.y; mk[2] = m.z; mk[3] = m.w;
            } else {
#pragma unroll
                for (int k = 0; k < kSelIpt; k++) {
                    const bool v = base + k < c;
                    key[k] = v ? in[base + k] : kEmpty;
                    mk[k] = v ? loser[cbase + base + k] : ep;
                }
            }
            u32 win = 0;
#pragma unroll
            for (int k = 0; k < kSelIpt; k++) {
                if (key[k] == kEmpty || mk[k] == ep) key[k] = kEmpty;
                else win++;
            }
            u64 agg;
            const u64 ex = block_exclusive_scan((u64)win, sm, &agg);
            if (threadIdx.x < 32) {
                const u64 pre = lookback_warp(status, (u32)tile, agg, tag, &ctl->flags);
                if (threadIdx.x == 0) s_prefix = pre;
            }
            {   // compacted into shared memory meanwhile
                u64 e = ex;
#pragma unroll
                for (int k = 0; k < kSelIpt; k++)
                    if (key[k] != kEmpty) s_win[e++] = key[k];
            }
            __syncthreads();
            const u64 pre = s_prefix;
            // the tile's winners: log rows dst_off + pre + i, consecutive threads, consecutive rows
            for (u32 i = threadIdx.x; i < agg; i += kThreads) {
                const u64 kk = s_win[i];
                const u64 r = pre + i;
                dk[dst_off + r] = kk;
                dv[dst_off + r] = tag_word | (id_ctr + r);
                for (int ps = 0; ps < a.passes; ps++)
                    atomicAdd(&s_hist[ps][(kk >> (ps * kRadixBits)) & (kRadix - 1)], 1u);
            }
            if (a.inst_base) {
                u64* row = a.inst_new + ctl->iteration * a.n_inst;
                for (u32 i0 = 0; i0 < agg; i0 += kThreads) {   // warp-uniform trip count
                    const u32 i = i0 + threadIdx.x;
                    const bool v = i < agg;
                    const u32 inst = v ? instance_of(a.inst_base, a.n_inst, s_win[i] >> a.inst_shift)
                                       : (0x80000000u | (u32)threadIdx.x);
                    const u32 peers = __match_any_sync(0xffffffffu, inst);
                    if (v && (peers & lanemask_lt()) == 0) atomicAdd(&row[inst], (u64)__popc(peers));
                }
            }
            if (tile == ntiles - 1 && threadIdx.x == 0) ctl->win_n[rule] = s_prefix + agg;
            __syncthreads();
        }
        if (a.passes) {
            __syncthreads();
            for (int i = threadIdx.x; i < a.passes * kRadix; i += kThreads) {
                const u32 v = (&s_hist[0][0])[i];
                if (v) atomicAdd(&ctl->sort_hist[out][i / kRadix][i % kRadix], (u64)v);
            }
        }
    }
    // the last block to finish runs the iteration end (after every write of this launch);
    // blocks past the last tile never write, so only min(grid, tiles) blocks take part
    const u32 parting = (u32)min((u64)gridDim.x, (active && c > 0) ? ntiles : (u64)1);
    if (blockIdx.x >= parting) return;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const u32 done = atomicAdd(&ctl->exit_ctr, 1u);
        if (done == parting - 1) {
            __threadfence();
            ctl->exit_ctr = 0;
            if (a.last) {
                end_of_iteration(ctl, plan, rm, history, cond, use_cond);
                if (a.tail_on && use_cond && tail_next(ctl, a)) cudaGraphSetConditional(cond, 0u);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// onesweep LSD radix pass over a relation's staged rows
// ---------------------------------------------------------------------------
constexpr int kSortIpt = 8;
constexpr int kSortTile = kThreads * kSortIpt;

// ---------------------------------------------------------------------------
// bitmap_select: the new tuples of a bitmap relation (all rules into it at
// once) into its log, in key order, one warp per row.  Takes part in the
// iteration like select_kernel: the same capacity check before any write, the
// same exit counter, the iteration end when it is the iteration's last launch.
// ---------------------------------------------------------------------------
struct BitSelectArgs {
    int rel;          // output relation slot
    int first_rule;   // the relation's first rule: credited with all its new tuples
    int last;         // this launch ends the iteration
    u64* dst_keys;
    u64* dst_ids;
    BitSeen bs;
    int bits;         // packed column width
    u64* inst_new;    // [iteration][instance] new tuples (with instances), else null
    u32 n_inst;
    u64 inst_iter_cap;
};

__global__ void __launch_bounds__(kThreads) bitmap_select_kernel(IterCtl* __restrict__ ctl, SccPlan plan, SccRelMap rm,
                                                                 BitSelectArgs a, u64* __restrict__ status,
                                                                 u64 status_cap, int tile_slot, u64* __restrict__ history,
                                                                 cudaGraphConditionalHandle cond, int use_cond)
{
    __shared__ u64 sm[kWarps + 1];
    __shared__ u64 s_cnt[kWarps];
    __shared__ u32 s_tile;
    __shared__ u64 s_prefix;
    const int out = a.rel, tslot = plan.rule_tag[a.first_rule];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const u64 rows = a.bs.n;
    const u64 ntiles = (rows + kWarps - 1) / kWarps;
    bool active = ctl->flags == 0;
    if (active && ntiles > status_cap) {   // never taken: status is sized for the rows
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(&ctl->flags, kFlagStatus);
        active = false;
    }
    if (active) {
        // select_kernel's check: room for every candidate of the iteration
        bool over = a.inst_new && ctl->iteration >= a.inst_iter_cap;
        for (int s = 0; s < plan.n_rels; s++) {
            u64 incoming = 0;
            for (int q = 0; q < rm.n_rules_in[s]; q++) incoming += ctl->cand_n[rm.rules_in[s][q]];
            if (incoming && ctl->full_n[s] + ctl->delta_n[s] + incoming > plan.log_cap[s]) over = true;
        }
        if (over) {
            if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(&ctl->flags, kFlagOverflow);
            active = false;
        }
    }
    if (active && blockIdx.x < ntiles) {
        u64 dst_off = ctl->full_n[out] + ctl->delta_n[out], id_ctr = ctl->intern[tslot];
        for (int q = 0; q < a.first_rule; q++)
            if (plan.rule_tag[q] == tslot) id_ctr += ctl->win_n[q];
        const u64 tag_word = plan.rel_tag_word[out];
        const u32 tag = iter_tag(ctl, tile_slot);
        u32* ctr = tile_counter(ctl, tile_slot);
        for (;;) {
            if (threadIdx.x == 0) s_tile = atomicAdd(ctr, 1u);
            __syncthreads();
            const u64 tile = s_tile;
            __syncthreads();
            if (tile >= ntiles) break;
            const u64 row = tile * kWarps + warp;
            const bool has = row < rows && a.bs.dirty[row];
            const u64 W = has && a.bs.row_word ? a.bs.row_words[row] : a.bs.words;
            const u64 vbase = has && a.bs.row_word ? a.bs.row_base[row] : 0;
            u32* frow = a.bs.fresh + (has && a.bs.row_word ? a.bs.row_word[row] : row * W);
            u64 cnt = 0;
            if (has)
                for (u64 w = lane; w < W; w += 32) cnt += __popc(frow[w]);
            for (int d = 16; d > 0; d >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, d);
            if (lane == 0) s_cnt[warp] = cnt;
            __syncthreads();
            u64 agg;
            const u64 ex = block_exclusive_scan(threadIdx.x < kWarps ? s_cnt[threadIdx.x] : 0, sm, &agg);
            __syncthreads();
            if (threadIdx.x < kWarps) s_cnt[threadIdx.x] = ex;   // row offsets inside the tile
            if (threadIdx.x < 32) {
                const u64 pre = lookback_warp(status, (u32)tile, agg, tag, &ctl->flags);
                if (threadIdx.x == 0) s_prefix = pre;
            }
            __syncthreads();
            if (has) {
                u64 pos = s_prefix + s_cnt[warp];
                for (u64 g = 0; g < W; g += 32) {
                    const u32 word = (g + lane < W) ? frow[g + lane] : 0u;
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
                        u32 lo = 0, hi = 31;
#pragma unroll
                        for (int step = 0; step < 5; step++) {
                            const u32 mid = (lo + hi) >> 1;
                            if (__shfl_sync(0xffffffffu, incl, mid) > t) hi = mid;
                            else lo = mid + 1;
                        }
                        const u32 wj = __shfl_sync(0xffffffffu, word, lo);
                        const u32 before = __shfl_sync(0xffffffffu, incl - c, lo);
                        if (t < group) {
                            const u32 bit = __fns(wj, 0, (int)(t - before) + 1);
                            const u64 c1 = vbase + (g + lo) * 32 + bit;
                            const u64 at = pos + t;
                            a.dst_keys[dst_off + at] = (row << a.bits) | c1;
                            a.dst_ids[dst_off + at] = tag_word | (id_ctr + at);
                        }
                    }
                    if (g + lane < W) frow[g + lane] = 0u;
                    pos += group;
                }
                if (lane == 0) {
                    a.bs.dirty[row] = 0;
                    if (a.inst_new)
                        atomicAdd((unsigned long long*)&a.inst_new[ctl->iteration * a.n_inst + a.bs.row_inst[row]],
                                  (unsigned long long)(pos - s_prefix - s_cnt[warp]));
                }
            }
            if (tile == ntiles - 1 && threadIdx.x == 0) {
                ctl->win_n[a.first_rule] = s_prefix + agg;
                for (int q = 0; q < rm.n_rules_in[out]; q++)
                    if (rm.rules_in[out][q] != a.first_rule) ctl->win_n[rm.rules_in[out][q]] = 0;
            }
            __syncthreads();
        }
    }
    const u32 parting = (u32)min((u64)gridDim.x, active ? ntiles : (u64)1);
    if (blockIdx.x >= parting) return;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const u32 done = atomicAdd(&ctl->exit_ctr, 1u);
        if (done == parting - 1) {
            __threadfence();
            ctl->exit_ctr = 0;
            if (a.last) end_of_iteration(ctl, plan, rm, history, cond, use_cond);
        }
    }
}

struct SortPassArgs {
    int rel;                  // relation slot
    int pass, shift;
    const u64* src_k;
    const u64* src_v;
    u64* dst_k;               // when dst_log: the log base (rows go to base + full_n + delta_n)
    u64* dst_v;
    int dst_log;
    u64 log_cap;              // rows the relation's log holds (dst_log)
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
        if (o + n > a.log_cap) {   // select checks this first; never write past the log
            if (threadIdx.x == 0) atomicOr(&ctl->flags, kFlagOverflow);
            return;
        }
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
        if (threadIdx.x == 0) s_tile = atomicAdd(tile_counter(ctl, tile_slot), 1u);
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

__global__ void scc_start_kernel(IterCtl* __restrict__ ctl) { ctl->t_start = global_ns(); }

// Order-independent digest of a tuple's data columns: depends only on the
// column values (not on the packing width), so runs with different widths agree.
__device__ __forceinline__ u64 tuple_digest(const u64* cols, int arity)
{
    u64 h = 0x9e3779b97f4a7c15ull * (u64)arity;
    for (int c = 0; c < arity; c++) h = mix64(h ^ (cols[c] + 0x632be59bd9b4e019ull * (u64)(c + 1)));
    return h;
}

// Per-instance count and digest (sum of tuple digests, values rebased to the
// instance) of packed rows.  Each warp walks a contiguous segment of rows
// (coalesced), every lane keeps a running (count, digest) for the instance of
// its last rows and flushes it when the instance changes; relation logs hold
// each instance's rows in long runs, so flushes are rare, and a row inside the
// current instance's value range skips the search over the bases.  Up to
// kSummarySmemInst instances accumulate in shared memory first.  ARITY > 0
// fixes the arity at compile time (columns in registers); 0 reads `arity`.
constexpr u32 kSummarySmemInst = 1024;
constexpr int kSummaryRowsPerLane = 16;

template <int ARITY>
__global__ void __launch_bounds__(kThreads) instance_summary_kernel(
    const u64* __restrict__ keys, u64 n, int arity_rt, int bits, const u64* __restrict__ base, u32 n_inst,
    u64* __restrict__ counts, u64* __restrict__ digests)
{
    const int arity = ARITY > 0 ? ARITY : arity_rt;
    constexpr int kCols = ARITY > 0 ? ARITY : kMaxArity;
    __shared__ u64 s_cnt[kSummarySmemInst];
    __shared__ u64 s_dig[kSummarySmemInst];
    const u32 m = base ? n_inst : 1;
    const bool in_smem = m <= kSummarySmemInst;
    if (in_smem)
        for (u32 i = threadIdx.x; i < m; i += blockDim.x) s_cnt[i] = s_dig[i] = 0;
    __syncthreads();
    u32 cur = 0xffffffffu;
    u64 cur_lo = 1, cur_hi = 0;   // value range of instance `cur` (empty: no instance yet)
    u64 c = 0, dsum = 0;
    auto flush = [&]() {
        if (!c) return;
        if (in_smem) {
            atomicAdd((unsigned long long*)&s_cnt[cur], (unsigned long long)c);
            atomicAdd((unsigned long long*)&s_dig[cur], (unsigned long long)dsum);
        } else {
            atomicAdd((unsigned long long*)&counts[cur], (unsigned long long)c);
            atomicAdd((unsigned long long*)&digests[cur], (unsigned long long)dsum);
        }
        c = 0;
        dsum = 0;
    };
    const int lane = threadIdx.x & 31;
    const u64 seg = 32ull * kSummaryRowsPerLane;
    const u64 warps = (u64)gridDim.x * (blockDim.x >> 5);
    for (u64 w = (u64)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); w * seg < n; w += warps) {
        for (int j = 0; j < kSummaryRowsPerLane; j++) {
            const u64 i = w * seg + (u64)j * 32 + lane;
            if (i >= n) break;
            const u64 k = keys[i];
            u64 cols[kCols];
#pragma unroll
            for (int q = 0; q < kCols; q++)
                if (q < arity) cols[q] = column_of(k, arity, q, bits);
            if (!(cols[0] >= cur_lo && cols[0] < cur_hi)) {
                const u32 inst = base ? instance_of(base, n_inst, cols[0]) : 0;
                if (inst != cur) {
                    flush();
                    cur = inst;
                }
                cur_lo = base ? __ldg(&base[inst]) : 0;
                cur_hi = base ? __ldg(&base[inst + 1]) : ~0ull;
            }
#pragma unroll
            for (int q = 0; q < kCols; q++)
                if (q < arity) cols[q] -= cur_lo;
            c++;
            dsum += tuple_digest(cols, arity);
        }
    }
    flush();
    if (!in_smem) return;
    __syncthreads();
    for (u32 i = threadIdx.x; i < m; i += blockDim.x)
        if (s_cnt[i]) {
            atomicAdd((unsigned long long*)&counts[i], (unsigned long long)s_cnt[i]);
            atomicAdd((unsigned long long*)&digests[i], (unsigned long long)s_dig[i]);
        }
}

// ---------------------------------------------------------------------------
// iteration end as its own launch (reference id order: after the sort passes)
// ---------------------------------------------------------------------------
__global__ void iter_end_kernel(IterCtl* __restrict__ ctl, SccPlan plan, SccRelMap rm, u64* __restrict__ history,
                                cudaGraphConditionalHandle cond, int use_cond)
{
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < (u64)kMaxSccRels * kMaxPasses * kRadix;
         i += (u64)gridDim.x * blockDim.x)
        (&ctl->sort_hist[0][0][0])[i] = 0;
    if (blockIdx.x == 0 && threadIdx.x == 0) end_of_iteration(ctl, plan, rm, history, cond, use_cond);
}

}  // namespace ra
