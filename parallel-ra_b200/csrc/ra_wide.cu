// Host side of the wide-tuple path (kernels in ra_wide.cuh).  Included into
// ra_engine.cu's translation unit: it uses ra_program, Relation and the
// engine's allocation, scan and error helpers.
//
// A program runs wide when some relation's tuples do not pack into one 63-bit
// key, a relation has more than kMaxArity columns or joins on zero columns, a
// join key exceeds the CSR index's 30 bits, or a rule copies an intern id into a
// data column.  Every relation version is then an
// array of arity + 1 u64 rows in trie order, and one iteration of an SCC is
// RAM::local_compute + local_insert_in_newt + local_insert_in_full
// (src/RAM/RA_tasks.cpp:305-555, 824-905; balanced_hash_relation.cpp:1120-1231):
//   1. each rule's candidates, in the reference's emission order (outer rows in
//      trie order, each one's inner matches in trie order; copies in input order),
//      written into its output relation's candidate buffer after the earlier rules';
//   2. per output relation: an index sort that puts equal candidates next to each
//      other in position order; the first of each group wins unless full or delta
//      holds it;
//   3. ids (tag << 46) | counter assigned to the winners rule by rule in the SCC's
//      rule order, the counters shared by the relations of one tag, as the
//      single-rank reference interns them (bucket 0);
//   4. newt sorted into trie order; full = full + delta (a rank merge), delta = newt.
// Intern ids therefore equal the reference's, and with them every data column
// that a rule copies out of an id (acopy).
//
// An iteration makes two host round trips (candidate counts; winner counts) and
// runs each phase for all of its small rules or relations in one batched launch
// (work lists as kernel parameters), so its cost is a few dozen launches
// however few tuples it moves.
//
// (Included inside the engine's anonymous namespace.)

// Scratch slots of the wide path (grow-only, contents not kept across calls).
enum WideSlot { kWsIdxA, kWsIdxB, kWsRows, kWsLo, kWsCnt, kWsOff, kWsPos, kWsFlag, kWsSmall, kWsTot, kWsCount };
static_assert(kWsCount <= 12, "wide scratch slots");

u64* wide_scratch(ra_program* p, int slot, u64 n)
{
    if (n > p->wbuf_cap[slot]) {
        dev_free(p, &p->wbuf[slot]);
        p->wbuf_cap[slot] = 0;
        const u64 nc = std::max<u64>(n + n / 2, 4096);
        dev_alloc(p, &p->wbuf[slot], nc);
        p->wbuf_cap[slot] = nc;
    }
    return p->wbuf[slot];
}

u32* wide_scratch32(ra_program* p, int slot, u64 n) { return (u32*)wide_scratch(p, slot, (n + 1) / 2); }

// Room for `rows` rows of W columns in *buf, keeping the first keep_rows rows.
void wide_reserve(ra_program* p, u64** buf, u64* cap, u64 rows, int W, u64 keep_rows)
{
    if (rows <= *cap && *buf) return;
    const u64 nc = std::max<u64>(rows + rows / 2, 256);
    *cap = std::min<u64>(*cap, keep_rows);   // a failed allocation leaves no stale capacity
    u64* nb;
    dev_alloc(p, &nb, nc * (u64)W);
    if (keep_rows && *buf) CK(cudaMemcpyAsync(nb, *buf, keep_rows * (u64)W * 8, cudaMemcpyDeviceToDevice, p->stream));
    dev_free(p, buf);
    *buf = nb;
    *cap = nc;
}

// Room for n u32 flags in *buf (contents not kept).
void wide_reserve32(ra_program* p, u32** buf, u64* cap, u64 n)
{
    if (n <= *cap && *buf) return;
    dev_free(p, buf);
    *cap = 0;
    const u64 nc = std::max<u64>(n + n / 2, 1024);
    dev_alloc(p, buf, nc);
    *cap = nc;
}

int wide_grid(u64 n) { return grid_for(std::max<u64>(n, 1)); }

// Exclusive scan of n values into out, the total into *total_dev, with no host
// round trip (one block for small inputs).
template <typename T>
void wide_scan_async(ra_program* p, const T* in, u64 n, u64* out, u64* total_dev)
{
    if (n <= (u64)kThreads * kWideScanPer) {
        wide_scan_small_kernel<T><<<1, kThreads, 0, p->stream>>>(in, n, out, total_dev);
        LAUNCHED();
        return;
    }
    scan_exclusive<T>(p, in, n, out, false);
    CK(cudaMemcpyAsync(total_dev, p->dscalar, 8, cudaMemcpyDeviceToDevice, p->stream));
}

// Indices 0..n-1 of `rows` sorted by (first ncmp columns, index); the result is
// one of the two index scratch slots.
const u64* wide_sort(ra_program* p, const u64* rows, int W, int ncmp, u64 n)
{
    u64* a = wide_scratch(p, kWsIdxA, n);
    u64* b = wide_scratch(p, kWsIdxB, n);
    if (n <= 64) {
        wide_tile_sort_kernel<64><<<1, kThreads, 0, p->stream>>>(rows, W, ncmp, n, a);
    } else if (n <= 256) {
        wide_tile_sort_kernel<256><<<1, kThreads, 0, p->stream>>>(rows, W, ncmp, n, a);
    } else {
        const u64 tiles = (n + kWideSortTile - 1) / kWideSortTile;
        wide_tile_sort_kernel<kWideSortTile><<<(unsigned)tiles, kThreads, 0, p->stream>>>(rows, W, ncmp, n, a);
    }
    LAUNCHED();
    for (u64 L = kWideSortTile; L < n; L *= 2) {
        wide_merge_pass_kernel<<<wide_grid(n), kThreads, 0, p->stream>>>(rows, W, ncmp, n, L, a, b);
        LAUNCHED();
        std::swap(a, b);
    }
    return a;
}

// Rows of `src` (n rows of W columns) sorted into trie order and made distinct,
// into *dst (capacity *cap); returns the row count.
u64 wide_sort_unique(ra_program* p, const u64* src, int W, u64 n, u64** dst, u64* cap)
{
    if (!n) return 0;
    const u64* idx = wide_sort(p, src, W, W, n);
    wide_reserve(p, dst, cap, n, W, 0);
    wide_gather_kernel<<<wide_grid(n * W), kThreads, 0, p->stream>>>(src, W, idx, n, *dst);
    LAUNCHED();
    u32* keep = wide_scratch32(p, kWsFlag, n);
    CK(cudaMemsetAsync(p->derr, 0, 4, p->stream));
    wide_dup_kernel<<<wide_grid(n), kThreads, 0, p->stream>>>(*dst, W, n, keep, p->derr);
    LAUNCHED();
    if (!(read_scalar(p, (const u64*)p->derr) & 0xffffffffull)) return n;
    u64* pos = wide_scratch(p, kWsPos, n);
    const u64 m = scan_exclusive<u32>(p, keep, n, pos);
    u64* tmp = wide_scratch(p, kWsRows, n * W);
    wide_compact_kernel<<<wide_grid(n), kThreads, 0, p->stream>>>(*dst, W, n, keep, pos, tmp);
    LAUNCHED();
    CK(cudaMemcpyAsync(*dst, tmp, m * (u64)W * 8, cudaMemcpyDeviceToDevice, p->stream));
    return m;
}

// *a = *a + b (both sorted, in trie order); the merged rows go to the spare
// buffer, which then becomes *a.
void wide_merge_into(ra_program* p, Relation& r, u64** a, u64* acap, u64* an, const u64* b, u64 bn)
{
    const int W = (int)r.arity + 1;
    if (!bn) return;
    if (!*an) {
        wide_reserve(p, a, acap, bn, W, 0);
        CK(cudaMemcpyAsync(*a, b, bn * (u64)W * 8, cudaMemcpyDeviceToDevice, p->stream));
        *an = bn;
        return;
    }
    const u64 n = *an + bn;
    wide_reserve(p, &r.wspare, &r.wspare_cap, n, W, 0);
    wide_merge_rows_kernel<<<wide_grid(n), kThreads, 0, p->stream>>>(*a, *an, b, bn, W, r.wspare);
    LAUNCHED();
    std::swap(*a, r.wspare);
    std::swap(*acap, r.wspare_cap);
    *an = n;
}

// relation::insert_delta_in_full (balanced_hash_relation.cpp:1120-1148)
void wide_delta_to_full(ra_program* p, Relation& r)
{
    if (!r.delta_n) return;
    wide_merge_into(p, r, &r.wfull, &r.wfull_cap, &r.full_n, r.wdelta, r.delta_n);
    r.delta_n = 0;
}

// relation::insert_full_in_delta (balanced_hash_relation.cpp:1152-1179)
void wide_full_to_delta(ra_program* p, Relation& r)
{
    if (!r.full_n) return;
    wide_merge_into(p, r, &r.wdelta, &r.wdelta_cap, &r.delta_n, r.wfull, r.full_n);
    r.full_n = 0;
}

// Restart (LIE::execute, lie.cpp:300-330): the relation's delta from the dump's
// <name>_delta rows, after any delta present joined full; no file, no delta.
void wide_load_restart_delta(ra_program* p, Relation& r)
{
    std::vector<u64> host;
    std::string path;
    if (!read_restart_rows(p, r, host, path)) return;
    wide_delta_to_full(p, r);
    const int W = (int)r.arity + 1;
    const u64 n = host.size() / (u64)W;
    if (!n) return;
    u64* raw;
    dev_alloc(p, &raw, host.size());
    CK(cudaMemcpyAsync(raw, host.data(), host.size() * 8, cudaMemcpyHostToDevice, p->stream));
    r.delta_n = wide_sort_unique(p, raw, W, n, &r.wdelta, &r.wdelta_cap);
    CK(cudaStreamSynchronize(p->stream));
    dev_free(p, &raw);
}

// Loaded rows (arity + 1 columns) into the relation's loaded version, in trie
// order and distinct on all columns, as populate_full inserts them
// (balanced_hash_relation.cpp:609-793).
void wide_load(ra_program* p, Relation& r)
{
    r.full_n = r.delta_n = r.newt_n = 0;
    if (!r.raw_n) return;
    const int W = (int)r.arity + 1;
    if (r.version == RA_DELTA) r.delta_n = wide_sort_unique(p, r.raw, W, r.raw_n, &r.wdelta, &r.wdelta_cap);
    else r.full_n = wide_sort_unique(p, r.raw, W, r.raw_n, &r.wfull, &r.wfull_cap);
}

// The rows of one version of a relation (sorted).
const u64* wide_version(Relation& r, int ver, u64* n)
{
    *n = ver == RA_DELTA ? r.delta_n : r.full_n;
    return ver == RA_DELTA ? r.wdelta : r.wfull;
}

// Candidate width of a relation written by an SCC's rules: data columns, or all
// columns for acopy targets (which carry their last column from the input).
int wide_cand_width(ra_program* p, const Scc& s, int out)
{
    int acopy = -1;
    for (const Rule& ru : s.rules) {
        if (ru.out != out) continue;
        const int a = ru.kind == RA_ACOPY ? 1 : 0;
        if (acopy >= 0 && acopy != a)
            fail(p, RA_E_UNSUPPORTED, "SCC %d: relation %s is written by acopy and by other rules", s.id,
                 p->rels[out].name.c_str());
        acopy = a;
    }
    return (int)p->rels[out].arity + (acopy == 1 ? 1 : 0);
}

// Projection of a rule onto its output's candidate columns, checked against the inputs.
WideProj wide_proj(ra_program* p, const Scc& s, const Rule& ru, int cw)
{
    WideProj pj{};
    const Relation& o = p->rels[ru.out];
    const Relation& a = p->rels[ru.in0];
    pj.n = (int)ru.proj.size();
    if (pj.n != cw || pj.n > kWideMaxCols)
        fail(p, RA_E_BADARG, "SCC %d: a rule into %s projects %d columns, the relation takes %d", s.id, o.name.c_str(),
             pj.n, cw);
    int span;
    if (ru.kind == kJoin) {
        const Relation& b = p->rels[ru.in1];
        if (a.jcc != b.jcc || a.jcc > a.arity || a.jcc > b.arity)
            fail(p, RA_E_BADARG, "SCC %d: join of %s and %s on different join columns", s.id, a.name.c_str(),
                 b.name.c_str());
        pj.left = ru.ver0 == RA_DELTA ? 1 : 0;
        pj.W0 = (int)a.arity + 1;
        pj.W1 = (int)b.arity + 1;
        pj.jcc = (int)a.jcc;
        span = pj.W0 + pj.W1 - pj.jcc;
    } else {
        span = (int)a.arity + 1;
    }
    for (int j = 0; j < pj.n; j++) {
        if (ru.proj[j] < 0 || ru.proj[j] >= span)
            fail(p, RA_E_BADARG, "SCC %d: projection column %d outside the rule's %d input columns", s.id, ru.proj[j],
                 span);
        pj.src[j] = ru.proj[j];
    }
    return pj;
}

struct WideOut {
    int rel;
    int cw;
    u64 n = 0;                      // candidates
    std::vector<int> rules;         // rule index of each segment
    std::vector<u64> seg_start;     // first candidate of each segment
    u64 winners = 0;
    std::vector<u64> seg_wins;      // winners before each segment, then the total
};

// Inputs of one rule in the running iteration.
struct WideRuleRun {
    bool active = false;
    const u64* outer = nullptr;     // join: outer rows; copy: input rows
    const u64* inner = nullptr;
    u64 no = 0, ni = 0;             // join: outer / inner rows; copy: input rows in `no`
    u64 off = 0;                    // this rule's region of the per-rule scratch
    WideProj pj{};
    u64 total = 0;                  // candidates
};

// One iteration: RAM::local_compute + local_insert_in_newt + local_insert_in_full,
// with two host round trips: after the candidate counts, and after the winners.
void wide_iteration(ra_program* p, Scc& s)
{
    const int nr = (int)s.rules.size();
    std::vector<WideOut> outs;
    outs.reserve(s.rules.size());
    std::vector<int> out_index(nr);
    for (int q = 0; q < nr; q++) {
        const int rel = s.rules[q].out;
        int k = 0;
        while (k < (int)outs.size() && outs[k].rel != rel) k++;
        if (k == (int)outs.size()) {
            WideOut o;
            o.rel = rel;
            o.cw = wide_cand_width(p, s, rel);
            Relation& R = p->rels[rel];
            if (R.wcand_w != o.cw) {   // the buffer's capacity counts rows of its last width
                dev_free(p, &R.wcand);
                R.wcand_cap = 0;
                R.wcand_w = o.cw;
            }
            outs.push_back(o);
        }
        out_index[q] = k;
        if ((int)outs[k].rules.size() >= kWideMaxSegs)
            fail(p, RA_E_UNSUPPORTED, "SCC %d: more than %d rules write relation %s", s.id, kWideMaxSegs,
                 p->rels[rel].name.c_str());
        outs[k].rules.push_back(q);
    }
    // inputs of every rule
    std::vector<WideRuleRun> rr(nr);
    u64 join_rows = 0, filter_rows = 0;
    for (int q = 0; q < nr; q++) {
        const Rule& ru = s.rules[q];
        WideRuleRun& r = rr[q];
        r.pj = wide_proj(p, s, ru, outs[out_index[q]].cw);
        Relation& a = p->rels[ru.in0];
        if (ru.kind == kJoin) {
            Relation& b = p->rels[ru.in1];
            if (ru.ver0 == RA_DELTA) {
                r.outer = wide_version(a, RA_DELTA, &r.no);
                r.inner = wide_version(b, ru.ver1, &r.ni);
            } else {
                r.outer = wide_version(b, ru.ver1, &r.no);
                r.inner = wide_version(a, RA_FULL, &r.ni);
            }
            r.active = r.no && r.ni;
            if (r.active) {
                r.off = join_rows;
                join_rows += r.no;
            }
        } else {
            r.outer = wide_version(a, ru.ver0, &r.no);
            r.active = r.no != 0;
            r.total = r.no;
            if (r.active && ru.kind == RA_COPY_FILTER) {
                r.off = filter_rows;
                filter_rows += r.no;
            }
        }
    }
    // 1. candidate counts (join ranges, filter passes), one round trip for all rules
    u64* tot = wide_scratch(p, kWsTot, (u64)nr + outs.size() * (kWideMaxSegs + 2));
    u64* lo = join_rows ? wide_scratch(p, kWsLo, join_rows) : nullptr;
    u64* cnt = join_rows ? wide_scratch(p, kWsCnt, join_rows) : nullptr;
    u64* off = join_rows ? wide_scratch(p, kWsOff, join_rows) : nullptr;
    u32* keep = filter_rows ? wide_scratch32(p, kWsFlag, filter_rows) : nullptr;
    u64* pos = filter_rows ? wide_scratch(p, kWsPos, filter_rows) : nullptr;
    bool counted = false;
    {
        PhaseTimer pt(p, 0);
        WideCountBatch cb{};
        auto flush_counts = [&]() {
            if (!cb.n) return;
            wide_count_batch_kernel<<<cb.n, kThreads, 0, p->stream>>>(cb);
            LAUNCHED();
            cb.n = 0;
        };
        for (int q = 0; q < nr; q++) {
            const Rule& ru = s.rules[q];
            WideRuleRun& r = rr[q];
            if (!r.active || (ru.kind != kJoin && ru.kind != RA_COPY_FILTER)) continue;
            counted = true;
            const bool join = ru.kind == kJoin;
            const int Wo = join ? (r.pj.left ? r.pj.W0 : r.pj.W1) : (int)p->rels[ru.in0].arity + 1;
            const int Wi = join ? (r.pj.left ? r.pj.W1 : r.pj.W0) : 0;
            if (r.no <= kWideBlockScan) {   // small: one block of the batched launch
                WideCountJob& j = cb.job[cb.n++];
                j = WideCountJob{r.outer, r.inner, r.no, r.ni, join ? lo + r.off : nullptr,
                                 join ? cnt + r.off : nullptr, join ? off + r.off : pos + r.off,
                                 join ? nullptr : keep + r.off, tot + q, Wo, Wi, join ? r.pj.jcc : 0,
                                 join ? -1 : ru.pred};
                if (cb.n == kWideJobs) flush_counts();
            } else if (join) {
                wide_join_count_kernel<<<wide_grid(r.no), kThreads, 0, p->stream>>>(r.outer, Wo, r.no, r.inner, Wi,
                                                                                    r.ni, r.pj.jcc, lo + r.off,
                                                                                    cnt + r.off);
                LAUNCHED();
                wide_scan_async<u64>(p, cnt + r.off, r.no, off + r.off, tot + q);
            } else {
                wide_filter_kernel<<<wide_grid(r.no), kThreads, 0, p->stream>>>(r.outer, Wo, r.no, ru.pred,
                                                                                keep + r.off);
                LAUNCHED();
                wide_scan_async<u32>(p, keep + r.off, r.no, pos + r.off, tot + q);
            }
        }
        flush_counts();
        if (counted) {
            std::vector<u64> h(nr);
            CK(cudaMemcpyAsync(h.data(), tot, nr * 8, cudaMemcpyDeviceToHost, p->stream));
            CK(cudaStreamSynchronize(p->stream));
            for (int q = 0; q < nr; q++)
                if (rr[q].active && (s.rules[q].kind == kJoin || s.rules[q].kind == RA_COPY_FILTER)) rr[q].total = h[q];
        }
    }
    // 2. candidates into each output relation's buffer, rule by rule, one flattened launch
    {
        PhaseTimer pt(p, 2);
        WideExpandBatch eb{};
        auto flush_expand = [&]() {
            if (!eb.n) return;
            wide_expand_batch_kernel<<<wide_grid(eb.total), kThreads, 0, p->stream>>>(eb);
            LAUNCHED();
            eb.n = 0;
            eb.total = 0;
        };
        for (WideOut& wo : outs) {
            Relation& R = p->rels[wo.rel];
            wo.n = 0;
            for (int q : wo.rules) {
                wo.seg_start.push_back(wo.n);
                if (rr[q].active) wo.n += rr[q].total;
            }
            if (wo.n) wide_reserve(p, &R.wcand, &R.wcand_cap, wo.n, wo.cw, 0);
        }
        for (WideOut& wo : outs) {
            Relation& R = p->rels[wo.rel];
            for (size_t k = 0; k < wo.rules.size(); k++) {
                const int q = wo.rules[k];
                const Rule& ru = s.rules[q];
                WideRuleRun& r = rr[q];
                if (!r.active || !r.total) continue;
                WideExpandJob& j = eb.job[eb.n++];
                j = WideExpandJob{};
                j.outer = r.outer;
                j.inner = r.inner;
                j.dst = R.wcand + wo.seg_start[k] * (u64)wo.cw;
                j.no = r.no;
                j.first = eb.total;
                j.n = r.pj.n;
                for (int c = 0; c < r.pj.n; c++) j.src[c] = (unsigned char)r.pj.src[c];
                if (ru.kind == kJoin) {
                    j.kind = 0;
                    j.lo = lo + r.off;
                    j.off = off + r.off;
                    j.left = r.pj.left;
                    j.W0 = r.pj.W0;
                    j.W1 = r.pj.W1;
                    j.jcc = r.pj.jcc;
                    p->stats.join_candidates += r.total;
                } else {
                    j.kind = 1;
                    j.Wi = (int)p->rels[ru.in0].arity + 1;
                    j.off = ru.kind == RA_COPY_FILTER ? pos + r.off : nullptr;
                }
                eb.total += r.total;
                if (eb.n == kWideJobs) flush_expand();
            }
        }
        flush_expand();
    }
    // 3. winners of every output relation, one round trip for all of them
    u64* picks = tot + nr;   // per relation: kWideMaxSegs + 1 picked counts, then its winner total
    bool any = false;
    {
        PhaseTimer pt(p, 3);
        // heads: the first of each group of equal candidates
        WideHeadBatch hb{};
        auto flush_heads = [&]() {
            if (!hb.n) return;
            wide_heads_batch_kernel<<<hb.n, kWideWideBlock, 0, p->stream>>>(hb);
            LAUNCHED();
            hb.n = 0;
        };
        for (size_t k = 0; k < outs.size(); k++) {
            WideOut& wo = outs[k];
            Relation& R = p->rels[wo.rel];
            if (!wo.n) continue;
            any = true;
            wide_reserve32(p, &R.wflag, &R.wflag_cap, wo.n);
            wide_reserve(p, &R.wpos, &R.wpos_cap, wo.n, 1, 0);
            if (wo.n <= kWideBlockSort) {
                hb.job[hb.n++] = WideHeadJob{R.wcand, R.wflag, wo.n, wo.cw};
                if (hb.n == kWideJobs) flush_heads();
                continue;
            }
            const u64* idx = wide_sort(p, R.wcand, wo.cw, wo.cw, wo.n);
            wide_head_flags_kernel<<<wide_grid(wo.n), kThreads, 0, p->stream>>>(R.wcand, wo.cw, idx, wo.n, R.wflag);
            LAUNCHED();
        }
        flush_heads();
        // membership of the heads in full and delta, one thread per candidate of every relation
        WideMemberBatch mb{};
        auto flush_member = [&]() {
            if (!mb.n) return;
            wide_member_batch_kernel<<<wide_grid(mb.total), kThreads, 0, p->stream>>>(mb);
            LAUNCHED();
            mb.n = 0;
            mb.total = 0;
        };
        for (WideOut& wo : outs) {
            Relation& R = p->rels[wo.rel];
            if (!wo.n) continue;
            mb.job[mb.n++] = WideMemberJob{R.wcand, R.wfull, R.wdelta, R.wflag, wo.n, R.full_n, R.delta_n, mb.total,
                                           wo.cw, (int)R.arity + 1};
            mb.total += wo.n;
            if (mb.n == kWideJobs) flush_member();
        }
        flush_member();
        // positions of the winners and each rule segment's winners-before count
        WideScanBatch sb{};
        int sseg = 0;
        auto flush_scan = [&]() {
            if (!sb.n) return;
            wide_scan_pick_batch_kernel<<<sb.n, kThreads, 0, p->stream>>>(sb);
            LAUNCHED();
            sb.n = 0;
            sseg = 0;
        };
        for (size_t k = 0; k < outs.size(); k++) {
            WideOut& wo = outs[k];
            Relation& R = p->rels[wo.rel];
            if (!wo.n) continue;
            u64* my = picks + k * (kWideMaxSegs + 2);
            const int nseg = (int)wo.rules.size();
            if (wo.n <= kWideBlockScan) {
                if (sseg + nseg > 2 * kWideJobs) flush_scan();
                sb.job[sb.n++] = WideScanJob{R.wflag, R.wpos, my, wo.n, sseg, nseg};
                for (int q = 0; q < nseg; q++) sb.seg_start[sseg + q] = wo.seg_start[q];
                sseg += nseg;
                if (sb.n == kWideJobs) flush_scan();
                continue;
            }
            wide_scan_async<u32>(p, R.wflag, wo.n, R.wpos, my + kWideMaxSegs + 1);
            WideSegs sg{};
            sg.n = nseg;
            for (int j = 0; j < sg.n; j++) sg.start[j] = wo.seg_start[j];
            sg.start[sg.n] = wo.n;
            wide_pick_kernel<<<1, kWideMaxSegs + 1, 0, p->stream>>>(R.wpos, wo.n, my + kWideMaxSegs + 1, sg, my);
            LAUNCHED();
        }
        flush_scan();
        std::vector<u64> h(outs.size() * (kWideMaxSegs + 2));
        if (any) {
            CK(cudaMemcpyAsync(h.data(), picks, h.size() * 8, cudaMemcpyDeviceToHost, p->stream));
            CK(cudaStreamSynchronize(p->stream));
        }
        for (size_t k = 0; k < outs.size(); k++) {
            WideOut& wo = outs[k];
            Relation& R = p->rels[wo.rel];
            wo.seg_wins.assign(wo.rules.size() + 1, 0);
            if (wo.n) {
                const u64* my = h.data() + k * (kWideMaxSegs + 2);
                for (size_t j = 0; j <= wo.rules.size(); j++) wo.seg_wins[j] = my[j];
                wo.winners = my[kWideMaxSegs + 1];
            }
            R.newt_n = wo.winners;
            if (wo.winners) wide_reserve(p, &R.wnewt, &R.wnewt_cap, wo.winners, (int)R.arity + 1, 0);
        }
    }
    // 4. ids: rule by rule in the SCC's order, each tag's counter shared by its relations
    std::vector<u64> id_base(nr, 0);
    for (int q = 0; q < nr; q++) {
        const Rule& ru = s.rules[q];
        if (ru.kind == RA_ACOPY) continue;
        WideOut& wo = outs[out_index[q]];
        const size_t k = std::find(wo.rules.begin(), wo.rules.end(), q) - wo.rules.begin();
        const u64 wins = wo.seg_wins[k + 1] - wo.seg_wins[k];
        u64& ctr = intern_counter(p, p->rels[ru.out].tag);
        id_base[q] = ((u64)p->rels[ru.out].tag << 46) | ctr;
        ctr += wins;
    }
    // 5. newt rows, sorted into trie order
    {
        PhaseTimer pt(p, 4);
        u64 small_rows = 0;   // scratch for the batched relations' unsorted rows
        for (WideOut& wo : outs)
            if (wo.winners && wo.winners <= kWideBlockSort) small_rows += wo.winners * (p->rels[wo.rel].arity + 1);
        u64* srows = small_rows ? wide_scratch(p, kWsRows, small_rows) : nullptr;
        u64 srow_at = 0;
        WideNewtBatch nb{};
        int nseg_at = 0;
        auto flush_newt = [&]() {
            if (!nb.n) return;
            wide_newt_batch_kernel<<<nb.n, kWideWideBlock, 0, p->stream>>>(nb);
            LAUNCHED();
            nb.n = 0;
            nseg_at = 0;
        };
        for (WideOut& wo : outs) {
            Relation& R = p->rels[wo.rel];
            if (!wo.winners) continue;
            const int W = (int)R.arity + 1;
            const int nseg = (int)wo.rules.size();
            p->stats.new_tuples += wo.winners;
            if (wo.winners <= kWideBlockSort) {
                if (nseg_at + nseg > 2 * kWideJobs) flush_newt();
                WideNewtJob& j = nb.job[nb.n++];
                j = WideNewtJob{R.wcand, R.wflag, R.wpos, srows + srow_at, R.wnewt, wo.n, wo.winners, wo.cw, W,
                                nseg_at, nseg};
                for (int k = 0; k < nseg; k++) {
                    nb.seg_start[nseg_at + k] = wo.seg_start[k];
                    nb.win_base[nseg_at + k] = wo.seg_wins[k];
                    nb.id_base[nseg_at + k] = id_base[wo.rules[k]];
                }
                nseg_at += nseg;
                srow_at += wo.winners * (u64)W;
                if (nb.n == kWideJobs) flush_newt();
                continue;
            }
            flush_newt();   // the large path reuses the row scratch
            srow_at = 0;
            WideSegs sg{};
            sg.n = nseg;
            for (int k = 0; k < sg.n; k++) {
                sg.start[k] = wo.seg_start[k];
                sg.win_base[k] = wo.seg_wins[k];
                sg.id_base[k] = id_base[wo.rules[k]];
            }
            sg.start[sg.n] = wo.n;
            u64* rows = wide_scratch(p, kWsRows, std::max<u64>(wo.winners * (u64)W, small_rows));
            srows = rows;
            wide_newt_kernel<<<wide_grid(wo.n), kThreads, 0, p->stream>>>(R.wcand, wo.cw, wo.n, R.wflag, R.wpos, sg,
                                                                           W, rows);
            LAUNCHED();
            const u64* idx = wide_sort(p, rows, W, W, wo.winners);
            wide_gather_kernel<<<wide_grid(wo.winners * W), kThreads, 0, p->stream>>>(rows, W, idx, wo.winners,
                                                                                     R.wnewt);
            LAUNCHED();
        }
        flush_newt();
    }
    // local_insert_in_full: full = full + delta (one flattened launch), delta = newt
    {
        PhaseTimer pt(p, 5);
        WideMergeBatch mb{};
        std::vector<int> merged;
        auto flush_merge = [&]() {
            if (!mb.n) return;
            wide_merge_batch_kernel<<<wide_grid(mb.total), kThreads, 0, p->stream>>>(mb);
            LAUNCHED();
            for (int ri : merged) {
                Relation& R = p->rels[ri];
                std::swap(R.wfull, R.wspare);
                std::swap(R.wfull_cap, R.wspare_cap);
                R.full_n += R.delta_n;
                R.delta_n = 0;
            }
            merged.clear();
            mb.n = 0;
            mb.total = 0;
        };
        for (int ri : s.rels) {
            Relation& R = p->rels[ri];
            if (!R.delta_n) continue;
            const int W = (int)R.arity + 1;
            wide_reserve(p, &R.wspare, &R.wspare_cap, R.full_n + R.delta_n, W, 0);
            mb.job[mb.n++] = WideMergeJob{R.wfull, R.wdelta, R.wspare, R.full_n, R.delta_n, mb.total, W};
            mb.total += R.full_n + R.delta_n;
            merged.push_back(ri);
            if (mb.n == kWideJobs) flush_merge();
        }
        flush_merge();
        for (int ri : s.rels) {
            Relation& R = p->rels[ri];
            std::swap(R.wdelta, R.wnewt);
            std::swap(R.wdelta_cap, R.wnewt_cap);
            R.delta_n = R.newt_n;
            R.newt_n = 0;
        }
    }
    p->stats.iterations++;
}

// RAM::execute_in_batches driven by LIE::execute (lie.cpp:355-432) for one SCC.
void run_scc_wide(ra_program* p, Scc& s)
{
    if (!p->rs_dir.empty()) {
        for (int ri : s.rels) wide_load_restart_delta(p, p->rels[ri]);
    } else {
        for (size_t i = 0; i < s.rels.size(); i++)
            if (s.init[i]) wide_full_to_delta(p, p->rels[s.rels[i]]);
    }
    std::vector<uint64_t> hist;
    for (;;) {
        uint32_t b = p->batch_size;
        while (b != 0) {
            wide_iteration(p, s);
            b--;
            if (!s.fixpoint) break;
        }
        uint32_t d = 0, f = 0;
        for (int ri : s.rels) {
            d += (uint32_t)p->rels[ri].delta_n;
            f += (uint32_t)p->rels[ri].full_n;
        }
        hist.push_back(d);
        hist.push_back(f);
        checkpoint_batch(p, s, !s.fixpoint || d == 0, host_counts(p));
        if (!s.fixpoint || d == 0) break;
    }
    CK(cudaStreamSynchronize(p->stream));
    p->pending_merge = s.rels;
    p->history.push_back((uint64_t)s.id);
    p->history.push_back(hist.size() / 2);
    p->history.insert(p->history.end(), hist.begin(), hist.end());
}

// Does this program need the wide path?  (The packed path's limits: arity and
// projections of at most kMaxArity columns, joins on at least one column, tuples
// within 63 packed bits, join keys within the CSR index's 30 bits.)
bool program_needs_wide(ra_program* p, int bits)
{
    for (const Relation& r : p->rels) {
        if (r.arity > (uint32_t)kMaxArity || r.jcc == 0) return true;
        if ((int)r.arity * bits > 63) return true;
    }
    for (const Scc& s : p->sccs)
        for (const Rule& ru : s.rules) {
            if (ru.proj.size() > (size_t)kMaxArity + (ru.kind == RA_ACOPY ? 1 : 0)) return true;
            const Relation& a = p->rels[ru.in0];
            if (ru.kind == kJoin) {
                const Relation& b = p->rels[ru.in1];
                if ((int)a.jcc * bits > 30) return true;
                // an intern id projected into a data column
                const int id0 = (int)a.arity, id1 = (int)(a.arity + 1 + b.arity - a.jcc);
                for (int x : ru.proj)
                    if (x == id0 || x == id1) return true;
            } else if (ru.kind != RA_ACOPY) {
                for (int x : ru.proj)
                    if (x == (int)a.arity) return true;
            }
        }
    return false;
}

void wide_free_relation(ra_program* p, Relation& r)
{
    dev_free(p, &r.wfull);
    dev_free(p, &r.wdelta);
    dev_free(p, &r.wnewt);
    dev_free(p, &r.wspare);
    dev_free(p, &r.wcand);
    dev_free(p, &r.wflag);
    dev_free(p, &r.wpos);
    r.wfull_cap = r.wdelta_cap = r.wnewt_cap = r.wspare_cap = r.wcand_cap = r.wflag_cap = r.wpos_cap = 0;
}
