/*
 * batch.cpp — many plans in one pass (no reference counterpart; the
 * reference runs one plan per execute() call).
 *
 * Plans are executed level by level: level(scan) = 0, level(join) =
 * 1 + max(level of its children). All joins of one level, across all plans,
 * are independent, so each phase of a level is one grouped, persistent
 * launch over all of them:
 *   decode (every base column of every plan, once, up front)
 *   build  (hist / scan / scatter / per-partition build over all hash joins)
 *   nested-loop collect (all joins with build sides <= 64 rows)
 *   probe  (one tile-ticket kernel over all joins; each join keeps its own
 *           match counter and output arrays)
 *   gather (row-id vectors of every intermediate)
 * and one host synchronisation per level reads every join's match count.
 * The root pages of all plans are written by one grouped launch (VARCHAR
 * columns by their own launches after one shared synchronisation).
 *
 * Results are the same as cj_execute on each plan: the same kernels' unit
 * bodies run on the same data, only scheduled together.
 *
 * Prepared batches (cj_batch_prepare / cj_batch_run) run the same executor
 * three ways: once as usual while it records every join's match count and
 * every VARCHAR column's page count (learn), then once under CUDA stream
 * capture with those counts as exact output sizes (capture): no host
 * synchronisation and no host read of a device value anywhere, every buffer
 * carved from one arena, every task table copied from pinned memory. The
 * captured graph is replayed by cj_batch_run: one launch for the whole
 * batch. Kernels in the graph compare each count with the recorded one and
 * raise DEV_ERR_STALE when they differ (the inputs changed).
 */
#include <algorithm>
#include <chrono>
#include <cstring>
#include <map>
#include <memory>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "exec_common.h"

namespace cj {
namespace {

struct JoinWork {
    size_t plan;
    uint64_t node;
    bool is_root;
    Relation *B, *P;
    RelCol bk, pk;
    bool nl;
    uint64_t cap;
    bool need_b, need_p;
    struct Out {
        bool from_build;
        const Relation *rel;
        RelCol col;
    };
    std::vector<Out> outs;
    DevPtr dir, tuples, part_buf, nlk, nlr, nlc, mb, mp, status, slots;
    unsigned long long *params = nullptr; /* direct-mapped table's parameters (device) */
    int log2_slots = 0, log2_parts = 0;
    uint64_t M = 0;
};

struct PlanState {
    const cj_plan_desc *plan = nullptr;
    int status = CJ_OK;
    std::string err;
    std::vector<int> level;
    std::map<uint64_t, Relation> rel; /* computed join outputs */
    std::vector<Relation> scans;      /* per node (scan nodes) */
    cj_result *result = nullptr;
    /* root */
    uint64_t root_rows = 0;
    std::vector<ColView> root_cols;
    std::vector<int32_t> root_types;
    std::vector<DevPtr> keep; /* match arrays the root views point into */
};

} // namespace

/* What a learning run records for the capture: match counts of every join
 * of every level, in the executor's work order, and page counts of every
 * VARCHAR output column, in materialisation order. */
struct BatchLearned {
    std::vector<std::vector<uint64_t>> level_M;
    std::vector<uint64_t> var_pages;
};

/* Pinned host memory, bump-allocated in 4 MiB blocks: the source of every
 * host-to-device copy captured into a graph (it must outlive the graph). */
struct PinnedBump {
    Context *ctx = nullptr;
    std::vector<PinnedPtr> blocks;
    size_t used = 0;
    void *take(size_t n) {
        n = (n + 15) & ~size_t(15);
        if (blocks.empty() || used + n > blocks.back()->bytes) {
            blocks.push_back(ctx->alloc_pinned(std::max<size_t>(n, 4u << 20)));
            used = 0;
        }
        void *p = static_cast<uint8_t *>(blocks.back()->ptr) + used;
        used += n;
        return p;
    }
};

namespace {

enum class Mode { Eager, Learn, Capture };

class BatchExecutor {
  public:
    BatchExecutor(Context &c, const cj_plan_desc *plans, size_t n, uint32_t flags, Mode mode = Mode::Eager,
                  BatchLearned *learned = nullptr, PinnedBump *bump = nullptr)
        : ctx(c), L(c.launch()), flags(flags), mode(mode), learned(learned), bump(bump) {
        ps.resize(n);
        for (size_t i = 0; i < n; ++i) ps[i].plan = &plans[i];
    }
    ~BatchExecutor() {
        for (auto &p : ps) delete p.result;
    }
    void run(cj_result **results, int32_t *statuses, cj_batch_stats *st);

  private:
    Context &ctx;
    Launch L;
    uint32_t flags;
    Mode mode;
    BatchLearned *learned;
    PinnedBump *bump;
    size_t level_ix = 0; /* levels run so far (index into learned->level_M) */
    size_t var_ix = 0;   /* VARCHAR columns planned so far                  */
    std::vector<PlanState> ps;
    std::map<std::tuple<size_t, uint64_t, uint64_t>, Decoded> decoded;
    cj_batch_stats stats{};
    uint64_t launches0 = 0;

    void ck(cudaError_t e, const char *w) { check_cuda(e, w); }
    template <typename T> DevPtr upload_tasks(const std::vector<T> &v) {
        DevPtr d = ctx.alloc(std::max<size_t>(v.size(), 1) * sizeof(T));
        if (!v.empty()) {
            const void *src = v.data();
            if (mode == Mode::Capture) { /* a captured copy needs a source that outlives the graph */
                void *h = bump->take(v.size() * sizeof(T));
                std::memcpy(h, v.data(), v.size() * sizeof(T));
                src = h;
            }
            ck(cudaMemcpyAsync(d->ptr, src, v.size() * sizeof(T), cudaMemcpyHostToDevice, ctx.stream), "tasks");
        }
        return d;
    }
    /* Device copy of recorded counts, then a check of `counts` against them. */
    void check_counts(const unsigned long long *counts, const std::vector<uint64_t> &want) {
        std::vector<unsigned long long> w(want.begin(), want.end());
        DevPtr d = upload_tasks(w);
        ck(launch_check_counts(L, counts, d->as<unsigned long long>(), (uint32_t)w.size(), ctx.d_status->stale,
                               num_checks++),
           "check_counts");
        keep_checks.push_back(d);
    }
    uint32_t num_checks = 0; /* checks captured so far (levels, then VARCHAR totals) */
    std::vector<DevPtr> keep_checks;
    int levels(PlanState &p, uint64_t node, int depth);
    void decode_all();
    Decoded &dec(size_t plan, uint64_t t, uint64_t c) { return decoded.at({plan, t, c}); }
    ColView view(size_t plan, const Relation &R, const RelCol &c, const uint32_t *ra) {
        return make_view(dec(plan, c.input, c.col), R, c, ra);
    }
    const Relation &relation(PlanState &p, uint64_t node) {
        if (p.plan->nodes[node].node_type == CJ_NODE_SCAN) return p.scans[node];
        return p.rel.at(node);
    }
    void run_level(int lvl);
    void materialize_roots();
};

int BatchExecutor::levels(PlanState &p, uint64_t node, int depth) {
    if (depth > (int)p.plan->num_nodes) fail(CJ_ERR_INVALID_PLAN, "plan has a cycle");
    if (p.level[node] >= 0) return p.level[node];
    const cj_plan_node &n = p.plan->nodes[node];
    int l = 0;
    if (n.node_type == CJ_NODE_HASH_JOIN)
        l = 1 + std::max(levels(p, n.left, depth + 1), levels(p, n.right, depth + 1));
    p.level[node] = l;
    return l;
}

void BatchExecutor::decode_all() {
    std::vector<DecodeTask> tasks;
    std::vector<std::tuple<size_t, uint64_t, uint64_t>> keys;
    uint64_t total_pages = 0;
    for (size_t i = 0; i < ps.size(); ++i) {
        PlanState &p = ps[i];
        if (p.status) continue;
        const cj_plan_desc &plan = *p.plan;
        for (uint64_t n = 0; n < plan.num_nodes; ++n) {
            if (p.level[n] < 0 || plan.nodes[n].node_type != CJ_NODE_SCAN) continue;
            const cj_plan_node &sn = plan.nodes[n];
            for (uint64_t a = 0; a < sn.num_output_attrs; ++a) {
                auto key = std::make_tuple(i, sn.base_table_id, sn.output_attrs[a].index);
                if (decoded.count(key)) continue;
                Decoded d;
                d.type = input_col_type(plan, sn.base_table_id, sn.output_attrs[a].index);
                d.rows = input_rows(plan, sn.base_table_id);
                if (d.rows > 0xFFFFFFFFull) fail(CJ_ERR_LIMIT, "table exceeds 2^32-1 rows");
                if (const cj_table *r = resident_input(plan, sn.base_table_id))
                    d.src = r->cols[sn.output_attrs[a].index];
                else if (mode == Mode::Capture)
                    fail(CJ_ERR_UNSUPPORTED, "a prepared batch needs device-resident inputs");
                else
                    upload_pages(ctx, plan.inputs[sn.base_table_id].columns[sn.output_attrs[a].index], d.src,
                                 &stats.h2d_bytes);
                const uint64_t words = std::max<uint64_t>((d.rows + 31) / 32, 1);
                d.valid = ctx.alloc(words * 4);
                ck(cudaMemsetAsync(d.valid->ptr, 0, words * 4, ctx.stream), "memset");
                if (d.type == CJ_VARCHAR) d.desc = ctx.alloc(d.rows * 8);
                else d.values = ctx.alloc(d.rows * (d.type == CJ_INT32 ? 4 : 8));
                DecodeTask t{};
                t.pages = d.src.dev;
                t.num_pages = d.src.num_pages;
                t.page_base = total_pages;
                t.rows = d.rows;
                t.type = d.type;
                t.values = d.values ? d.values->ptr : nullptr;
                t.desc = d.desc ? d.desc->as<uint64_t>() : nullptr;
                t.valid = d.valid->as<uint32_t>();
                total_pages += t.num_pages;
                tasks.push_back(t);
                keys.push_back(key);
                decoded.emplace(key, std::move(d));
            }
        }
    }
    if (tasks.empty()) return;
    DevPtr td = upload_tasks(tasks);
    DevPtr rows_pp = ctx.alloc(std::max<uint64_t>(total_pages, 1) * 4);
    DevPtr row_start = ctx.alloc((total_pages + 1) * 8);
    DevPtr tmp = ctx.alloc(scan_temp_bytes(total_pages));
    ck(launch_decode_grouped(L, td->as<DecodeTask>(), (uint32_t)tasks.size(), total_pages, rows_pp->as<uint32_t>(),
                             row_start->as<uint64_t>(), tmp->ptr),
       "decode_grouped");
}

void BatchExecutor::run_level(int lvl) {
    std::vector<JoinWork> work;
    for (size_t i = 0; i < ps.size(); ++i) {
        PlanState &p = ps[i];
        if (p.status) continue;
        const cj_plan_desc &plan = *p.plan;
        for (uint64_t n = 0; n < plan.num_nodes; ++n) {
            if (p.level[n] != lvl || plan.nodes[n].node_type != CJ_NODE_HASH_JOIN) continue;
            const cj_plan_node &node = plan.nodes[n];
            JoinWork w;
            w.plan = i;
            w.node = n;
            w.is_root = n == plan.root;
            Relation &Lr = const_cast<Relation &>(relation(p, node.left));
            Relation &Rr = const_cast<Relation &>(relation(p, node.right));
            const bool bl = Lr.rows <= Rr.rows; /* join_setup.h:108-136 */
            w.B = bl ? &Lr : &Rr;
            w.P = bl ? &Rr : &Lr;
            const uint64_t battr = bl ? node.left_attr : node.right_attr;
            const uint64_t pattr = bl ? node.right_attr : node.left_attr;
            if (battr >= w.B->cols.size() || pattr >= w.P->cols.size())
                fail(CJ_ERR_INVALID_PLAN, "join key index out of range");
            w.bk = w.B->cols[battr];
            w.pk = w.P->cols[pattr];
            auto key_ok = [](int32_t t) { return t == CJ_INT32 || t == CJ_INT64; };
            if (!key_ok(w.bk.type) || !key_ok(w.pk.type)) fail(CJ_ERR_UNSUPPORTED, "join keys must be INT32 or INT64");
            if (w.B->rows > 0xFFFFFFFFull || w.P->rows > 0xFFFFFFFFull)
                fail(CJ_ERR_LIMIT, "relation exceeds 2^32-1 rows");
            const uint64_t lsz = Lr.cols.size();
            w.need_b = w.need_p = false;
            for (uint64_t a = 0; a < node.num_output_attrs; ++a) {
                const cj_attr &at = node.output_attrs[a];
                if (at.index >= lsz + Rr.cols.size()) fail(CJ_ERR_INVALID_PLAN, "output attribute out of range");
                const Relation *side = at.index < lsz ? &Lr : &Rr;
                RelCol c = side->cols[at.index < lsz ? at.index : at.index - lsz];
                if (c.type != at.type) fail(CJ_ERR_INVALID_PLAN, "output attribute type differs from its column");
                bool fb = side == w.B;
                if (key_from_probe_side(fb, c, w.bk, w.pk)) {
                    fb = false;
                    side = w.P;
                    c = w.pk;
                }
                w.need_b |= fb;
                w.need_p |= !fb;
                w.outs.push_back({fb, side, c});
            }
            const uint64_t nl_max =
                std::min<int64_t>(std::max<int64_t>(ctx.opt.nested_loop_max_build, 0), kNestedLoopMax);
            w.nl = w.B->rows <= nl_max;
            w.cap = w.P->rows;
            work.push_back(std::move(w));
        }
    }
    if (work.empty()) return;
    stats.num_joins += work.size();

    /* ---- build: hash tables and nested-loop build sides ---- */
    std::vector<BuildTask> btasks;
    std::vector<NlCollectTask> ntasks;
    uint32_t chunks = 0, parts = 0, max_parts = 1, max_slots = 1;
    uint64_t cells = 0;
    for (auto &w : work) {
        if (!w.B->rows || !w.P->rows) continue;
        const ColView bv = view(w.plan, *w.B, w.bk, nullptr);
        if (w.nl) {
            w.nlk = ctx.alloc(kNestedLoopMax * 8);
            w.nlr = ctx.alloc(kNestedLoopMax * 4);
            w.nlc = ctx.alloc(4);
            ntasks.push_back({bv, (uint32_t)w.B->rows, w.nlk->as<int64_t>(), w.nlr->as<uint32_t>(), w.nlc->as<uint32_t>()});
            continue;
        }
        BuildPlan bp;
        bp.num_rows = (uint32_t)w.B->rows;
        bp.log2_slots = std::max(11, ceil_log2(w.B->rows));
        const int spp = std::min(build_log2_spp(ctx, w.B->rows), bp.log2_slots);
        bp.log2_parts = std::min(bp.log2_slots - spp, 12);
        if (bp.log2_slots - bp.log2_parts > 14) fail(CJ_ERR_LIMIT, "build side too large for one radix pass");
        w.log2_slots = bp.log2_slots;
        w.log2_parts = bp.log2_parts;
        const int kb = w.bk.type == CJ_INT32 ? 4 : 8;
        w.dir = ctx.alloc(build_dir_bytes(bp.log2_slots, kb));
        w.tuples = ctx.alloc(w.B->rows * build_tuple_bytes(kb));
        w.part_buf = ctx.alloc(w.B->rows * build_tuple_bytes(kb));
        BuildGeometry g = build_geometry(build_launch(ctx, w.B->rows), bp);
        BuildTask t{};
        t.key = bv;
        t.n = bp.num_rows;
        t.log2_slots = bp.log2_slots;
        t.log2_parts = bp.log2_parts;
        t.grid = g.grid;
        t.chunk = g.chunk;
        t.chunk_base = chunks;
        t.part_base = parts;
        t.cell_base = cells;
        t.dir = w.dir->as<uint64_t>();
        t.tuples = w.tuples->ptr;
        t.part_buf = w.part_buf->ptr;
        chunks += g.grid;
        parts += 1u << bp.log2_parts;
        cells += g.cells;
        max_parts = std::max(max_parts, 1u << bp.log2_parts);
        max_slots = std::max(max_slots, 1u << (bp.log2_slots - bp.log2_parts));
        btasks.push_back(t);
    }
    /* Unique keys spread over at most dense_keys x rows values also get a
     * direct-mapped table (built beside the hash table, which stays the
     * fallback): the device decides per join whether it is usable, and the
     * probe takes it when it is (one random access per probe row). */
    std::vector<DirectTask> dtasks;
    std::vector<size_t> didx;
    uint32_t key_blocks = 0, fill_blocks = 0;
    for (size_t k = 0; k < work.size(); ++k) {
        auto &w = work[k];
        if (w.nl || !w.B->rows || !w.P->rows || ctx.opt.dense_keys <= 0) continue;
        const uint64_t max_span = std::min<uint64_t>((uint64_t)ctx.opt.dense_keys * w.B->rows, 1ull << 28);
        w.slots = ctx.alloc(max_span * 4);
        DirectTask t{};
        t.key = view(w.plan, *w.B, w.bk, nullptr);
        t.n = (uint32_t)w.B->rows;
        t.key_blocks = (uint32_t)((w.B->rows + kDirectBlockRows - 1) / kDirectBlockRows);
        t.key_base = key_blocks;
        t.fill_blocks = (uint32_t)((max_span + kDirectFillSlots - 1) / kDirectFillSlots);
        t.fill_base = fill_blocks;
        t.max_span = max_span;
        t.slots = w.slots->as<uint32_t>();
        key_blocks += t.key_blocks;
        fill_blocks += t.fill_blocks;
        dtasks.push_back(t);
        didx.push_back(k);
    }
    DevPtr dparams;
    if (!dtasks.empty()) {
        std::vector<unsigned long long> init(dtasks.size() * kDirectParams, 0ull);
        for (size_t j = 0; j < dtasks.size(); ++j) init[j * kDirectParams] = ~0ull;
        dparams = upload_tasks(init);
        for (size_t j = 0; j < dtasks.size(); ++j) {
            dtasks[j].params = dparams->as<unsigned long long>() + j * kDirectParams;
            work[didx[j]].params = dtasks[j].params;
        }
        keep_checks.push_back(dparams);
    }
    stats.num_hash_joins += btasks.size();
    stats.num_nested_loop_joins += ntasks.size();
    DevPtr dt = upload_tasks(dtasks);
    ck(launch_direct_build_grouped(L, dt->as<DirectTask>(), (uint32_t)dtasks.size(), key_blocks, fill_blocks),
       "direct_build_grouped");
    DevPtr bt = upload_tasks(btasks), nt = upload_tasks(ntasks);
    DevPtr btmp = ctx.alloc(build_grouped_temp_bytes(cells));
    ck(launch_build_grouped(L, bt->as<BuildTask>(), (uint32_t)btasks.size(), chunks, parts, cells, max_parts, max_slots,
                            ctx.d_bloom, btmp->ptr),
       "build_grouped");
    ck(launch_nl_collect_grouped(L, nt->as<NlCollectTask>(), (uint32_t)ntasks.size()), "nl_collect_grouped");

    /* ---- probe: one ticketed launch over the tiles of every join ---- */
    const std::vector<uint64_t> *known = nullptr; /* capture: the recorded counts */
    if (mode == Mode::Capture) {
        if (level_ix >= learned->level_M.size() || learned->level_M[level_ix].size() != work.size())
            fail(CJ_ERR_INTERNAL, "prepared batch: level shape differs from the learning run");
        known = &learned->level_M[level_ix];
        for (size_t k = 0; k < work.size(); ++k) work[k].cap = (*known)[k];
    }
    for (int attempt = 0; attempt < 2; ++attempt) {
        std::vector<ProbeTask> ptasks;
        std::vector<size_t> pidx;
        uint32_t tiles = 0;
        for (size_t k = 0; k < work.size(); ++k) {
            auto &w = work[k];
            if (!w.B->rows || !w.P->rows) continue;
            if (attempt == 1 && w.M <= w.cap) continue;
            if (attempt == 1) {
                stats.probe_reruns++;
                w.cap = w.M;
            }
            pidx.push_back(k);
        }
        if (pidx.empty()) break;
        const size_t nwords = pidx.size() + 1; /* ticket, then one match counter per join */
        DevPtr words = ctx.alloc(nwords * 8);
        ck(cudaMemsetAsync(words->ptr, 0, nwords * 8, ctx.stream), "memset");
        unsigned long long *wp = words->as<unsigned long long>();
        unsigned int *ticket = reinterpret_cast<unsigned int *>(wp);
        size_t off = 1;
        for (size_t k : pidx) {
            auto &w = work[k];
            w.mb = w.need_b ? ctx.alloc(w.cap * 4) : nullptr;
            w.mp = w.need_p ? ctx.alloc(w.cap * 4) : nullptr;
            ProbeTask t{};
            t.pkey = view(w.plan, *w.P, w.pk, nullptr);
            t.n_probe = (uint32_t)w.P->rows;
            t.kind = w.nl ? 1 : (w.params ? 2 : 0);
            t.slots = w.slots ? w.slots->as<uint32_t>() : nullptr;
            t.params = w.params;
            t.build_key_type = w.bk.type;
            t.log2_slots = w.log2_slots;
            t.dir = w.dir ? w.dir->as<uint64_t>() : nullptr;
            t.tuples = w.tuples ? w.tuples->ptr : nullptr;
            t.nl_keys = w.nlk ? w.nlk->as<int64_t>() : nullptr;
            t.nl_rids = w.nlr ? w.nlr->as<uint32_t>() : nullptr;
            t.nl_count = w.nlc ? w.nlc->as<uint32_t>() : nullptr;
            t.out.build_rids = w.mb ? w.mb->as<uint32_t>() : nullptr;
            t.out.probe_rids = w.mp ? w.mp->as<uint32_t>() : nullptr;
            t.out.capacity = (w.need_b || w.need_p) ? w.cap : 0;
            t.out.counter = wp + off++;
            t.num_tiles = probe_tiles(t.n_probe);
            t.tile_base = tiles;
            tiles += t.num_tiles;
            ptasks.push_back(t);
        }
        DevPtr pt = upload_tasks(ptasks);
        ck(launch_probe_grouped(L, pt->as<ProbeTask>(), (uint32_t)ptasks.size(), tiles, ticket, ctx.d_bloom),
           "probe_grouped");
        if (known) {
            /* capture: outputs were sized to the recorded counts; the graph
             * checks them instead of reading them back */
            std::vector<uint64_t> want;
            for (size_t k : pidx) want.push_back((*known)[k]);
            check_counts(wp + 1, want);
            for (size_t k : pidx) work[k].M = (*known)[k];
            keep_checks.push_back(words);
            keep_checks.push_back(pt);
            break;
        }
        std::vector<unsigned long long> counts(nwords);
        ck(cudaMemcpyAsync(counts.data(), words->ptr, counts.size() * 8, cudaMemcpyDeviceToHost, ctx.stream), "counts");
        ctx.sync_status();
        stats.syncs++;
        bool overflow = false;
        for (size_t j = 0; j < pidx.size(); ++j) {
            auto &w = work[pidx[j]];
            w.M = counts[ptasks[j].out.counter - wp];
            if (w.M > 0xFFFFFFFFull) fail(CJ_ERR_LIMIT, "join result exceeds 2^32-1 rows");
            if (w.M > w.cap && (w.need_b || w.need_p)) overflow = true;
        }
        if (!overflow) break;
    }
    if (mode == Mode::Learn) {
        std::vector<uint64_t> Ms;
        for (auto &w : work) Ms.push_back(w.M);
        learned->level_M.push_back(std::move(Ms));
    }
    ++level_ix;
    for (auto &w : work) {
        w.dir.reset();
        w.tuples.reset();
        w.part_buf.reset();
        w.slots.reset();
        stats.probe_rows += w.P->rows;
        stats.matches += w.M;
    }

    /* ---- outputs: intermediates by one grouped gather; roots remembered ---- */
    std::vector<GatherTask> gtasks;
    uint64_t gchunks = 0;
    for (auto &w : work) {
        PlanState &p = ps[w.plan];
        if (w.is_root) {
            p.root_rows = w.M;
            for (auto &o : w.outs) {
                const DevPtr &m = o.from_build ? w.mb : w.mp;
                p.root_cols.push_back(view(w.plan, *o.rel, o.col, m ? m->as<uint32_t>() : nullptr));
                p.root_types.push_back(o.col.type);
                if (m) p.keep.push_back(m);
                for (auto &v : o.rel->vecs) p.keep.push_back(v);
            }
            continue;
        }
        Relation res;
        res.rows = w.M;
        std::map<std::pair<int, int>, int> vecmap;
        for (auto &o : w.outs) {
            auto key = std::make_pair(o.from_build ? 0 : 1, o.col.vec);
            auto it = vecmap.find(key);
            int vi;
            if (it != vecmap.end()) {
                vi = it->second;
            } else {
                const DevPtr &match = o.from_build ? w.mb : w.mp;
                DevPtr nv;
                if (w.M == 0) {
                    nv = ctx.alloc(0);
                } else if (o.col.vec < 0) {
                    nv = match;
                } else {
                    nv = ctx.alloc(w.M * 4);
                    GatherTask g{o.rel->vecs[o.col.vec]->as<uint32_t>(), match->as<uint32_t>(), nv->as<uint32_t>(), w.M,
                                 gchunks};
                    gchunks += (w.M + kGatherChunk - 1) / kGatherChunk;
                    gtasks.push_back(g);
                }
                vi = (int)res.vecs.size();
                res.vecs.push_back(nv);
                vecmap[key] = vi;
            }
            res.cols.push_back({o.col.type, o.col.input, o.col.col, vi, true});
        }
        p.rel[w.node] = std::move(res);
    }
    DevPtr gt = upload_tasks(gtasks);
    ck(launch_gather_grouped(L, gt->as<GatherTask>(), (uint32_t)gtasks.size(), gchunks), "gather_grouped");
}

void BatchExecutor::materialize_roots() {
    const uint32_t TR = (uint32_t)std::max<int64_t>(64, std::min<int64_t>(ctx.opt.varchar_tile_rows, 8192));
    std::vector<PageTask> ptasks;
    uint64_t pages = 0;
    struct VarJob {
        size_t plan, col;
        DevPtr temp;
    };
    std::vector<VarJob> var;
    for (size_t i = 0; i < ps.size(); ++i) {
        PlanState &p = ps[i];
        if (p.status) continue;
        auto *res = new cj_result;
        p.result = res;
        res->ctx = &ctx;
        res->num_rows = p.root_rows;
        res->types = p.root_types;
        const size_t nc = p.root_cols.size();
        res->num_pages.assign(nc, 0);
        res->dev_pages.resize(nc);
        res->host_cols.assign(nc, nullptr);
        if (!p.root_rows) continue;
        for (size_t c = 0; c < nc; ++c) {
            if (p.root_types[c] == CJ_VARCHAR) {
                var.push_back({i, c, ctx.alloc(varchar_temp_bytes(p.root_rows, TR))});
                continue;
            }
            const uint32_t R = rows_per_page_fixed(p.root_types[c]);
            res->num_pages[c] = (p.root_rows + R - 1) / R;
            res->dev_pages[c] = ctx.alloc(res->num_pages[c] * kPageSize);
            ptasks.push_back({p.root_cols[c], p.root_rows, res->dev_pages[c]->as<uint8_t>(), pages});
            pages += res->num_pages[c];
        }
    }
    DevPtr pt = upload_tasks(ptasks);
    ck(launch_write_fixed_grouped(L, pt->as<PageTask>(), (uint32_t)ptasks.size(), pages), "write_fixed_grouped");
    if (!var.empty()) {
        DevPtr totals = ctx.alloc(var.size() * 8);
        for (size_t k = 0; k < var.size(); ++k) {
            PlanState &p = ps[var[k].plan];
            ck(launch_varchar_plan(L, p.root_cols[var[k].col], p.root_rows, TR, var[k].temp->ptr,
                                   totals->as<unsigned long long>() + k),
               "varchar_plan");
        }
        std::vector<unsigned long long> host(var.size());
        if (mode == Mode::Capture) {
            if (learned->var_pages.size() != var.size())
                fail(CJ_ERR_INTERNAL, "prepared batch: VARCHAR columns differ from the learning run");
            for (size_t k = 0; k < var.size(); ++k) host[k] = learned->var_pages[k];
            check_counts(totals->as<unsigned long long>(), learned->var_pages);
            keep_checks.push_back(totals);
        } else {
            ck(cudaMemcpyAsync(host.data(), totals->ptr, host.size() * 8, cudaMemcpyDeviceToHost, ctx.stream),
               "copy");
            ctx.sync_status();
            stats.syncs++;
            if (mode == Mode::Learn) learned->var_pages.assign(host.begin(), host.end());
        }
        for (size_t k = 0; k < var.size(); ++k) {
            PlanState &p = ps[var[k].plan];
            cj_result *res = p.result;
            const size_t c = var[k].col;
            res->num_pages[c] = host[k];
            res->dev_pages[c] = ctx.alloc(host[k] * kPageSize);
            ck(launch_varchar_write(L, p.root_cols[c], p.root_rows, TR, var[k].temp->ptr,
                                    res->dev_pages[c]->as<uint8_t>()),
               "varchar_write");
        }
    }
    if (flags & CJ_EXEC_RESULT_ON_DEVICE) return;
    for (auto &p : ps) {
        if (!p.result) continue;
        uint64_t total = 0;
        for (uint64_t np : p.result->num_pages) total += np;
        if (!total) continue;
        /* one block per plan, of the size a plan run alone takes, so that
         * blocks go back to the pool as their results are freed and serve
         * single-plan and grouped executions alike */
        p.result->host = ctx.alloc_pinned(total * kPageSize);
        uint8_t *h = static_cast<uint8_t *>(p.result->host->ptr);
        for (size_t c = 0; c < p.result->num_pages.size(); ++c) {
            p.result->host_cols[c] = h;
            const size_t bytes = p.result->num_pages[c] * kPageSize;
            if (bytes)
                ck(cudaMemcpyAsync(h, p.result->dev_pages[c]->ptr, bytes, cudaMemcpyDeviceToHost, ctx.stream),
                   "download");
            h += bytes;
            stats.d2h_bytes += bytes;
        }
    }
}

void BatchExecutor::run(cj_result **results, int32_t *statuses, cj_batch_stats *st) {
    auto t0 = std::chrono::steady_clock::now();
    launches0 = launches_so_far();
    int maxl = 0;
    for (auto &p : ps) {
        try {
            validate_plan(ctx, *p.plan);
            p.level.assign(p.plan->num_nodes, -1);
            maxl = std::max(maxl, levels(p, p.plan->root, 0));
            p.scans.resize(p.plan->num_nodes);
            for (uint64_t n = 0; n < p.plan->num_nodes; ++n)
                if (p.level[n] >= 0 && p.plan->nodes[n].node_type == CJ_NODE_SCAN)
                    p.scans[n] = scan_relation(*p.plan, p.plan->nodes[n]);
        } catch (const Error &e) {
            p.status = e.code;
            p.err = e.msg;
        }
    }
    decode_all();
    /* scan roots */
    for (size_t i = 0; i < ps.size(); ++i) {
        PlanState &p = ps[i];
        if (p.status) continue;
        const cj_plan_node &root = p.plan->nodes[p.plan->root];
        if (root.node_type != CJ_NODE_SCAN) continue;
        const Relation &s = p.scans[p.plan->root];
        p.root_rows = s.rows;
        for (auto &c : s.cols) {
            p.root_cols.push_back(view(i, s, c, nullptr));
            p.root_types.push_back(c.type);
        }
    }
    for (int lvl = 1; lvl <= maxl; ++lvl) {
        nvtxRangePushA("cj:batch_level");
        struct Pop {
            ~Pop() { nvtxRangePop(); }
        } pop;
        run_level(lvl);
    }
    nvtxRangePushA("cj:batch_materialize");
    {
        struct Pop {
            ~Pop() { nvtxRangePop(); }
        } pop;
        materialize_roots();
    }
    if (mode != Mode::Capture) {
        ctx.sync_status();
        stats.syncs++;
    }
    for (size_t i = 0; i < ps.size(); ++i) {
        results[i] = ps[i].result;
        ps[i].result = nullptr;
        if (statuses) statuses[i] = ps[i].status;
    }
    auto t1 = std::chrono::steady_clock::now();
    stats.num_plans = ps.size();
    stats.num_levels = (uint64_t)maxl;
    stats.kernel_launches = launches_so_far() - launches0;
    stats.total_us = std::chrono::duration<double, std::micro>(t1 - t0).count();
    if (st) *st = stats;
}

} // namespace

void execute_batch(Context &ctx, const cj_plan_desc *plans, size_t n, uint32_t flags, cj_result **results,
                   int32_t *statuses, cj_batch_stats *stats) {
    for (size_t i = 0; i < n; ++i) results[i] = nullptr;
    BatchExecutor ex(ctx, plans, n, flags);
    ex.run(results, statuses, stats);
}

} // namespace cj

/* A batch captured as one CUDA graph over buffers it owns. */
struct cj_prepared {
    cj::Context *ctx = nullptr;
    std::vector<cj_plan_desc> plans;
    uint32_t flags = 0;
    cj::DevPtr arena;            /* every device buffer of the graph   */
    cj::PinnedBump bump;         /* sources of the captured task copies */
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<cj_result *> templates; /* the results' layout, in the arena */
    cj_batch_stats capture_stats{};
    ~cj_prepared() {
        for (auto *r : templates) delete r;
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
    }
};

namespace cj {

cj_prepared *prepare_batch(Context &ctx, const cj_plan_desc *plans, size_t n, uint32_t flags) {
    for (size_t i = 0; i < n; ++i)
        for (uint64_t t = 0; t < plans[i].num_inputs; ++t)
            if (!resident_input(plans[i], t))
                fail(CJ_ERR_UNSUPPORTED, "a prepared batch needs device-resident inputs (cj_table)");
    /* A VARCHAR column's page count depends on the order of its rows (the
     * writer packs each tile's strings greedily), and a probe's output
     * order differs from run to run (tiles reserve their output as they
     * finish): a graph cannot size such pages from a learned count.
     * Fixed-width pages (ceil(rows / rows per page)) do not depend on it. */
    for (size_t i = 0; i < n; ++i) {
        if (plans[i].root >= plans[i].num_nodes || !plans[i].nodes) continue; /* the learn run reports it */
        const cj_plan_node &root = plans[i].nodes[plans[i].root];
        for (uint64_t a = 0; a < root.num_output_attrs; ++a)
            if (root.output_attrs && root.output_attrs[a].type == CJ_VARCHAR)
                fail(CJ_ERR_UNSUPPORTED, "a prepared batch writes fixed-width results only (plan " + std::to_string(i) +
                                             " outputs VARCHAR, whose page count depends on the row order)");
    }
    auto prep = std::make_unique<cj_prepared>();
    prep->ctx = &ctx;
    prep->plans.assign(plans, plans + n);
    prep->flags = flags;
    prep->bump.ctx = &ctx;
    /* 1. learn: run once, recording every count; its allocations bound the
     *    arena (the capture allocates the same buffers, outputs no larger) */
    BatchLearned learned;
    {
        std::vector<cj_result *> res(n, nullptr);
        std::vector<int32_t> sts(n, CJ_OK);
        const uint64_t bytes0 = ctx.alloc_bytes;
        BatchExecutor ex(ctx, prep->plans.data(), n, flags, Mode::Learn, &learned);
        try {
            ex.run(res.data(), sts.data(), nullptr);
        } catch (...) {
            for (auto *r : res) delete r;
            throw;
        }
        for (auto *r : res) delete r;
        for (size_t i = 0; i < n; ++i)
            if (sts[i] != CJ_OK) fail(sts[i], "plan " + std::to_string(i) + " of the batch failed validation");
        const uint64_t need = ctx.alloc_bytes - bytes0;
        check_cuda(cudaStreamSynchronize(ctx.stream), "stream synchronize");
        prep->arena = ctx.alloc(need + need / 8 + (8u << 20));
    }
    /* 2. capture the whole batch into one graph over the arena */
    ctx.arena_base = prep->arena->as<uint8_t>();
    ctx.arena_size = prep->arena->bytes;
    ctx.arena_used = 0;
    struct ArenaOff {
        Context &c;
        ~ArenaOff() { c.arena_base = nullptr; }
    } arena_off{ctx};
    check_cuda(cudaStreamBeginCapture(ctx.stream, cudaStreamCaptureModeRelaxed), "begin capture");
    prep->templates.assign(n, nullptr);
    try {
        std::vector<int32_t> sts(n, CJ_OK);
        BatchExecutor ex(ctx, prep->plans.data(), n, flags, Mode::Capture, &learned, &prep->bump);
        ex.run(prep->templates.data(), sts.data(), &prep->capture_stats);
    } catch (...) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(ctx.stream, &g);
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        throw;
    }
    check_cuda(cudaStreamEndCapture(ctx.stream, &prep->graph), "end capture");
    check_cuda(cudaGraphInstantiate(&prep->exec, prep->graph, 0), "graph instantiate");
    return prep.release();
}

void run_prepared(cj_prepared &p, cj_result **results, cj_batch_stats *stats) {
    Context &ctx = *p.ctx;
    auto t0 = std::chrono::steady_clock::now();
    check_cuda(cudaGraphLaunch(p.exec, ctx.stream), "graph launch");
    ctx.sync_status();
    for (size_t i = 0; i < p.templates.size(); ++i) {
        const cj_result *t = p.templates[i];
        auto *r = new cj_result(*t); /* pages are the prepared batch's: shared, not copied */
        r->keep = p.arena;
        results[i] = r;
    }
    auto t1 = std::chrono::steady_clock::now();
    if (stats) {
        *stats = p.capture_stats;
        stats->syncs = 1;
        stats->total_us = std::chrono::duration<double, std::micro>(t1 - t0).count();
    }
}

} // namespace cj

extern "C" {

int cj_batch_prepare(cj_context *ctx, const cj_plan_desc *plans, uint64_t num_plans, uint32_t flags,
                     cj_prepared **out) {
    if (!ctx || !out || (num_plans && !plans)) return cj::set_last_error(CJ_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    cudaSetDevice(ctx->device);
    try {
        *out = cj::prepare_batch(*ctx, plans, (size_t)num_plans, flags);
    } catch (const cj::Error &e) {
        cudaStreamSynchronize(ctx->stream);
        cudaGetLastError();
        return cj::set_last_error(e.code, e.msg);
    } catch (const std::bad_alloc &) {
        return cj::set_last_error(CJ_ERR_OUT_OF_MEMORY, "host allocation failed");
    } catch (...) {
        return cj::set_last_error(CJ_ERR_INTERNAL, "unexpected exception");
    }
    cj::clear_last_error();
    return CJ_OK;
}

int cj_batch_run(cj_prepared *p, cj_result **results, cj_batch_stats *stats) {
    if (!p || (!p->templates.empty() && !results)) return cj::set_last_error(CJ_ERR_INVALID_ARGUMENT, "null argument");
    cudaSetDevice(p->ctx->device);
    try {
        cj::run_prepared(*p, results, stats);
    } catch (const cj::Error &e) {
        cudaGetLastError();
        return cj::set_last_error(e.code, e.msg);
    } catch (const std::bad_alloc &) {
        return cj::set_last_error(CJ_ERR_OUT_OF_MEMORY, "host allocation failed");
    }
    cj::clear_last_error();
    return CJ_OK;
}

void cj_prepared_free(cj_prepared *p) {
    if (!p) return;
    cudaSetDevice(p->ctx->device);
    cudaStreamSynchronize(p->ctx->stream);
    delete p;
}

} // extern "C"
