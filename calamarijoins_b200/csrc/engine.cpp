/*
 * engine.cpp — plan executor: the depth-first join recursion of the
 * reference (src/execute.cpp:84-325) over device-resident relations.
 *
 * A relation is either a scan (rows are base-table rows) or the output of
 * a join. Join outputs are late-materialised: instead of copying values
 * (construct_intermediate.h:121-220) a join output keeps one u32 row-id
 * vector per contributing base table, and each of its columns names its
 * base column and the vector that reaches it. Values are read only by the
 * kernels that need them: join keys by build/probe, projected columns by
 * the root's page writers.
 */
#include <algorithm>
#include <chrono>
#include <cstring>
#include <functional>
#include <map>
#include <set>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "engine.h"

#include "exec_common.h"

namespace cj {
namespace {

enum Phase { PH_UPLOAD, PH_DECODE, PH_BUILD, PH_PROBE, PH_NL, PH_INTER, PH_MAT, PH_DOWNLOAD, PH_COUNT };
/* NVTX range names of the phases (host-side ranges around the enqueueing of
 * each phase; visible in Nsight Systems timelines). */
constexpr const char *kPhaseNames[PH_COUNT] = {"cj:upload", "cj:decode",       "cj:build",       "cj:probe",
                                               "cj:nested_loop", "cj:intermediate", "cj:materialize",
                                               "cj:download"};

class Executor {
  public:
    Executor(Context &c, const cj_plan_desc &p, uint32_t f) : ctx(c), plan(p), flags(f), L(c.launch()) {}
    ~Executor() {
        /* Pages still being uploaded (an error came first) are freed on the
         * kernel stream: order those frees after the copies. */
        for (auto &kv : prefetched) {
            cudaStreamWaitEvent(ctx.stream, kv.second.done, 0);
            ctx.put_event(kv.second.done);
        }
        for (auto &pe : phase_events) {
            ctx.put_event(pe.a);
            ctx.put_event(pe.b);
        }
    }
    cj_result *run(cj_exec_stats *st);

  private:
    struct PhaseEv {
        int phase;
        cudaEvent_t a, b;
    };
    class PhaseScope {
      public:
        PhaseScope(Executor &e, int ph) : e_(e), ph_(ph) {
            nvtxRangePushA(kPhaseNames[ph]);
            a_ = e.ctx.get_event();
            cudaEventRecord(a_, e.ctx.stream);
        }
        ~PhaseScope() {
            cudaEvent_t b = e_.ctx.get_event();
            cudaEventRecord(b, e_.ctx.stream);
            e_.phase_events.push_back({ph_, a_, b});
            nvtxRangePop();
        }

      private:
        Executor &e_;
        int ph_;
        cudaEvent_t a_;
    };
    /* Per-kernel timing when profiling is on. */
    class KScope {
      public:
        KScope(Executor &e, const char *name) : e_(e) {
            if (!e.ctx.opt.profile_kernels) return;
            auto it = e.ctx.profile_index.find(name);
            if (it == e.ctx.profile_index.end()) {
                slot_ = e.ctx.profile.size();
                e.ctx.profile.push_back({name, 0, 0.0});
                e.ctx.profile_index[name] = slot_;
            } else {
                slot_ = it->second;
            }
            a_ = e.ctx.get_event();
            cudaEventRecord(a_, e.ctx.stream);
            on_ = true;
        }
        ~KScope() {
            if (!on_) return;
            cudaEvent_t b = e_.ctx.get_event();
            cudaEventRecord(b, e_.ctx.stream);
            e_.ctx.pending.push_back({slot_, a_, b});
        }

      private:
        Executor &e_;
        size_t slot_ = 0;
        cudaEvent_t a_ = nullptr;
        bool on_ = false;
    };

    Context &ctx;
    const cj_plan_desc &plan;
    uint32_t flags;
    Launch L;
    std::map<std::pair<uint64_t, uint64_t>, Decoded> decoded;
    /* Host columns whose pages are on their way on the upload stream. */
    struct Prefetched {
        ColumnPages pages;
        cudaEvent_t done = nullptr;
    };
    std::map<std::pair<uint64_t, uint64_t>, Prefetched> prefetched;
    std::vector<PhaseEv> phase_events;
    cj_exec_stats stats{};
    bool synced_last = false; /* the last thing enqueued was a synchronisation */
    /* Brings the status block to the host, counting the synchronisation. */
    void sync() {
        ctx.sync_status();
        stats.host_syncs++;
    }
    /* A result written with a device-side row count (materialize with
     * rows_dev): its rows and pages once the count is known. */
    void finish_counted(cj_result &r, uint64_t rows) {
        r.num_rows = rows;
        uint64_t pages = 0;
        for (size_t c = 0; c < r.types.size(); ++c) {
            const uint32_t R = rows_per_page_fixed(r.types[c]);
            r.num_pages[c] = (rows + R - 1) / R;
            if (!rows) r.dev_pages[c].reset();
            pages += r.num_pages[c];
        }
        stats.output_rows = rows;
        stats.output_pages = pages;
    }

    const cj_table *resident(uint64_t t) const { return resident_input(plan, t); }
    uint64_t table_rows(uint64_t t) const { return input_rows(plan, t); }
    int32_t column_type(uint64_t t, uint64_t c) const { return input_col_type(plan, t, c); }

    void validate();
    void prefetch();
    Decoded &decode(uint64_t t, uint64_t c);
    Relation resolve(uint64_t node, int depth);
    Relation exec_join(uint64_t node, int depth, bool is_root, cj_result **out);
    ColView view(const Relation &R, const RelCol &c, const uint32_t *rid_a);
    /* An output column of the root: its relation column and the match row
     * ids that select its rows (null for a scan root). Decoded on use. */
    struct OutCol {
        const Relation *rel; /* null: the values are already in `pages` */
        RelCol col;
        const uint32_t *rid_a;
        DevPtr pages; /* result pages written by the probe (no NULL) */
    };
    ColView out_view(const OutCol &oc) { return view(*oc.rel, oc.col, oc.rid_a); }
    cj_result *materialize(const std::vector<OutCol> &cols, const std::vector<int32_t> &types, uint64_t rows,
                           const unsigned long long *rows_dev = nullptr);
    void ck(cudaError_t e, const char *what) { check_cuda(e, what); }
};

void Executor::validate() { validate_plan(ctx, plan); }

/* Starts the upload of every host column the plan will decode, on the
 * context's upload stream, in the order the kernels need them: join keys
 * bottom-up, then the root's outputs. The kernel stream waits for a
 * column's copy only when it decodes that column, so later columns (the
 * payloads) cross PCIe while the joins below the root run. */
void Executor::prefetch() {
    using TC = std::pair<uint64_t, uint64_t>;
    std::vector<TC> order;
    std::set<TC> seen;
    auto add = [&](const TC &tc) {
        if (seen.insert(tc).second) order.push_back(tc);
    };
    std::function<std::vector<TC>(uint64_t, int)> cols = [&](uint64_t node, int depth) -> std::vector<TC> {
        if (depth > (int)plan.num_nodes) fail(CJ_ERR_INVALID_PLAN, "plan has a cycle");
        const cj_plan_node &n = plan.nodes[node];
        std::vector<TC> out;
        if (n.node_type == CJ_NODE_SCAN) {
            for (uint64_t a = 0; a < n.num_output_attrs; ++a) out.push_back({n.base_table_id, n.output_attrs[a].index});
            return out;
        }
        std::vector<TC> both = cols(n.left, depth + 1);
        const std::vector<TC> r = cols(n.right, depth + 1);
        if (n.left_attr < both.size()) add(both[n.left_attr]);
        if (n.right_attr < r.size()) add(r[n.right_attr]);
        both.insert(both.end(), r.begin(), r.end());
        for (uint64_t a = 0; a < n.num_output_attrs; ++a)
            if (n.output_attrs[a].index < both.size()) out.push_back(both[n.output_attrs[a].index]);
        return out;
    };
    for (const TC &tc : cols(plan.root, 0)) add(tc);
    cudaEvent_t first = nullptr;
    for (const TC &tc : order) {
        if (resident(tc.first)) continue;
        if (!first) {
            first = ctx.get_event();
            ck(cudaEventRecord(first, ctx.h2d_stream), "event record");
        }
        Prefetched pf;
        upload_pages(ctx, plan.inputs[tc.first].columns[tc.second], pf.pages, &stats.h2d_bytes, ctx.h2d_stream);
        pf.done = ctx.get_event();
        ck(cudaEventRecord(pf.done, ctx.h2d_stream), "event record");
        prefetched.emplace(tc, std::move(pf));
    }
    if (first) {
        cudaEvent_t last = ctx.get_event();
        ck(cudaEventRecord(last, ctx.h2d_stream), "event record");
        phase_events.push_back({PH_UPLOAD, first, last});
    }
}

Decoded &Executor::decode(uint64_t t, uint64_t c) {
    auto key = std::make_pair(t, c);
    auto it = decoded.find(key);
    if (it != decoded.end()) return it->second;
    Decoded d;
    d.type = column_type(t, c);
    d.rows = table_rows(t);
    if (d.rows > 0xFFFFFFFFull) fail(CJ_ERR_LIMIT, "table exceeds 2^32-1 rows (u32 row ids)");
    auto pf = prefetched.find(key);
    if (const cj_table *r = resident(t)) {
        d.src = r->cols[c];
    } else if (pf != prefetched.end()) {
        d.src = pf->second.pages;
        ck(cudaStreamWaitEvent(ctx.stream, pf->second.done, 0), "stream wait");
        ctx.put_event(pf->second.done);
        prefetched.erase(pf);
    } else {
        PhaseScope ph(*this, PH_UPLOAD);
        upload_pages(ctx, plan.inputs[t].columns[c], d.src, &stats.h2d_bytes);
    }
    PhaseScope ph(*this, PH_DECODE);
    const uint64_t np = d.src.num_pages;
    DevPtr rows_pp = ctx.alloc(std::max<uint64_t>(np, 1) * 4);
    DevPtr row_start = ctx.alloc((np + 1) * 8);
    DevPtr partials = ctx.alloc(page_index_blocks(L, np) * 8);
    d.col_flags = ctx.alloc(8); /* COL_* flags, then the index's finished-block count */
    ck(cudaMemsetAsync(d.col_flags->ptr, 0, 8, ctx.stream), "memset");
    {
        KScope k(*this, "page_index");
        ck(launch_page_index(L, d.src.dev, np, d.type, d.rows, rows_pp->as<uint32_t>(), partials->as<uint64_t>(),
                             row_start->as<uint64_t>(), d.col_flags->as<uint32_t>()),
           "page_index");
    }
    const uint64_t words = (d.rows + 31) / 32;
    d.valid = ctx.alloc(std::max<uint64_t>(words, 1) * 4);
    ck(cudaMemsetAsync(d.valid->ptr, 0, std::max<uint64_t>(words, 1) * 4, ctx.stream), "memset");
    if (d.type == CJ_VARCHAR) {
        d.desc = ctx.alloc(d.rows * 8);
        KScope k(*this, "decode_varchar");
        ck(launch_decode_varchar(L, d.src.dev, np, row_start->as<uint64_t>(), d.rows, d.desc->as<uint64_t>(),
                                 d.valid->as<uint32_t>()),
           "decode_varchar");
    } else {
        const uint64_t w = d.type == CJ_INT32 ? 4 : 8;
        d.values = ctx.alloc(d.rows * w);
        KScope k(*this, d.type == CJ_INT32 ? "decode_int32" : "decode_8byte");
        ck(launch_decode_fixed(L, d.src.dev, np, d.type, row_start->as<uint64_t>(), d.rows, d.values->ptr,
                               d.valid->as<uint32_t>(), d.col_flags->as<uint32_t>()),
           "decode_fixed");
    }
    return decoded.emplace(key, std::move(d)).first->second;
}

ColView Executor::view(const Relation &R, const RelCol &c, const uint32_t *rid_a) {
    return make_view(decode(c.input, c.col), R, c, rid_a);
}

Relation Executor::resolve(uint64_t node, int depth) {
    if (depth > (int)plan.num_nodes) fail(CJ_ERR_INVALID_PLAN, "plan has a cycle");
    const cj_plan_node &n = plan.nodes[node];
    if (n.node_type == CJ_NODE_SCAN) return scan_relation(plan, n);
    return exec_join(node, depth, false, nullptr);
}

Relation Executor::exec_join(uint64_t node_idx, int depth, bool is_root, cj_result **out) {
    const cj_plan_node &n = plan.nodes[node_idx];
    Relation Lr = resolve(n.left, depth + 1);
    Relation Rr = resolve(n.right, depth + 1);

    /* select_build_probe_side (join_setup.h:108-136): the smaller relation
     * builds, left wins ties; the plan's build_left hint is not used. */
    const bool build_left = Lr.rows <= Rr.rows;
    Relation &B = build_left ? Lr : Rr;
    Relation &P = build_left ? Rr : Lr;
    const uint64_t battr = build_left ? n.left_attr : n.right_attr;
    const uint64_t pattr = build_left ? n.right_attr : n.left_attr;
    if (battr >= B.cols.size() || pattr >= P.cols.size()) fail(CJ_ERR_INVALID_PLAN, "join key index out of range");
    const RelCol bk = B.cols[battr], pk = P.cols[pattr];
    auto key_ok = [](int32_t t) { return t == CJ_INT32 || t == CJ_INT64; };
    if (!key_ok(bk.type) || !key_ok(pk.type)) fail(CJ_ERR_UNSUPPORTED, "join keys must be INT32 or INT64");
    if (B.rows > 0xFFFFFFFFull || P.rows > 0xFFFFFFFFull) fail(CJ_ERR_LIMIT, "relation exceeds 2^32-1 rows");

    /* Output columns over (left ++ right) and which match side each needs
     * (determine_collection_mode, join_setup.h:146-173). */
    struct OutRef {
        bool from_build;
        const Relation *rel;
        RelCol col;
        bool from_keys = false; /* root: read from the keys the probe writes */
    };
    std::vector<OutRef> outs;
    bool need_b = false, need_p = false;
    const uint64_t lsz = Lr.cols.size();
    for (uint64_t a = 0; a < n.num_output_attrs; ++a) {
        const cj_attr &at = n.output_attrs[a];
        if (at.index >= lsz + Rr.cols.size()) fail(CJ_ERR_INVALID_PLAN, "output attribute out of range");
        const Relation *side = at.index < lsz ? &Lr : &Rr;
        RelCol c = side->cols[at.index < lsz ? at.index : at.index - lsz];
        if (c.type != at.type) fail(CJ_ERR_INVALID_PLAN, "output attribute type differs from its column");
        bool fb = side == &B;
        if (key_from_probe_side(fb, c, bk, pk)) {
            fb = false;
            side = &P;
            c = pk;
        }
        need_b |= fb;
        need_p |= !fb;
        outs.push_back({fb, side, c});
    }

    stats.num_joins++;
    stats.probe_rows += P.rows;
    uint64_t M = 0;
    /* At the root, outputs of the probe key (and of the build key, which is
     * read through the probe side) are written by the probe itself, straight
     * into their places in the result pages (matched keys are never NULL):
     * no gather, no copy; every such column shares those pages. */
    bool emit_keys = false;
    if (is_root) {
        need_p = false;
        for (auto &o : outs) {
            if (!o.from_build && o.rel == &P && same_column(o.col, pk)) {
                o.from_keys = true;
                emit_keys = true;
            } else if (!o.from_build) {
                need_p = true;
            }
        }
    }
    const bool collect = need_b || need_p || emit_keys;
    const int32_t key_bytes = pk.type == CJ_INT32 ? 4 : 8;
    DevPtr mb, mp, mk;
    /* The root's result columns: the pages the probe wrote the keys into, or
     * a relation column and the match row ids that select its rows. */
    auto root_columns = [&](std::vector<OutCol> &cols, std::vector<int32_t> &types) {
        for (auto &o : outs) {
            OutCol oc{o.rel, o.col, nullptr, nullptr};
            if (o.from_keys) {
                oc.rel = nullptr;
                oc.pages = mk; /* o.col.type == the probe key's type */
            } else {
                oc.rid_a = o.from_build ? (mb ? mb->as<uint32_t>() : nullptr) : (mp ? mp->as<uint32_t>() : nullptr);
            }
            cols.push_back(oc);
            types.push_back(o.col.type);
        }
    };
    if (B.rows && P.rows) {
        const ColView bv = view(B, bk, nullptr);
        const ColView pv = view(P, pk, nullptr);
        if (is_root) {
            /* The root's other output columns whose pages are already in
             * HBM are indexed (and decoded, if they must be) now, while the
             * kernels above run, rather than after the probe's
             * synchronisation, where the GPU would wait for the host to
             * enqueue them. Columns still uploading stay lazy, so that the
             * result downloads overlap their uploads. */
            for (const auto &o : outs)
                if (!o.from_keys && resident(o.col.input)) decode(o.col.input, o.col.col);
        }
        const uint64_t nl_max = std::min<int64_t>(std::max<int64_t>(ctx.opt.nested_loop_max_build, 0), kNestedLoopMax);
        const bool nl = B.rows <= nl_max;
        DevPtr dir, tuples, nlk, nlr, nlc, slots;
        int log2_slots = 0;
        bool inline_dir = true;
        unsigned long long *d_params = &ctx.d_status->aux[0];
        bool direct = false; /* direct-mapped table tried (the device decides) */
        bool open = false;   /* open-addressing table tried (the device decides) */
        DevPtr open_slots;
        uint64_t open_n = 0;
        /* Unique INT32 keys too spread out for the direct-mapped table: an
         * open-addressing table (one slot walk per probe row, against a
         * directory entry and a tuple range). Tried only after the
         * direct-mapped table turned out unusable; a repeated key sends the
         * join on to the hash table. */
        auto build_open = [&]() -> bool {
            if (bk.type != CJ_INT32 || B.rows > kOpenMaxRows) return false;
            open_n = (std::max<uint64_t>(2 * B.rows, 1024) + 3) & ~3ull; /* groups of 4 slots */
            open_slots = ctx.alloc(open_n * 8);
            ck(cudaMemsetAsync(d_params + kOpenDup, 0, 8, ctx.stream), "memset");
            KScope k(*this, "open_build");
            ck(launch_open_build(L, bv, (uint32_t)B.rows, open_slots->as<unsigned long long>(), open_n,
                                 d_params + kOpenDup),
               "open_build");
            return true;
        };
        auto build_hash = [&]() {
            BuildPlan bp;
            bp.num_rows = (uint32_t)B.rows;
            bp.log2_slots = std::max(11, ceil_log2(B.rows)); /* hashtable.h:255-264 */
            /* 2^11 directory slots per partition by default (the slot
             * counters of one partition fit shared memory); the partition
             * bits are spread over one radix pass, or two above 12 bits
             * (build sides of more than 2^23 rows) */
            const int log2_spp = std::min(std::min(build_log2_spp(ctx, B.rows), 14), bp.log2_slots);
            bp.log2_parts = bp.log2_slots - log2_spp;
            log2_slots = bp.log2_slots;
            const int kb = bk.type == CJ_INT32 ? 4 : 8;
            const Launch LB = build_launch(ctx, B.rows);
            bp.inline_first = kb == 4 && build_dir_bytes(bp.log2_slots, 4, true) + B.rows * build_tuple_bytes(4) <=
                                             (uint64_t)ctx.opt.inline_dir_max_bytes;
            inline_dir = bp.inline_first;
            dir = ctx.alloc(build_dir_bytes(bp.log2_slots, kb, bp.inline_first));
            tuples = ctx.alloc(B.rows * build_tuple_bytes(kb));
            DevPtr tmp = ctx.alloc(build_temp_bytes(LB, bp, kb));
            KScope k(*this, "build");
            ck(launch_build(LB, bp, bv, ctx.d_bloom, dir->as<uint64_t>(), tuples->ptr, tmp->ptr), "build");
        };
        if (nl) {
            stats.num_nested_loop_joins++;
            PhaseScope ph(*this, PH_NL);
            nlk = ctx.alloc(kNestedLoopMax * 8);
            nlr = ctx.alloc(kNestedLoopMax * 4);
            nlc = ctx.alloc(4);
            KScope k(*this, "nl_collect");
            ck(launch_nl_collect(L, bv, (uint32_t)B.rows, nlk->as<int64_t>(), nlr->as<uint32_t>(),
                                 nlc->as<uint32_t>()),
               "nl_collect");
        } else {
            stats.num_hash_joins++;
            PhaseScope ph(*this, PH_BUILD);
            if (ctx.opt.dense_keys > 0) {
                /* Unique keys spread over at most dense_keys x rows values get
                 * a direct-mapped table: one random access per probe row
                 * instead of a directory entry and a tuple. The device works
                 * out the key range and whether the table is usable; the
                 * host learns it at the probe's own synchronisation and then,
                 * if it was not, builds the hash table. */
                /* 4 bytes per slot: at 8 x rows, 32 B per build row, against
                 * about 16-24 B for the hash table, for one random access
                 * per probe row instead of two; at most 2^28 slots (1 GiB) */
                const uint64_t max_span = std::min<uint64_t>((uint64_t)ctx.opt.dense_keys * B.rows, 1ull << 28);
                ck(cudaMemsetAsync(d_params, 0xFF, 8, ctx.stream), "memset");
                ck(cudaMemsetAsync(d_params + 1, 0, (kDirectParams - 1) * 8, ctx.stream), "memset");
                slots = ctx.alloc(max_span * 4);
                KScope k(*this, "direct_build");
                ck(launch_direct_build(L, bv, (uint32_t)B.rows, max_span, slots->as<uint32_t>(), d_params),
                   "direct_build");
                direct = true;
            }
            if (!direct) build_hash();
        }
        /* Allocates the match outputs for `cap` pairs and launches the probe
         * of the table built above. */
        auto launch_probe = [&](uint64_t cap) {
            mb = need_b ? ctx.alloc(cap * 4) : nullptr;
            mp = need_p ? ctx.alloc(cap * 4) : nullptr;
            /* the key columns' result pages, sized for the capacity */
            const uint32_t key_rpp = rows_per_page_fixed(pk.type);
            mk = emit_keys ? ctx.alloc((cap + key_rpp - 1) / key_rpp * kPageSize) : nullptr;
            MatchOut mo;
            mo.build_rids = mb ? mb->as<uint32_t>() : nullptr;
            mo.probe_rids = mp ? mp->as<uint32_t>() : nullptr;
            mo.key_pages = mk ? mk->as<uint8_t>() : nullptr;
            mo.key_bytes = key_bytes;
            mo.capacity = collect ? cap : 0;
            mo.counter = &ctx.d_status->counter;
            DevPtr sched = ctx.alloc(probe_sched_bytes((uint32_t)P.rows));
            {
                PhaseScope ph(*this, nl ? PH_NL : PH_PROBE);
                if (nl) {
                    KScope k(*this, "nl_probe");
                    ck(launch_nl_probe_tiles(L, pv, (uint32_t)P.rows, nlk->as<int64_t>(), nlr->as<uint32_t>(),
                                             nlc->as<uint32_t>(), mo, sched->ptr),
                       "nl_probe");
                } else if (open) {
                    KScope k(*this, "probe_open");
                    ck(launch_probe_tiles_open(L, pv, (uint32_t)P.rows, open_slots->as<unsigned long long>(), open_n,
                                               d_params + kOpenDup, mo, sched->ptr),
                       "probe_open");
                } else if (direct) {
                    KScope k(*this, "probe_array");
                    ck(launch_probe_tiles_array(L, pv, (uint32_t)P.rows, slots->as<uint32_t>(), d_params, mo,
                                                sched->ptr),
                       "probe_array");
                } else {
                    KScope k(*this, "probe_hash");
                    ck(launch_probe_tiles_hash(probe_launch(ctx, P.rows), pv, (uint32_t)P.rows, bk.type,
                                               dir->as<uint64_t>(), tuples->ptr, log2_slots, ctx.d_bloom, mo,
                                               sched->ptr, inline_dir),
                       "probe");
                }
            }
        };
        /* keys too spread out (aux[3] = 1) or a key repeats (2): the
         * direct-mapped table is unusable (its probe did nothing); an
         * open-addressing table for spread-out keys, else the hash table */
        auto replace_direct = [&]() {
            direct = false;
            slots.reset();
            PhaseScope ph(*this, PH_BUILD);
            open = ctx.h_status->aux[3] == 1 && build_open();
            if (!open) build_hash();
        };
        uint64_t cap = P.rows;
        bool all_fixed = true;
        for (const auto &o : outs) all_fixed &= o.col.type != CJ_VARCHAR;
        if (is_root && direct && collect && all_fixed && (flags & CJ_EXEC_RESULT_ON_DEVICE) && ctx.opt.defer_count) {
            /* Unique build keys at the root, result left in HBM, no VARCHAR
             * output: at most one match per probe row, so the result is sized
             * for P.rows and its pages are written with the match count read
             * on the device. The execution's one host synchronisation comes
             * last; only if the device refused the direct-mapped table does
             * the join go on as below. */
            launch_probe(cap);
            std::vector<OutCol> cols;
            std::vector<int32_t> types;
            root_columns(cols, types);
            std::unique_ptr<cj_result> r(materialize(cols, types, cap, &ctx.d_status->counter));
            sync();
            if (!ctx.h_status->aux[3]) {
                M = ctx.h_status->counter;
                finish_counted(*r, M);
                stats.num_direct_joins++;
                stats.matches += M;
                synced_last = true;
                *out = r.release();
                return Relation{};
            }
            r.reset();
            replace_direct();
        }
        for (;;) {
            launch_probe(cap);
            sync();
            if (direct && ctx.h_status->aux[3]) {
                replace_direct();
                continue;
            }
            if (open && ctx.h_status->aux[kOpenDup]) {
                /* a key repeats: the probe did nothing; hash table */
                open = false;
                open_slots.reset();
                PhaseScope ph(*this, PH_BUILD);
                build_hash();
                continue;
            }
            M = ctx.h_status->counter;
            if (M <= cap || !collect) break;
            if (M > 0xFFFFFFFFull) fail(CJ_ERR_LIMIT, "join result exceeds 2^32-1 rows");
            stats.probe_reruns++;
            cap = M;
        }
        if (direct) stats.num_direct_joins++;
        if (open) stats.num_open_joins++;
    }
    if (M > 0xFFFFFFFFull) fail(CJ_ERR_LIMIT, "join result exceeds 2^32-1 rows");
    stats.matches += M;

    if (is_root) {
        std::vector<OutCol> cols;
        std::vector<int32_t> types;
        root_columns(cols, types);
        *out = materialize(cols, types, M);
        return Relation{};
    }

    /* Intermediate: one row-id vector per (side, source vector). */
    Relation res;
    res.rows = M;
    std::map<std::pair<int, int>, int> vecmap;
    PhaseScope ph(*this, PH_INTER);
    for (auto &o : outs) {
        const int side = o.from_build ? 0 : 1;
        auto key = std::make_pair(side, o.col.vec);
        auto it = vecmap.find(key);
        int vi;
        if (it != vecmap.end()) {
            vi = it->second;
        } else {
            const DevPtr &match = o.from_build ? mb : mp;
            DevPtr nv;
            if (M == 0) {
                nv = ctx.alloc(0);
            } else if (o.col.vec < 0) {
                nv = match; /* scan side: the match row ids are base rows */
            } else {
                nv = ctx.alloc(M * 4);
                KScope k(*this, "gather_rids");
                ck(launch_gather_u32(L, o.rel->vecs[o.col.vec]->as<uint32_t>(), match->as<uint32_t>(), M,
                                     nv->as<uint32_t>()),
                   "gather");
            }
            vi = (int)res.vecs.size();
            res.vecs.push_back(nv);
            vecmap[key] = vi;
        }
        res.cols.push_back({o.col.type, o.col.input, o.col.col, vi, true});
    }
    return res;
}

/* Writes the root's result pages. For a host result each column's pages
 * go down on the context's download stream as soon as its writer is done,
 * so the copy of one column overlaps the writing of the next. */
cj_result *Executor::materialize(const std::vector<OutCol> &cols, const std::vector<int32_t> &types,
                                 uint64_t rows, const unsigned long long *rows_dev) {
    auto *res = new cj_result;
    std::unique_ptr<cj_result> guard(res);
    res->ctx = &ctx;
    res->num_rows = rows;
    res->types = types;
    const size_t nc = cols.size();
    res->num_pages.assign(nc, 0);
    res->dev_pages.resize(nc);
    res->host_cols.assign(nc, nullptr);
    const bool to_host = !(flags & CJ_EXEC_RESULT_ON_DEVICE);
    if (rows_dev) {
        /* rows is a capacity and the count is on the device: fixed-width
         * columns left in HBM only (their pages do not depend on the count
         * beyond the last one) */
        for (int32_t t : types)
            if (t == CJ_VARCHAR) fail(CJ_ERR_INTERNAL, "device-counted result with a VARCHAR column");
        if (to_host) fail(CJ_ERR_INTERNAL, "device-counted result for the host");
    }
    /* Orders the kernel stream (and so every later free) after the copies
     * issued so far, also when an error leaves this scope early. */
    struct DownloadJoin {
        Context &ctx;
        cudaEvent_t first = nullptr, last = nullptr;
        bool timed = false; /* events handed to the phase timer */
        ~DownloadJoin() {
            if (!first) return;
            if (!last) {
                last = ctx.get_event();
                cudaEventRecord(last, ctx.d2h_stream);
            }
            cudaStreamWaitEvent(ctx.stream, last, 0);
            if (!timed) {
                ctx.put_event(first);
                ctx.put_event(last);
            }
        }
    } dl{ctx};
    {
        PhaseScope ph(*this, PH_MAT);
        const uint32_t TR = (uint32_t)std::max<int64_t>(64, std::min<int64_t>(ctx.opt.varchar_tile_rows, 8192));
        std::vector<DevPtr> vtemp(nc);
        DevPtr totals;
        size_t nvar = 0;
        for (size_t c = 0; c < nc; ++c)
            if (types[c] == CJ_VARCHAR) ++nvar;
        if (rows && nvar) {
            totals = ctx.alloc(nvar * 8);
            size_t k = 0;
            for (size_t c = 0; c < nc; ++c) {
                if (types[c] != CJ_VARCHAR) continue;
                vtemp[c] = ctx.alloc(varchar_temp_bytes(rows, TR));
                const ColView cv = out_view(cols[c]);
                KScope ks(*this, "varchar_plan");
                ck(launch_varchar_plan(L, cv, rows, TR, vtemp[c]->ptr,
                                       totals->as<unsigned long long>() + k),
                   "varchar_plan");
                ++k;
            }
            std::vector<unsigned long long> host(nvar);
            ck(cudaMemcpyAsync(host.data(), totals->ptr, nvar * 8, cudaMemcpyDeviceToHost, ctx.stream), "copy");
            sync();
            k = 0;
            for (size_t c = 0; c < nc; ++c)
                if (types[c] == CJ_VARCHAR) res->num_pages[c] = host[k++];
        }
        uint64_t total_pages = 0;
        for (size_t c = 0; c < nc; ++c) {
            if (rows && types[c] != CJ_VARCHAR) {
                const uint32_t R = rows_per_page_fixed(types[c]);
                res->num_pages[c] = (rows + R - 1) / R;
            }
            total_pages += res->num_pages[c];
        }
        stats.output_rows = rows;
        stats.output_pages = total_pages;
        /* Columns that share device pages (the join keys written by the
         * probe) share one host copy too: downloaded once. */
        std::vector<int64_t> alias(nc, -1);
        for (size_t c = 0; c < nc; ++c)
            for (size_t k = 0; k < c && alias[c] < 0; ++k)
                if (cols[c].pages && cols[k].pages == cols[c].pages) alias[c] = (int64_t)k;
        uint64_t host_pages = 0;
        for (size_t c = 0; c < nc; ++c)
            if (alias[c] < 0) host_pages += res->num_pages[c];
        if (to_host && host_pages) {
            res->host = ctx.alloc_pinned(host_pages * kPageSize);
            uint8_t *h = static_cast<uint8_t *>(res->host->ptr);
            for (size_t c = 0; c < nc; ++c) {
                if (alias[c] >= 0) {
                    res->host_cols[c] = res->host_cols[alias[c]];
                    continue;
                }
                res->host_cols[c] = h;
                h += res->num_pages[c] * kPageSize;
            }
        }
        for (size_t c = 0; c < nc; ++c) {
            if (!rows) continue;
            if (cols[c].pages) {
                /* values already in place: headers and bitmaps, once per
                 * shared page array */
                res->dev_pages[c] = cols[c].pages;
                if (alias[c] < 0) {
                    KScope ks(*this, "finish_pages");
                    ck(launch_finish_dense_pages(L, cols[c].pages->as<uint8_t>(), rows, types[c], rows_dev),
                       "finish_pages");
                }
            } else {
                /* decoded here, not before the loop: the kernel stream waits
                 * for a column's upload only when its pages are written */
                const ColView cv = out_view(cols[c]);
                res->dev_pages[c] = ctx.alloc(res->num_pages[c] * kPageSize);
                if (types[c] != CJ_VARCHAR) {
                    KScope ks(*this, types[c] == CJ_INT32 ? "write_pages_int32" : "write_pages_8byte");
                    ck(launch_write_fixed_pages(L, cv, rows, res->dev_pages[c]->as<uint8_t>(), rows_dev),
                       "write_fixed");
                } else {
                    KScope ks(*this, "varchar_write");
                    ck(launch_varchar_write(L, cv, rows, TR, vtemp[c]->ptr, res->dev_pages[c]->as<uint8_t>()),
                       "varchar_write");
                }
            }
            const size_t bytes = res->num_pages[c] * kPageSize;
            if (to_host && bytes && alias[c] < 0) {
                cudaEvent_t written = ctx.get_event();
                ck(cudaEventRecord(written, ctx.stream), "event record");
                ck(cudaStreamWaitEvent(ctx.d2h_stream, written, 0), "stream wait");
                ctx.put_event(written);
                if (!dl.first) {
                    dl.first = ctx.get_event();
                    ck(cudaEventRecord(dl.first, ctx.d2h_stream), "event record");
                }
                ck(cudaMemcpyAsync(res->host_cols[c], res->dev_pages[c]->ptr, bytes, cudaMemcpyDeviceToHost,
                                   ctx.d2h_stream),
                   "download");
                stats.d2h_bytes += bytes;
            }
        }
    }
    if (dl.first) {
        dl.last = ctx.get_event();
        ck(cudaEventRecord(dl.last, ctx.d2h_stream), "event record");
        phase_events.push_back({PH_DOWNLOAD, dl.first, dl.last});
        dl.timed = true;
    }
    return guard.release();
}

cj_result *Executor::run(cj_exec_stats *st) {
    auto t0 = std::chrono::steady_clock::now();
    const uint64_t launches0 = launches_so_far();
    validate();
    prefetch();
    cj_result *res = nullptr;
    const cj_plan_node &root = plan.nodes[plan.root];
    if (root.node_type == CJ_NODE_SCAN) {
        /* A scan root (the reference requires a join root) returns the
         * projected table. */
        Relation s = scan_relation(plan, root);
        if (s.rows > 0xFFFFFFFFull) fail(CJ_ERR_LIMIT, "table exceeds 2^32-1 rows");
        std::vector<OutCol> cols;
        std::vector<int32_t> types;
        for (auto &c : s.cols) {
            cols.push_back({&s, c, nullptr, nullptr});
            types.push_back(c.type);
        }
        res = materialize(cols, types, s.rows);
    } else {
        exec_join(plan.root, 0, true, &res);
    }
    std::unique_ptr<cj_result> guard(res);
    if (!synced_last) sync();
    double ph_us[PH_COUNT] = {0};
    for (auto &pe : phase_events) {
        float ms = 0;
        if (cudaEventElapsedTime(&ms, pe.a, pe.b) == cudaSuccess) ph_us[pe.phase] += ms * 1000.0;
    }
    cudaGetLastError();
    if (ctx.opt.profile_kernels) ctx.resolve_profile();
    auto t1 = std::chrono::steady_clock::now();
    stats.upload_us = ph_us[PH_UPLOAD];
    stats.decode_us = ph_us[PH_DECODE];
    stats.build_us = ph_us[PH_BUILD];
    stats.probe_us = ph_us[PH_PROBE];
    stats.nested_loop_us = ph_us[PH_NL];
    stats.intermediate_us = ph_us[PH_INTER];
    stats.materialize_us = ph_us[PH_MAT];
    stats.download_us = ph_us[PH_DOWNLOAD];
    stats.total_us = std::chrono::duration<double, std::micro>(t1 - t0).count();
    stats.kernel_launches = launches_so_far() - launches0;
    if (st) *st = stats;
    return guard.release();
}

} // namespace

cj_result *execute_plan(Context &ctx, const cj_plan_desc &plan, uint32_t flags, cj_exec_stats *stats) {
    struct Range {
        Range() { nvtxRangePushA("cj_execute"); }
        ~Range() { nvtxRangePop(); }
    } range;
    Executor ex(ctx, plan, flags);
    return ex.run(stats);
}

} // namespace cj
