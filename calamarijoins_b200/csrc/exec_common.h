/*
 * exec_common.h — types shared by the one-plan executor (engine.cpp) and
 * the batch executor (batch.cpp).
 */
#pragma once

#include <map>
#include <string>
#include <vector>

#include "engine.h"

namespace cj {

inline int ceil_log2(uint64_t x) {
    int l = 0;
    while ((1ull << l) < x) ++l;
    return l;
}

/* Hash directory slots per radix partition (log2) for a build of `rows`
 * rows: the option when set, else the autotuner's entry, else 2^11. */
inline int build_log2_spp(const Context &ctx, uint64_t rows) {
    if (ctx.opt.slots_per_partition > 0) return ceil_log2((uint64_t)ctx.opt.slots_per_partition);
    const int t = ctx.tuning.for_rows(rows).log2_spp;
    return t > 0 ? t : 11;
}
/* Launch parameters of a hash build / a hash probe over `rows` rows: the
 * CJ_OPT_CTAS_PER_SM option when set, else the autotuner's entry, else the
 * kernels' defaults. */
inline Launch build_launch(const Context &ctx, uint64_t rows) {
    Launch L = ctx.launch();
    L.part_ctas_per_sm = ctx.opt.ctas_per_sm > 0 ? (int)ctx.opt.ctas_per_sm : ctx.tuning.for_rows(rows).part_ctas;
    return L;
}
inline Launch probe_launch(const Context &ctx, uint64_t rows) {
    Launch L = ctx.launch();
    L.ctas_per_sm = ctx.opt.ctas_per_sm > 0 ? (int)ctx.opt.ctas_per_sm : ctx.tuning.for_rows(rows).probe_ctas;
    return L;
}

/* A base column decoded into dense device arrays. */
struct Decoded {
    int32_t type = CJ_INT32;
    uint64_t rows = 0;
    ColumnPages src;
    DevPtr values, valid, desc;
    DevPtr col_flags; /* u32 COL_* flags from the page headers; null: not computed */
};

/* A column of a relation: base column (input, col) reached through row-id
 * vector `vec` of the relation (-1: the relation row is the base row). */
struct RelCol {
    int32_t type;
    uint64_t input;
    uint64_t col;
    int vec;
    bool sentinel; /* value left a non-root join: INT32_MIN reads as NULL */
};

inline bool same_column(const RelCol &a, const RelCol &b) {
    return a.input == b.input && a.col == b.col && a.vec == b.vec;
}

/* On every output row of an equi-join the build key equals the probe key.
 * When both keys have one type, an output of the build key is read through
 * the probe side instead: its row ids run in probe order, the build side's
 * are random, and a join whose build side contributes nothing else needs no
 * build row ids at all. (NULL and, after a non-root join, INT32_MIN never
 * match, so the two columns agree on every output row, NULL flags too.) */
inline bool key_from_probe_side(bool from_build, const RelCol &c, const RelCol &bk, const RelCol &pk) {
    return from_build && same_column(c, bk) && bk.type == pk.type;
}

/* A scan (rows are base rows) or a join output (late-materialised: one
 * u32 row-id vector per contributing base table). */
struct Relation {
    uint64_t rows = 0;
    std::vector<DevPtr> vecs;
    std::vector<RelCol> cols;
};

inline const cj_table *resident_input(const cj_plan_desc &plan, uint64_t t) {
    return plan.resident_inputs ? plan.resident_inputs[t] : nullptr;
}
inline uint64_t input_rows(const cj_plan_desc &plan, uint64_t t) {
    const cj_table *r = resident_input(plan, t);
    return r ? r->num_rows : plan.inputs[t].num_rows;
}
inline uint64_t input_cols(const cj_plan_desc &plan, uint64_t t) {
    const cj_table *r = resident_input(plan, t);
    return r ? r->cols.size() : plan.inputs[t].num_columns;
}
inline int32_t input_col_type(const cj_plan_desc &plan, uint64_t t, uint64_t c) {
    const cj_table *r = resident_input(plan, t);
    return r ? r->cols[c].type : plan.inputs[t].columns[c].type;
}

inline Relation scan_relation(const cj_plan_desc &plan, const cj_plan_node &n) {
    Relation r;
    r.rows = input_rows(plan, n.base_table_id);
    for (uint64_t a = 0; a < n.num_output_attrs; ++a)
        r.cols.push_back({n.output_attrs[a].type, n.base_table_id, n.output_attrs[a].index, -1, false});
    return r;
}

inline ColView make_view(const Decoded &d, const Relation &R, const RelCol &c, const uint32_t *rid_a) {
    ColView v{};
    v.type = c.type;
    v.values = d.values ? d.values->ptr : nullptr;
    v.valid = d.valid->as<uint32_t>();
    v.str_desc = d.desc ? d.desc->as<uint64_t>() : nullptr;
    v.pages = d.src.dev;
    v.rid_a = rid_a;
    v.rid_b = c.vec >= 0 ? R.vecs[c.vec]->as<uint32_t>() : nullptr;
    v.null_sentinel = (c.sentinel && c.type == CJ_INT32) ? 1 : 0;
    v.col_flags = d.col_flags ? d.col_flags->as<uint32_t>() : nullptr;
    return v;
}

/* Structural checks of a plan description (indices, types, children). */
inline void validate_plan(const Context &ctx, const cj_plan_desc &plan) {
    if (plan.num_nodes == 0 || !plan.nodes) fail(CJ_ERR_INVALID_PLAN, "plan has no nodes");
    if (plan.root >= plan.num_nodes) fail(CJ_ERR_INVALID_PLAN, "root index out of range");
    if (plan.num_inputs && !plan.inputs && !plan.resident_inputs)
        fail(CJ_ERR_INVALID_PLAN, "plan has inputs but no input tables");
    for (uint64_t t = 0; t < plan.num_inputs; ++t) {
        const cj_table *r = resident_input(plan, t);
        if (!r && !plan.inputs) fail(CJ_ERR_INVALID_PLAN, "input " + std::to_string(t) + " missing");
        /* a resident table is complete when it is handed out (its upload
         * or filter synchronises), so any context of the same device may
         * read it; its owner must outlive the plans that do */
        if (r && r->ctx != &ctx && r->ctx->device != ctx.device)
            fail(CJ_ERR_INVALID_ARGUMENT, "resident table of another device");
        if (!r) {
            const cj_table_desc &td = plan.inputs[t];
            if (td.num_columns && !td.columns) fail(CJ_ERR_INVALID_PLAN, "table without column array");
            for (uint64_t c = 0; c < td.num_columns; ++c)
                if (td.columns[c].type < CJ_INT32 || td.columns[c].type > CJ_VARCHAR)
                    fail(CJ_ERR_INVALID_PLAN, "unknown column type");
        }
    }
    for (uint64_t i = 0; i < plan.num_nodes; ++i) {
        const cj_plan_node &n = plan.nodes[i];
        if (n.num_output_attrs && !n.output_attrs) fail(CJ_ERR_INVALID_PLAN, "node without attr array");
        for (uint64_t a = 0; a < n.num_output_attrs; ++a)
            if (n.output_attrs[a].type < CJ_INT32 || n.output_attrs[a].type > CJ_VARCHAR)
                fail(CJ_ERR_INVALID_PLAN, "unknown attribute type");
        if (n.node_type == CJ_NODE_SCAN) {
            if (n.base_table_id >= plan.num_inputs) fail(CJ_ERR_INVALID_PLAN, "scan of missing table");
            for (uint64_t a = 0; a < n.num_output_attrs; ++a) {
                const cj_attr &at = n.output_attrs[a];
                if (at.index >= input_cols(plan, n.base_table_id)) fail(CJ_ERR_INVALID_PLAN, "scan column out of range");
                if (input_col_type(plan, n.base_table_id, at.index) != at.type)
                    fail(CJ_ERR_INVALID_PLAN, "scan attribute type differs from column type");
            }
        } else if (n.node_type == CJ_NODE_HASH_JOIN) {
            if (n.left >= plan.num_nodes || n.right >= plan.num_nodes)
                fail(CJ_ERR_INVALID_PLAN, "join child out of range");
        } else {
            fail(CJ_ERR_INVALID_PLAN, "unknown node type");
        }
    }
}

} // namespace cj
