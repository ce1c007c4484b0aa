/*
 * execute.cpp — drop-in replacement for CalamariJoins' src/execute.cpp.
 *
 * Implements the reference's three entry points (include/data_model/
 * plan.h:380-385) on top of libcj_b200.so: the Plan is flattened into the
 * POD cj_plan_desc (page pointers are passed through, never copied on the
 * host), executed on the GPU, and the result pages are placed in one
 * anonymous mapping owned by a MappedMemory (plan.h:10-44) shared by every
 * result column, so ~Column (plan.h:126-135) unmaps it when the last column
 * is destroyed. Unlike the reference's arena pages (reset by the next
 * execute(), src/execute.cpp:313) the result stays valid as long as the
 * caller keeps it.
 *
 * Build: compile this file instead of src/execute.cpp with
 *   -I<repo>/include  and link  <repo>/calamarijoins_b200/libcj_b200.so
 */
#include <data_model/plan.h>

#include <sys/mman.h>

#include <cstring>
#include <stdexcept>
#include <string>
#include <variant>
#include <vector>

#include "cj_b200.h"

namespace Contest {

namespace {

[[noreturn]] void raise(int status) {
    std::string msg = std::string("cj_b200 status ") + std::to_string(status) + ": " + cj_last_error();
    if (status == CJ_ERR_OUT_OF_MEMORY) throw std::bad_alloc();
    throw std::runtime_error(msg);
}

} // namespace

void *build_context() {
    cj_context *ctx = nullptr;
    int rc = cj_context_create(-1, &ctx);
    if (rc != CJ_OK) raise(rc);
    return ctx;
}

void destroy_context(void *context) { cj_context_destroy(static_cast<cj_context *>(context)); }

ColumnarTable execute(const Plan &plan, void *context, TimingStats *stats_out) {
    cj_context *ctx = static_cast<cj_context *>(context);
    bool own_ctx = false;
    if (!ctx) { /* callers that pass nullptr still get a device context */
        ctx = static_cast<cj_context *>(build_context());
        own_ctx = true;
    }
    struct CtxGuard {
        cj_context *c;
        bool own;
        ~CtxGuard() {
            if (own) cj_context_destroy(c);
        }
    } guard{ctx, own_ctx};

    /* Plan -> cj_plan_desc */
    std::vector<std::vector<cj_attr>> attrs(plan.nodes.size());
    std::vector<cj_plan_node> nodes(plan.nodes.size());
    for (size_t i = 0; i < plan.nodes.size(); ++i) {
        const PlanNode &pn = plan.nodes[i];
        for (auto &[idx, type] : pn.output_attrs) attrs[i].push_back({idx, static_cast<int32_t>(type), 0});
        cj_plan_node &d = nodes[i];
        std::memset(&d, 0, sizeof(d));
        d.num_output_attrs = attrs[i].size();
        d.output_attrs = attrs[i].data();
        if (const auto *scan = std::get_if<ScanNode>(&pn.data)) {
            d.node_type = CJ_NODE_SCAN;
            d.base_table_id = scan->base_table_id;
        } else {
            const auto &j = std::get<JoinNode>(pn.data);
            d.node_type = CJ_NODE_HASH_JOIN;
            d.build_left = j.build_left ? 1 : 0;
            d.left = j.left;
            d.right = j.right;
            d.left_attr = j.left_attr;
            d.right_attr = j.right_attr;
        }
    }
    std::vector<std::vector<cj_column_desc>> cols(plan.inputs.size());
    std::vector<cj_table_desc> tables(plan.inputs.size());
    for (size_t t = 0; t < plan.inputs.size(); ++t) {
        const ColumnarTable &in = plan.inputs[t];
        for (const Column &c : in.columns) {
            cj_column_desc cd;
            cd.type = static_cast<int32_t>(c.type);
            cd.reserved = 0;
            cd.num_pages = c.pages.size();
            cd.pages = reinterpret_cast<const void *const *>(c.pages.data());
            cols[t].push_back(cd);
        }
        tables[t] = {in.num_rows, cols[t].size(), cols[t].data()};
    }
    cj_plan_desc desc;
    desc.num_nodes = nodes.size();
    desc.nodes = nodes.data();
    desc.num_inputs = tables.size();
    desc.inputs = tables.data();
    desc.resident_inputs = nullptr;
    desc.root = plan.root;

    cj_result *res = nullptr;
    cj_timing_stats ts;
    /* The library downloads each result column into its pinned host memory
     * as soon as the column's pages are written (overlapped with the next
     * column's writer); the pages are then copied into the mapping the
     * returned table owns. */
    int rc = cj_execute(ctx, &desc, CJ_EXEC_DEFAULT, &res, &ts, nullptr);
    if (rc != CJ_OK) raise(rc);

    /* Result -> ColumnarTable over one mapping */
    ColumnarTable out;
    uint64_t nrows = 0, ncols = 0;
    cj_result_num_rows(res, &nrows);
    cj_result_num_columns(res, &ncols);
    out.num_rows = nrows;
    std::vector<int32_t> types(ncols);
    std::vector<uint64_t> npages(ncols);
    uint64_t total = 0;
    for (uint64_t c = 0; c < ncols; ++c) {
        cj_result_column(res, c, &types[c], &npages[c], nullptr);
        total += npages[c];
    }
    void *mem = nullptr;
    if (total) {
        mem = mmap(nullptr, total * PAGE_SIZE, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_ANONYMOUS, -1, 0);
        if (mem == MAP_FAILED) {
            cj_result_free(res);
            throw std::bad_alloc();
        }
        madvise(mem, total * PAGE_SIZE, MADV_HUGEPAGE); /* fewer first-touch faults in the copy */
    }
    MappedMemory *mapping = total ? new MappedMemory(mem, total * PAGE_SIZE) : nullptr;
    auto *base = static_cast<std::byte *>(mem);
    for (uint64_t c = 0; c < ncols; ++c) {
        out.columns.emplace_back(static_cast<DataType>(types[c]));
        Column &col = out.columns.back();
        if (!npages[c]) continue;
        rc = cj_result_copy_column(res, c, base, npages[c] * PAGE_SIZE);
        if (rc != CJ_OK) {
            cj_result_free(res);
            raise(rc);
        }
        for (uint64_t p = 0; p < npages[c]; ++p) col.pages.push_back(reinterpret_cast<Page *>(base + p * PAGE_SIZE));
        col.assign_mapped_memory(mapping);
        base += npages[c] * PAGE_SIZE;
    }
    if (mapping && mapping->refs == 0) delete mapping; /* no column took it */
    cj_result_free(res);
    if (stats_out) {
        stats_out->hashtable_build_ms = ts.hashtable_build_ms;
        stats_out->hash_join_probe_ms = ts.hash_join_probe_ms;
        stats_out->nested_loop_join_ms = ts.nested_loop_join_ms;
        stats_out->materialize_ms = ts.materialize_ms;
        stats_out->setup_ms = ts.setup_ms;
        stats_out->total_execution_ms = ts.total_execution_ms;
        stats_out->intermediate_ms = ts.intermediate_ms;
    }
    return out;
}

} // namespace Contest
