/*
 * ref_bridge.cpp — C entry points over the reference's own
 * Contest::execute() (CalamariJoins src/execute.cpp), compiled from the
 * reference's sources by oracle/build_oracle.py into oracle/_ref/.
 *
 * TEST INFRASTRUCTURE ONLY: it lets tests pin the oracle against the real
 * reference, and lets bench.py time the reference on the host cores. It
 * builds a reference `Plan` (include/data_model/plan.h:149-185) from the
 * same POD plan description the product takes, runs the reference, and
 * copies the result pages out before the reference's arena is reset by its
 * next call (src/execute.cpp:313).
 */
#include <data_model/plan.h>

#include <chrono>
#include <cstring>
#include <exception>
#include <new>
#include <vector>

#include "../include/cj_b200.h"

namespace Contest {
/* Defined in the reference's src/execute.cpp. */
void *build_context();
void destroy_context(void *);
ColumnarTable execute(const Plan &plan, void *context, TimingStats *stats_out);
} // namespace Contest

namespace {

/* Input pages belong to the caller: a MappedMemory whose reference count
 * never reaches zero keeps ~Column (plan.h:126-135) from deleting them. */
MappedMemory *borrowed_pages() {
    static MappedMemory *m = [] {
        auto *p = new MappedMemory(nullptr, 0);
        p->refs = 1ull << 40;
        return p;
    }();
    return m;
}

DataType to_dt(int32_t t) { return static_cast<DataType>(t); }

} // namespace

struct cjref_result {
    uint64_t num_rows = 0;
    std::vector<int32_t> types;
    std::vector<std::vector<unsigned char>> pages; /* consecutive pages */
};

extern "C" {

int cjref_thread_count(void) { return SPC__THREAD_COUNT; }

int cjref_execute(const cj_plan_desc *d, cjref_result **out,
                  cj_timing_stats *timing, double *wall_ms) {
    if (!d || !out) return CJ_ERR_INVALID_ARGUMENT;
    try {
        Plan plan;
        for (uint64_t i = 0; i < d->num_nodes; ++i) {
            const cj_plan_node &n = d->nodes[i];
            std::vector<std::tuple<size_t, DataType>> attrs;
            for (uint64_t a = 0; a < n.num_output_attrs; ++a)
                attrs.emplace_back(n.output_attrs[a].index,
                                   to_dt(n.output_attrs[a].type));
            if (n.node_type == CJ_NODE_SCAN)
                plan.new_scan_node(n.base_table_id, std::move(attrs));
            else
                plan.new_join_node(n.build_left != 0, n.left, n.right,
                                   n.left_attr, n.right_attr,
                                   std::move(attrs));
        }
        for (uint64_t t = 0; t < d->num_inputs; ++t) {
            const cj_table_desc &td = d->inputs[t];
            ColumnarTable table;
            table.num_rows = td.num_rows;
            for (uint64_t c = 0; c < td.num_columns; ++c) {
                const cj_column_desc &cd = td.columns[c];
                table.columns.emplace_back(to_dt(cd.type));
                Column &col = table.columns.back();
                for (uint64_t p = 0; p < cd.num_pages; ++p)
                    col.pages.push_back(reinterpret_cast<Page *>(
                        const_cast<void *>(cd.pages[p])));
                col.assign_mapped_memory(borrowed_pages());
            }
            plan.inputs.emplace_back(std::move(table));
        }
        plan.root = d->root;

        Contest::TimingStats stats;
        void *ctx = Contest::build_context();
        auto t0 = std::chrono::steady_clock::now();
        ColumnarTable res = Contest::execute(plan, ctx, &stats);
        auto t1 = std::chrono::steady_clock::now();
        Contest::destroy_context(ctx);

        auto *r = new cjref_result;
        r->num_rows = res.num_rows;
        for (auto &col : res.columns) {
            r->types.push_back(static_cast<int32_t>(col.type));
            std::vector<unsigned char> buf(col.pages.size() * PAGE_SIZE);
            for (size_t p = 0; p < col.pages.size(); ++p)
                std::memcpy(buf.data() + p * PAGE_SIZE, col.pages[p]->data,
                            PAGE_SIZE);
            r->pages.push_back(std::move(buf));
        }
        if (timing) {
            timing->hashtable_build_ms = stats.hashtable_build_ms;
            timing->hash_join_probe_ms = stats.hash_join_probe_ms;
            timing->nested_loop_join_ms = stats.nested_loop_join_ms;
            timing->materialize_ms = stats.materialize_ms;
            timing->setup_ms = stats.setup_ms;
            timing->total_execution_ms = stats.total_execution_ms;
            timing->intermediate_ms = stats.intermediate_ms;
        }
        if (wall_ms)
            *wall_ms =
                std::chrono::duration<double, std::milli>(t1 - t0).count();
        *out = r;
        return CJ_OK;
    } catch (const std::bad_alloc &) {
        return CJ_ERR_OUT_OF_MEMORY;
    } catch (...) {
        return CJ_ERR_INTERNAL;
    }
}

uint64_t cjref_result_num_rows(const cjref_result *r) { return r ? r->num_rows : 0; }
uint64_t cjref_result_num_columns(const cjref_result *r) { return r ? r->types.size() : 0; }

int cjref_result_column(const cjref_result *r, uint64_t c, int32_t *type,
                        uint64_t *num_pages, const void **pages) {
    if (!r || c >= r->types.size()) return CJ_ERR_INVALID_ARGUMENT;
    if (type) *type = r->types[c];
    if (num_pages) *num_pages = r->pages[c].size() / PAGE_SIZE;
    if (pages) *pages = r->pages[c].data();
    return CJ_OK;
}

void cjref_result_free(cjref_result *r) { delete r; }

} /* extern "C" */
