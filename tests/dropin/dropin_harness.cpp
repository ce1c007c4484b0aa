/*
 * dropin_harness.cpp — runs one plan through the drop-in execute.cpp using
 * the reference's own Plan / ColumnarTable types (include/data_model/
 * plan.h), so the path a reference caller takes (Contest::build_context,
 * Contest::execute, Contest::destroy_context) is exercised end to end.
 *
 * Input file (little endian):
 *   u64 nodes; per node: i32 kind (0 join, 1 scan), i32 build_left,
 *     u64 table, left, right, left_attr, right_attr, u64 nattrs,
 *     nattrs x (u64 index, i32 type)
 *   u64 inputs; per input: u64 rows, u64 cols; per column: i32 type,
 *     u64 pages, pages x 8192 bytes
 *   u64 root
 * Output file: u64 rows, u64 cols; per column: i32 type, u64 pages, pages.
 * Usage: dropin_harness <in> <out>
 */
#include <data_model/plan.h>

#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <vector>

namespace {

struct Reader {
    FILE *f;
    template <typename T> T get() {
        T v;
        if (std::fread(&v, sizeof(T), 1, f) != 1) throw std::runtime_error("short read");
        return v;
    }
};

template <typename T> void put(FILE *f, T v) { std::fwrite(&v, sizeof(T), 1, f); }

} // namespace

int main(int argc, char **argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s <plan-in> <result-out>\n", argv[0]);
        return 2;
    }
    try {
        FILE *fi = std::fopen(argv[1], "rb");
        if (!fi) throw std::runtime_error("cannot open input");
        Reader r{fi};
        Plan plan;
        uint64_t nn = r.get<uint64_t>();
        for (uint64_t i = 0; i < nn; ++i) {
            int32_t kind = r.get<int32_t>(), bl = r.get<int32_t>();
            uint64_t table = r.get<uint64_t>(), left = r.get<uint64_t>(), right = r.get<uint64_t>();
            uint64_t la = r.get<uint64_t>(), ra = r.get<uint64_t>(), na = r.get<uint64_t>();
            std::vector<std::tuple<size_t, DataType>> attrs;
            for (uint64_t a = 0; a < na; ++a) {
                uint64_t idx = r.get<uint64_t>();
                int32_t t = r.get<int32_t>();
                attrs.emplace_back(idx, static_cast<DataType>(t));
            }
            if (kind == 1)
                plan.new_scan_node(table, std::move(attrs));
            else
                plan.new_join_node(bl != 0, left, right, la, ra, std::move(attrs));
        }
        uint64_t ni = r.get<uint64_t>();
        for (uint64_t t = 0; t < ni; ++t) {
            ColumnarTable table;
            table.num_rows = r.get<uint64_t>();
            uint64_t nc = r.get<uint64_t>();
            for (uint64_t c = 0; c < nc; ++c) {
                int32_t type = r.get<int32_t>();
                uint64_t np = r.get<uint64_t>();
                table.columns.emplace_back(static_cast<DataType>(type));
                for (uint64_t p = 0; p < np; ++p) {
                    Page *pg = table.columns.back().new_page();
                    if (std::fread(pg->data, PAGE_SIZE, 1, fi) != 1) throw std::runtime_error("short page");
                }
            }
            plan.inputs.emplace_back(std::move(table));
        }
        plan.root = r.get<uint64_t>();
        std::fclose(fi);

        void *ctx = Contest::build_context();
        Contest::TimingStats stats;
        ColumnarTable result = Contest::execute(plan, ctx, &stats);
        Contest::destroy_context(ctx);

        FILE *fo = std::fopen(argv[2], "wb");
        if (!fo) throw std::runtime_error("cannot open output");
        put<uint64_t>(fo, result.num_rows);
        put<uint64_t>(fo, result.columns.size());
        for (auto &col : result.columns) {
            put<int32_t>(fo, static_cast<int32_t>(col.type));
            put<uint64_t>(fo, col.pages.size());
            for (auto *pg : col.pages) std::fwrite(pg->data, PAGE_SIZE, 1, fo);
        }
        std::fclose(fo);
        return 0;
    } catch (const std::exception &e) {
        std::fprintf(stderr, "dropin_harness: %s\n", e.what());
        return 1;
    }
}
