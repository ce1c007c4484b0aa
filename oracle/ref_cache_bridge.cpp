/* Bridge to the reference's own `.tbl` cache code (TEST INFRASTRUCTURE):
 * Table::from_cache (src/build_table.cpp:140-197) reads a cache file and
 * DumpTable::dump (include/data_access/table.h:136-221) writes one, so that
 * the library's reader and writer (cj_table_load_cache, cj_cache_read_meta,
 * cj_table_write_cache) are checked against the reference's, not against a
 * restatement. Built by oracle/build_oracle.py. */
#include <cstring>
#include <fstream>

#include <data_access/table.h>
#include <data_model/plan.h>

#include "../include/cj_b200.h"

struct cjref_cache {
    ColumnarTable table;
};

extern "C" {

/* Table::from_cache on `path`; the table stays mapped until cjref_cache_free. */
int cjref_cache_read(const char *path, cjref_cache **out) {
    try {
        auto *c = new cjref_cache{Table::from_cache(path)};
        *out = c;
        return 0;
    } catch (...) {
        return 1;
    }
}
uint64_t cjref_cache_num_rows(const cjref_cache *c) { return c->table.num_rows; }
uint64_t cjref_cache_num_columns(const cjref_cache *c) { return c->table.columns.size(); }
/* Column c: its type, page count and page pointers (num_pages of them). */
int cjref_cache_column(const cjref_cache *c, uint64_t col, int32_t *type, uint64_t *num_pages,
                       const void **pages, uint64_t capacity) {
    if (col >= c->table.columns.size()) return 1;
    const Column &cl = c->table.columns[col];
    *type = (int32_t)cl.type;
    *num_pages = cl.pages.size();
    for (uint64_t p = 0; p < cl.pages.size() && p < capacity; ++p) pages[p] = cl.pages[p];
    return 0;
}
void cjref_cache_free(cjref_cache *c) { delete c; }

/* DumpTable::dump of host pages into `path`. */
int cjref_cache_write(const cj_table_desc *t, const char *path) {
    try {
        ColumnarTable table;
        table.num_rows = t->num_rows;
        for (uint64_t c = 0; c < t->num_columns; ++c) {
            table.columns.emplace_back((DataType)t->columns[c].type);
            for (uint64_t p = 0; p < t->columns[c].num_pages; ++p)
                table.columns.back().pages.push_back((Page *)t->columns[c].pages[p]);
        }
        std::ofstream out(path, std::ios::binary);
        DumpTable(&table).dump(out);
        out.close();
        for (auto &c : table.columns) c.pages.clear(); /* the pages are the caller's */
        return out.good() ? 0 : 1;
    } catch (...) {
        return 1;
    }
}

} // extern "C"
