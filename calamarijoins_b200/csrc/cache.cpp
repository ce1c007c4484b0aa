/*
 * cache.cpp — the reference's `.tbl` table cache and a catalog of resident
 * tables.
 *
 * File format (the reference writes it with DumpTable::dump,
 * include/data_access/table.h:136-221, and maps it with Table::from_cache,
 * src/build_table.cpp:140-197): one 8 KiB header page holding TableMeta
 * (table.h:30-35: u64 num_rows, u64 num_cols, 16 x 4-byte DataType, 16 x
 * u64 page counts; 208 bytes) followed by zeros, then the pages of column 0,
 * of column 1, ... back to back. At most 16 columns.
 *
 * cj_table_load_cache reads such a file straight into a resident table (the
 * pages go to HBM once and plans then name the table instead of shipping its
 * pages); cj_table_write_cache writes one from host pages; a catalog keeps
 * resident tables by name, so a driver can load a directory of caches once
 * and build every plan's inputs from it.
 */
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "engine.h"

namespace {

constexpr uint64_t kMaxCacheColumns = 16;

/* TableMeta of the reference (include/data_access/table.h:30-35). */
struct FileMeta {
    uint64_t num_rows;
    uint64_t num_cols;
    int32_t types[kMaxCacheColumns];
    uint64_t num_pages[kMaxCacheColumns];
};
static_assert(sizeof(FileMeta) == 208, "TableMeta is 208 bytes");

int api_error(int code, const std::string &msg) { return cj::set_last_error(code, msg); }

/* Checks a header against the file size; fills `m`. */
int check_meta(const FileMeta &m, uint64_t file_bytes, const std::string &path) {
    if (m.num_cols > kMaxCacheColumns)
        return api_error(CJ_ERR_MALFORMED_PAGE, path + ": header names " + std::to_string(m.num_cols) +
                                                    " columns (at most 16)");
    uint64_t pages = 0;
    for (uint64_t c = 0; c < m.num_cols; ++c) {
        if (m.types[c] < CJ_INT32 || m.types[c] > CJ_VARCHAR)
            return api_error(CJ_ERR_MALFORMED_PAGE, path + ": unknown type in column " + std::to_string(c));
        if (m.num_pages[c] > file_bytes / cj::kPageSize)
            return api_error(CJ_ERR_MALFORMED_PAGE, path + ": page count beyond the file");
        pages += m.num_pages[c];
    }
    if (file_bytes != (pages + 1) * cj::kPageSize)
        return api_error(CJ_ERR_MALFORMED_PAGE, path + ": " + std::to_string(file_bytes) + " bytes, the header calls for " +
                                                    std::to_string((pages + 1) * cj::kPageSize));
    return CJ_OK;
}

/* A read-only mapping of a whole file. */
struct Mapping {
    void *addr = MAP_FAILED;
    size_t bytes = 0;
    ~Mapping() {
        if (addr != MAP_FAILED) munmap(addr, bytes);
    }
};

int map_file(const char *path, Mapping &map) {
    const int fd = open(path, O_RDONLY);
    if (fd < 0) return api_error(CJ_ERR_INVALID_ARGUMENT, std::string("cannot open ") + path);
    struct stat sb;
    if (fstat(fd, &sb) != 0 || sb.st_size < (off_t)cj::kPageSize) {
        close(fd);
        return api_error(CJ_ERR_MALFORMED_PAGE, std::string(path) + ": shorter than one header page");
    }
    map.bytes = (size_t)sb.st_size;
    map.addr = mmap(nullptr, map.bytes, PROT_READ, MAP_PRIVATE, fd, 0);
    close(fd);
    if (map.addr == MAP_FAILED) return api_error(CJ_ERR_INVALID_ARGUMENT, std::string("cannot map ") + path);
    return CJ_OK;
}

} // namespace

struct cj_catalog {
    cj_context *ctx = nullptr;
    std::map<std::string, cj_table *> tables;
    std::vector<std::string> order;
};

extern "C" {

int cj_cache_read_meta(const char *path, cj_cache_meta *meta) {
    if (!path || !meta) return api_error(CJ_ERR_INVALID_ARGUMENT, "null argument");
    Mapping map;
    int rc = map_file(path, map);
    if (rc != CJ_OK) return rc;
    FileMeta m;
    std::memcpy(&m, map.addr, sizeof(m));
    rc = check_meta(m, map.bytes, path);
    if (rc != CJ_OK) return rc;
    meta->num_rows = m.num_rows;
    meta->num_columns = m.num_cols;
    for (uint64_t c = 0; c < kMaxCacheColumns; ++c) {
        meta->types[c] = c < m.num_cols ? m.types[c] : 0;
        meta->num_pages[c] = c < m.num_cols ? m.num_pages[c] : 0;
    }
    cj::clear_last_error();
    return CJ_OK;
}

int cj_table_write_cache(const cj_table_desc *table, const char *path) {
    if (!table || !path || (table->num_columns && !table->columns))
        return api_error(CJ_ERR_INVALID_ARGUMENT, "null argument");
    if (table->num_columns > kMaxCacheColumns)
        return api_error(CJ_ERR_LIMIT, "a cache file holds at most 16 columns");
    FileMeta m;
    std::memset(&m, 0, sizeof(m));
    m.num_rows = table->num_rows;
    m.num_cols = table->num_columns;
    for (uint64_t c = 0; c < table->num_columns; ++c) {
        const cj_column_desc &cd = table->columns[c];
        if (cd.type < CJ_INT32 || cd.type > CJ_VARCHAR) return api_error(CJ_ERR_INVALID_ARGUMENT, "unknown column type");
        if (cd.num_pages && !cd.pages) return api_error(CJ_ERR_INVALID_ARGUMENT, "column without page array");
        m.types[c] = cd.type;
        m.num_pages[c] = cd.num_pages;
    }
    FILE *f = std::fopen(path, "wb");
    if (!f) return api_error(CJ_ERR_INVALID_ARGUMENT, std::string("cannot create ") + path);
    std::vector<unsigned char> header(cj::kPageSize, 0);
    std::memcpy(header.data(), &m, sizeof(m));
    bool ok = std::fwrite(header.data(), 1, header.size(), f) == header.size();
    for (uint64_t c = 0; ok && c < table->num_columns; ++c)
        for (uint64_t p = 0; ok && p < table->columns[c].num_pages; ++p) {
            const void *pg = table->columns[c].pages[p];
            ok = pg && std::fwrite(pg, 1, cj::kPageSize, f) == cj::kPageSize;
        }
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) return api_error(CJ_ERR_INVALID_ARGUMENT, std::string("writing ") + path + " failed");
    cj::clear_last_error();
    return CJ_OK;
}

int cj_table_load_cache(cj_context *ctx, const char *path, cj_table **out) {
    if (!ctx || !path || !out) return api_error(CJ_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    Mapping map;
    int rc = map_file(path, map);
    if (rc != CJ_OK) return rc;
    FileMeta m;
    std::memcpy(&m, map.addr, sizeof(m));
    rc = check_meta(m, map.bytes, path);
    if (rc != CJ_OK) return rc;
    /* the mapped pages, described as a host table, go through the same
     * upload as cj_table_upload */
    const uint8_t *data = static_cast<const uint8_t *>(map.addr) + cj::kPageSize;
    std::vector<std::vector<const void *>> ptrs(m.num_cols);
    std::vector<cj_column_desc> cols(m.num_cols);
    for (uint64_t c = 0; c < m.num_cols; ++c) {
        ptrs[c].resize(m.num_pages[c]);
        for (uint64_t p = 0; p < m.num_pages[c]; ++p, data += cj::kPageSize) ptrs[c][p] = data;
        cols[c].type = m.types[c];
        cols[c].reserved = 0;
        cols[c].num_pages = m.num_pages[c];
        cols[c].pages = ptrs[c].empty() ? nullptr : ptrs[c].data();
    }
    cj_table_desc desc;
    desc.num_rows = m.num_rows;
    desc.num_columns = m.num_cols;
    desc.columns = cols.empty() ? nullptr : cols.data();
    return cj_table_upload(ctx, &desc, out); /* synchronises before the mapping goes */
}

int cj_catalog_create(cj_context *ctx, cj_catalog **out) {
    if (!ctx || !out) return api_error(CJ_ERR_INVALID_ARGUMENT, "null argument");
    *out = new cj_catalog;
    (*out)->ctx = ctx;
    cj::clear_last_error();
    return CJ_OK;
}

void cj_catalog_destroy(cj_catalog *cat) {
    if (!cat) return;
    for (auto &kv : cat->tables) cj_table_free(kv.second);
    delete cat;
}

int cj_catalog_add(cj_catalog *cat, const char *name, cj_table *table) {
    if (!cat || !name || !table) return api_error(CJ_ERR_INVALID_ARGUMENT, "null argument");
    if (cat->tables.count(name)) return api_error(CJ_ERR_INVALID_ARGUMENT, std::string("table ") + name + " exists");
    cat->tables[name] = table;
    cat->order.push_back(name);
    cj::clear_last_error();
    return CJ_OK;
}

int cj_catalog_load(cj_catalog *cat, const char *name, const char *path) {
    if (!cat || !name || !path) return api_error(CJ_ERR_INVALID_ARGUMENT, "null argument");
    if (cat->tables.count(name)) return api_error(CJ_ERR_INVALID_ARGUMENT, std::string("table ") + name + " exists");
    cj_table *t = nullptr;
    const int rc = cj_table_load_cache(cat->ctx, path, &t);
    if (rc != CJ_OK) return rc;
    return cj_catalog_add(cat, name, t);
}

int cj_catalog_get(const cj_catalog *cat, const char *name, cj_table **table) {
    if (!cat || !name || !table) return api_error(CJ_ERR_INVALID_ARGUMENT, "null argument");
    auto it = cat->tables.find(name);
    if (it == cat->tables.end()) return api_error(CJ_ERR_INVALID_ARGUMENT, std::string("no table ") + name);
    *table = it->second;
    cj::clear_last_error();
    return CJ_OK;
}

int cj_catalog_size(const cj_catalog *cat, uint64_t *count) {
    if (!cat || !count) return api_error(CJ_ERR_INVALID_ARGUMENT, "null argument");
    *count = cat->order.size();
    return CJ_OK;
}

int cj_catalog_name(const cj_catalog *cat, uint64_t index, const char **name) {
    if (!cat || !name || index >= cat->order.size()) return api_error(CJ_ERR_INVALID_ARGUMENT, "bad index");
    *name = cat->order[index].c_str();
    return CJ_OK;
}

} /* extern "C" */
