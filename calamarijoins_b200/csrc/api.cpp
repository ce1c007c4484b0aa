/*
 * api.cpp — the C ABI (include/cj_b200.h). Every entry point catches
 * internal errors and returns a status code; nothing throws across it.
 */
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>
#include <string>

#include "engine.h"

namespace {

int set_error(int code, const std::string &msg) { return cj::set_last_error(code, msg); }

#define API_BEGIN try {
#define API_END                                                                 \
    }                                                                           \
    catch (const cj::Error &e) {                                                \
        return set_error(e.code, e.msg);                                        \
    }                                                                           \
    catch (const std::bad_alloc &) {                                            \
        return set_error(CJ_ERR_OUT_OF_MEMORY, "host allocation failed");       \
    }                                                                           \
    catch (...) {                                                               \
        return set_error(CJ_ERR_INTERNAL, "unexpected exception");              \
    }                                                                           \
    cj::clear_last_error();                                                       \
    return CJ_OK;

void set_device(const cj::Context *ctx) { cudaSetDevice(ctx->device); }

} // namespace

extern "C" {

const char *cj_last_error(void) { return cj::last_error(); }

const char *cj_version(void) { return "cj_b200 1 sm_100a"; }

int cj_context_create(int device, cj_context **out) {
    if (!out) return set_error(CJ_ERR_INVALID_ARGUMENT, "out is null");
    *out = nullptr;
    API_BEGIN
    *out = static_cast<cj_context *>(cj::create_context(device, nullptr));
    API_END
}

void cj_context_destroy(cj_context *ctx) {
    if (!ctx) return;
    set_device(ctx);
    delete ctx;
}

int cj_context_set_option(cj_context *ctx, int32_t option, int64_t value) {
    if (!ctx) return set_error(CJ_ERR_INVALID_ARGUMENT, "ctx is null");
    switch (option) {
    case CJ_OPT_NESTED_LOOP_MAX_BUILD: ctx->opt.nested_loop_max_build = value; break;
    case CJ_OPT_SLOTS_PER_PARTITION:
        if (value < 0 || (value & (value - 1))) return set_error(CJ_ERR_INVALID_ARGUMENT, "not a power of two");
        ctx->opt.slots_per_partition = value;
        break;
    case CJ_OPT_PROFILE_KERNELS: ctx->opt.profile_kernels = value; break;
    case CJ_OPT_BLOCK_THREADS: ctx->opt.block_threads = value; break;
    case CJ_OPT_VARCHAR_TILE_ROWS:
        if (value < 64 || value > 8192) return set_error(CJ_ERR_INVALID_ARGUMENT, "tile rows in [64, 8192]");
        ctx->opt.varchar_tile_rows = value;
        break;
    case CJ_OPT_CTAS_PER_SM: ctx->opt.ctas_per_sm = value; break;
    case CJ_OPT_DENSE_KEYS:
        if (value < 0 || value > 64) return set_error(CJ_ERR_INVALID_ARGUMENT, "dense key factor in [0, 64]");
        ctx->opt.dense_keys = value;
        break;
    case CJ_OPT_BUFFER_CACHE_BYTES:
        if (value < 0) return set_error(CJ_ERR_INVALID_ARGUMENT, "cache bytes must be >= 0");
        if (ctx->pool && !ctx->owns_pool && value) return set_error(CJ_ERR_INVALID_ARGUMENT, "server workers keep no cache");
        ctx->opt.buffer_cache_bytes = value;
        set_device(ctx);
        ctx->trim_buffers();
        break;
    case CJ_OPT_FAIL_ALLOC_AT:
        if (value < 0) return set_error(CJ_ERR_INVALID_ARGUMENT, "allocation index must be >= 0");
        ctx->opt.fail_alloc_at = value;
        break;
    default: return set_error(CJ_ERR_INVALID_ARGUMENT, "unknown option");
    }
    return CJ_OK;
}

int cj_context_get_option(const cj_context *ctx, int32_t option, int64_t *value) {
    if (!ctx || !value) return set_error(CJ_ERR_INVALID_ARGUMENT, "null argument");
    switch (option) {
    case CJ_OPT_NESTED_LOOP_MAX_BUILD: *value = ctx->opt.nested_loop_max_build; break;
    case CJ_OPT_SLOTS_PER_PARTITION: *value = ctx->opt.slots_per_partition; break;
    case CJ_OPT_PROFILE_KERNELS: *value = ctx->opt.profile_kernels; break;
    case CJ_OPT_BLOCK_THREADS: *value = ctx->opt.block_threads; break;
    case CJ_OPT_VARCHAR_TILE_ROWS: *value = ctx->opt.varchar_tile_rows; break;
    case CJ_OPT_CTAS_PER_SM: *value = ctx->opt.ctas_per_sm; break;
    case CJ_OPT_DENSE_KEYS: *value = ctx->opt.dense_keys; break;
    case CJ_OPT_BUFFER_CACHE_BYTES: *value = ctx->opt.buffer_cache_bytes; break;
    case CJ_OPT_FAIL_ALLOC_AT: *value = ctx->opt.fail_alloc_at; break;
    default: return set_error(CJ_ERR_INVALID_ARGUMENT, "unknown option");
    }
    return CJ_OK;
}

int cj_profile_reset(cj_context *ctx) {
    if (!ctx) return set_error(CJ_ERR_INVALID_ARGUMENT, "ctx is null");
    set_device(ctx);
    cudaStreamSynchronize(ctx->stream);
    ctx->resolve_profile();
    ctx->profile.clear();
    ctx->profile_index.clear();
    return CJ_OK;
}

int cj_profile_count(const cj_context *ctx, uint64_t *n) {
    if (!ctx || !n) return set_error(CJ_ERR_INVALID_ARGUMENT, "null argument");
    *n = ctx->profile.size();
    return CJ_OK;
}

int cj_profile_entry(const cj_context *ctx, uint64_t index, const char **name, uint64_t *launches,
                     double *total_us) {
    if (!ctx || index >= ctx->profile.size()) return set_error(CJ_ERR_INVALID_ARGUMENT, "bad index");
    const auto &p = ctx->profile[index];
    if (name) *name = p.name.c_str();
    if (launches) *launches = p.launches;
    if (total_us) *total_us = p.total_us;
    return CJ_OK;
}

int cj_context_stream(const cj_context *ctx, void **stream) {
    if (!ctx || !stream) return set_error(CJ_ERR_INVALID_ARGUMENT, "null argument");
    *stream = ctx->stream;
    return CJ_OK;
}

int cj_context_memory(const cj_context *ctx, uint64_t *used, uint64_t *reserved) {
    if (!ctx) return set_error(CJ_ERR_INVALID_ARGUMENT, "ctx is null");
    API_BEGIN
    set_device(ctx);
    cj::check_cuda(cudaStreamSynchronize(ctx->stream), "sync");
    uint64_t u = 0, r = 0;
    cj::check_cuda(cudaMemPoolGetAttribute(ctx->pool, cudaMemPoolAttrUsedMemCurrent, &u), "pool attr");
    cj::check_cuda(cudaMemPoolGetAttribute(ctx->pool, cudaMemPoolAttrReservedMemCurrent, &r), "pool attr");
    if (used) *used = u;
    if (reserved) *reserved = r;
    API_END
}

/* ------------------------------------------------------------------ */
int cj_table_upload(cj_context *ctx, const cj_table_desc *table, cj_table **out) {
    if (!ctx || !table || !out) return set_error(CJ_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    API_BEGIN
    set_device(ctx);
    auto t = std::make_unique<cj_table>();
    t->ctx = ctx;
    t->num_rows = table->num_rows;
    if (table->num_columns && !table->columns) cj::fail(CJ_ERR_INVALID_ARGUMENT, "no column array");
    for (uint64_t c = 0; c < table->num_columns; ++c) {
        const cj_column_desc &cd = table->columns[c];
        if (cd.type < CJ_INT32 || cd.type > CJ_VARCHAR) cj::fail(CJ_ERR_INVALID_ARGUMENT, "unknown column type");
        cj::ColumnPages cp;
        cj::upload_pages(*ctx, cd, cp, nullptr);
        t->cols.push_back(cp);
    }
    cj::check_cuda(cudaStreamSynchronize(ctx->stream), "upload");
    *out = t.release();
    API_END
}

int cj_table_from_device(cj_context *ctx, uint64_t num_rows, uint64_t num_columns, const int32_t *types,
                         const uint64_t *num_pages, const void *const *device_pages, cj_table **out) {
    if (!ctx || !out || (num_columns && (!types || !num_pages || !device_pages)))
        return set_error(CJ_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    API_BEGIN
    auto t = std::make_unique<cj_table>();
    t->ctx = ctx;
    t->num_rows = num_rows;
    for (uint64_t c = 0; c < num_columns; ++c) {
        if (types[c] < CJ_INT32 || types[c] > CJ_VARCHAR) cj::fail(CJ_ERR_INVALID_ARGUMENT, "unknown column type");
        cj::ColumnPages cp;
        cp.type = types[c];
        cp.num_pages = num_pages[c];
        cp.dev = static_cast<const uint8_t *>(device_pages[c]);
        if (cp.num_pages && !cp.dev) cj::fail(CJ_ERR_INVALID_ARGUMENT, "null device pages");
        t->cols.push_back(cp);
    }
    *out = t.release();
    API_END
}

int cj_table_column_pages(const cj_table *table, uint64_t column, const void **device_pages,
                          uint64_t *num_pages) {
    if (!table || column >= table->cols.size()) return set_error(CJ_ERR_INVALID_ARGUMENT, "bad column");
    if (device_pages) *device_pages = table->cols[column].dev;
    if (num_pages) *num_pages = table->cols[column].num_pages;
    return CJ_OK;
}

int cj_table_copy_column(const cj_table *table, uint64_t column, void *dst, uint64_t dst_bytes) {
    if (!table || column >= table->cols.size()) return set_error(CJ_ERR_INVALID_ARGUMENT, "bad column");
    const uint64_t bytes = table->cols[column].num_pages * CJ_PAGE_SIZE;
    if (bytes && !dst) return set_error(CJ_ERR_INVALID_ARGUMENT, "null destination");
    if (dst_bytes < bytes) return set_error(CJ_ERR_INVALID_ARGUMENT, "destination too small");
    if (!bytes) return CJ_OK;
    API_BEGIN
    set_device(table->ctx);
    cj::check_cuda(cudaMemcpyAsync(dst, table->cols[column].dev, bytes, cudaMemcpyDeviceToHost, table->ctx->stream),
                   "download");
    cj::check_cuda(cudaStreamSynchronize(table->ctx->stream), "download");
    API_END
}

void cj_table_free(cj_table *table) {
    if (!table) return;
    set_device(table->ctx);
    delete table;
}

/* ------------------------------------------------------------------ */
int cj_execute(cj_context *ctx, const cj_plan_desc *plan, uint32_t flags, cj_result **out,
               cj_timing_stats *timing, cj_exec_stats *stats) {
    if (!ctx || !plan || !out) return set_error(CJ_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    set_device(ctx);
    try {
        cj_exec_stats st{};
        cj_result *r = cj::execute_plan(*ctx, *plan, flags, &st);
        *out = r;
        if (stats) *stats = st;
        if (timing) {
            /* TimingStats fields are whole milliseconds (plan.h:370-378) */
            timing->hashtable_build_ms = (int64_t)(st.build_us / 1000.0);
            timing->hash_join_probe_ms = (int64_t)(st.probe_us / 1000.0);
            timing->nested_loop_join_ms = (int64_t)(st.nested_loop_us / 1000.0);
            timing->materialize_ms = (int64_t)((st.materialize_us + st.download_us) / 1000.0);
            timing->setup_ms = (int64_t)((st.upload_us + st.decode_us) / 1000.0);
            timing->total_execution_ms = (int64_t)(st.total_us / 1000.0);
            timing->intermediate_ms = (int64_t)(st.intermediate_us / 1000.0);
        }
    } catch (const cj::Error &e) {
        cudaStreamSynchronize(ctx->stream);
        cudaGetLastError();
        return set_error(e.code, e.msg);
    } catch (const std::bad_alloc &) {
        cudaStreamSynchronize(ctx->stream);
        return set_error(CJ_ERR_OUT_OF_MEMORY, "host allocation failed");
    } catch (...) {
        cudaStreamSynchronize(ctx->stream);
        return set_error(CJ_ERR_INTERNAL, "unexpected exception");
    }
    cj::clear_last_error();
    return CJ_OK;
}

int cj_execute_batch(cj_context *ctx, const cj_plan_desc *plans, uint64_t n, uint32_t flags, cj_result **results,
                     int32_t *statuses, cj_batch_stats *stats) {
    if (!ctx || (n && (!plans || !results))) return set_error(CJ_ERR_INVALID_ARGUMENT, "null argument");
    set_device(ctx);
    try {
        cj::execute_batch(*ctx, plans, (size_t)n, flags, results, statuses, stats);
    } catch (const cj::Error &e) {
        cudaStreamSynchronize(ctx->stream);
        cudaGetLastError();
        return set_error(e.code, e.msg);
    } catch (const std::bad_alloc &) {
        cudaStreamSynchronize(ctx->stream);
        return set_error(CJ_ERR_OUT_OF_MEMORY, "host allocation failed");
    } catch (...) {
        cudaStreamSynchronize(ctx->stream);
        return set_error(CJ_ERR_INTERNAL, "unexpected exception");
    }
    cj::clear_last_error();
    return CJ_OK;
}

int cj_result_num_rows(const cj_result *r, uint64_t *n) {
    if (!r || !n) return set_error(CJ_ERR_INVALID_ARGUMENT, "null argument");
    *n = r->num_rows;
    return CJ_OK;
}

int cj_result_num_columns(const cj_result *r, uint64_t *n) {
    if (!r || !n) return set_error(CJ_ERR_INVALID_ARGUMENT, "null argument");
    *n = r->types.size();
    return CJ_OK;
}

int cj_result_column(const cj_result *r, uint64_t c, int32_t *type, uint64_t *num_pages, const void **host_pages) {
    if (!r || c >= r->types.size()) return set_error(CJ_ERR_INVALID_ARGUMENT, "bad column");
    if (type) *type = r->types[c];
    if (num_pages) *num_pages = r->num_pages[c];
    if (host_pages) *host_pages = r->host_cols.empty() ? nullptr : r->host_cols[c];
    return CJ_OK;
}

int cj_result_column_device(const cj_result *r, uint64_t c, const void **device_pages) {
    if (!r || c >= r->types.size() || !device_pages) return set_error(CJ_ERR_INVALID_ARGUMENT, "bad column");
    *device_pages = r->dev_pages[c] ? r->dev_pages[c]->ptr : nullptr;
    return CJ_OK;
}

/* Host-to-host copy split over up to 8 threads for large blocks (one core
 * copies, and first-touches fresh destination pages, at a fraction of the
 * host's memory bandwidth). */
static void parallel_copy(void *dst, const void *src, uint64_t bytes) {
    const uint64_t kMinPerThread = 32ull << 20;
    unsigned nt = (unsigned)std::min<uint64_t>(8, bytes / kMinPerThread);
    if (nt < 2) {
        std::memcpy(dst, src, bytes);
        return;
    }
    const uint64_t per = (bytes / nt + 4095) & ~uint64_t(4095);
    std::vector<std::thread> ts;
    for (unsigned t = 0; t < nt; ++t) {
        const uint64_t b = t * per;
        if (b >= bytes) break;
        const uint64_t n = std::min(per, bytes - b);
        ts.emplace_back([=] { std::memcpy(static_cast<uint8_t *>(dst) + b, static_cast<const uint8_t *>(src) + b, n); });
    }
    for (auto &t : ts) t.join();
}

int cj_result_copy_column(const cj_result *r, uint64_t c, void *dst, uint64_t dst_bytes) {
    if (!r || c >= r->types.size() || (!dst && r->num_pages[c]))
        return set_error(CJ_ERR_INVALID_ARGUMENT, "bad argument");
    const uint64_t bytes = r->num_pages[c] * CJ_PAGE_SIZE;
    if (dst_bytes < bytes) return set_error(CJ_ERR_INVALID_ARGUMENT, "destination too small");
    if (!bytes) return CJ_OK;
    API_BEGIN
    set_device(r->ctx);
    if (!r->host_cols.empty() && r->host_cols[c]) {
        parallel_copy(dst, r->host_cols[c], bytes);
    } else {
        cj::check_cuda(cudaMemcpyAsync(dst, r->dev_pages[c]->ptr, bytes, cudaMemcpyDeviceToHost, r->ctx->stream),
                       "download");
        cj::check_cuda(cudaStreamSynchronize(r->ctx->stream), "download");
    }
    API_END
}

void cj_result_free(cj_result *r) {
    if (!r) return;
    set_device(r->ctx);
    delete r;
}

int cj_host_alloc(uint64_t bytes, void **out) {
    if (!out) return set_error(CJ_ERR_INVALID_ARGUMENT, "out is null");
    *out = nullptr;
    cudaError_t e = cudaHostAlloc(out, bytes ? bytes : 1, cudaHostAllocPortable);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *out = nullptr;
        return set_error(e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver ? CJ_ERR_NO_DEVICE
                                                                                      : CJ_ERR_OUT_OF_MEMORY,
                         cudaGetErrorString(e));
    }
    return CJ_OK;
}

void cj_host_free(void *p) {
    if (p) cudaFreeHost(p);
}

} /* extern "C" */
