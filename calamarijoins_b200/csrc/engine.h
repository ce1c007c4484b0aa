/*
 * engine.h — host side of the library: the context (device, streams,
 * stream-ordered memory pool, pinned staging, per-kernel profiler), device
 * buffers, resident tables and results.
 *
 * The reference's context is a process-wide mmap arena reset on every
 * execute() plus a persistent thread pool (include/platform/arena.h:88-372,
 * worker_pool.h:44-149). Here the context owns a CUDA memory pool from
 * which every per-plan buffer is taken and returned in stream order, so
 * memory is recycled between plans without device synchronisation.
 */
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "cj_internal.h"

namespace cj {

/* Internal error: thrown inside the library, turned into a status code at
 * the C ABI. */
struct Error {
    int code;
    std::string msg;
};
[[noreturn]] void fail(int code, const std::string &msg);
/* Records the calling thread's last error (cj_last_error) and returns code. */
int set_last_error(int code, const std::string &msg);
void clear_last_error();
const char *last_error();
void check_cuda(cudaError_t e, const char *what);

struct Options {
    int64_t nested_loop_max_build = 64;
    int64_t slots_per_partition = 0; /* 0 = auto (2048) */
    int64_t profile_kernels = 0;
    int64_t block_threads = 0;
    int64_t varchar_tile_rows = 2048;
    int64_t ctas_per_sm = 0;
    int64_t dense_keys = 8; /* max key span / build rows for a direct-mapped table; 0 = off */
    int64_t buffer_cache_bytes = 16ll << 30; /* freed device buffers kept for reuse */
    int64_t fail_alloc_at = 0; /* injected failure of the N-th device allocation from now; 0 = off */
    /* INT32-key hash tables whose directory (16-byte entries) and tuples
     * together stay within this many bytes keep each slot's first tuple in
     * its entry; larger ones use 8-byte entries, so that more of the table
     * stays in L2 (environment CJ_INLINE_DIR_MAX_BYTES) */
    int64_t inline_dir_max_bytes = 256ll << 20;
    /* a root over unique build keys with its result left in HBM writes the
     * result with the match count read on the device, without a host
     * synchronisation after the probe (environment CJ_DEFER_COUNT=0: off) */
    int64_t defer_count = 1;
};

struct Context;

/* A device allocation of the context, ordered on its kernel stream. */
struct DevBuf {
    Context *ctx = nullptr;
    void *ptr = nullptr;
    size_t bytes = 0;
    size_t cls = 0;     /* bytes actually held (size class) */
    bool arena = false; /* carved from the context's arena: not freed alone */
    ~DevBuf();
    template <typename T> T *as() const { return reinterpret_cast<T *>(ptr); }
};
using DevPtr = std::shared_ptr<DevBuf>;

/* Cache of page-locked host blocks by size class (cudaHostAlloc is slow:
 * freed blocks are kept for reuse). A context has its own; the worker
 * contexts of a server share one, so that no worker pays for allocating
 * blocks another has already made. */
struct PinnedPool {
    std::multimap<size_t, void *> free;
    std::mutex mu;
    std::atomic<uint64_t> host_allocs{0}, host_alloc_bytes{0}; /* cudaHostAlloc calls made */
    /* Optional arena reserved up front (a server's host_cache_bytes):
     * blocks are carved from it first fit, and freed ranges merge with
     * their neighbours, so any mix of sizes is served without allocating
     * while it has room. */
    uint8_t *arena = nullptr;
    size_t arena_bytes = 0;
    std::map<size_t, size_t> arena_free; /* offset -> length */
    void reserve(size_t bytes);          /* throws Error */
    void *arena_take(size_t bytes);      /* mu held; nullptr when no range fits */
    void arena_give(void *p, size_t bytes); /* mu held */
    ~PinnedPool();
};

/* Page-locked host block from a pinned pool. */
struct PinnedBlock {
    std::shared_ptr<PinnedPool> pool;
    void *ptr = nullptr;
    size_t bytes = 0;
    bool in_arena = false;
    ~PinnedBlock();
};
using PinnedPtr = std::shared_ptr<PinnedBlock>;

struct KernelProfile {
    std::string name;
    uint64_t launches = 0;
    double total_us = 0;
};

struct Context {
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;     /* kernels, allocation, frees       */
    cudaStream_t h2d_stream = nullptr; /* input pages ahead of the kernels */
    cudaStream_t d2h_stream = nullptr; /* result pages behind the kernels  */
    cudaMemPool_t pool = nullptr;
    bool owns_pool = true;            /* false: pool shared with a server   */
    uint16_t *d_bloom = nullptr;      /* 2048 Bloom tags                  */
    StatusBlock *d_status = nullptr;  /* device status word + counters     */
    StatusBlock *h_status = nullptr;  /* pinned mirror                     */
    void *staging[2] = {nullptr, nullptr};
    cudaEvent_t staging_ev[2] = {nullptr, nullptr};
    size_t staging_bytes = 16u << 20;
    Options opt;
    Tuning tuning; /* autotuned launch parameters (cj_autotune / CJ_TUNING_FILE) */

    std::shared_ptr<PinnedPool> pinned; /* pinned host blocks by size class */

    /* Freed device buffers by size class. Every use of a context buffer is
     * ordered on the kernel stream (copy streams wait on it and it waits on
     * them), so a buffer freed at some point of that order can serve a
     * later allocation at once: no driver call in the steady state. */
    std::multimap<size_t, void *> dev_free;
    size_t dev_cached = 0;
    std::mutex dev_mu;
    void release(void *ptr, size_t cls);
    void trim_buffers(); /* returns every cached buffer to the pool */

    /* Bump arena (a prepared batch's buffers): while arena_base is set,
     * alloc() carves 256-byte-aligned buffers from it instead of the pool;
     * they are never freed one by one. alloc_bytes sums the size classes
     * of every allocation (what an arena for the same work needs). */
    uint8_t *arena_base = nullptr;
    size_t arena_size = 0, arena_used = 0;
    uint64_t alloc_bytes = 0;

    /* profiler */
    std::vector<KernelProfile> profile;
    std::map<std::string, size_t> profile_index;
    std::vector<cudaEvent_t> event_pool;
    struct PendingTiming {
        size_t slot;
        cudaEvent_t a, b;
    };
    std::vector<PendingTiming> pending;

    ~Context();

    Launch launch() const {
        Launch L;
        L.stream = stream;
        L.num_sms = num_sms;
        L.block_threads = (int)opt.block_threads;
        L.dev_errors = &d_status->errors;
        return L;
    }
    DevPtr alloc(size_t bytes);
    PinnedPtr alloc_pinned(size_t bytes);
    cudaEvent_t get_event();
    void put_event(cudaEvent_t e);
    /* Copies the status block to the host, waits for the stream and throws
     * on any device-side error bit. */
    void sync_status();
    void resolve_profile();
};

/* Device pages of one column. */
struct ColumnPages {
    int32_t type = CJ_INT32;
    uint64_t num_pages = 0;
    const uint8_t *dev = nullptr;
    DevPtr owner; /* null when the memory is adopted from the caller */
};

void upload_pages(Context &ctx, const cj_column_desc &cd, ColumnPages &out, uint64_t *h2d_bytes,
                  cudaStream_t stream = nullptr);

/* Creates a context on `device`; with `shared_pool` non-null the context
 * allocates from that pool instead of creating its own. Throws Error. */
Context *create_context(int device, cudaMemPool_t shared_pool,
                        std::shared_ptr<PinnedPool> shared_pinned = nullptr);
/* Reads a tuning file written by cj_autotune; num_sms > 0 must match the
 * file's SM count. Throws Error. */
Tuning load_tuning_file(const char *path, int num_sms);
/* Creates a device memory pool that keeps freed memory for reuse. */
cudaMemPool_t create_pool(int device);

} // namespace cj



struct cj_table {
    cj::Context *ctx = nullptr;
    uint64_t num_rows = 0;
    std::vector<cj::ColumnPages> cols;
};

struct cj_result {
    cj::Context *ctx = nullptr;
    uint64_t num_rows = 0;
    std::vector<int32_t> types;
    std::vector<uint64_t> num_pages;
    std::vector<cj::DevPtr> dev_pages;
    cj::PinnedPtr host;
    std::vector<uint8_t *> host_cols;
    cj::DevPtr keep; /* memory the pages live in, when not their own (a prepared batch's arena) */
};

struct cj_context : cj::Context {};

namespace cj {
cj_result *execute_plan(Context &ctx, const cj_plan_desc &plan, uint32_t flags, cj_exec_stats *stats);
void execute_batch(Context &ctx, const cj_plan_desc *plans, size_t n, uint32_t flags, cj_result **results,
                   int32_t *statuses, cj_batch_stats *stats);
}
