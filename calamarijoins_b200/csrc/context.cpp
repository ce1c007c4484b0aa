/*
 * context.cpp — context resources: stream-ordered device pool, pinned
 * pool, events, status block, page upload.
 */
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <memory>
#include <string>

#include "engine.h"

#include <atomic>

namespace cj {

static std::atomic<uint64_t> g_launches{0};
void count_launches(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
uint64_t launches_so_far() { return g_launches.load(std::memory_order_relaxed); }

void fail(int code, const std::string &msg) { throw Error{code, msg}; }

static thread_local std::string g_last_error;
int set_last_error(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}
void clear_last_error() { g_last_error.clear(); }
const char *last_error() { return g_last_error.c_str(); }

void check_cuda(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return;
    int code = (e == cudaErrorMemoryAllocation) ? CJ_ERR_OUT_OF_MEMORY : CJ_ERR_CUDA;
    fail(code, std::string(what) + ": " + cudaGetErrorString(e));
}

DevBuf::~DevBuf() {
    if (ptr && ctx && !arena) ctx->release(ptr, cls);
}

/* Four size classes per power of two (at most 25 % above the request),
 * 256 bytes at least. */
static size_t device_class(size_t bytes) {
    if (bytes <= 256) return 256;
    int l = 63 - __builtin_clzll((unsigned long long)bytes - 1); /* 2^l < bytes <= 2^(l+1) */
    const size_t quarter = (size_t)1 << (l > 2 ? l - 2 : 0);
    return (bytes + quarter - 1) / quarter * quarter;
}

void Context::release(void *p, size_t c) {
    {
        std::lock_guard<std::mutex> g(dev_mu);
        if (opt.buffer_cache_bytes > 0 && dev_cached + c <= (size_t)opt.buffer_cache_bytes) {
            dev_free.emplace(c, p);
            dev_cached += c;
            return;
        }
    }
    cudaFreeAsync(p, stream);
}

void Context::trim_buffers() {
    std::lock_guard<std::mutex> g(dev_mu);
    for (auto &kv : dev_free) cudaFreeAsync(kv.second, stream);
    dev_free.clear();
    dev_cached = 0;
}

PinnedBlock::~PinnedBlock() {
    if (!ptr || !pool) return;
    std::lock_guard<std::mutex> g(pool->mu);
    if (in_arena) pool->arena_give(ptr, bytes);
    else pool->free.emplace(bytes, ptr);
}

PinnedPool::~PinnedPool() {
    for (auto &kv : free) cudaFreeHost(kv.second);
    if (arena) cudaFreeHost(arena);
}

constexpr size_t kArenaAlign = 64u << 10; /* arena blocks start and end on 64 KB */

void PinnedPool::reserve(size_t bytes) {
    std::lock_guard<std::mutex> g(mu);
    if (arena || !bytes) return;
    bytes = (bytes + kArenaAlign - 1) & ~(kArenaAlign - 1);
    void *p = nullptr;
    if (cudaHostAlloc(&p, bytes, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        fail(CJ_ERR_OUT_OF_MEMORY, "page-locked host cache of " + std::to_string(bytes) + " bytes failed");
    }
    host_allocs.fetch_add(1, std::memory_order_relaxed);
    host_alloc_bytes.fetch_add(bytes, std::memory_order_relaxed);
    arena = static_cast<uint8_t *>(p);
    arena_bytes = bytes;
    arena_free.emplace(0, bytes);
}

void *PinnedPool::arena_take(size_t bytes) {
    for (auto it = arena_free.begin(); it != arena_free.end(); ++it) {
        if (it->second < bytes) continue;
        const size_t off = it->first, left = it->second - bytes;
        arena_free.erase(it);
        if (left) arena_free.emplace(off + bytes, left);
        return arena + off;
    }
    return nullptr;
}

void PinnedPool::arena_give(void *p, size_t bytes) {
    size_t off = static_cast<uint8_t *>(p) - arena;
    auto next = arena_free.lower_bound(off);
    if (next != arena_free.end() && off + bytes == next->first) {
        bytes += next->second;
        next = arena_free.erase(next);
    }
    if (next != arena_free.begin()) {
        auto prev = std::prev(next);
        if (prev->first + prev->second == off) {
            prev->second += bytes;
            return;
        }
    }
    arena_free.emplace(off, bytes);
}

DevPtr Context::alloc(size_t bytes) {
    auto b = std::make_shared<DevBuf>();
    b->ctx = this;
    b->bytes = bytes;
    if (bytes == 0) return b;
    if (opt.fail_alloc_at > 0 && --opt.fail_alloc_at == 0) /* injected fault (CJ_OPT_FAIL_ALLOC_AT) */
        fail(CJ_ERR_OUT_OF_MEMORY, "device allocation of " + std::to_string(bytes) + " bytes failed (injected)");
    const size_t cls = device_class(bytes);
    alloc_bytes += cls;
    if (arena_base) {
        const size_t off = (arena_used + 255) & ~size_t(255);
        if (off + bytes > arena_size) fail(CJ_ERR_OUT_OF_MEMORY, "prepared batch arena exhausted");
        b->ptr = arena_base + off;
        b->arena = true;
        arena_used = off + bytes;
        return b;
    }
    b->cls = cls;
    {
        std::lock_guard<std::mutex> g(dev_mu);
        auto it = dev_free.find(cls);
        if (it != dev_free.end()) {
            b->ptr = it->second;
            dev_free.erase(it);
            dev_cached -= cls;
            return b;
        }
    }
    cudaError_t e = cudaMallocFromPoolAsync(&b->ptr, cls, pool, stream);
    if (e != cudaSuccess) {
        /* cached buffers of other sizes go back to the pool, then retry */
        cudaGetLastError();
        trim_buffers();
        cudaStreamSynchronize(stream);
        e = cudaMallocFromPoolAsync(&b->ptr, cls, pool, stream);
    }
    if (e != cudaSuccess) {
        b->ptr = nullptr;
        cudaGetLastError();
        fail(CJ_ERR_OUT_OF_MEMORY, "device allocation of " + std::to_string(bytes) + " bytes failed");
    }
    return b;
}

static size_t pinned_class(size_t bytes) {
    size_t c = 1u << 20;
    while (c < bytes) c <<= 1;
    return c;
}

PinnedPtr Context::alloc_pinned(size_t bytes) {
    auto b = std::make_shared<PinnedBlock>();
    b->pool = pinned;
    if (bytes == 0) return b;
    size_t cls = pinned_class(bytes);
    {
        std::lock_guard<std::mutex> g(pinned->mu);
        if (pinned->arena) {
            const size_t need = (bytes + kArenaAlign - 1) & ~(kArenaAlign - 1);
            if (void *p = pinned->arena_take(need)) {
                b->ptr = p;
                b->bytes = need;
                b->in_arena = true;
                return b;
            }
        }
        /* best fit: the smallest cached block of this class or up to two
         * classes larger (a block of 4x the request at most) */
        auto it = pinned->free.lower_bound(cls);
        if (it != pinned->free.end() && it->first <= 4 * cls) {
            b->ptr = it->second;
            b->bytes = it->first;
            pinned->free.erase(it);
            return b;
        }
    }
    void *p = nullptr;
    cudaError_t e = cudaHostAlloc(&p, cls, cudaHostAllocDefault);
    if (e != cudaSuccess) {
        cudaGetLastError();
        fail(CJ_ERR_OUT_OF_MEMORY, "pinned allocation of " + std::to_string(cls) + " bytes failed");
    }
    pinned->host_allocs.fetch_add(1, std::memory_order_relaxed);
    pinned->host_alloc_bytes.fetch_add(cls, std::memory_order_relaxed);
    b->ptr = p;
    b->bytes = cls;
    return b;
}

cudaEvent_t Context::get_event() {
    if (!event_pool.empty()) {
        cudaEvent_t e = event_pool.back();
        event_pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    check_cuda(cudaEventCreate(&e), "cudaEventCreate");
    return e;
}

void Context::put_event(cudaEvent_t e) { event_pool.push_back(e); }

void Context::sync_status() {
    check_cuda(cudaMemcpyAsync(h_status, d_status, sizeof(StatusBlock), cudaMemcpyDeviceToHost, stream),
               "status copy");
    check_cuda(cudaStreamSynchronize(stream), "stream synchronize");
    unsigned int err = h_status->errors;
    if (err) {
        /* clear for the next call */
        cudaMemsetAsync(&d_status->errors, 0, sizeof(unsigned int), stream);
        cudaStreamSynchronize(stream);
        std::string what;
        if (err & DEV_ERR_PAGE_HEADER) what += " page header inconsistent;";
        if (err & DEV_ERR_VARCHAR_OFFSETS) what += " VARCHAR offsets out of range;";
        if (err & DEV_ERR_LONG_CHAIN) what += " long-string continuation without start;";
        if (err & DEV_ERR_BAD_PAGE_KIND) what += " special page in fixed-width column;";
        if (err & DEV_ERR_ROW_COUNT) what += " pages hold a row count other than the table's;";
        if (err & DEV_ERR_INTERNAL) what += " internal;";
        if (err & DEV_ERR_STALE)
            what += " match counts differ from the prepared batch's (inputs changed): check " +
                    std::to_string(h_status->stale[0] >> 32) + " entry " + std::to_string(h_status->stale[0] & 0xFFFFFFFFu) +
                    " counted " + std::to_string(h_status->stale[1]) + ", recorded " + std::to_string(h_status->stale[2]) +
                    ";";
        int code = (err & DEV_ERR_INTERNAL) ? CJ_ERR_INTERNAL
                   : (err & DEV_ERR_STALE)  ? CJ_ERR_INVALID_ARGUMENT
                                            : CJ_ERR_MALFORMED_PAGE;
        fail(code, "device reported:" + what);
    }
}

void Context::resolve_profile() {
    for (auto &p : pending) {
        float ms = 0;
        if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
            profile[p.slot].launches += 1;
            profile[p.slot].total_us += ms * 1000.0;
        }
        put_event(p.a);
        put_event(p.b);
    }
    pending.clear();
    cudaGetLastError();
}

Context::~Context() {
    trim_buffers();
    if (h2d_stream) cudaStreamSynchronize(h2d_stream);
    if (d2h_stream) cudaStreamSynchronize(d2h_stream);
    if (stream) cudaStreamSynchronize(stream);
    for (auto &p : pending) {
        cudaEventDestroy(p.a);
        cudaEventDestroy(p.b);
    }
    for (auto e : event_pool) cudaEventDestroy(e);
    for (int i = 0; i < 2; ++i) {
        if (staging_ev[i]) cudaEventDestroy(staging_ev[i]);
        if (staging[i]) cudaFreeHost(staging[i]);
    }
    if (h_status) cudaFreeHost(h_status);
    if (d_status) cudaFree(d_status);
    if (d_bloom) cudaFree(d_bloom);
    if (pool && owns_pool) cudaMemPoolDestroy(pool);
    if (stream) cudaStreamDestroy(stream);
    if (h2d_stream) cudaStreamDestroy(h2d_stream);
    if (d2h_stream) cudaStreamDestroy(d2h_stream);
}

static void make_bloom(uint16_t *out) {
    /* The 2048 smallest 16-bit values with exactly five bits set, ascending:
     * the Bloom tag table of the reference (include/join_execution/
     * bloom_tags.h:35-263), regenerated. */
    int n = 0;
    for (uint32_t v = 0; v < 65536 && n < 2048; ++v)
        if (__builtin_popcount(v) == 5) out[n++] = (uint16_t)v;
}

static int64_t env_opt(const char *name, int64_t dflt) {
    const char *v = std::getenv(name);
    if (!v || !*v) return dflt;
    return std::strtoll(v, nullptr, 10);
}

cudaMemPool_t create_pool(int device) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t pool = nullptr;
    check_cuda(cudaMemPoolCreate(&pool, &props), "cudaMemPoolCreate");
    uint64_t keep = UINT64_MAX;
    check_cuda(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep), "pool attr");
    return pool;
}

Context *create_context(int device, cudaMemPool_t shared_pool, std::shared_ptr<PinnedPool> shared_pinned) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        cudaGetLastError();
        fail(CJ_ERR_NO_DEVICE, "no CUDA device visible");
    }
    if (device < 0) check_cuda(cudaGetDevice(&device), "cudaGetDevice");
    if (device >= n) fail(CJ_ERR_INVALID_ARGUMENT, "device ordinal out of range");
    check_cuda(cudaSetDevice(device), "cudaSetDevice");
    std::unique_ptr<Context> c(new cj_context());
    c->device = device;
    c->pinned = shared_pinned ? shared_pinned : std::make_shared<PinnedPool>();
    check_cuda(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device), "attr");
    check_cuda(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "stream");
    check_cuda(cudaStreamCreateWithFlags(&c->h2d_stream, cudaStreamNonBlocking), "stream");
    check_cuda(cudaStreamCreateWithFlags(&c->d2h_stream, cudaStreamNonBlocking), "stream");
    if (shared_pool) {
        c->pool = shared_pool;
        c->owns_pool = false;
    } else {
        c->pool = create_pool(device);
    }
    uint16_t bloom[2048];
    make_bloom(bloom);
    check_cuda(cudaMalloc(&c->d_bloom, sizeof(bloom)), "cudaMalloc");
    check_cuda(cudaMemcpy(c->d_bloom, bloom, sizeof(bloom), cudaMemcpyHostToDevice), "bloom upload");
    check_cuda(cudaMalloc(&c->d_status, sizeof(StatusBlock)), "cudaMalloc");
    check_cuda(cudaMemset(c->d_status, 0, sizeof(StatusBlock)), "memset");
    check_cuda(cudaHostAlloc(reinterpret_cast<void **>(&c->h_status), sizeof(StatusBlock), 0), "host");
    std::memset(c->h_status, 0, sizeof(StatusBlock));
    for (int i = 0; i < 2; ++i) {
        check_cuda(cudaHostAlloc(&c->staging[i], c->staging_bytes, 0), "staging");
        check_cuda(cudaEventCreateWithFlags(&c->staging_ev[i], cudaEventDisableTiming), "event");
    }
    c->opt.nested_loop_max_build = env_opt("CJ_NESTED_LOOP_MAX_BUILD", c->opt.nested_loop_max_build);
    c->opt.slots_per_partition = env_opt("CJ_SLOTS_PER_PARTITION", c->opt.slots_per_partition);
    c->opt.profile_kernels = env_opt("CJ_PROFILE_KERNELS", c->opt.profile_kernels);
    c->opt.block_threads = env_opt("CJ_BLOCK_THREADS", c->opt.block_threads);
    c->opt.varchar_tile_rows = env_opt("CJ_VARCHAR_TILE_ROWS", c->opt.varchar_tile_rows);
    c->opt.ctas_per_sm = env_opt("CJ_CTAS_PER_SM", c->opt.ctas_per_sm);
    c->opt.dense_keys = std::max<int64_t>(0, std::min<int64_t>(64, env_opt("CJ_DENSE_KEYS", c->opt.dense_keys)));
    c->opt.buffer_cache_bytes = std::max<int64_t>(0, env_opt("CJ_BUFFER_CACHE_BYTES", c->opt.buffer_cache_bytes));
    c->opt.inline_dir_max_bytes = std::max<int64_t>(0, env_opt("CJ_INLINE_DIR_MAX_BYTES", c->opt.inline_dir_max_bytes));
    c->opt.defer_count = env_opt("CJ_DEFER_COUNT", c->opt.defer_count);
    if (shared_pool) c->opt.buffer_cache_bytes = 0; /* contexts sharing a pool share through it */
    if (const char *tf = std::getenv("CJ_TUNING_FILE"); tf && *tf) c->tuning = load_tuning_file(tf, c->num_sms);
    return c.release();
}

/* Host pages -> one consecutive device array. A run of pages that are
 * already consecutive in host memory goes in one cudaMemcpyAsync (full PCIe
 * speed when the memory is page-locked); scattered pages are gathered into
 * one of two pinned staging buffers while the other is in flight. The
 * copies go on `stream` (the context's stream when null); the device array
 * is allocated on the context's stream and `stream` is ordered after that. */
void upload_pages(Context &ctx, const cj_column_desc &cd, ColumnPages &out, uint64_t *h2d_bytes,
                  cudaStream_t stream) {
    out.type = cd.type;
    out.num_pages = cd.num_pages;
    if (cd.num_pages == 0) return;
    if (!cd.pages) fail(CJ_ERR_INVALID_ARGUMENT, "column has pages but no page array");
    const size_t P = kPageSize;
    out.owner = ctx.alloc(cd.num_pages * P);
    uint8_t *dev = out.owner->as<uint8_t>();
    out.dev = dev;
    const cudaStream_t s = stream ? stream : ctx.stream;
    if (s != ctx.stream) {
        cudaEvent_t ready = ctx.get_event();
        check_cuda(cudaEventRecord(ready, ctx.stream), "event record");
        check_cuda(cudaStreamWaitEvent(s, ready, 0), "stream wait");
        ctx.put_event(ready);
    }
    const uint64_t per_buf = ctx.staging_bytes / P;
    int buf = 0;
    uint64_t fill = 0, fill_first = 0;
    auto flush = [&]() {
        if (!fill) return;
        check_cuda(cudaMemcpyAsync(dev + fill_first * P, ctx.staging[buf], fill * P, cudaMemcpyHostToDevice, s),
                   "page upload");
        check_cuda(cudaEventRecord(ctx.staging_ev[buf], s), "event record");
        buf ^= 1;
        fill = 0;
    };
    uint64_t i = 0;
    const uint64_t np = cd.num_pages;
    while (i < np) {
        const uint8_t *p0 = static_cast<const uint8_t *>(cd.pages[i]);
        if (!p0) fail(CJ_ERR_INVALID_ARGUMENT, "null page pointer");
        uint64_t j = i + 1;
        while (j < np && static_cast<const uint8_t *>(cd.pages[j]) == p0 + (j - i) * P) ++j;
        const uint64_t run = j - i;
        if (run * P >= (1u << 20)) {
            flush();
            check_cuda(cudaMemcpyAsync(dev + i * P, p0, run * P, cudaMemcpyHostToDevice, s), "page upload");
        } else {
            for (uint64_t k = i; k < j; ++k) {
                if (fill == 0) {
                    check_cuda(cudaEventSynchronize(ctx.staging_ev[buf]), "staging wait");
                    fill_first = k;
                }
                std::memcpy(static_cast<uint8_t *>(ctx.staging[buf]) + fill * P, cd.pages[k], P);
                if (++fill == per_buf) flush();
            }
        }
        i = j;
    }
    flush();
    if (h2d_bytes) *h2d_bytes += np * P;
}

} // namespace cj
