/*
 * noalloc.cu — cj_hash_join_noalloc: the radix-partitioned hash build and
 * the tiled probe of a single equi-join on INT32 key arrays that already
 * sit in device memory, without allocating anything.
 *
 * Some callers cannot let a library allocate device memory: an engine that
 * owns every byte of the GPU through its own allocator or fixed budget, or
 * a host process whose allocator must not be bypassed. The regular path
 * (cj_execute) takes its hash table, partition buffers and tile scratch
 * from the context's memory pool; this entry point takes them from one
 * file-scope device array instead, of fixed size kNoAllocScratchBytes,
 * which every GPU that loads the library holds until the process exits.
 * The caller passes inputs and outputs; nothing else is needed.
 *
 * The array's name is only a host-side stand-in in host code, so its device
 * address is fetched once per device with cudaGetSymbolAddress, while that
 * device is current, on the first call on that device (that first call
 * should therefore be made before any stream capture). All calls share the
 * array and it keeps the previous call's contents: the parts that must
 * start at zero (tile ticket, match counter) are cleared by every call, and
 * the directory and tuples are rewritten in full; two calls whose work
 * overlaps on the GPU (different streams or threads at the same time) race
 * on it.
 *
 * Output order: the probe hands out tiles from an atomic ticket and each
 * tile reserves its output range with one atomicAdd, so pairs keep probe
 * order only within a tile; across tiles the order is unspecified, and when
 * capacity is below the match count the pairs written are an arbitrary
 * subset of them (call again with capacity >= *d_count for all of them).
 */
#include <cstring>
#include <mutex>
#include <string>

#include "engine.h"

namespace {

constexpr uint64_t kNoAllocMaxBuild = 1ull << 18;  /* 262,144 build rows     */
constexpr uint64_t kNoAllocMaxProbe = 1ull << 27;  /* 134,217,728 probe rows */
constexpr size_t kNoAllocScratchBytes = 12u << 20; /* 12 MiB per device     */
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

struct DeviceScratch {
    bool ready = false;
    unsigned char *base = nullptr; /* device address of g_noalloc_scratch */
    int num_sms = 0;
};
DeviceScratch g_dev[kMaxDevices];
std::mutex g_mu;

/* layout: [reserved word | Bloom tags | directory | tuples | build scratch |
 * probe scratch], each 256-byte aligned. The build and probe kernels of
 * this path raise no device error bits; the launch's error word points at
 * the reserved word only because the launch descriptor requires one. */
constexpr size_t kErrOff = 0;
constexpr size_t kBloomOff = 256;
constexpr size_t kDirOff = kBloomOff + 4096;

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

int ceil_log2(uint64_t x) {
    int l = 0;
    while ((1ull << l) < x) ++l;
    return l;
}

/* Once per device, with that device current: resolve the array's device
 * address and fill the Bloom tag table (the 2048 smallest 16-bit values
 * with five bits set). */
int setup(int dev, DeviceScratch **out) {
    std::lock_guard<std::mutex> lk(g_mu);
    DeviceScratch &d = g_dev[dev];
    if (!d.ready) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return cj::set_last_error(CJ_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        }
        uint16_t tags[2048];
        int n = 0;
        for (uint32_t v = 0; v < 65536 && n < 2048; ++v)
            if (__builtin_popcount(v) == 5) tags[n++] = (uint16_t)v;
        e = cudaMemcpy(static_cast<unsigned char *>(p) + kBloomOff, tags, sizeof(tags), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&d.num_sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return cj::set_last_error(CJ_ERR_CUDA, std::string("scratch set-up: ") + cudaGetErrorString(e));
        }
        d.base = static_cast<unsigned char *>(p);
        d.ready = true;
    }
    *out = &d;
    return CJ_OK;
}

int cuda_status(cudaError_t e, const char *what) {
    cudaGetLastError();
    return cj::set_last_error(CJ_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

} // namespace

extern "C" int cj_hash_join_noalloc(const int32_t *build_keys, const uint32_t *build_valid, uint32_t n_build,
                                    const int32_t *probe_keys, const uint32_t *probe_valid, uint32_t n_probe,
                                    uint32_t *out_build_rows, uint32_t *out_probe_rows, uint64_t capacity,
                                    unsigned long long *d_count, uint64_t *h_count, void *stream) {
    if (!d_count || (n_build && (!build_keys || !build_valid)) || (n_probe && (!probe_keys || !probe_valid)) ||
        (capacity && (!out_build_rows || !out_probe_rows)))
        return cj::set_last_error(CJ_ERR_INVALID_ARGUMENT, "null argument");
    if (n_build > kNoAllocMaxBuild || n_probe > kNoAllocMaxProbe)
        return cj::set_last_error(CJ_ERR_LIMIT, "cj_hash_join_noalloc takes at most 262144 build rows and "
                                                "134217728 probe rows (fixed 12 MiB scratch)");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_status(e, "cudaGetDevice");
    if (dev >= kMaxDevices) return cj::set_last_error(CJ_ERR_LIMIT, "device ordinal too large");
    DeviceScratch *ds = nullptr;
    int rc = setup(dev, &ds);
    if (rc != CJ_OK) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    cj::Launch L;
    L.stream = s;
    L.num_sms = ds->num_sms;
    L.block_threads = 0;
    L.dev_errors = reinterpret_cast<unsigned int *>(ds->base + kErrOff);

    if (n_build && n_probe) {
        cj::BuildPlan bp;
        bp.num_rows = n_build;
        bp.log2_slots = ceil_log2(n_build) > 11 ? ceil_log2(n_build) : 11;
        bp.log2_parts = bp.log2_slots - 11 < 12 ? bp.log2_slots - 11 : 12;
        const size_t dir_bytes = align256(cj::build_dir_bytes(bp.log2_slots, 4));
        const size_t tup_off = kDirOff + dir_bytes;
        const size_t build_off = tup_off + align256((size_t)n_build * cj::build_tuple_bytes(4));
        const size_t probe_off = build_off + align256(cj::build_temp_bytes(L, bp, 4));
        const size_t end = probe_off + cj::probe_sched_bytes(n_probe);
        if (end > kNoAllocScratchBytes)
            return cj::set_last_error(CJ_ERR_LIMIT, "join needs " + std::to_string(end) +
                                                        " bytes of scratch; the fixed array holds " +
                                                        std::to_string(kNoAllocScratchBytes));
        cj::ColView bk{};
        bk.values = build_keys;
        bk.valid = build_valid;
        bk.type = CJ_INT32;
        cj::ColView pk{};
        pk.values = probe_keys;
        pk.valid = probe_valid;
        pk.type = CJ_INT32;
        const uint16_t *bloom = reinterpret_cast<const uint16_t *>(ds->base + kBloomOff);
        uint64_t *dir = reinterpret_cast<uint64_t *>(ds->base + kDirOff);
        void *tuples = ds->base + tup_off;
        e = cj::launch_build(L, bp, bk, bloom, dir, tuples, ds->base + build_off);
        if (e != cudaSuccess) return cuda_status(e, "build");
        cj::MatchOut mo;
        mo.build_rids = out_build_rows;
        mo.probe_rids = out_probe_rows;
        mo.capacity = capacity;
        mo.counter = d_count;
        e = cj::launch_probe_tiles_hash(L, pk, n_probe, CJ_INT32, dir, tuples, bp.log2_slots, bloom, mo,
                                        ds->base + probe_off);
        if (e != cudaSuccess) return cuda_status(e, "probe");
    } else {
        e = cudaMemsetAsync(d_count, 0, sizeof(unsigned long long), s);
        if (e != cudaSuccess) return cuda_status(e, "cudaMemsetAsync");
    }
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e, "cudaStreamSynchronize");
    if (h_count) {
        e = cudaMemcpy(h_count, d_count, sizeof(uint64_t), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_status(e, "cudaMemcpy");
    }
    cj::clear_last_error();
    return CJ_OK;
}
