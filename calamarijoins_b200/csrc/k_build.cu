/*
 * k_build.cu — unchained hash-table build with Bloom tags on sm_100a.
 *
 * The table is the reference's UnchainedHashtable (include/join_execution/
 * hashtable.h:63-506): a power-of-two directory of u64 entries over a
 * contiguous, slot-ordered tuple array, each entry carrying the OR of the
 * slot's 16-bit Bloom tags (:197-246). Directory size = pow2 >= max(2048,
 * build rows) (:255-264). The reference stores the slot's END offset
 * (end << 16 | tags) and reads [dir[s-1] >> 16, dir[s] >> 16) (:298-313),
 * two dependent loads per probe; here an entry holds
 *     start (bits 63..32) | count (31..16, saturated at 0xFFFF) | tags (15..0)
 * so one load gives the candidate range. A saturated count is bounded by
 * the next entry's start; one sentinel entry after the last slot holds the
 * total tuple count as its start, so the directory has slots + 1 entries.
 *
 * Build = radix partition + per-partition counting sort, the reference's
 * two-pass build (:405-505) mapped to the GPU:
 *   1. k_part_hist    one CTA per contiguous chunk of build rows builds a
 *                     shared-memory histogram over the P partitions (top
 *                     log2(P) hash bits) and stores it column-major in a
 *                     P x G matrix;
 *   2. exclusive scan of the matrix gives every (partition, CTA) pair its
 *                     output range: a stable, atomic-free partitioning;
 *   3. k_part_scatter each CTA re-reads its chunk and scatters {key, row id}
 *                     tuples, ranking rows of one partition within a warp
 *                     with __match_any_sync (warp-aggregated scatter);
 *   4. k_part_build   one CTA per partition counts its S slots in shared
 *                     memory, ORs the Bloom tags, scans, writes its S
 *                     directory entries and scatters the tuples into slot
 *                     order (build_partition, hashtable.h:197-246).
 * NULL keys are skipped (hashtable.h:439-478).
 */
#include <algorithm>
#include <atomic>
#include <mutex>

#include "cj_device.cuh"

#define CJ_DEV_HOST_INLINE __host__ __device__ __forceinline__

namespace cj {
namespace {

constexpr int kBuildThreads = 256;
/* Radix histogram and scatter passes: 512 threads per CTA, at most four
 * CTAs per SM, each over a contiguous chunk of at least kPartMinRows build
 * rows (64 warps per SM stream the keys; fewer chunks keep the partition x
 * chunk offset matrix and its scan small). */
constexpr int kPartThreads = 512;
constexpr uint32_t kPartMinRows = 2048;
constexpr int kPartCtasPerSm = 4;
/* Radix bits one pass can take: 2^12 shared-memory counters (16 KB) per
 * CTA. More partition bits than that are split over two passes: the first
 * over the build keys (top b1 bits), the second refining every first-pass
 * partition by the next b2 bits (k_part_refine), b1 >= 8 so that the second
 * pass has at least 256 partitions to spread over the SMs. */
constexpr int kMaxPassBits = 12;
constexpr int kMinFirstPassBits = 8;
CJ_DEV_HOST_INLINE int first_pass_bits(int log2_parts) {
    if (log2_parts <= kMaxPassBits) return log2_parts;
    const int b2 = log2_parts - kMinFirstPassBits < kMaxPassBits ? log2_parts - kMinFirstPassBits : kMaxPassBits;
    return log2_parts - b2;
}

struct PartGeom {
    uint32_t n;        /* build relation rows                */
    int log2_parts;
    int log2_slots;
    uint32_t grid;     /* CTAs of the hist / scatter passes  */
    uint32_t chunk;    /* rows per CTA                       */
};

CJ_DEV uint32_t part_of(uint64_t h, int log2_parts) {
    return log2_parts ? (uint32_t)(h >> (64 - log2_parts)) : 0u;
}

/* ---- per-unit bodies (shared by the single-join and grouped kernels) ---- */

/* Histogram of one chunk of build rows over the partitions; column-major
 * into `matrix` (P x g.grid). */
CJ_DEV void hist_chunk(const ColView &key, const PartGeom &g, uint32_t chunk, uint32_t *__restrict__ matrix,
                       uint32_t *s_hist) {
    const uint32_t P = 1u << g.log2_parts;
    for (uint32_t b = threadIdx.x; b < P; b += blockDim.x) s_hist[b] = 0;
    __syncthreads();
    const uint64_t r0 = (uint64_t)chunk * g.chunk;
    const uint64_t r1 = min((uint64_t)g.n, r0 + g.chunk);
    for (uint64_t i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
        int64_t k;
        if (load_key(key, (uint32_t)i, &k)) atomicAdd(&s_hist[part_of(hash_key(k), g.log2_parts)], 1u);
    }
    __syncthreads();
    for (uint32_t b = threadIdx.x; b < P; b += blockDim.x) matrix[(uint64_t)b * g.grid + chunk] = s_hist[b];
    __syncthreads();
}

/* Scatter of one chunk into the partitioned buffer. `offsets` is the
 * exclusive scan of the matrix, `off_base` subtracted from every entry.
 * The rows of one partition inside a warp are ranked with
 * __match_any_sync and the group's leader reserves their places with one
 * shared-memory atomicAdd on the partition's cursor: each tuple is written
 * as soon as its key is read, with no block barrier in the loop and no
 * rows held in registers. The order of a chunk's tuples inside a partition
 * is therefore not row order; nothing depends on it (the per-partition
 * build sorts them by slot, and the order of equal-slot tuples, like the
 * order of a join's output rows, is unspecified). */
template <typename K>
CJ_DEV void scatter_chunk(const ColView &key, const PartGeom &g, uint32_t chunk, const uint64_t *__restrict__ offsets,
                          uint64_t off_base, Tuple<K> *__restrict__ out, uint32_t *smem) {
    const uint32_t P = 1u << g.log2_parts;
    uint32_t *s_cursor = smem; /* next output position per partition */
    for (uint32_t b = threadIdx.x; b < P; b += blockDim.x)
        s_cursor[b] = (uint32_t)(offsets[(uint64_t)b * g.grid + chunk] - off_base);
    __syncthreads();
    const uint64_t r0 = (uint64_t)chunk * g.chunk;
    const uint64_t r1 = min((uint64_t)g.n, r0 + g.chunk);
    /* whole warps iterate together (match_any needs every lane) */
    const uint64_t span = (r1 > r0 ? r1 - r0 : 0);
    const uint64_t iters = (span + blockDim.x - 1) / blockDim.x;
    for (uint64_t k = 0; k < iters; ++k) {
        const uint64_t i = r0 + k * blockDim.x + threadIdx.x;
        int64_t kv = 0;
        const bool v = i < r1 && load_key(key, (uint32_t)i, &kv);
        const uint32_t p = v ? part_of(hash_key(kv), g.log2_parts) : 0xffffffffu;
        const uint32_t peers = __match_any_sync(0xffffffffu, p);
        const uint32_t leader = __ffs(peers) - 1;
        uint32_t base = 0;
        if (v && lane_id() == leader) base = atomicAdd(&s_cursor[p], (uint32_t)__popc(peers));
        base = __shfl_sync(0xffffffffu, base, leader);
        if (v) {
            Tuple<K> tp;
            tp.key = (K)kv;
            tp.rid = (uint32_t)i;
            out[base + __popc(peers & lanemask_lt())] = tp;
        }
    }
    __syncthreads();
}

/* Counting sort of one partition into slot order + its directory entries
 * (build_partition, hashtable.h:197-246). */
template <typename K>
CJ_DEV void build_partition(const Tuple<K> *__restrict__ in, const uint64_t *__restrict__ offsets, uint64_t off_base,
                            uint32_t grid_hist, int log2_parts, int log2_slots, uint32_t p, const uint16_t *s_bloom,
                            uint64_t *__restrict__ dir, Tuple<K> *__restrict__ out, uint32_t *s_cnt, uint32_t *s_tag,
                            uint32_t *wbuf, bool inline_first) {
    const uint32_t S = 1u << (log2_slots - log2_parts);
    for (uint32_t s = threadIdx.x; s < S; s += blockDim.x) {
        s_cnt[s] = 0;
        s_tag[s] = 0;
    }
    __syncthreads();
    const uint64_t ps = offsets[(uint64_t)p * grid_hist] - off_base;
    const uint64_t pe = offsets[(uint64_t)(p + 1) * grid_hist] - off_base;
    for (uint64_t t = ps + threadIdx.x; t < pe; t += blockDim.x) {
        uint64_t h = hash_key((int64_t)in[t].key);
        uint32_t ls = slot_of(h, log2_slots) & (S - 1);
        atomicAdd(&s_cnt[ls], 1u);
        atomicOr(&s_tag[ls], (uint32_t)s_bloom[bloom_index(h)]);
    }
    __syncthreads();
    /* exclusive scan of the S counts: each thread owns S/blockDim slots */
    const uint32_t per = (S + blockDim.x - 1) / blockDim.x;
    const uint32_t s0 = threadIdx.x * per;
    uint32_t sum = 0;
    for (uint32_t k = 0; k < per; ++k)
        if (s0 + k < S) sum += s_cnt[s0 + k];
    uint32_t tot;
    uint32_t pre = block_exclusive_scan<uint32_t>(sum, wbuf, &tot);
    const bool kInline = sizeof(K) == 4 && inline_first; /* DirEntry32: first tuple in the entry */
    DirEntry32 *dir16 = reinterpret_cast<DirEntry32 *>(dir);
    for (uint32_t k = 0; k < per; ++k) {
        uint32_t s = s0 + k;
        if (s >= S) break;
        uint32_t c = s_cnt[s];
        const uint64_t start = ps + pre;
        const uint64_t word = (start << 32) | ((uint64_t)min(c, 0xFFFFu) << 16) | (uint64_t)(s_tag[s] & 0xFFFFu);
        if (kInline) dir16[(uint64_t)p * S + s].word = word;
        else dir[(uint64_t)p * S + s] = word;
        s_cnt[s] = pre; /* becomes the scatter cursor */
        s_tag[s] = pre; /* the slot's first position */
        pre += c;
    }
    if (threadIdx.x == 0 && p == (1u << log2_parts) - 1) { /* sentinel */
        if (kInline) dir16[(uint64_t)(p + 1) * S].word = pe << 32;
        else dir[(uint64_t)(p + 1) * S] = pe << 32;
    }
    __syncthreads();
    for (uint64_t t = ps + threadIdx.x; t < pe; t += blockDim.x) {
        Tuple<K> tp = in[t];
        uint32_t ls = slot_of(hash_key((int64_t)tp.key), log2_slots) & (S - 1);
        uint32_t pos = atomicAdd(&s_cnt[ls], 1u);
        out[ps + pos] = tp;
        if (kInline && pos == s_tag[ls]) { /* the slot's first tuple, also in its entry */
            dir16[(uint64_t)p * S + ls].key0 = (int32_t)tp.key;
            dir16[(uint64_t)p * S + ls].rid0 = tp.rid;
        }
    }
    __syncthreads();
}

/* Second radix pass: one CTA per first-pass partition (a contiguous range
 * of `in`, bounded by offsets[p1 * grid_hist]) counts its tuples over the
 * next b2 hash bits in shared memory, scans the counts into the global
 * partition starts part_start[p1 * 2^b2 + q], and scatters the tuples into
 * `out` with warp-aggregated shared-memory cursors. Afterwards `out` is
 * ordered by the top b1 + b2 hash bits, as one pass over 2^(b1 + b2)
 * partitions would have left it, and part_start (2^(b1+b2) + 1 entries)
 * bounds each partition for k_part_build. */
template <typename K>
__global__ void __launch_bounds__(kPartThreads)
    k_part_refine(const Tuple<K> *__restrict__ in, const uint64_t *__restrict__ offsets, uint32_t grid_hist, int b1,
                  int b2, Tuple<K> *__restrict__ out, uint64_t *__restrict__ part_start) {
    extern __shared__ uint32_t s_cnt[];
    __shared__ uint32_t wbuf[kPartThreads / 32 + 1];
    const uint32_t Q = 1u << b2;
    const uint32_t P1 = 1u << b1;
    const int top = b1 + b2;
    for (uint32_t p1 = blockIdx.x; p1 < P1; p1 += gridDim.x) {
        const uint64_t ps = offsets[(uint64_t)p1 * grid_hist], pe = offsets[(uint64_t)(p1 + 1) * grid_hist];
        for (uint32_t q = threadIdx.x; q < Q; q += blockDim.x) s_cnt[q] = 0;
        __syncthreads();
        const uint64_t iters = (pe - ps + blockDim.x - 1) / blockDim.x;
        for (uint64_t k = 0; k < iters; ++k) {
            const uint64_t t = ps + k * blockDim.x + threadIdx.x;
            const bool v = t < pe;
            const uint32_t q = v ? (uint32_t)(hash_key((int64_t)in[t].key) >> (64 - top)) & (Q - 1) : 0xffffffffu;
            const uint32_t peers = __match_any_sync(0xffffffffu, q);
            if (v && lane_id() == (uint32_t)(__ffs(peers) - 1)) atomicAdd(&s_cnt[q], (uint32_t)__popc(peers));
        }
        __syncthreads();
        /* exclusive scan of the Q counts, each thread a run of them */
        const uint32_t per = (Q + blockDim.x - 1) / blockDim.x;
        const uint32_t q0 = threadIdx.x * per;
        uint32_t sum = 0;
        for (uint32_t j = 0; j < per; ++j)
            if (q0 + j < Q) sum += s_cnt[q0 + j];
        uint32_t tot;
        uint32_t pre = block_exclusive_scan<uint32_t>(sum, wbuf, &tot);
        for (uint32_t j = 0; j < per; ++j) {
            const uint32_t q = q0 + j;
            if (q >= Q) break;
            const uint32_t c = s_cnt[q];
            part_start[(uint64_t)p1 * Q + q] = ps + pre;
            s_cnt[q] = (uint32_t)(ps + pre); /* tuple counts stay below 2^32 */
            pre += c;
        }
        if (p1 == P1 - 1 && threadIdx.x == 0) part_start[(uint64_t)P1 * Q] = pe;
        __syncthreads();
        for (uint64_t k = 0; k < iters; ++k) {
            const uint64_t t = ps + k * blockDim.x + threadIdx.x;
            const bool v = t < pe;
            Tuple<K> tp;
            uint32_t q = 0xffffffffu;
            if (v) {
                tp = in[t];
                q = (uint32_t)(hash_key((int64_t)tp.key) >> (64 - top)) & (Q - 1);
            }
            const uint32_t peers = __match_any_sync(0xffffffffu, q);
            const uint32_t leader = __ffs(peers) - 1;
            uint32_t base = 0;
            if (v && lane_id() == leader) base = atomicAdd(&s_cnt[q], (uint32_t)__popc(peers));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (v) out[base + __popc(peers & lanemask_lt())] = tp;
        }
        __syncthreads();
    }
}

/* ---- single-join kernels ---- */
__global__ void __launch_bounds__(kPartThreads)
    k_part_hist(ColView key, PartGeom g, uint32_t *__restrict__ matrix) {
    extern __shared__ uint32_t s_hist[];
    hist_chunk(key, g, blockIdx.x, matrix, s_hist);
}

template <typename K>
__global__ void __launch_bounds__(kPartThreads)
    k_part_scatter(ColView key, PartGeom g, const uint64_t *__restrict__ offsets, Tuple<K> *__restrict__ out) {
    extern __shared__ uint32_t smem[];
    scatter_chunk<K>(key, g, blockIdx.x, offsets, 0, out, smem);
}

template <typename K>
__global__ void __launch_bounds__(kBuildThreads)
    k_part_build(const Tuple<K> *__restrict__ in, const uint64_t *__restrict__ offsets, uint32_t grid_hist,
                 int log2_parts, int log2_slots, const uint16_t *__restrict__ g_bloom, uint64_t *__restrict__ dir,
                 Tuple<K> *__restrict__ out, int inline_first) {
    extern __shared__ uint32_t smem[];
    __shared__ uint16_t s_bloom[2048];
    __shared__ uint32_t wbuf[kBuildThreads / 32 + 1];
    const uint32_t P = 1u << log2_parts;
    const uint32_t S = 1u << (log2_slots - log2_parts);
    load_bloom(s_bloom, g_bloom);
    for (uint32_t p = blockIdx.x; p < P; p += gridDim.x)
        build_partition<K>(in, offsets, 0, grid_hist, log2_parts, log2_slots, p, s_bloom, dir, out, smem, smem + S,
                           wbuf, inline_first != 0);
}

/* ---- grouped kernels: every hash join of a batch level ---- */
CJ_DEV uint32_t find_task(const BuildTask *tasks, uint32_t ntasks, uint32_t unit, bool by_partition) {
    uint32_t lo = 0, hi = ntasks;
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        uint32_t b = by_partition ? tasks[mid].part_base : tasks[mid].chunk_base;
        if (b <= unit) lo = mid;
        else hi = mid;
    }
    return lo;
}

CJ_DEV PartGeom task_geom(const BuildTask &T) {
    PartGeom g;
    g.n = T.n;
    g.log2_parts = T.log2_parts;
    g.log2_slots = T.log2_slots;
    g.grid = T.grid;
    g.chunk = T.chunk;
    return g;
}

__global__ void __launch_bounds__(kPartThreads)
    k_part_hist_grouped(const BuildTask *__restrict__ tasks, uint32_t ntasks, uint32_t *__restrict__ matrix) {
    extern __shared__ uint32_t s_hist[];
    __shared__ uint32_t s_task;
    if (threadIdx.x == 0) s_task = find_task(tasks, ntasks, blockIdx.x, false);
    __syncthreads();
    const BuildTask &T = tasks[s_task];
    hist_chunk(T.key, task_geom(T), blockIdx.x - T.chunk_base, matrix + T.cell_base, s_hist);
}

__global__ void __launch_bounds__(kPartThreads)
    k_part_scatter_grouped(const BuildTask *__restrict__ tasks, uint32_t ntasks,
                           const uint64_t *__restrict__ offsets) {
    extern __shared__ uint32_t smem[];
    __shared__ uint32_t s_task;
    if (threadIdx.x == 0) s_task = find_task(tasks, ntasks, blockIdx.x, false);
    __syncthreads();
    const BuildTask &T = tasks[s_task];
    const uint64_t *off = offsets + T.cell_base;
    if (T.key.type == CJ_INT32)
        scatter_chunk<int32_t>(T.key, task_geom(T), blockIdx.x - T.chunk_base, off, off[0],
                               reinterpret_cast<Tuple<int32_t> *>(T.part_buf), smem);
    else
        scatter_chunk<int64_t>(T.key, task_geom(T), blockIdx.x - T.chunk_base, off, off[0],
                               reinterpret_cast<Tuple<int64_t> *>(T.part_buf), smem);
}

__global__ void __launch_bounds__(kBuildThreads)
    k_part_build_grouped(const BuildTask *__restrict__ tasks, uint32_t ntasks, uint32_t total_parts,
                         const uint64_t *__restrict__ offsets, const uint16_t *__restrict__ g_bloom) {
    extern __shared__ uint32_t smem[];
    __shared__ uint16_t s_bloom[2048];
    __shared__ uint32_t wbuf[kBuildThreads / 32 + 1];
    __shared__ uint32_t s_task;
    load_bloom(s_bloom, g_bloom);
    for (uint32_t u = blockIdx.x; u < total_parts; u += gridDim.x) {
        __syncthreads();
        if (threadIdx.x == 0) s_task = find_task(tasks, ntasks, u, true);
        __syncthreads();
        const BuildTask &T = tasks[s_task];
        const uint32_t S = 1u << (T.log2_slots - T.log2_parts);
        const uint64_t *off = offsets + T.cell_base;
        if (T.key.type == CJ_INT32)
            build_partition<int32_t>(reinterpret_cast<const Tuple<int32_t> *>(T.part_buf), off, off[0], T.grid,
                                     T.log2_parts, T.log2_slots, u - T.part_base, s_bloom, T.dir,
                                     reinterpret_cast<Tuple<int32_t> *>(T.tuples), smem, smem + S, wbuf, true);
        else
            build_partition<int64_t>(reinterpret_cast<const Tuple<int64_t> *>(T.part_buf), off, off[0], T.grid,
                                     T.log2_parts, T.log2_slots, u - T.part_base, s_bloom, T.dir,
                                     reinterpret_cast<Tuple<int64_t> *>(T.tuples), smem, smem + S, wbuf, true);
    }
}

PartGeom geometry(const Launch &L, const BuildPlan &bp) {
    PartGeom g;
    g.n = bp.num_rows;
    g.log2_parts = first_pass_bits(bp.log2_parts);
    g.log2_slots = bp.log2_slots;
    uint64_t chunks = ((uint64_t)bp.num_rows + kPartMinRows - 1) / kPartMinRows;
    uint64_t grid = (uint64_t)L.num_sms * (L.part_ctas_per_sm > 0 ? L.part_ctas_per_sm : kPartCtasPerSm);
    if (chunks < grid) grid = chunks;
    if (grid == 0) grid = 1;
    g.grid = (uint32_t)grid;
    g.chunk = (uint32_t)(((uint64_t)bp.num_rows + grid - 1) / grid);
    return g;
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

template <typename K>
cudaError_t build_impl(const Launch &L, const BuildPlan &bp, const ColView &key,
                       const uint16_t *bloom, uint64_t *dir, Tuple<K> *tuples, void *temp) {
    PartGeom g = geometry(L, bp);
    const int b1 = g.log2_parts, b2 = bp.log2_parts - b1; /* b2 > 0: a second pass */
    const uint64_t P1 = 1ull << b1;
    const uint64_t cells = P1 * g.grid;
    char *t = reinterpret_cast<char *>(temp);
    uint32_t *matrix = reinterpret_cast<uint32_t *>(t);
    t += align256(cells * sizeof(uint32_t));
    uint64_t *offsets = reinterpret_cast<uint64_t *>(t);
    t += align256((cells + 1) * sizeof(uint64_t));
    Tuple<K> *part_buf = reinterpret_cast<Tuple<K> *>(t);
    t += align256((size_t)bp.num_rows * sizeof(Tuple<K>));
    Tuple<K> *part_buf2 = nullptr;
    uint64_t *part_start = nullptr;
    if (b2 > 0) {
        part_buf2 = reinterpret_cast<Tuple<K> *>(t);
        t += align256((size_t)bp.num_rows * sizeof(Tuple<K>));
        part_start = reinterpret_cast<uint64_t *>(t);
        t += align256(((1ull << bp.log2_parts) + 1) * sizeof(uint64_t));
    }
    void *scan_tmp = t;

    const size_t hist_smem = P1 * sizeof(uint32_t);
    k_part_hist<<<g.grid, kPartThreads, hist_smem, L.stream>>>(key, g, matrix);
    count_launches(1);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    e = scan_u32_to_u64(L, matrix, offsets, cells, scan_tmp);
    if (e != cudaSuccess) return e;
    const size_t scat_smem = P1 * sizeof(uint32_t);
    k_part_scatter<K><<<g.grid, kPartThreads, scat_smem, L.stream>>>(key, g, offsets, part_buf);
    count_launches(1);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const Tuple<K> *parts = part_buf;
    const uint64_t *bounds = offsets;
    uint32_t bounds_stride = g.grid;
    if (b2 > 0) {
        const unsigned grid_r = (unsigned)std::min<uint64_t>(P1, (uint64_t)L.num_sms * 4);
        k_part_refine<K><<<grid_r, kPartThreads, (1u << b2) * sizeof(uint32_t), L.stream>>>(
            part_buf, offsets, g.grid, b1, b2, part_buf2, part_start);
        count_launches(1);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        parts = part_buf2;
        bounds = part_start;
        bounds_stride = 1;
    }
    const uint64_t P = 1ull << bp.log2_parts;
    const uint64_t S = 1ull << (bp.log2_slots - bp.log2_parts);
    const size_t build_smem = 2 * S * sizeof(uint32_t);
    unsigned grid_b = (unsigned)(P < (uint64_t)L.num_sms * 16 ? P : (uint64_t)L.num_sms * 16);
    k_part_build<K><<<grid_b, kBuildThreads, build_smem, L.stream>>>(
        parts, bounds, bounds_stride, bp.log2_parts, bp.log2_slots, bloom, dir, tuples, bp.inline_first ? 1 : 0);
    count_launches(1);
    return cudaGetLastError();
}

/* ---- direct-mapped table (unique keys over a dense range) ---- */
CJ_DEV unsigned long long warp_min_u64(unsigned long long v) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, d));
    return v;
}
CJ_DEV unsigned long long warp_max_u64(unsigned long long v) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, d));
    return v;
}

/* Block-wide min / max / count of the non-NULL keys of rows i0, i0 +
 * stride, ... below i1, folded into range[0..2] by atomics. */
CJ_DEV void key_range_rows(const ColView &key, uint64_t i0, uint64_t i1, uint64_t stride,
                           unsigned long long *range) {
    __shared__ unsigned long long s_min[kBuildThreads / 32], s_max[kBuildThreads / 32];
    __shared__ unsigned int s_cnt[kBuildThreads / 32];
    unsigned long long mn = ~0ull, mx = 0ull;
    unsigned int cnt = 0;
    for (uint64_t i = i0; i < i1; i += stride) {
        int64_t k;
        if (load_key(key, (uint32_t)i, &k)) {
            const unsigned long long b = (unsigned long long)k ^ (1ull << 63);
            mn = min(mn, b);
            mx = max(mx, b);
            ++cnt;
        }
    }
    mn = warp_min_u64(mn);
    mx = warp_max_u64(mx);
    cnt = __reduce_add_sync(0xffffffffu, cnt);
    const uint32_t warp = threadIdx.x >> 5;
    if (lane_id() == 0) {
        s_min[warp] = mn;
        s_max[warp] = mx;
        s_cnt[warp] = cnt;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < kBuildThreads / 32; ++w) {
            mn = min(mn, s_min[w]);
            mx = max(mx, s_max[w]);
            cnt += s_cnt[w];
        }
        if (cnt) {
            atomicMin(range, mn);
            atomicMax(range + 1, mx);
            atomicAdd(range + 2, (unsigned long long)cnt);
        }
    }
}

__global__ void __launch_bounds__(kBuildThreads)
    k_key_range(ColView key, uint32_t n, unsigned long long *range) {
    key_range_rows(key, (uint64_t)blockIdx.x * blockDim.x + threadIdx.x, n, (uint64_t)gridDim.x * blockDim.x,
                   range);
}

/* params: [0] min ^ 2^63, [1] max ^ 2^63, [2] count (from k_key_range),
 * [3] unusable (1: span too wide, 2: a key repeats), [4] lo, [5] span. */
__global__ void k_array_prep(unsigned long long *p, uint64_t max_span) {
    if (p[2] == 0) return; /* no non-NULL key: span 0, nothing matches */
    const unsigned long long width = p[1] - p[0]; /* max - min: the bias cancels */
    if (width >= max_span) {
        p[3] = 1ull;
        return;
    }
    if (p[2] > width + 1) { /* more keys than values in their range: one repeats */
        p[3] = 2ull;
        return;
    }
    p[4] = p[0] ^ (1ull << 63);
    p[5] = width + 1;
}

__global__ void k_array_fill(uint32_t *__restrict__ slots, const unsigned long long *p) {
    const uint64_t span = p[5];
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < span; i += (uint64_t)gridDim.x * blockDim.x)
        slots[i] = kArrayEmpty;
}

__global__ void k_array_build(ColView key, uint32_t n, uint32_t *__restrict__ slots, unsigned long long *p) {
    if (p[3]) return;
    const uint64_t lo = p[4], span = p[5];
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        int64_t k;
        if (!load_key(key, (uint32_t)i, &k)) continue;
        const uint64_t off = (uint64_t)k - lo;
        if (off >= span) continue; /* cannot happen: lo and span come from these keys */
        if (atomicCAS(slots + off, kArrayEmpty, (uint32_t)i) != kArrayEmpty) p[3] = 2ull; /* a key repeats */
    }
}

/* ---- grouped direct-mapped builds (every candidate join of a batch level) ---- */
CJ_DEV uint32_t find_direct_task(const DirectTask *tasks, uint32_t ntasks, uint32_t block, bool fill) {
    uint32_t lo = 0, hi = ntasks;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if ((fill ? tasks[mid].fill_base : tasks[mid].key_base) <= block) lo = mid;
        else hi = mid;
    }
    return lo;
}

__global__ void __launch_bounds__(kBuildThreads)
    k_key_range_grouped(const DirectTask *__restrict__ tasks, uint32_t ntasks) {
    __shared__ uint32_t s_task;
    if (threadIdx.x == 0) s_task = find_direct_task(tasks, ntasks, blockIdx.x, false);
    __syncthreads();
    const DirectTask &T = tasks[s_task];
    const uint64_t r0 = (uint64_t)(blockIdx.x - T.key_base) * kDirectBlockRows;
    const uint64_t r1 = min((uint64_t)T.n, r0 + kDirectBlockRows);
    key_range_rows(T.key, r0 + threadIdx.x, r1, blockDim.x, T.params);
}

__global__ void k_array_prep_grouped(const DirectTask *__restrict__ tasks, uint32_t ntasks) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntasks) return;
    unsigned long long *p = tasks[t].params;
    if (p[2] == 0) return;
    const unsigned long long width = p[1] - p[0];
    if (width >= tasks[t].max_span) {
        p[3] = 1ull;
        return;
    }
    if (p[2] > width + 1) { /* more keys than values in their range: one repeats */
        p[3] = 2ull;
        return;
    }
    p[4] = p[0] ^ (1ull << 63);
    p[5] = width + 1;
}

__global__ void __launch_bounds__(kBuildThreads)
    k_array_fill_grouped(const DirectTask *__restrict__ tasks, uint32_t ntasks) {
    __shared__ uint32_t s_task;
    if (threadIdx.x == 0) s_task = find_direct_task(tasks, ntasks, blockIdx.x, true);
    __syncthreads();
    const DirectTask &T = tasks[s_task];
    const uint64_t span = T.params[3] ? 0ull : T.params[5];
    const uint64_t i0 = (uint64_t)(blockIdx.x - T.fill_base) * kDirectFillSlots;
    const uint64_t i1 = min(span, i0 + kDirectFillSlots);
    for (uint64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) T.slots[i] = kArrayEmpty;
}

__global__ void __launch_bounds__(kBuildThreads)
    k_array_build_grouped(const DirectTask *__restrict__ tasks, uint32_t ntasks) {
    __shared__ uint32_t s_task;
    if (threadIdx.x == 0) s_task = find_direct_task(tasks, ntasks, blockIdx.x, false);
    __syncthreads();
    const DirectTask &T = tasks[s_task];
    unsigned long long *p = T.params;
    if (p[3]) return;
    const uint64_t lo = p[4], span = p[5];
    const uint64_t r0 = (uint64_t)(blockIdx.x - T.key_base) * kDirectBlockRows;
    const uint64_t r1 = min((uint64_t)T.n, r0 + kDirectBlockRows);
    for (uint64_t i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
        int64_t k;
        if (!load_key(T.key, (uint32_t)i, &k)) continue;
        const uint64_t off = (uint64_t)k - lo;
        if (off >= span) continue;
        if (atomicCAS(T.slots + off, kArrayEmpty, (uint32_t)i) != kArrayEmpty) p[3] = 2ull;
    }
}

/* ---- open-addressing table (unique INT32 keys, any spread) ---- */
constexpr unsigned long long kOpenEmpty = ~0ull; /* row 2^32-1 never exists */

__global__ void k_open_fill(unsigned long long *__restrict__ slots, uint64_t nslots) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nslots;
         i += (uint64_t)gridDim.x * blockDim.x)
        slots[i] = kOpenEmpty;
}

/* Each non-NULL key claims the first empty slot from its hash on (at most
 * half the slots fill, so a free one is always found); meeting its own key
 * on the way means the key repeats. A slot is read before it is CASed
 * (slots only go from empty to full, so a full one read from L2 is final):
 * the copies of a heavily repeated key see it taken without hammering one
 * address with atomics, and once a repeat is flagged every thread stops. */
__global__ void k_open_insert(ColView key, uint32_t n, unsigned long long *__restrict__ slots, uint32_t nslots,
                              unsigned long long *dup) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        if (*reinterpret_cast<volatile unsigned long long *>(dup)) return;
        int64_t k;
        if (!load_key(key, (uint32_t)i, &k)) continue;
        const unsigned long long v = ((unsigned long long)(uint32_t)k << 32) | (unsigned long long)i;
        uint32_t h = open_slot(k, nslots);
        for (uint32_t step = 0; step < nslots; ++step) {
            unsigned long long cur = __ldcg(slots + h);
            if (cur == kOpenEmpty) {
                cur = atomicCAS(slots + h, kOpenEmpty, v);
                if (cur == kOpenEmpty) break;
            }
            if ((uint32_t)(cur >> 32) == (uint32_t)k) {
                *dup = 1ull;
                break;
            }
            if (++h == nslots) h = 0;
        }
    }
}

/* cudaFuncSetAttribute applies to the current device only: track which
 * devices have had the limits raised. */
constexpr int kMaxAttrDevices = 64;
std::atomic<bool> g_attrs_set[kMaxAttrDevices];
std::mutex g_attrs_mu;
void set_smem_attrs() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxAttrDevices) {
        cudaGetLastError();
        dev = 0;
    }
    if (g_attrs_set[dev].load(std::memory_order_acquire)) return;
    std::lock_guard<std::mutex> lk(g_attrs_mu);
    if (g_attrs_set[dev].load(std::memory_order_relaxed)) return;
    cudaFuncSetAttribute(k_part_hist, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
    cudaFuncSetAttribute(k_part_scatter<int32_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
    cudaFuncSetAttribute(k_part_scatter<int64_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
    cudaFuncSetAttribute(k_part_build<int32_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
    cudaFuncSetAttribute(k_part_build<int64_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
    cudaFuncSetAttribute(k_part_hist_grouped, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
    cudaFuncSetAttribute(k_part_scatter_grouped, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
    cudaFuncSetAttribute(k_part_build_grouped, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
    cudaFuncSetAttribute(k_part_refine<int32_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
    cudaFuncSetAttribute(k_part_refine<int64_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
    g_attrs_set[dev].store(true, std::memory_order_release);
}

} // namespace

size_t build_temp_bytes(const Launch &L, const BuildPlan &bp, int key_bytes) {
    PartGeom g = geometry(L, bp);
    uint64_t cells = (1ull << g.log2_parts) * g.grid;
    size_t tuple = key_bytes == 4 ? sizeof(Tuple<int32_t>) : sizeof(Tuple<int64_t>);
    size_t b = align256(cells * 4) + align256((cells + 1) * 8) + align256((size_t)bp.num_rows * tuple) +
               scan_temp_bytes(cells) + 256;
    if (bp.log2_parts > g.log2_parts) /* second pass: its output and the partition starts */
        b += align256((size_t)bp.num_rows * tuple) + align256(((1ull << bp.log2_parts) + 1) * 8);
    return b;
}

BuildGeometry build_geometry(const Launch &L, const BuildPlan &bp) {
    PartGeom g = geometry(L, bp);
    BuildGeometry out;
    out.grid = g.grid;
    out.chunk = g.chunk;
    out.cells = (1ull << bp.log2_parts) * g.grid;
    return out;
}

cudaError_t launch_build_grouped(const Launch &L, const BuildTask *tasks_dev, uint32_t ntasks, uint32_t total_chunks,
                                 uint32_t total_parts, uint64_t total_cells, uint32_t max_parts, uint32_t max_slots,
                                 const uint16_t *bloom, void *temp) {
    set_smem_attrs();
    if (!ntasks) return cudaSuccess;
    char *t = reinterpret_cast<char *>(temp);
    uint32_t *matrix = reinterpret_cast<uint32_t *>(t);
    t += align256(total_cells * sizeof(uint32_t));
    uint64_t *offsets = reinterpret_cast<uint64_t *>(t);
    t += align256((total_cells + 1) * sizeof(uint64_t));
    k_part_hist_grouped<<<total_chunks, kPartThreads, max_parts * sizeof(uint32_t), L.stream>>>(tasks_dev, ntasks,
                                                                                                  matrix);
    count_launches(1);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    e = scan_u32_to_u64(L, matrix, offsets, total_cells, t);
    if (e != cudaSuccess) return e;
    k_part_scatter_grouped<<<total_chunks, kPartThreads, max_parts * sizeof(uint32_t), L.stream>>>(
        tasks_dev, ntasks, offsets);
    count_launches(1);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    unsigned grid_b = (unsigned)std::min<uint64_t>(total_parts, (uint64_t)L.num_sms * 16);
    k_part_build_grouped<<<grid_b, kBuildThreads, 2 * max_slots * sizeof(uint32_t), L.stream>>>(
        tasks_dev, ntasks, total_parts, offsets, bloom);
    count_launches(1);
    return cudaGetLastError();
}

size_t build_grouped_temp_bytes(uint64_t total_cells) {
    return align256(total_cells * 4) + align256((total_cells + 1) * 8) + scan_temp_bytes(total_cells) + 256;
}

cudaError_t launch_direct_build(const Launch &L, const ColView &key, uint32_t n, uint64_t max_span, uint32_t *slots,
                                unsigned long long *params) {
    if (n == 0) return cudaSuccess;
    uint64_t g = ((uint64_t)n + kBuildThreads * 8 - 1) / (kBuildThreads * 8);
    g = std::min<uint64_t>(std::max<uint64_t>(g, 1), (uint64_t)L.num_sms * 8);
    k_key_range<<<(unsigned)g, kBuildThreads, 0, L.stream>>>(key, n, params);
    k_array_prep<<<1, 1, 0, L.stream>>>(params, max_span);
    g = std::min<uint64_t>(std::max<uint64_t>((max_span + 255) / 256, 1), (uint64_t)L.num_sms * 8);
    k_array_fill<<<(unsigned)g, 256, 0, L.stream>>>(slots, params);
    g = std::min<uint64_t>(((uint64_t)n + 255) / 256, (uint64_t)L.num_sms * 8);
    k_array_build<<<(unsigned)g, 256, 0, L.stream>>>(key, n, slots, params);
    count_launches(4);
    return cudaGetLastError();
}

cudaError_t launch_direct_build_grouped(const Launch &L, const DirectTask *tasks_dev, uint32_t ntasks,
                                        uint32_t total_key_blocks, uint32_t total_fill_blocks) {
    if (!ntasks) return cudaSuccess;
    if (total_key_blocks) k_key_range_grouped<<<total_key_blocks, kBuildThreads, 0, L.stream>>>(tasks_dev, ntasks);
    k_array_prep_grouped<<<(ntasks + 127) / 128, 128, 0, L.stream>>>(tasks_dev, ntasks);
    if (total_fill_blocks) k_array_fill_grouped<<<total_fill_blocks, kBuildThreads, 0, L.stream>>>(tasks_dev, ntasks);
    if (total_key_blocks) k_array_build_grouped<<<total_key_blocks, kBuildThreads, 0, L.stream>>>(tasks_dev, ntasks);
    count_launches(4);
    return cudaGetLastError();
}

cudaError_t launch_open_build(const Launch &L, const ColView &key, uint32_t n, unsigned long long *slots,
                              uint64_t nslots, unsigned long long *dup) {
    if (nslots < 2ull * n || nslots > 0xFFFFFFFFull) return cudaErrorInvalidValue; /* free slots; u32 indices */
    uint64_t g = std::min<uint64_t>(std::max<uint64_t>((nslots + 255) / 256, 1), (uint64_t)L.num_sms * 8);
    k_open_fill<<<(unsigned)g, 256, 0, L.stream>>>(slots, nslots);
    g = std::min<uint64_t>(std::max<uint64_t>(((uint64_t)n + 255) / 256, 1), (uint64_t)L.num_sms * 8);
    k_open_insert<<<(unsigned)g, 256, 0, L.stream>>>(key, n, slots, (uint32_t)nslots, dup);
    count_launches(2);
    return cudaGetLastError();
}

size_t build_tuple_bytes(int key_bytes) {
    return key_bytes == 4 ? sizeof(Tuple<int32_t>) : sizeof(Tuple<int64_t>);
}

cudaError_t launch_build(const Launch &L, const BuildPlan &bp, const ColView &key,
                         const uint16_t *bloom, uint64_t *dir, void *tuples, void *temp) {
    set_smem_attrs();
    if (key.type == CJ_INT32)
        return build_impl<int32_t>(L, bp, key, bloom, dir, reinterpret_cast<Tuple<int32_t> *>(tuples), temp);
    return build_impl<int64_t>(L, bp, key, bloom, dir, reinterpret_cast<Tuple<int64_t> *>(tuples), temp);
}

} // namespace cj
