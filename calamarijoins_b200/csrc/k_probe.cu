/*
 * k_probe.cu — hash probe and nested-loop join on sm_100a.
 *
 * Both are one persistent kernel over probe tiles (NT x ITEMS rows):
 *   - a CTA takes tiles in order from an atomic ticket, so every earlier
 *     tile is already owned by a running CTA;
 *   - each lane counts the matches of ITEMS rows (keys read once, streamed
 *     with evict-first loads so the hash table stays in L2);
 *   - warp scans and a block scan give every row its offset inside the tile;
 *   - the tile's base offset comes from a decoupled look-back over the
 *     preceding tiles' published totals (bounded wait: a stuck predecessor
 *     sets DEV_ERR_LOOKBACK instead of hanging);
 *   - each lane writes its rows' (build row id, probe row id) pairs.
 * Matches therefore come out in probe-row order with no contended atomic,
 * and the last tile publishes the total match count.
 *
 * Hash probe: Bloom-tag test on the directory entry, then a scan of the
 * slot's contiguous tuple range (find_indices, include/join_execution/
 * hashtable.h:298-313; probe_columnar / probe_intermediate, hash_join.h:
 * 87-244). NULL probe keys are skipped (hash_join.h:119, 215-218).
 *
 * Nested loop: the (<= 64) non-NULL build keys sit in shared memory and
 * every warp sweeps them for 32 probe rows at once, the GPU form of the
 * reference's register-resident build side (nested_loop.h:107-244,
 * simd_compare.h:46-163).
 */
#include "cj_device.cuh"

namespace cj {

namespace {

constexpr int kProbeThreads = 256;
constexpr int kProbeItems = 8;
constexpr uint32_t kTileRows = kProbeThreads * kProbeItems;
constexpr unsigned long long kFlagAgg = 1ull << 62;
constexpr unsigned long long kFlagPre = 2ull << 62;
constexpr unsigned long long kValMask = (1ull << 62) - 1;
constexpr uint64_t kSpinLimit = 1ull << 24;

struct TileSched {
    unsigned int *ticket;         /* zeroed before launch              */
    unsigned long long *status;   /* num_tiles entries, zeroed         */
    uint32_t num_tiles;
};

/* Publishes this tile's aggregate, accumulates the predecessors' and
 * returns the exclusive prefix (single thread). */
CJ_DEV unsigned long long tile_lookback(const TileSched &ts, uint32_t tile, uint32_t agg,
                                        unsigned int *err) {
    if (tile == 0) {
        atomicExch(ts.status, kFlagPre | (unsigned long long)agg);
        return 0;
    }
    atomicExch(ts.status + tile, kFlagAgg | (unsigned long long)agg);
    unsigned long long excl = 0;
    int64_t p = (int64_t)tile - 1;
    uint64_t spins = 0;
    while (p >= 0) {
        unsigned long long v = *reinterpret_cast<volatile unsigned long long *>(ts.status + p);
        unsigned long long f = v & ~kValMask;
        if (f == 0) {
            if (++spins > kSpinLimit) {
                atomicOr(err, DEV_ERR_LOOKBACK);
                break;
            }
            __nanosleep(64);
            continue;
        }
        excl += v & kValMask;
        if (f == kFlagPre) break;
        --p;
    }
    atomicExch(ts.status + tile, kFlagPre | (excl + agg));
    return excl;
}

/* ---------------- matchers ---------------- */
template <typename KB> struct HashMatcher {
    HashTableView<KB> ht;
    const uint16_t *g_bloom;
    struct Shared {
        uint16_t bloom[2048];
    };
    struct State {
        uint32_t s, e;
    };
    CJ_DEV void init(Shared &sh) const { load_bloom(sh.bloom, g_bloom); }
    CJ_DEV uint32_t count(const Shared &sh, int64_t key, State &st) const {
        uint64_t h = hash_key(key);
        uint32_t slot = slot_of(h, ht.log2_slots);
        uint64_t entry = __ldg(ht.dir + slot);
        uint32_t tag = sh.bloom[bloom_index(h)];
        st.s = st.e = 0;
        if ((entry & tag) != tag) return 0;
        st.e = (uint32_t)(entry >> 16);
        st.s = slot ? (uint32_t)(__ldg(ht.dir + slot - 1) >> 16) : 0u;
        uint32_t c = 0;
        for (uint32_t j = st.s; j < st.e; ++j) c += (int64_t)ht.tuples[j].key == key;
        return c;
    }
    CJ_DEV void write(const Shared &, int64_t key, const State &st, unsigned long long pos,
                      uint32_t probe_row, const MatchOut &out) const {
        for (uint32_t j = st.s; j < st.e; ++j) {
            Tuple<KB> t = ht.tuples[j];
            if ((int64_t)t.key != key) continue;
            if (pos < out.capacity) {
                if (out.build_rids) out.build_rids[pos] = t.rid;
                if (out.probe_rids) out.probe_rids[pos] = probe_row;
            }
            ++pos;
        }
    }
};

struct LoopMatcher {
    const int64_t *g_keys;
    const uint32_t *g_rids;
    const uint32_t *g_count;
    struct Shared {
        int64_t keys[kNestedLoopMax];
        uint32_t rids[kNestedLoopMax];
        uint32_t n;
    };
    struct State {};
    CJ_DEV void init(Shared &sh) const {
        uint32_t n = *g_count;
        if (threadIdx.x == 0) sh.n = n;
        for (uint32_t b = threadIdx.x; b < n; b += blockDim.x) {
            sh.keys[b] = g_keys[b];
            sh.rids[b] = g_rids[b];
        }
    }
    CJ_DEV uint32_t count(const Shared &sh, int64_t key, State &) const {
        uint32_t c = 0;
        for (uint32_t b = 0; b < sh.n; ++b) c += sh.keys[b] == key;
        return c;
    }
    CJ_DEV void write(const Shared &sh, int64_t key, const State &, unsigned long long pos,
                      uint32_t probe_row, const MatchOut &out) const {
        for (uint32_t b = 0; b < sh.n; ++b) {
            if (sh.keys[b] != key) continue;
            if (pos < out.capacity) {
                if (out.build_rids) out.build_rids[pos] = sh.rids[b];
                if (out.probe_rids) out.probe_rids[pos] = probe_row;
            }
            ++pos;
        }
    }
};

struct ProbeSmem {
    uint32_t warp[kProbeThreads / 32 + 1];
    uint32_t tile;
    uint32_t task;
    unsigned long long base;
};

/* One probe tile: count, scan, look back, write. Block-wide. */
template <class M>
CJ_DEV void probe_tile(const ColView &pkey, uint32_t n, const M &m, const typename M::Shared &sh,
                       const MatchOut &out, unsigned long long *status, uint32_t num_tiles, uint32_t tile,
                       unsigned int *err, ProbeSmem &ps) {
    const uint32_t warp = threadIdx.x >> 5, lane = lane_id();
    const uint64_t row0 = (uint64_t)tile * kTileRows + (uint64_t)warp * 32 * kProbeItems;
    int64_t key[kProbeItems];
    uint32_t cnt[kProbeItems], pre[kProbeItems];
    typename M::State st[kProbeItems];
    uint32_t wrun = 0;
#pragma unroll
    for (int it = 0; it < kProbeItems; ++it) {
        uint64_t i = row0 + (uint64_t)it * 32 + lane;
        cnt[it] = 0;
        key[it] = 0;
        if (i < n && load_key_stream(pkey, (uint32_t)i, &key[it])) cnt[it] = m.count(sh, key[it], st[it]);
        uint32_t incl = warp_inclusive_scan(cnt[it]);
        pre[it] = wrun + incl - cnt[it];
        wrun += __shfl_sync(0xffffffffu, incl, 31);
    }
    if (lane == 0) ps.warp[warp] = wrun;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < kProbeThreads / 32 ? ps.warp[lane] : 0u;
        uint32_t wi = warp_inclusive_scan(w);
        if (lane < kProbeThreads / 32) ps.warp[lane] = wi - w;
        if (lane == 31) ps.warp[kProbeThreads / 32] = wi;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        TileSched ts{nullptr, status, num_tiles};
        uint32_t agg = ps.warp[kProbeThreads / 32];
        unsigned long long b = tile_lookback(ts, tile, agg, err);
        ps.base = b;
        if (tile == num_tiles - 1) *out.counter = b + agg;
    }
    __syncthreads();
    const unsigned long long base = ps.base + ps.warp[warp];
#pragma unroll
    for (int it = 0; it < kProbeItems; ++it) {
        if (!cnt[it]) continue;
        uint64_t i = row0 + (uint64_t)it * 32 + lane;
        m.write(sh, key[it], st[it], base + pre[it], (uint32_t)i, out);
    }
    __syncthreads();
}

template <class M>
__global__ void __launch_bounds__(kProbeThreads)
    k_probe_tiles(ColView pkey, uint32_t n, M m, MatchOut out, TileSched ts, unsigned int *err) {
    __shared__ typename M::Shared sh;
    __shared__ ProbeSmem ps;
    m.init(sh);
    __syncthreads();
    for (;;) {
        if (threadIdx.x == 0) ps.tile = atomicAdd(ts.ticket, 1u);
        __syncthreads();
        const uint32_t tile = ps.tile;
        if (tile >= ts.num_tiles) break;
        probe_tile(pkey, n, m, sh, out, ts.status, ts.num_tiles, tile, err, ps);
    }
}

/* Grouped probe: the tiles of every join of a batch level in one
 * persistent launch. Task k owns global tiles [tile_base[k],
 * tile_base[k+1]); tickets are global, so a tile's predecessors in its
 * own join always hold earlier tickets. */
struct GroupedShared {
    union {
        HashMatcher<int32_t>::Shared h;
        LoopMatcher::Shared l;
    };
};

__global__ void __launch_bounds__(kProbeThreads)
    k_probe_grouped(const ProbeTask *__restrict__ tasks, uint32_t ntasks, uint32_t total_tiles,
                    unsigned int *ticket, const uint16_t *__restrict__ g_bloom, unsigned int *err) {
    __shared__ GroupedShared sh;
    __shared__ ProbeSmem ps;
    __shared__ uint32_t loaded_task;
    if (threadIdx.x == 0) loaded_task = 0xffffffffu;
    load_bloom(sh.h.bloom, g_bloom);
    __syncthreads();
    bool bloom_live = true;
    for (;;) {
        if (threadIdx.x == 0) {
            uint32_t t = atomicAdd(ticket, 1u);
            ps.tile = t;
            /* task = last k with tile_base[k] <= t */
            uint32_t lo = 0, hi = ntasks;
            while (hi - lo > 1) {
                uint32_t mid = (lo + hi) >> 1;
                if (tasks[mid].tile_base <= t) lo = mid;
                else hi = mid;
            }
            ps.task = lo;
        }
        __syncthreads();
        const uint32_t gt = ps.tile;
        if (gt >= total_tiles) break;
        const ProbeTask &T = tasks[ps.task];
        const uint32_t tile = gt - T.tile_base;
        if (T.kind == 1) {
            LoopMatcher m{T.nl_keys, T.nl_rids, T.nl_count};
            if (loaded_task != ps.task) {
                __syncthreads();
                m.init(sh.l);
                __syncthreads();
                if (threadIdx.x == 0) loaded_task = ps.task;
                bloom_live = false;
                __syncthreads();
            }
            probe_tile(T.pkey, T.n_probe, m, sh.l, T.out, T.status, T.num_tiles, tile, err, ps);
        } else {
            if (!bloom_live) {
                __syncthreads();
                load_bloom(sh.h.bloom, g_bloom);
                if (threadIdx.x == 0) loaded_task = 0xffffffffu;
                bloom_live = true;
                __syncthreads();
            }
            if (T.build_key_type == CJ_INT32) {
                HashMatcher<int32_t> m{{T.dir, reinterpret_cast<const Tuple<int32_t> *>(T.tuples), T.log2_slots},
                                       g_bloom};
                probe_tile(T.pkey, T.n_probe, m, sh.h, T.out, T.status, T.num_tiles, tile, err, ps);
            } else {
                HashMatcher<int64_t> m{{T.dir, reinterpret_cast<const Tuple<int64_t> *>(T.tuples), T.log2_slots},
                                       g_bloom};
                probe_tile(T.pkey, T.n_probe, m,
                           *reinterpret_cast<const HashMatcher<int64_t>::Shared *>(&sh.h), T.out, T.status,
                           T.num_tiles, tile, err, ps);
            }
        }
    }
}

/* Compacts the non-NULL build keys (<= 64 rows) in row order. */
__global__ void k_nl_collect(ColView bkey, uint32_t n, int64_t *keys, uint32_t *rids,
                             uint32_t *count) {
    __shared__ uint32_t s_w0;
    const uint32_t i = threadIdx.x;
    int64_t k = 0;
    bool v = i < n && load_key(bkey, i, &k);
    uint32_t ball = __ballot_sync(0xffffffffu, v);
    uint32_t off = __popc(ball & lanemask_lt());
    if (threadIdx.x == 31) s_w0 = __popc(ball);
    __syncthreads();
    if (threadIdx.x >= 32) off += s_w0;
    if (v) {
        keys[off] = k;
        rids[off] = i;
    }
    if (threadIdx.x == 63) *count = off + (v ? 1u : 0u);
}

} // namespace

static size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

size_t probe_sched_bytes(uint32_t n_probe) {
    uint32_t tiles = (n_probe + kTileRows - 1) / kTileRows;
    return 256 + align256((size_t)tiles * sizeof(unsigned long long));
}

template <class M>
static cudaError_t run_tiles(const Launch &L, const ColView &pkey, uint32_t n, const M &m,
                             const MatchOut &out, void *sched_mem) {
    TileSched ts;
    ts.num_tiles = (n + kTileRows - 1) / kTileRows;
    ts.ticket = reinterpret_cast<unsigned int *>(sched_mem);
    ts.status = reinterpret_cast<unsigned long long *>(reinterpret_cast<char *>(sched_mem) + 256);
    cudaError_t e = cudaMemsetAsync(sched_mem, 0, probe_sched_bytes(n), L.stream);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(out.counter, 0, sizeof(unsigned long long), L.stream);
    if (e != cudaSuccess) return e;
    if (n == 0) return cudaSuccess;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_probe_tiles<M>, kProbeThreads, 0);
    if (per_sm < 1) per_sm = 1;
    uint64_t grid = (uint64_t)L.num_sms * per_sm;
    if (grid > ts.num_tiles) grid = ts.num_tiles;
    k_probe_tiles<M><<<(unsigned)grid, kProbeThreads, 0, L.stream>>>(pkey, n, m, out, ts, L.dev_errors);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_probe_tiles_hash(const Launch &L, const ColView &pkey, uint32_t n_probe,
                                    int32_t build_key_type, const uint64_t *dir,
                                    const void *tuples, int log2_slots, const uint16_t *bloom,
                                    const MatchOut &out, void *sched_mem) {
    if (build_key_type == CJ_INT32) {
        HashMatcher<int32_t> m{{dir, reinterpret_cast<const Tuple<int32_t> *>(tuples), log2_slots}, bloom};
        return run_tiles(L, pkey, n_probe, m, out, sched_mem);
    }
    HashMatcher<int64_t> m{{dir, reinterpret_cast<const Tuple<int64_t> *>(tuples), log2_slots}, bloom};
    return run_tiles(L, pkey, n_probe, m, out, sched_mem);
}

cudaError_t launch_nl_collect(const Launch &L, const ColView &bkey, uint32_t n_build,
                              int64_t *keys, uint32_t *rids, uint32_t *count) {
    if (n_build > kNestedLoopMax) return cudaErrorInvalidValue;
    k_nl_collect<<<1, 64, 0, L.stream>>>(bkey, n_build, keys, rids, count);
    count_launches(1);
    return cudaGetLastError();
}

uint32_t probe_tiles(uint32_t n_probe) { return (n_probe + kTileRows - 1) / kTileRows; }

cudaError_t launch_probe_grouped(const Launch &L, const ProbeTask *tasks_dev, uint32_t ntasks, uint32_t total_tiles,
                                 unsigned int *ticket, const uint16_t *bloom) {
    if (total_tiles == 0) return cudaSuccess;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_probe_grouped, kProbeThreads, 0);
    if (per_sm < 1) per_sm = 1;
    uint64_t grid = (uint64_t)L.num_sms * per_sm;
    if (grid > total_tiles) grid = total_tiles;
    k_probe_grouped<<<(unsigned)grid, kProbeThreads, 0, L.stream>>>(tasks_dev, ntasks, total_tiles, ticket, bloom,
                                                                       L.dev_errors);
    count_launches(1);
    return cudaGetLastError();
}

__global__ void k_nl_collect_grouped(const NlCollectTask *__restrict__ tasks) {
    const NlCollectTask &T = tasks[blockIdx.x];
    __shared__ uint32_t s_w0;
    const uint32_t i = threadIdx.x;
    int64_t k = 0;
    bool v = i < T.n_build && load_key(T.bkey, i, &k);
    uint32_t ball = __ballot_sync(0xffffffffu, v);
    uint32_t off = __popc(ball & lanemask_lt());
    if (threadIdx.x == 31) s_w0 = __popc(ball);
    __syncthreads();
    if (threadIdx.x >= 32) off += s_w0;
    if (v) {
        T.keys[off] = k;
        T.rids[off] = i;
    }
    if (threadIdx.x == 63) *T.count = off + (v ? 1u : 0u);
}

cudaError_t launch_nl_collect_grouped(const Launch &L, const NlCollectTask *tasks_dev, uint32_t ntasks) {
    if (!ntasks) return cudaSuccess;
    k_nl_collect_grouped<<<ntasks, 64, 0, L.stream>>>(tasks_dev);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_nl_probe_tiles(const Launch &L, const ColView &pkey, uint32_t n_probe,
                                  const int64_t *keys, const uint32_t *rids,
                                  const uint32_t *count, const MatchOut &out, void *sched_mem) {
    LoopMatcher m{keys, rids, count};
    return run_tiles(L, pkey, n_probe, m, out, sched_mem);
}

} // namespace cj
