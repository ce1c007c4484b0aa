/*
 * k_probe.cu — hash probe and nested-loop join on sm_100a.
 *
 * Both are one persistent kernel over probe tiles of 256 x kItems rows:
 *   - a CTA takes tiles from an atomic ticket;
 *   - each lane handles kItems rows, one dependent chain each (key ->
 *     directory entry -> candidate tuples), kept short and register-light so
 *     that eight CTAs share an SM and their loads overlap;
 *   - for every match count it remembers the first matching build row, so
 *     the common case (at most one match) writes without a second lookup;
 *   - warp scans and a block scan place every row's matches inside the tile,
 *     and one atomicAdd per tile on the match counter reserves the tile's
 *     output range (rows stay in probe order inside a tile);
 *   - the counter ends as the total match count; pairs past the output
 *     capacity are counted but not written, so the caller can size a re-run.
 *
 * Hash probe: Bloom-tag test on the directory entry, then the slot's
 * contiguous tuple range (find_indices, include/join_execution/hashtable.h:
 * 298-313; probe_columnar / probe_intermediate, hash_join.h:87-244). NULL
 * probe keys are skipped (hash_join.h:119, 215-218).
 *
 * Nested loop: the (<= 64) non-NULL build keys sit in shared memory and each
 * warp sweeps them for 32 probe rows at once, the GPU form of the reference's
 * register-resident build side (nested_loop.h:107-244, simd_compare.h:46-163).
 */
#include "cj_device.cuh"

namespace cj {
namespace {

/* 2 rows per thread at 8 CTAs per SM measured fastest on the 4M x 64M
 * workload (825 us vs 870 us for 4 rows, 1218 us for 8 rows at 4 CTAs). */
#ifndef CJ_PROBE_ITEMS
#define CJ_PROBE_ITEMS 2
#endif
#ifndef CJ_PROBE_MIN_BLOCKS
#define CJ_PROBE_MIN_BLOCKS 8
#endif
#ifndef CJ_HASH_MIN_BLOCKS
#define CJ_HASH_MIN_BLOCKS 8
#endif
/* The grouped kernel carries every matcher's code and the shared memory of
 * both tile shapes (35 KB): at 5 CTAs per SM (48 registers, 80 bytes of
 * spills) it ran C4 faster than at 4 (64 registers, no spills) and at 6 (40
 * registers, 252 bytes of spills). The hash matchers alone spill a little at
 * 8 CTAs but ran 11 % slower at 6 without spills: occupancy wins there. */
#ifndef CJ_GROUPED_MIN_BLOCKS
#define CJ_GROUPED_MIN_BLOCKS 5
#endif
constexpr int kProbeThreads = 256;
constexpr int kProbeItems = CJ_PROBE_ITEMS; /* rows per thread (hash, nested loop)      */
/* The grouped kernel's tile: four rows per thread. A usable direct-mapped
 * table probes it at once (ArrayMatcherT<4>, one light chain per row); hash
 * tables and nested loops probe it as two halves of kProbeItems rows per
 * thread, as their own kernels do. */
constexpr int kGroupedItems = 4;
constexpr uint32_t kTileRows = kProbeThreads * kGroupedItems;
static_assert(kGroupedItems == 2 * kProbeItems, "a grouped tile is two hash / nested-loop tiles");
constexpr int kProbeMinBlocks = CJ_PROBE_MIN_BLOCKS; /* 8 x 256 threads = 64 warps/SM */

struct TileSched {
    unsigned int *ticket; /* zeroed before launch */
    uint32_t num_tiles;
};

/* ---------------- matchers ---------------- */

CJ_DEV bool wants_key(const MatchOut &out) { return out.key_pages != nullptr; }

/* The join key of match `pos`, when the caller asked for it, straight into
 * its place in the key columns' result pages: value q sits at byte
 * 4 + 4q + 256 (q / 1984) (INT32: a page is 7936 value bytes and 256
 * others) or 8 + 8q + 136 (q / 1007) (8-byte keys). */
CJ_DEV void put_key(const MatchOut &out, unsigned long long pos, int64_t key) {
    if (!out.key_pages) return;
    const uint64_t q = (uint32_t)pos; /* pos < capacity < 2^32 */
    if (out.key_bytes == 4)
        __stcs(reinterpret_cast<int32_t *>(out.key_pages + 4 + 4 * q + 256 * (q / kRowsPerPageInt32)), (int32_t)key);
    else
        __stcs(reinterpret_cast<long long *>(out.key_pages + 8 + 8 * q + 136 * (q / kRowsPerPage8B)), (long long)key);
}

/* Directory entry word: start of the slot's tuples (bits 63..32), their
 * count (31..16, saturated at 0xFFFF: then the next entry's start bounds
 * them) and the OR of their Bloom tags (15..0). INT32-key tables hold the
 * slot's first tuple in the entry too (DirEntry32, 16 bytes, one sector):
 * a row whose slot has one tuple is answered by that one random load. */
template <typename KB, bool kInlineDir = (sizeof(KB) == 4)> struct HashMatcher {
    static constexpr bool kAtMostOne = false;
    static constexpr bool kInline = kInlineDir && sizeof(KB) == 4;
    /* A probe row whose slot holds more tuples than this is counted and
     * written by its whole warp (warp_count / warp_write), 32 tuples a
     * step, instead of by its own lane alone: a heavy-hitter key with
     * 10^5 build rows costs its warp 10^5 / 32 steps, not one lane 10^5. */
    static constexpr bool kHeavy = true;
    static constexpr uint32_t kHeavyRun = 64;
    static constexpr int kMinBlocks = CJ_HASH_MIN_BLOCKS;
    static constexpr int kItems = kProbeItems;
    CJ_DEV HashMatcher resolved() const { return *this; }
    HashTableView<KB> ht;
    const uint16_t *g_bloom;
    struct Shared {
        uint16_t bloom[2048];
    };
    struct Entry {
        uint32_t s, n;   /* tuple range                      */
        int32_t key0;    /* inline first tuple (INT32 keys)  */
        uint32_t rid0;
    };
    CJ_DEV bool skip() const { return false; }
    CJ_DEV void init(Shared &sh) const { load_bloom(sh.bloom, g_bloom); }
    /* The slot's tuple range, empty when the Bloom tags rule the key out. */
    CJ_DEV Entry entry(const Shared &sh, int64_t key) const {
        const uint64_t h = hash_key(key);
        const uint32_t slot = slot_of(h, ht.log2_slots);
        Entry en{0, 0, 0, 0};
        uint64_t e;
        if (kInline) {
            const uint4 v = __ldg(reinterpret_cast<const uint4 *>(ht.dir) + slot);
            e = (uint64_t)v.x | ((uint64_t)v.y << 32);
            en.key0 = (int32_t)v.z;
            en.rid0 = v.w;
        } else {
            e = __ldg(ht.dir + slot);
        }
        const uint32_t tag = sh.bloom[bloom_index(h)];
        en.s = (uint32_t)(e >> 32);
        if (((uint32_t)e & tag) != tag) return en;
        en.n = (uint32_t)(e >> 16) & 0xFFFFu;
        if (en.n == 0xFFFFu) {
            const uint64_t nx = kInline ? __ldg(reinterpret_cast<const unsigned long long *>(
                                              reinterpret_cast<const DirEntry32 *>(ht.dir) + slot + 1))
                                        : __ldg(ht.dir + slot + 1);
            en.n = (uint32_t)(nx >> 32) - en.s;
        }
        return en;
    }
    /* heavy: the slot is longer than kHeavyRun; the count is left to
     * warp_count (0 returned). */
    CJ_DEV uint32_t count(const Shared &sh, int64_t key, uint32_t &first, uint32_t &second, bool &heavy) const {
        const Entry en = entry(sh, key);
        if (en.n > kHeavyRun) {
            heavy = true;
            return 0;
        }
        uint32_t c = 0, j = 0;
        if (kInline && en.n) { /* tuple 0 came with the entry */
            if ((int64_t)en.key0 == key) {
                first = en.rid0;
                c = 1;
            }
            j = 1;
        }
        for (; j < en.n; ++j) {
            const Tuple<KB> t = ht.tuples[en.s + j];
            if ((int64_t)t.key == key) {
                if (!c) first = t.rid;
                else if (c == 1) second = t.rid;
                ++c;
            }
        }
        return c;
    }
    CJ_DEV void write_all(const Shared &sh, int64_t key, unsigned long long pos, uint32_t prow,
                          const MatchOut &out) const {
        const Entry en = entry(sh, key);
        for (uint32_t j = 0; j < en.n; ++j) {
            const Tuple<KB> t = ht.tuples[en.s + j];
            if ((int64_t)t.key != key) continue;
            if (pos < out.capacity) {
                if (out.build_rids) out.build_rids[pos] = t.rid;
                if (out.probe_rids) out.probe_rids[pos] = prow;
                put_key(out, pos, key);
            }
            ++pos;
        }
    }
    /* Warp-wide (every lane calls it with the same key): the key's matches
     * among its slot's tuples, each lane taking every 32nd tuple. */
    CJ_DEV uint32_t warp_count(const Shared &sh, int64_t key) const {
        const Entry en = entry(sh, key);
        uint32_t c = 0;
        for (uint32_t j = lane_id(); j < en.n; j += 32) c += (int64_t)ht.tuples[en.s + j].key == key ? 1u : 0u;
        return warp_sum(c);
    }
    /* Warp-wide: the key's matches written from `pos` on, in slot order,
     * 32 tuples a step (a ballot places each step's matches). */
    CJ_DEV void warp_write(const Shared &sh, int64_t key, unsigned long long pos, uint32_t prow,
                           const MatchOut &out) const {
        const Entry en = entry(sh, key);
        for (uint32_t j0 = 0; j0 < en.n; j0 += 32) {
            const uint32_t j = j0 + lane_id();
            Tuple<KB> t{};
            bool hit = false;
            if (j < en.n) {
                t = ht.tuples[en.s + j];
                hit = (int64_t)t.key == key;
            }
            const uint32_t b = __ballot_sync(0xffffffffu, hit);
            if (hit) {
                const unsigned long long p = pos + __popc(b & lanemask_lt());
                if (p < out.capacity) {
                    if (out.build_rids) out.build_rids[p] = t.rid;
                    if (out.probe_rids) out.probe_rids[p] = prow;
                    put_key(out, p, key);
                }
            }
            pos += __popc(b);
        }
    }
};

/* Direct-mapped table: slots[key - lo] holds the build row of `key`, or
 * kArrayEmpty. Unique build keys only: a duplicate found while building
 * sets *dup, and a probe launched over such a table does nothing (the
 * caller then builds the hash table instead). */
template <int kItemsT> struct ArrayMatcherT {
    static constexpr bool kAtMostOne = true; /* unique keys: 0 or 1 match per row */
    static constexpr bool kHeavy = false;
    static constexpr int kMinBlocks = kProbeMinBlocks;
    static constexpr int kItems = kItemsT;
    const uint32_t *slots;
    const unsigned long long *params; /* [3] unusable, [4] lo, [5] span */
    uint64_t lo = 0, span = 0;        /* read from params by resolved() */
    struct Shared {
        uint32_t unused;
    };
    CJ_DEV bool skip() const { return params[3] != 0ull; }
    CJ_DEV ArrayMatcherT resolved() const {
        ArrayMatcherT m = *this;
        m.lo = params[4];
        m.span = params[5];
        return m;
    }
    CJ_DEV void init(Shared &) const {}
    CJ_DEV uint32_t count(const Shared &, int64_t key, uint32_t &first) const {
        const uint64_t off = (uint64_t)key - lo; /* keys below lo wrap past span */
        if (off >= span) return 0;
        const uint32_t r = __ldg(slots + off);
        if (r == kArrayEmpty) return 0;
        first = r;
        return 1;
    }
    CJ_DEV void write_all(const Shared &sh, int64_t key, unsigned long long pos, uint32_t prow,
                          const MatchOut &out) const {
        uint32_t r;
        if (count(sh, key, r) && pos < out.capacity) {
            if (out.build_rids) out.build_rids[pos] = r;
            if (out.probe_rids) out.probe_rids[pos] = prow;
            put_key(out, pos, key);
        }
    }
};

/* One light chain per row: 4 rows per thread fit 32 registers (387 us vs
 * 434 us for 2 on 64M probe rows). The grouped kernel's tiles are 2 rows
 * per thread for every matcher (ArrayMatcherT<kProbeItems>). */
using ArrayMatcher = ArrayMatcherT<4>;

/* Open-addressing table of unique INT32 keys (launch_open_build): walk the
 * slots from the key's hash until the key or an empty slot. The walk reads
 * the aligned group of four slots (one 32-byte sector) around its position
 * with two independent 16-byte loads and examines the group's slots from
 * there on, so most rows are answered by one round trip instead of one per
 * slot (the slot count is a multiple of 4: a group never runs past the
 * end). */
struct OpenMatcher {
    static constexpr bool kAtMostOne = true; /* unique keys */
    static constexpr bool kHeavy = false;
    static constexpr int kItems = 4;
    static constexpr int kMinBlocks = kProbeMinBlocks;
    const unsigned long long *slots;
    uint32_t nslots; /* < 2^32 and a multiple of 4 (launch_probe_tiles_open checks) */
    const unsigned long long *dup;
    struct Shared {
        uint32_t unused;
    };
    CJ_DEV bool skip() const { return *dup != 0ull; }
    CJ_DEV OpenMatcher resolved() const { return *this; }
    CJ_DEV void init(Shared &) const {}
    CJ_DEV uint32_t count(const Shared &, int64_t key, uint32_t &first) const {
        if (key != (int64_t)(int32_t)key) return 0; /* no INT32 build key equals it */
        const uint32_t k32 = (uint32_t)(int32_t)key;
        uint32_t h = open_slot(key, nslots);
        for (uint32_t step = 0; step < nslots;) {
            const uint32_t g0 = h & ~3u;
            const ulonglong2 *grp = reinterpret_cast<const ulonglong2 *>(slots + g0);
            const ulonglong2 a = __ldg(grp), b = __ldg(grp + 1);
#pragma unroll
            for (uint32_t q = 0; q < 4; ++q) {
                if (q < (h & 3u)) continue;
                const unsigned long long v = q == 0 ? a.x : q == 1 ? a.y : q == 2 ? b.x : b.y;
                if (v == ~0ull) return 0;
                if ((uint32_t)(v >> 32) == k32) {
                    first = (uint32_t)v;
                    return 1;
                }
                ++step;
            }
            h = g0 + 4;
            if (h >= nslots) h = 0;
        }
        return 0;
    }
    CJ_DEV void write_all(const Shared &sh, int64_t key, unsigned long long pos, uint32_t prow,
                          const MatchOut &out) const {
        uint32_t r;
        if (count(sh, key, r) && pos < out.capacity) {
            if (out.build_rids) out.build_rids[pos] = r;
            if (out.probe_rids) out.probe_rids[pos] = prow;
            put_key(out, pos, key);
        }
    }
};

struct LoopMatcher {
    static constexpr bool kAtMostOne = false;
    static constexpr bool kHeavy = false;
    static constexpr int kMinBlocks = kProbeMinBlocks;
    static constexpr int kItems = kProbeItems;
    CJ_DEV LoopMatcher resolved() const { return *this; }
    const int64_t *g_keys;
    const uint32_t *g_rids;
    const uint32_t *g_count;
    struct Shared {
        int64_t keys[kNestedLoopMax];
        uint32_t rids[kNestedLoopMax];
        uint32_t n;
    };
    CJ_DEV bool skip() const { return false; }
    CJ_DEV void init(Shared &sh) const {
        const uint32_t n = *g_count;
        if (threadIdx.x == 0) sh.n = n;
        for (uint32_t b = threadIdx.x; b < n; b += blockDim.x) {
            sh.keys[b] = g_keys[b];
            sh.rids[b] = g_rids[b];
        }
    }
    CJ_DEV uint32_t count(const Shared &sh, int64_t key, uint32_t &first, uint32_t &second) const {
        uint32_t c = 0;
        for (uint32_t b = 0; b < sh.n; ++b)
            if (sh.keys[b] == key) {
                if (!c) first = sh.rids[b];
                else if (c == 1) second = sh.rids[b];
                ++c;
            }
        return c;
    }
    CJ_DEV void write_all(const Shared &sh, int64_t key, unsigned long long pos, uint32_t prow,
                          const MatchOut &out) const {
        for (uint32_t b = 0; b < sh.n; ++b) {
            if (sh.keys[b] != key) continue;
            if (pos < out.capacity) {
                if (out.build_rids) out.build_rids[pos] = sh.rids[b];
                if (out.probe_rids) out.probe_rids[pos] = prow;
                put_key(out, pos, key);
            }
            ++pos;
        }
    }
};

/* Per-row state between the counting and the writing pass lives in shared
 * memory, not registers, so the kernel fits 32 registers (8 CTAs per SM). */
template <int kItemsT> struct ProbeSmemT {
    static constexpr uint32_t kRows = kProbeThreads * kItemsT;
    uint32_t first[kRows]; /* first matching build row (one- and two-match rows) */
    uint32_t second[kRows]; /* second matching build row (two-match rows)        */
    int64_t key[kRows];    /* the row's key, when the matches carry it   */
    uint32_t pre[kRows];   /* row's match offset within its warp        */
    uint32_t warp[kProbeThreads / 32 + 1];
    uint32_t tile;
    uint32_t task;
    unsigned long long base;
};

/* One probe tile. Block-wide. */
template <class M>
CJ_DEV void probe_tile(const ColView &pkey, uint32_t n, const M &m, const typename M::Shared &sh,
                       const MatchOut &out, uint32_t tile, ProbeSmemT<M::kItems> &ps) {
    constexpr int kItems = M::kItems;
    constexpr uint32_t kRows = ProbeSmemT<M::kItems>::kRows;
    const uint32_t warp = threadIdx.x >> 5, lane = lane_id();
    const uint64_t row0 = (uint64_t)tile * kRows + (uint64_t)warp * 32 * kItems;
    /* 3 bits per item: 0 no match, 1 one, 2 two (both build rows kept), 3
     * more (the write pass walks the slot again), 4 heavy slot (the warp
     * writes it) */
    uint32_t kinds = 0;
    uint32_t wrun = 0;
#pragma unroll
    for (int it = 0; it < kItems; ++it) {
        const uint64_t i = row0 + (uint64_t)it * 32 + lane;
        const uint32_t si = warp * 32 * kItems + it * 32 + lane;
        int64_t key = 0;
        uint32_t c = 0, first = 0, second = 0;
        bool heavy = false;
        if (i < n && load_key_stream(pkey, (uint32_t)i, &key)) {
            if constexpr (M::kHeavy) c = m.count(sh, key, first, second, heavy);
            else if constexpr (!M::kAtMostOne) c = m.count(sh, key, first, second);
            else c = m.count(sh, key, first);
        }
        if constexpr (M::kHeavy) {
            /* the warp counts each heavy row's slot together */
            uint32_t hb = __ballot_sync(0xffffffffu, heavy);
            while (hb) {
                const int L = __ffs(hb) - 1;
                hb &= hb - 1;
                const uint32_t cnt = m.warp_count(sh, (int64_t)__shfl_sync(0xffffffffu, (long long)key, L));
                if ((int)lane == L) c = cnt;
            }
        }
        const uint32_t kind = c == 0 ? 0u : (heavy ? 4u : (c <= 2 ? c : 3u));
        kinds |= kind << (3 * it);
        ps.first[si] = first;
        if (!M::kAtMostOne) ps.second[si] = second;
        if (wants_key(out) && (kind == 1u || kind == 2u)) ps.key[si] = key;
        if (M::kAtMostOne) {
            const uint32_t ball = __ballot_sync(0xffffffffu, c != 0);
            ps.pre[si] = wrun + __popc(ball & lanemask_lt());
            wrun += __popc(ball);
        } else {
            const uint32_t incl = warp_inclusive_scan(c);
            ps.pre[si] = wrun + incl - c;
            wrun += __shfl_sync(0xffffffffu, incl, 31);
        }
    }
    if (lane == 0) ps.warp[warp] = wrun;
    __syncthreads();
    if (warp == 0) {
        const uint32_t w = lane < kProbeThreads / 32 ? ps.warp[lane] : 0u;
        const uint32_t wi = warp_inclusive_scan(w);
        if (lane < kProbeThreads / 32) ps.warp[lane] = wi - w;
        if (lane == 31) {
            ps.base = wi ? atomicAdd(out.counter, (unsigned long long)wi) : 0ull;
        }
    }
    __syncthreads();
    const unsigned long long base = ps.base + ps.warp[warp];
#pragma unroll
    for (int it = 0; it < kItems; ++it) {
        const uint32_t k = (kinds >> (3 * it)) & 7u;
        const uint32_t prow = (uint32_t)(row0 + (uint64_t)it * 32 + lane);
        const uint32_t si = warp * 32 * kItems + it * 32 + lane;
        const unsigned long long pos = base + ps.pre[si];
        if (k == 1 || k == 2) {
            if (pos < out.capacity) {
                if (out.build_rids) out.build_rids[pos] = ps.first[si];
                if (out.probe_rids) out.probe_rids[pos] = prow;
                if (wants_key(out)) put_key(out, pos, ps.key[si]);
            }
            if (!M::kAtMostOne && k == 2 && pos + 1 < out.capacity) {
                if (out.build_rids) out.build_rids[pos + 1] = ps.second[si];
                if (out.probe_rids) out.probe_rids[pos + 1] = prow;
                if (wants_key(out)) put_key(out, pos + 1, ps.key[si]);
            }
        } else if (k == 3) {
            int64_t key;
            load_key(pkey, prow, &key);
            m.write_all(sh, key, pos, prow, out);
        }
        if constexpr (M::kHeavy) {
            /* heavy rows: the warp writes each one's matches together */
            uint32_t hb = __ballot_sync(0xffffffffu, k == 4u);
            while (hb) {
                const int L = __ffs(hb) - 1;
                hb &= hb - 1;
                const uint32_t prow_l = __shfl_sync(0xffffffffu, prow, L);
                const unsigned long long pos_l = __shfl_sync(0xffffffffu, pos, L);
                int64_t key_l = 0;
                load_key(pkey, prow_l, &key_l);
                m.warp_write(sh, key_l, pos_l, prow_l, out);
            }
        }
    }
    __syncthreads();
}

template <class M>
__global__ void __launch_bounds__(kProbeThreads, M::kMinBlocks)
    k_probe_tiles(ColView pkey_arg, uint32_t n, M m_arg, MatchOut out, TileSched ts) {
    __shared__ typename M::Shared sh;
    __shared__ ProbeSmemT<M::kItems> ps;
    if (m_arg.skip()) return;
    const M m = m_arg.resolved();
    const ColView pkey = resolve_view(pkey_arg);
    m.init(sh);
    __syncthreads();
    for (;;) {
        if (threadIdx.x == 0) ps.tile = atomicAdd(ts.ticket, 1u);
        __syncthreads();
        const uint32_t tile = ps.tile;
        if (tile >= ts.num_tiles) break;
        probe_tile(pkey, n, m, sh, out, tile, ps);
    }
}

/* Grouped probe: the tiles of every join of a batch level in one
 * persistent launch; task k owns global tiles [tile_base[k], tile_base[k+1]). */
struct GroupedShared {
    union {
        HashMatcher<int32_t>::Shared h;
        LoopMatcher::Shared l;
    };
};

__global__ void __launch_bounds__(kProbeThreads, CJ_GROUPED_MIN_BLOCKS)
    k_probe_grouped(const ProbeTask *__restrict__ tasks, uint32_t ntasks, uint32_t total_tiles,
                    unsigned int *ticket, const uint16_t *__restrict__ g_bloom) {
    __shared__ GroupedShared sh;
    __shared__ ProbeSmemT<kProbeItems> ps;   /* ticket, task, and the halves' row state */
    __shared__ ProbeSmemT<kGroupedItems> pw; /* row state of a whole-tile direct probe   */
    static_assert(HashMatcher<int32_t>::kItems == kProbeItems && LoopMatcher::kItems == kProbeItems,
                  "hash and nested-loop tasks probe half tiles");
    __shared__ uint32_t loaded_task;
    if (threadIdx.x == 0) loaded_task = 0xffffffffu;
    load_bloom(sh.h.bloom, g_bloom);
    __syncthreads();
    bool bloom_live = true;
    for (;;) {
        if (threadIdx.x == 0) {
            const uint32_t t = atomicAdd(ticket, 1u);
            ps.tile = t;
            uint32_t lo = 0, hi = ntasks;
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
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
        if (T.kind == 2 && T.params[3] == 0ull) {
            /* a direct-mapped table the build found usable (unique keys
             * over a dense range); otherwise the task's hash table below */
            const ArrayMatcherT<kGroupedItems> m = ArrayMatcherT<kGroupedItems>{T.slots, T.params}.resolved();
            ArrayMatcherT<kGroupedItems>::Shared none;
            probe_tile(T.pkey, T.n_probe, m, none, T.out, tile, pw);
        } else if (T.kind == 1) {
            LoopMatcher m{T.nl_keys, T.nl_rids, T.nl_count};
            if (loaded_task != ps.task) {
                __syncthreads();
                m.init(sh.l);
                __syncthreads();
                if (threadIdx.x == 0) loaded_task = ps.task;
                bloom_live = false;
                __syncthreads();
            }
            probe_tile(T.pkey, T.n_probe, m, sh.l, T.out, 2 * tile, ps);
            probe_tile(T.pkey, T.n_probe, m, sh.l, T.out, 2 * tile + 1, ps);
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
                probe_tile(T.pkey, T.n_probe, m, sh.h, T.out, 2 * tile, ps);
                probe_tile(T.pkey, T.n_probe, m, sh.h, T.out, 2 * tile + 1, ps);
            } else {
                HashMatcher<int64_t> m{{T.dir, reinterpret_cast<const Tuple<int64_t> *>(T.tuples), T.log2_slots},
                                       g_bloom};
                const auto &hs = *reinterpret_cast<const HashMatcher<int64_t>::Shared *>(&sh.h);
                probe_tile(T.pkey, T.n_probe, m, hs, T.out, 2 * tile, ps);
                probe_tile(T.pkey, T.n_probe, m, hs, T.out, 2 * tile + 1, ps);
            }
        }
    }
}

/* Compacts the non-NULL build keys (<= 64 rows) in row order. */
CJ_DEV void nl_collect(const ColView &bkey, uint32_t n, int64_t *keys, uint32_t *rids, uint32_t *count,
                       uint32_t *s_w0) {
    const uint32_t i = threadIdx.x;
    int64_t k = 0;
    const bool v = i < n && load_key(bkey, i, &k);
    const uint32_t ball = __ballot_sync(0xffffffffu, v);
    uint32_t off = __popc(ball & lanemask_lt());
    if (threadIdx.x == 31) *s_w0 = __popc(ball);
    __syncthreads();
    if (threadIdx.x >= 32) off += *s_w0;
    if (v) {
        keys[off] = k;
        rids[off] = i;
    }
    if (threadIdx.x == 63) *count = off + (v ? 1u : 0u);
}

__global__ void k_nl_collect(ColView bkey, uint32_t n, int64_t *keys, uint32_t *rids, uint32_t *count) {
    __shared__ uint32_t s_w0;
    nl_collect(bkey, n, keys, rids, count, &s_w0);
}

__global__ void k_nl_collect_grouped(const NlCollectTask *__restrict__ tasks) {
    __shared__ uint32_t s_w0;
    const NlCollectTask &T = tasks[blockIdx.x];
    nl_collect(T.bkey, T.n_build, T.keys, T.rids, T.count, &s_w0);
}

template <class M>
cudaError_t run_tiles(const Launch &L, const ColView &pkey, uint32_t n, const M &m, const MatchOut &out,
                      void *sched_mem) {
    TileSched ts;
    ts.num_tiles = (n + ProbeSmemT<M::kItems>::kRows - 1) / ProbeSmemT<M::kItems>::kRows;
    ts.ticket = reinterpret_cast<unsigned int *>(sched_mem);
    cudaError_t e = cudaMemsetAsync(sched_mem, 0, sizeof(unsigned int), L.stream);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(out.counter, 0, sizeof(unsigned long long), L.stream);
    if (e != cudaSuccess) return e;
    if (n == 0) return cudaSuccess;
    static const int per_sm = [] { /* once per matcher: a driver query per launch costs host time */
        int n = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_probe_tiles<M>, kProbeThreads, 0);
        return n < 1 ? 1 : n;
    }();
    const int ctas = L.ctas_per_sm > 0 && L.ctas_per_sm < per_sm ? L.ctas_per_sm : per_sm;
    uint64_t grid = (uint64_t)L.num_sms * ctas;
    if (grid > ts.num_tiles) grid = ts.num_tiles;
    k_probe_tiles<M><<<(unsigned)grid, kProbeThreads, 0, L.stream>>>(pkey, n, m, out, ts);
    count_launches(1);
    return cudaGetLastError();
}

} // namespace

size_t probe_sched_bytes(uint32_t) { return 256; }

uint32_t probe_tiles(uint32_t n_probe) { return (n_probe + kTileRows - 1) / kTileRows; }

cudaError_t launch_probe_tiles_hash(const Launch &L, const ColView &pkey, uint32_t n_probe, int32_t build_key_type,
                                    const uint64_t *dir, const void *tuples, int log2_slots, const uint16_t *bloom,
                                    const MatchOut &out, void *sched_mem, bool inline_dir) {
    if (build_key_type == CJ_INT32 && inline_dir) {
        HashMatcher<int32_t, true> m{{dir, reinterpret_cast<const Tuple<int32_t> *>(tuples), log2_slots}, bloom};
        return run_tiles(L, pkey, n_probe, m, out, sched_mem);
    }
    if (build_key_type == CJ_INT32) {
        HashMatcher<int32_t, false> m{{dir, reinterpret_cast<const Tuple<int32_t> *>(tuples), log2_slots}, bloom};
        return run_tiles(L, pkey, n_probe, m, out, sched_mem);
    }
    HashMatcher<int64_t> m{{dir, reinterpret_cast<const Tuple<int64_t> *>(tuples), log2_slots}, bloom};
    return run_tiles(L, pkey, n_probe, m, out, sched_mem);
}

cudaError_t launch_probe_tiles_array(const Launch &L, const ColView &pkey, uint32_t n_probe, const uint32_t *slots,
                                     const unsigned long long *params, const MatchOut &out, void *sched_mem) {
    ArrayMatcher m{slots, params};
    return run_tiles(L, pkey, n_probe, m, out, sched_mem);
}

cudaError_t launch_probe_tiles_open(const Launch &L, const ColView &pkey, uint32_t n_probe,
                                    const unsigned long long *slots, uint64_t nslots,
                                    const unsigned long long *dup, const MatchOut &out, void *sched_mem) {
    if (nslots > 0xFFFFFFFFull || nslots % 4 || reinterpret_cast<uintptr_t>(slots) % 16) return cudaErrorInvalidValue;
    OpenMatcher m{slots, (uint32_t)nslots, dup};
    return run_tiles(L, pkey, n_probe, m, out, sched_mem);
}

cudaError_t launch_nl_collect(const Launch &L, const ColView &bkey, uint32_t n_build, int64_t *keys, uint32_t *rids,
                              uint32_t *count) {
    if (n_build > kNestedLoopMax) return cudaErrorInvalidValue;
    k_nl_collect<<<1, 64, 0, L.stream>>>(bkey, n_build, keys, rids, count);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_nl_probe_tiles(const Launch &L, const ColView &pkey, uint32_t n_probe, const int64_t *keys,
                                  const uint32_t *rids, const uint32_t *count, const MatchOut &out,
                                  void *sched_mem) {
    LoopMatcher m{keys, rids, count};
    return run_tiles(L, pkey, n_probe, m, out, sched_mem);
}

cudaError_t launch_probe_grouped(const Launch &L, const ProbeTask *tasks_dev, uint32_t ntasks, uint32_t total_tiles,
                                 unsigned int *ticket, const uint16_t *bloom) {
    if (total_tiles == 0) return cudaSuccess;
    static const int per_sm = [] {
        int n = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_probe_grouped, kProbeThreads, 0);
        return n < 1 ? 1 : n;
    }();
    uint64_t grid = (uint64_t)L.num_sms * per_sm;
    if (grid > total_tiles) grid = total_tiles;
    k_probe_grouped<<<(unsigned)grid, kProbeThreads, 0, L.stream>>>(tasks_dev, ntasks, total_tiles, ticket, bloom);
    count_launches(1);
    return cudaGetLastError();
}

namespace {
__global__ void k_check_counts(const unsigned long long *__restrict__ counts,
                               const unsigned long long *__restrict__ expected, uint32_t n, unsigned int *errors,
                               unsigned long long *detail, uint32_t check_id) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (counts[i] != expected[i]) {
            /* the first mismatch found records where (check, entry) and
             * the two counts */
            if (!(atomicOr(errors, (unsigned int)DEV_ERR_STALE) & DEV_ERR_STALE) && detail) {
                detail[0] = ((unsigned long long)check_id << 32) | i;
                detail[1] = counts[i];
                detail[2] = expected[i];
            }
        }
}
} // namespace

cudaError_t launch_check_counts(const Launch &L, const unsigned long long *counts, const unsigned long long *expected,
                                uint32_t n, unsigned long long *detail, uint32_t check_id) {
    if (!n) return cudaSuccess;
    k_check_counts<<<(n + 255) / 256, 256, 0, L.stream>>>(counts, expected, n, L.dev_errors, detail, check_id);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_nl_collect_grouped(const Launch &L, const NlCollectTask *tasks_dev, uint32_t ntasks) {
    if (!ntasks) return cudaSuccess;
    k_nl_collect_grouped<<<ntasks, 64, 0, L.stream>>>(tasks_dev);
    count_launches(1);
    return cudaGetLastError();
}

} // namespace cj
