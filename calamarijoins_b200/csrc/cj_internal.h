/*
 * cj_internal.h — types shared by the host engine and the sm_100a kernels.
 *
 * Device data layout (all in HBM, one allocation per array):
 *   pages        a column's 8 KiB pages, consecutive, exactly as on the host
 *   row_start    u64[num_pages + 1], first row of each page (prefix sum of
 *                the rows each page holds: n_rows, 1 for a long-string start
 *                page 0xffff, 0 for a continuation page 0xfffe)
 *   values       dense fixed-width values, one per row (0 where NULL)
 *   valid        validity bitmap, u32 words, bit r = row r present
 *   str_desc     VARCHAR: one u64 per row, see CJ_DESC_* below
 *   rid vectors  u32 row ids (late materialisation of intermediates)
 *   hash table   u64 directory ((end << 16) | 16-bit Bloom tag) and a
 *                slot-ordered tuple array {key, row id}
 */
#pragma once

#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

#include "../../include/cj_b200.h"

namespace cj {

constexpr uint32_t kPageSize = CJ_PAGE_SIZE;
constexpr uint32_t kMaxShortString = kPageSize - 7; /* plan.h:331 */
constexpr uint32_t kLongChunk = kPageSize - 4;      /* plan.h:301 */
constexpr uint32_t kRowsPerPageInt32 = 1984;        /* ColumnInserter<int32_t> fill */
constexpr uint32_t kRowsPerPage8B = 1007;           /* ColumnInserter<int64_t/double> */

/* VARCHAR row descriptor.
 *   short string: bit 63 = 0, bits 62..24 = byte offset of the first
 *                 character inside the column's page blob, bits 23..0 =
 *                 length (<= 8185)
 *   long string:  bit 63 = 1, bits 62..24 = index of its 0xffff page,
 *                 bits 23..0 = number of pages in the chain (the 0xffff
 *                 page and the 0xfffe pages that follow it)
 *   NULL rows hold 0 (the validity bitmap says NULL). */
constexpr uint64_t CJ_DESC_LONG = 1ull << 63;
__host__ __device__ inline uint64_t desc_short(uint64_t off, uint32_t len) {
    return (off << 24) | len;
}
__host__ __device__ inline uint64_t desc_long(uint64_t page, uint32_t chain) {
    return CJ_DESC_LONG | (page << 24) | chain;
}
__host__ __device__ inline bool desc_is_long(uint64_t d) { return (d >> 63) != 0; }
__host__ __device__ inline uint64_t desc_pos(uint64_t d) { return (d >> 24) & ((1ull << 39) - 1); }
__host__ __device__ inline uint32_t desc_len(uint64_t d) { return (uint32_t)(d & 0xFFFFFFu); }

/* Error bits the kernels raise in the device status word. */
enum DevError : uint32_t {
    DEV_ERR_PAGE_HEADER = 1u << 0,   /* n_values > n_rows or page overflow */
    DEV_ERR_VARCHAR_OFFSETS = 1u << 1,
    DEV_ERR_LONG_CHAIN = 1u << 2,    /* 0xfffe page without a 0xffff start */
    DEV_ERR_BAD_PAGE_KIND = 1u << 3, /* 0xffff/0xfffe page in a fixed column */
    DEV_ERR_ROW_COUNT = 1u << 5,     /* pages hold more/fewer rows than the
                                        table declares                       */
    DEV_ERR_STALE = 1u << 6,         /* a prepared batch's counts no longer
                                        match its inputs                     */
    DEV_ERR_INTERNAL = 1u << 31
};

/* Small pinned block the host reads at each synchronisation point. */
struct StatusBlock {
    unsigned int errors;          /* DevError bits                          */
    unsigned int pad;
    unsigned long long counter;   /* match counter of the last probe        */
    unsigned long long aux[8];    /* [0, kDirectParams): direct-mapped table
                                     parameters; [kOpenDup]: a repeated key
                                     in the open-addressing table          */
    unsigned long long stale[3];  /* DEV_ERR_STALE: check index, count found,
                                     count recorded (one of the mismatches) */
};

/* How a kernel reads one column of a relation: row i of the relation is
 * row rid_b[rid_a[i]] of the decoded base column (each indirection is
 * skipped when its pointer is null). */
struct ColView {
    const void *values;
    const uint32_t *valid;
    const uint64_t *str_desc;
    const uint8_t *pages;
    const uint32_t *rid_a;
    const uint32_t *rid_b;
    int32_t type;
    int32_t null_sentinel; /* INT32: INT32_MIN reads as NULL (value_t) */
    const uint32_t *col_flags; /* device word of COL_* bits from the page
                                  headers; null: unknown (read the decoded
                                  values and validity)                   */
};

/* Column flags, set by the page-row pass. A fixed-width column whose word
 * is 0 has no NULL and every page but the last holds exactly
 * kRowsPerPageInt32 / kRowsPerPage8B rows (the fill of the reference's
 * ColumnInserter): row r is value r % R of page r / R, so it is read from
 * the pages and not decoded at all. */
enum ColFlag : uint32_t {
    COL_HAS_NULLS = 1u,  /* some page stores fewer values than rows      */
    COL_NOT_DIRECT = 2u, /* VARCHAR, or pages not filled as above        */
};

template <typename K> struct Tuple;
template <> struct alignas(8) Tuple<int32_t> {
    int32_t key;
    uint32_t rid;
};
template <> struct alignas(16) Tuple<int64_t> {
    int64_t key;
    uint32_t rid;
    uint32_t pad;
};

/* Directory entry of a table with INT32 keys: the entry word (start of the
 * slot's tuples << 32 | count << 16 | Bloom tags) and the slot's first
 * tuple inline, 16 bytes in one sector: a probe row whose slot holds one
 * tuple needs one random access. Tables with INT64 keys keep 8-byte entries
 * (the word alone). */
struct alignas(16) DirEntry32 {
    uint64_t word;
    int32_t key0;
    uint32_t rid0;
};

template <typename K> struct HashTableView {
    const uint64_t *dir; /* DirEntry32[] for K = int32_t, entry words for int64_t */
    const Tuple<K> *tuples;
    int log2_slots;
};

/* Output of a probe / nested-loop launch. */
struct MatchOut {
    uint32_t *build_rids = nullptr; /* null: not collected (RIGHT_ONLY)  */
    uint32_t *probe_rids = nullptr; /* null: not collected (LEFT_ONLY)   */
    uint8_t *key_pages = nullptr;   /* null, or the join key written straight
                                       into 8 KiB result pages: value pos % R
                                       of page pos / R (R = 1984 or 1007 by
                                       key_bytes); launch_finish_dense_pages
                                       adds headers and bitmaps */
    int32_t key_bytes = 4;
    unsigned long long capacity = 0;
    unsigned long long *counter = nullptr;
};

/* Kernels launched by this process (every launcher adds its launches). */
void count_launches(uint64_t n);
uint64_t launches_so_far();

/* ----------------------------------------------------------------------- */
/* Kernel launchers (defined in the .cu files; all enqueue on `s`).         */
/* ----------------------------------------------------------------------- */
struct Launch {
    cudaStream_t stream;
    int num_sms;
    int block_threads; /* 0 = kernel default */
    unsigned int *dev_errors;
    int ctas_per_sm = 0;      /* persistent probe grids: CTAs per SM (0 = as many as fit) */
    int part_ctas_per_sm = 0; /* radix histogram / scatter passes: CTAs per SM (0 = 4)     */
};

/* Tuned launch parameters per size class of a relation's row count (the
 * autotuner's table). Classes split at 2^12, 2^15, 2^18, 2^21 and 2^24
 * rows. A zero entry means "the default". */
constexpr int kTuneClasses = 6;
inline int tune_class(uint64_t rows) {
    int c = 0;
    for (int t : {12, 15, 18, 21, 24})
        if (rows >= (1ull << t)) ++c;
    return c;
}
struct TuneEntry {
    int log2_spp = 0;    /* hash directory slots per radix partition (log2) */
    int part_ctas = 0;   /* radix passes: CTAs per SM                        */
    int probe_ctas = 0;  /* hash probe: CTAs per SM                          */
};
struct Tuning {
    bool loaded = false;
    TuneEntry cls[kTuneClasses];
    const TuneEntry &for_rows(uint64_t rows) const { return cls[tune_class(rows)]; }
};

/* Scan */
size_t scan_temp_bytes(size_t n);
/* out[i] = sum(in[0..i)), out[n] = total; in and out may not alias. */
cudaError_t scan_u32_to_u64(const Launch &L, const uint32_t *in, uint64_t *out,
                            size_t n, void *temp);

/* Decode */
/* Page index of one column: rows_pp[p] = rows of page p, row_start[p] =
 * rows before page p (row_start[num_pages] = total; only the total when
 * the column is read in place), state[0] |= the column's COL_* flags;
 * a total other than `rows` raises DEV_ERR_ROW_COUNT and sets
 * COL_NOT_DIRECT. state (2 words) must be zero; partials holds
 * page_index_blocks(num_pages) entries. Two launches. */
uint64_t page_index_blocks(const Launch &L, uint64_t num_pages);
cudaError_t launch_page_index(const Launch &L, const uint8_t *pages, uint64_t num_pages, int32_t type,
                              uint64_t rows, uint32_t *rows_pp, uint64_t *partials, uint64_t *row_start,
                              uint32_t *state);
/* Rows past max_rows are never written; a page that would write them
 * raises DEV_ERR_ROW_COUNT instead. Does nothing when *col_flags is 0
 * (readers then take the values from the pages). */
cudaError_t launch_decode_fixed(const Launch &L, const uint8_t *pages,
                                uint64_t num_pages, int32_t type,
                                const uint64_t *row_start, uint64_t max_rows,
                                void *values, uint32_t *valid, const uint32_t *col_flags);
cudaError_t launch_decode_varchar(const Launch &L, const uint8_t *pages,
                                  uint64_t num_pages,
                                  const uint64_t *row_start, uint64_t max_rows,
                                  uint64_t *desc, uint32_t *valid);
/* Grouped decode of many columns: task k's pages are global pages
 * [page_base, page_base + num_pages). rows_pp / row_start are scratch of
 * total_pages / total_pages + 1 entries; scan_temp of
 * scan_temp_bytes(total_pages). */
struct DecodeTask {
    const uint8_t *pages;
    uint64_t num_pages;
    uint64_t page_base;
    uint64_t rows;
    int32_t type;
    int32_t pad;
    void *values;
    uint64_t *desc;
    uint32_t *valid; /* zeroed */
};
cudaError_t launch_decode_grouped(const Launch &L, const DecodeTask *tasks_dev, uint32_t ntasks,
                                  uint64_t total_pages, uint32_t *rows_pp, uint64_t *row_start,
                                  void *scan_temp);

/* Build */
struct BuildPlan {
    int log2_slots;      /* directory = 2^log2_slots entries + 1          */
    int log2_parts;      /* radix partition bits in all: one pass up to 12
                            bits, two passes above (launch_build)         */
    uint32_t num_rows;   /* rows of the build relation                    */
    bool inline_first = true; /* INT32 keys: 16-byte entries holding the
                                 slot's first tuple (DirEntry32), else the
                                 8-byte word alone                        */
};
/* Directory entry word: start (63..32) | count (31..16, saturated) | tags
 * (15..0); INT32 keys add the first tuple (DirEntry32); one sentinel entry
 * after the last slot. */
inline size_t build_dir_bytes(int log2_slots, int key_bytes, bool inline_first = true) {
    return ((1ull << log2_slots) + 1) * (key_bytes == 4 && inline_first ? sizeof(DirEntry32) : sizeof(uint64_t));
}
size_t build_temp_bytes(const Launch &L, const BuildPlan &bp, int key_bytes);
size_t build_tuple_bytes(int key_bytes);
cudaError_t launch_build(const Launch &L, const BuildPlan &bp, const ColView &key,
                         const uint16_t *bloom, uint64_t *dir, void *tuples,
                         void *temp);

/* Grouped build over the hash joins of one batch level. Each task
 * partitions its own rows into its own part_buf; chunk_base / part_base /
 * cell_base place its chunks, partitions and histogram cells in the global
 * numbering (prefix sums over the tasks). */
struct BuildGeometry {
    uint32_t grid;  /* chunks of the hist / scatter passes */
    uint32_t chunk; /* rows per chunk                      */
    uint64_t cells; /* partitions x chunks                 */
};
BuildGeometry build_geometry(const Launch &L, const BuildPlan &bp);
struct BuildTask {
    ColView key;
    uint32_t n;
    int32_t log2_slots;
    int32_t log2_parts;
    uint32_t grid;
    uint32_t chunk;
    uint32_t chunk_base;
    uint32_t part_base;
    uint64_t cell_base;
    uint64_t *dir;
    void *tuples;
    void *part_buf; /* n tuples of scratch */
};
size_t build_grouped_temp_bytes(uint64_t total_cells);
cudaError_t launch_build_grouped(const Launch &L, const BuildTask *tasks_dev, uint32_t ntasks, uint32_t total_chunks,
                                 uint32_t total_parts, uint64_t total_cells, uint32_t max_parts, uint32_t max_slots,
                                 const uint16_t *bloom, void *temp);

/* Direct-mapped build for unique keys spread densely over [lo, lo + span):
 * slots[key - lo] = build row, decided on the device. `params` (6 u64, set
 * by the caller to {~0, 0, 0, 0, 0, 0}) receives [0] min and [1] max of the
 * non-NULL keys (XOR 2^63: unsigned order is signed order), [2] their count,
 * [3] non-zero when the table cannot be used (1: span above max_span, 2: a
 * repeated key), [4] lo, [5] span. `slots` holds max_span entries. Four launches, no
 * host round trip. */
constexpr uint32_t kArrayEmpty = 0xFFFFFFFFu;
constexpr int kDirectParams = 6;
cudaError_t launch_direct_build(const Launch &L, const ColView &key, uint32_t n, uint64_t max_span, uint32_t *slots,
                                unsigned long long *params);
/* Probe of a direct-mapped table; does nothing when params[3] is set. */
cudaError_t launch_probe_tiles_array(const Launch &L, const ColView &pkey, uint32_t n_probe, const uint32_t *slots,
                                     const unsigned long long *params, const MatchOut &out, void *sched);

/* Open-addressing table for unique INT32 build keys too spread out for a
 * direct-mapped table: `nslots` 8-byte slots (key << 32 | build row, all
 * ones when empty; at most half of them full), linear probing from the
 * key's hash scaled to [0, nslots). The build sets *dup when a key repeats
 * (the table cannot be used); the probe then does nothing. Two launches. */
constexpr int kOpenDup = kDirectParams;
constexpr uint64_t kOpenMaxRows = 1ull << 28;
cudaError_t launch_open_build(const Launch &L, const ColView &key, uint32_t n, unsigned long long *slots,
                              uint64_t nslots, unsigned long long *dup);
cudaError_t launch_probe_tiles_open(const Launch &L, const ColView &pkey, uint32_t n_probe,
                                    const unsigned long long *slots, uint64_t nslots,
                                    const unsigned long long *dup, const MatchOut &out, void *sched);

/* Probe and nested loop share one tiled kernel; `sched` is scratch of
 * probe_sched_bytes(n_probe) bytes (the tile ticket). */
size_t probe_sched_bytes(uint32_t n_probe);
/* inline_dir: the table was built with BuildPlan::inline_first (INT32
 * keys only; ignored for INT64). */
cudaError_t launch_probe_tiles_hash(const Launch &L, const ColView &pkey, uint32_t n_probe,
                                    int32_t build_key_type, const uint64_t *dir,
                                    const void *tuples, int log2_slots, const uint16_t *bloom,
                                    const MatchOut &out, void *sched, bool inline_dir = true);

/* Nested loop (build side <= 64 rows) */
constexpr uint32_t kNestedLoopMax = 64;
cudaError_t launch_nl_collect(const Launch &L, const ColView &bkey, uint32_t n_build,
                              int64_t *keys, uint32_t *rids, uint32_t *count);
cudaError_t launch_nl_probe_tiles(const Launch &L, const ColView &pkey, uint32_t n_probe,
                                  const int64_t *keys, const uint32_t *rids,
                                  const uint32_t *count, const MatchOut &out, void *sched);

/* Grouped probe over the joins of one batch level. */
struct ProbeTask {
    ColView pkey;
    uint32_t n_probe;
    int32_t kind;           /* 0 hash, 1 nested loop, 2 direct-mapped table
                               when usable (params[3] == 0), else hash     */
    int32_t build_key_type; /* hash: CJ_INT32 / CJ_INT64 tuples            */
    int32_t log2_slots;
    const uint64_t *dir;
    const void *tuples;
    const int64_t *nl_keys;
    const uint32_t *nl_rids;
    const uint32_t *nl_count;
    const uint32_t *slots;              /* kind 2: direct-mapped table      */
    const unsigned long long *params;   /* kind 2: its kDirectParams words  */
    MatchOut out;               /* out.counter zeroed before launch         */
    uint32_t num_tiles;
    uint32_t tile_base;         /* first global tile of this task           */
};
/* Grouped direct-mapped builds (launch_direct_build for every task): task k
 * owns blocks [block_base, block_base + blocks) of each pass; params hold
 * kDirectParams words per task, set to {~0, 0, 0, 0, 0, 0} before. */
struct DirectTask {
    ColView key;
    uint32_t n;
    uint32_t key_blocks;   /* blocks over the keys                         */
    uint32_t key_base;
    uint32_t fill_blocks;  /* blocks over max_span slots                   */
    uint32_t fill_base;
    uint64_t max_span;
    uint32_t *slots;
    unsigned long long *params;
};
cudaError_t launch_direct_build_grouped(const Launch &L, const DirectTask *tasks_dev, uint32_t ntasks,
                                        uint32_t total_key_blocks, uint32_t total_fill_blocks);
constexpr uint32_t kDirectBlockRows = 256 * 8; /* key rows per block of the grouped passes */
constexpr uint32_t kDirectFillSlots = 256 * 16; /* slots per block of the grouped fill     */
uint32_t probe_tiles(uint32_t n_probe);
/* `ticket` must be zeroed, and each task's counter. */
cudaError_t launch_probe_grouped(const Launch &L, const ProbeTask *tasks_dev, uint32_t ntasks,
                                 uint32_t total_tiles, unsigned int *ticket, const uint16_t *bloom);
struct NlCollectTask {
    ColView bkey;
    uint32_t n_build;
    int64_t *keys;
    uint32_t *rids;
    uint32_t *count;
};
cudaError_t launch_nl_collect_grouped(const Launch &L, const NlCollectTask *tasks_dev, uint32_t ntasks);

/* Raises DEV_ERR_STALE unless counts[i] == expected[i] for every i < n. */
cudaError_t launch_check_counts(const Launch &L, const unsigned long long *counts,
                                const unsigned long long *expected, uint32_t n,
                                unsigned long long *detail, uint32_t check_id);

/* Headers (n_rows = n_values), zero gaps and all-ones bitmaps of the
 * ceil(rows / R) pages of a NULL-free fixed-width column whose values are
 * already in place (R by type, as rows_per_page_fixed). */
/* The page writers below take `rows` as the rows to write, or, with
 * `rows_dev` set, as the capacity the pages were sized for while the count
 * itself is read on the device from *rows_dev (a match counter the host has
 * not read yet). */
cudaError_t launch_finish_dense_pages(const Launch &L, uint8_t *pages, uint64_t rows, int32_t type,
                                      const unsigned long long *rows_dev = nullptr);

/* Intermediates: out[i] = src[idx[i]] */
cudaError_t launch_gather_u32(const Launch &L, const uint32_t *src,
                              const uint32_t *idx, uint64_t n, uint32_t *out);

/* Grouped variants for batches: each task's units are numbered from
 * page_base / chunk_base in a global sequence (prefix sums over tasks). */
constexpr uint64_t kGatherChunk = 8192;
struct GatherTask {
    const uint32_t *src;
    const uint32_t *idx;
    uint32_t *out;
    uint64_t n;
    uint64_t chunk_base;
};
cudaError_t launch_gather_grouped(const Launch &L, const GatherTask *tasks_dev, uint32_t ntasks,
                                  uint64_t total_chunks);
struct PageTask {
    ColView col;
    uint64_t rows;
    uint8_t *out;
    uint64_t page_base;
};
cudaError_t launch_write_fixed_grouped(const Launch &L, const PageTask *tasks_dev, uint32_t ntasks,
                                      uint64_t total_pages);

/* Output pages */
uint32_t rows_per_page_fixed(int32_t type);
cudaError_t launch_write_fixed_pages(const Launch &L, const ColView &col,
                                     uint64_t rows, uint8_t *out_pages,
                                     const unsigned long long *rows_dev = nullptr);
size_t varchar_temp_bytes(uint64_t rows, uint32_t tile_rows);
/* Pass 1: page count per tile; total pages into *total_pages_dev. */
cudaError_t launch_varchar_plan(const Launch &L, const ColView &col, uint64_t rows,
                                uint32_t tile_rows, void *temp,
                                unsigned long long *total_pages_dev);
/* Pass 2: write pages (out_pages sized by pass 1's total). */
cudaError_t launch_varchar_write(const Launch &L, const ColView &col, uint64_t rows,
                                 uint32_t tile_rows, void *temp, uint8_t *out_pages);

} // namespace cj
