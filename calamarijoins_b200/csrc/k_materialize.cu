/*
 * k_materialize.cu — late materialisation: gather matched rows back into
 * 8 KiB result pages.
 *
 * The reference materialises the root join through per-thread page
 * builders (include/materialization/materialize.h:85-321,
 * page_builders.h:92-391) and non-root joins into 4-byte value_t columns
 * (construct_intermediate.h:121-220). Here non-root joins only gather u32
 * row-id vectors (k_gather_u32); values are read once, by the root's page
 * writers, through up to two row-id indirections.
 *
 * Fixed-width pages (k_write_fixed): output page p holds rows
 * [p*R, p*R+R) with R = 1984 (INT32) or 1007 (INT64 / FP64), the fill of
 * ColumnInserter<T> (plan.h:241-250), so every page fits whatever the NULL
 * pattern. One CTA writes one page: all of the page's loads issued at
 * once; a page without NULLs is stored straight from registers (values in
 * row order, header, zero gap, all-ones bitmap); a page with NULLs is built
 * in shared memory (values compacted by one ballot/scan over the validity
 * bits, bitmap at the page end, gap zeroed) and written with 16-byte
 * streaming stores.
 *
 * VARCHAR pages (k_varchar_plan / k_varchar_write): rows are cut into tiles;
 * within a tile pages are packed greedily in row order like
 * ColumnInserter<std::string> (plan.h:340-369): a page takes rows while
 * 4 + 2*n_values + chars + ceil(n_rows/8) <= 8192, found by binary search on
 * the tile's prefix sums. A string longer than 8185 bytes arrives as a chain
 * of long-string pages and is copied verbatim, as VarcharPageBuilder::
 * copy_long_string_pages does (page_builders.h:345-362). Pass 1 counts each
 * tile's pages, a scan places them, pass 2 writes them.
 */
#include <algorithm>

#include "cj_device.cuh"

namespace cj {
namespace {

constexpr int kMatThreads = 256;

CJ_DEV uint32_t rows_per_page_dev(int32_t type) { return type == CJ_INT32 ? kRowsPerPageInt32 : kRowsPerPage8B; }

__global__ void k_gather_u32(const uint32_t *__restrict__ src, const uint32_t *__restrict__ idx,
                             uint64_t n, uint32_t *__restrict__ out) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = __ldg(src + __ldcs(idx + i));
}

constexpr int kMatMinBlocks = 8; /* page writers: 8 x 256 threads per SM */

struct PageSmem {
    uint4 page[kPageSize / 16]; /* zero between pages: copy-out clears it */
    uint32_t cnt[64];           /* non-NULL rows per (slab, warp), then offsets */
    uint32_t total;
};

/* Builds output page `pg` (rows [pg*R, pg*R+R)) of a fixed-width column in
 * shared memory and stores it. Block-wide; sm.page must be zero on entry and
 * is zero again on return.
 *
 * Thread t takes rows t, t+256, ... of the page (kSlabs of them) and issues
 * all their loads (row ids, then validity words and values) before using
 * any, so a page costs one dependent round trip, not one per 256 rows. One
 * scan over the (slab, warp) counts then places the non-NULL values. */
template <typename T>
CJ_DEV void write_fixed_page(const ColView &col, uint64_t rows, uint32_t R, uint64_t pg, uint8_t *__restrict__ out,
                             PageSmem &sm) {
    constexpr uint32_t DB = sizeof(T) == 4 ? 4u : 8u;
    constexpr int kSlabs = (int)(((sizeof(T) == 4 ? kRowsPerPageInt32 : kRowsPerPage8B) + kMatThreads - 1) / kMatThreads);
    constexpr int kWarps = kMatThreads / 32;
    static_assert(kSlabs * kWarps <= 64, "cnt holds 64 (slab, warp) counts");
    uint8_t *sp = reinterpret_cast<uint8_t *>(sm.page);
    const uint32_t warp = threadIdx.x >> 5, lane = lane_id();
    const uint64_t r0 = pg * R;
    const uint32_t nr = (uint32_t)min((uint64_t)R, rows - r0);


    uint32_t br[kSlabs];
#pragma unroll
    for (int k = 0; k < kSlabs; ++k) {
        const uint32_t r = k * kMatThreads + threadIdx.x;
        br[k] = 0xffffffffu;
        if (r < nr) br[k] = col.rid_a ? __ldcs(col.rid_a + r0 + r) : (uint32_t)(r0 + r);
    }
    if (col.rid_b) {
#pragma unroll
        for (int k = 0; k < kSlabs; ++k)
            if (br[k] != 0xffffffffu) br[k] = __ldg(col.rid_b + br[k]);
    }
    T val[kSlabs];
    uint32_t vm = 0; /* bit k: row of slab k is non-NULL */
    /* a column without NULLs needs no validity loads (one random load per
     * row instead of two when the row ids are random); a direct column is
     * read from its pages */
    const bool all_valid = col_all_valid(col);
    const bool direct = col_direct(col);
#pragma unroll
    for (int k = 0; k < kSlabs; ++k) {
        val[k] = T(0);
        if (br[k] != 0xffffffffu) {
            const bool v = all_valid || valid_bit(col.valid, br[k]);
            val[k] = direct ? page_value<T>(col.pages, br[k]) : __ldg(reinterpret_cast<const T *>(col.values) + br[k]);
            if (v && !(sizeof(T) == 4 && col.null_sentinel && (int32_t)val[k] == INT32_MIN)) vm |= 1u << k;
        }
    }

    const uint32_t bm_bytes = (nr + 7) / 8;

    /* No NULL on this page (always, for a column without NULLs): a value's
     * place is its row, so the page is stored straight from registers, with
     * no compaction, no shared memory and no barrier. Same bytes as below:
     * header, values, zero gap, bitmap of nr ones. */
    uint32_t live = 0;
#pragma unroll
    for (int k = 0; k < kSlabs; ++k)
        if (k * kMatThreads + threadIdx.x < nr) live |= 1u << k;
    const bool null_free_col = all_valid && !(sizeof(T) == 4 && col.null_sentinel);
    if (null_free_col || !__syncthreads_or(vm != live)) {
        uint8_t *dst = out + pg * kPageSize;
        T *dv = reinterpret_cast<T *>(dst + DB);
#pragma unroll
        for (int k = 0; k < kSlabs; ++k) {
            const uint32_t r = k * kMatThreads + threadIdx.x;
            if (r < nr) __stcs(dv + r, val[k]);
        }
        if (threadIdx.x == 0) {
            if (DB == 8) __stcs(reinterpret_cast<unsigned long long *>(dst), (unsigned long long)nr * 0x10001ull);
            else __stcs(reinterpret_cast<unsigned int *>(dst), nr * 0x10001u);
        }
        const uint32_t bm0 = kPageSize - bm_bytes;
        for (uint32_t b = DB + nr * (uint32_t)sizeof(T) + threadIdx.x; b < kPageSize; b += blockDim.x) {
            uint8_t v = 0;
            if (b >= bm0) {
                const uint32_t i = b - bm0;
                v = (i + 1) * 8 <= nr ? 0xFFu : (uint8_t)((1u << (nr - i * 8)) - 1u);
            }
            dst[b] = v;
        }
        return;
    }

    uint8_t *bm = sp + kPageSize - bm_bytes;
#pragma unroll
    for (int k = 0; k < kSlabs; ++k) {
        const uint32_t ball = __ballot_sync(0xffffffffu, (vm >> k) & 1u);
        if (lane == 0) sm.cnt[k * kWarps + warp] = __popc(ball);
        if (lane < 4) {
            const uint32_t byte = (k * kMatThreads + warp * 32) / 8 + lane;
            if (byte < bm_bytes) bm[byte] = (uint8_t)(ball >> (8 * lane));
        }
    }
    __syncthreads();
    if (warp == 0) {
        const uint32_t i0 = 2 * lane, i1 = 2 * lane + 1, n = kSlabs * kWarps;
        const uint32_t a = i0 < n ? sm.cnt[i0] : 0u, b = i1 < n ? sm.cnt[i1] : 0u;
        const uint32_t incl = warp_inclusive_scan(a + b);
        if (i0 < n) sm.cnt[i0] = incl - a - b;
        if (i1 < n) sm.cnt[i1] = incl - b;
        if (lane == 31) sm.total = incl;
    }
    __syncthreads();
    T *vals = reinterpret_cast<T *>(sp + DB);
    const uint32_t lt = lanemask_lt();
#pragma unroll
    for (int k = 0; k < kSlabs; ++k) {
        const uint32_t ball = __ballot_sync(0xffffffffu, (vm >> k) & 1u);
        if ((vm >> k) & 1u) vals[sm.cnt[k * kWarps + warp] + __popc(ball & lt)] = val[k];
    }
    if (threadIdx.x == 0) {
        reinterpret_cast<uint16_t *>(sp)[0] = (uint16_t)nr;
        reinterpret_cast<uint16_t *>(sp)[1] = (uint16_t)sm.total;
    }
    __syncthreads();
    uint4 *dst = reinterpret_cast<uint4 *>(out + pg * kPageSize);
    const uint4 zero = make_uint4(0, 0, 0, 0);
    for (uint32_t k = threadIdx.x; k < kPageSize / 16; k += blockDim.x) {
        __stcs(dst + k, sm.page[k]);
        sm.page[k] = zero;
    }
    __syncthreads();
}

CJ_DEV void zero_page(PageSmem &sm) {
    for (uint32_t k = threadIdx.x; k < kPageSize / 16; k += blockDim.x) sm.page[k] = make_uint4(0, 0, 0, 0);
    __syncthreads();
}

/* Rows to write: `rows`, or, when `rows_dev` is set, the count it holds
 * (at most `rows`, the capacity the pages were sized for). */
CJ_DEV uint64_t live_rows(uint64_t rows, const unsigned long long *rows_dev) {
    if (!rows_dev) return rows;
    const uint64_t n = *rows_dev;
    return n < rows ? n : rows;
}

template <typename T>
__global__ void __launch_bounds__(kMatThreads, kMatMinBlocks)
    k_write_fixed(ColView col, uint64_t rows, const unsigned long long *rows_dev, uint32_t R,
                  uint8_t *__restrict__ out) {
    __shared__ PageSmem sm;
    rows = live_rows(rows, rows_dev);
    const uint64_t num_pages = (rows + R - 1) / R;
    if (blockIdx.x >= num_pages) return;
    zero_page(sm);
    for (uint64_t pg = blockIdx.x; pg < num_pages; pg += gridDim.x) write_fixed_page<T>(col, rows, R, pg, out, sm);
}

/* Finishes pages whose values are in place (a NULL-free column written by
 * the probe): header, zero gap after the values, bitmap of nr ones. */
template <typename T>
__global__ void k_finish_dense_pages(uint8_t *__restrict__ pages, uint64_t rows, const unsigned long long *rows_dev) {
    constexpr uint32_t R = sizeof(T) == 4 ? kRowsPerPageInt32 : kRowsPerPage8B;
    constexpr uint32_t DB = sizeof(T) == 4 ? 4u : 8u;
    rows = live_rows(rows, rows_dev);
    const uint64_t num_pages = (rows + R - 1) / R;
    for (uint64_t pg = blockIdx.x; pg < num_pages; pg += gridDim.x) {
        uint8_t *dst = pages + pg * kPageSize;
        const uint32_t nr = (uint32_t)min((uint64_t)R, rows - pg * R);
        if (threadIdx.x == 0) {
            if (DB == 8) __stcs(reinterpret_cast<unsigned long long *>(dst), (unsigned long long)nr * 0x10001ull);
            else __stcs(reinterpret_cast<unsigned int *>(dst), nr * 0x10001u);
        }
        const uint32_t bm_bytes = (nr + 7) / 8, bm0 = kPageSize - bm_bytes;
        for (uint32_t b = DB + nr * (uint32_t)sizeof(T) + threadIdx.x; b < kPageSize; b += blockDim.x) {
            uint8_t v = 0;
            if (b >= bm0) {
                const uint32_t i = b - bm0;
                v = (i + 1) * 8 <= nr ? 0xFFu : (uint8_t)((1u << (nr - i * 8)) - 1u);
            }
            dst[b] = v;
        }
    }
}

/* Grouped page writer: every fixed-width output column of a batch. */
__global__ void __launch_bounds__(kMatThreads, kMatMinBlocks)
    k_write_fixed_grouped(const PageTask *__restrict__ tasks, uint32_t ntasks, uint64_t total_pages) {
    __shared__ PageSmem sm;
    __shared__ uint32_t s_task;
    zero_page(sm);
    for (uint64_t gp = blockIdx.x; gp < total_pages; gp += gridDim.x) {
        if (threadIdx.x == 0) {
            uint32_t lo = 0, hi = ntasks;
            while (hi - lo > 1) {
                uint32_t mid = (lo + hi) >> 1;
                if (tasks[mid].page_base <= gp) lo = mid;
                else hi = mid;
            }
            s_task = lo;
        }
        __syncthreads();
        const PageTask &T = tasks[s_task];
        const uint64_t pg = gp - T.page_base;
        if (T.col.type == CJ_INT32)
            write_fixed_page<int32_t>(T.col, T.rows, rows_per_page_dev(CJ_INT32), pg, T.out, sm);
        else
            write_fixed_page<long long>(T.col, T.rows, rows_per_page_dev(CJ_INT64), pg, T.out, sm);
    }
}

/* Grouped row-id gather: task k covers global chunks [chunk_base, ...). */
__global__ void k_gather_grouped(const GatherTask *__restrict__ tasks, uint32_t ntasks, uint64_t total_chunks) {
    __shared__ uint32_t s_task;
    for (uint64_t gc = blockIdx.x; gc < total_chunks; gc += gridDim.x) {
        if (threadIdx.x == 0) {
            uint32_t lo = 0, hi = ntasks;
            while (hi - lo > 1) {
                uint32_t mid = (lo + hi) >> 1;
                if (tasks[mid].chunk_base <= gc) lo = mid;
                else hi = mid;
            }
            s_task = lo;
        }
        __syncthreads();
        const GatherTask &T = tasks[s_task];
        const uint64_t r0 = (gc - T.chunk_base) * kGatherChunk;
        const uint64_t r1 = min(T.n, r0 + kGatherChunk);
        for (uint64_t i = r0 + threadIdx.x; i < r1; i += blockDim.x) T.out[i] = __ldg(T.src + __ldcs(T.idx + i));
        __syncthreads();
    }
}

/* ---------------- VARCHAR ---------------- */
struct VarSmem {
    uint64_t *desc;     /* TR   row descriptors (0 = NULL)                 */
    uint32_t *lpre;     /* TR+1 prefix of short-string bytes               */
    uint32_t *vpre;     /* TR+1 prefix of short non-NULL rows              */
    uint32_t *longpre;  /* TR+1 prefix of long-string rows                 */
    uint32_t *seg;      /* TR+1 first row of each segment                  */
    uint32_t *segpg;    /* TR+1 first output page of each segment          */
};

CJ_DEV VarSmem carve(uint8_t *base, uint32_t TR) {
    VarSmem s;
    s.desc = reinterpret_cast<uint64_t *>(base);
    uint32_t *u = reinterpret_cast<uint32_t *>(base + (size_t)TR * 8);
    s.lpre = u;
    s.vpre = u + (TR + 1);
    s.longpre = u + 2 * (TR + 1);
    s.seg = u + 3 * (TR + 1);
    s.segpg = u + 4 * (TR + 1);
    return s;
}

/* Loads the tile's descriptors, builds the prefix sums and cuts the tile
 * into segments (one normal page, or one long string's chain). Returns the
 * segment count; the page count is in s.segpg[nseg]. Block-wide. */
CJ_DEV uint32_t plan_tile(const ColView &col, uint64_t r0, uint32_t nt, uint32_t TR,
                          const VarSmem &s, uint32_t *wbuf, uint32_t *s_nseg) {
    const bool all_valid = col_all_valid(col);
    for (uint32_t r = threadIdx.x; r < nt; r += blockDim.x) {
        uint32_t br = base_row(col, (uint32_t)(r0 + r));
        s.desc[r] = (all_valid || valid_bit(col.valid, br)) ? __ldg(col.str_desc + br) : 0ull;
    }
    __syncthreads();
    const uint32_t per = (TR + blockDim.x - 1) / blockDim.x;
    const uint32_t q0 = threadIdx.x * per;
    uint32_t lsum = 0, vsum = 0, gsum = 0;
    for (uint32_t k = 0; k < per; ++k) {
        uint32_t r = q0 + k;
        if (r >= nt) break;
        uint64_t d = s.desc[r];
        if (!d) continue;
        if (desc_is_long(d)) ++gsum;
        else {
            lsum += desc_len(d);
            ++vsum;
        }
    }
    uint32_t ltot, vtot, gtot;
    uint32_t lp = block_exclusive_scan<uint32_t>(lsum, wbuf, &ltot);
    uint32_t vp = block_exclusive_scan<uint32_t>(vsum, wbuf, &vtot);
    uint32_t gp = block_exclusive_scan<uint32_t>(gsum, wbuf, &gtot);
    for (uint32_t k = 0; k < per; ++k) {
        uint32_t r = q0 + k;
        if (r >= nt) break;
        s.lpre[r] = lp;
        s.vpre[r] = vp;
        s.longpre[r] = gp;
        uint64_t d = s.desc[r];
        if (d) {
            if (desc_is_long(d)) ++gp;
            else {
                lp += desc_len(d);
                ++vp;
            }
        }
    }
    if (threadIdx.x == 0) {
        s.lpre[nt] = ltot;
        s.vpre[nt] = vtot;
        s.longpre[nt] = gtot;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t a = 0, ns = 0, np = 0;
        while (a < nt) {
            s.seg[ns] = a;
            s.segpg[ns] = np;
            uint64_t d = s.desc[a];
            if (d && desc_is_long(d)) {
                np += desc_len(d);
                a += 1;
            } else {
                uint32_t lo = a + 1, hi = nt;
                while (lo < hi) {
                    uint32_t mid = (lo + hi + 1) >> 1;
                    uint32_t n = mid - a;
                    bool ok = s.longpre[mid] == s.longpre[a] && n <= 65533u &&
                              4u + 2u * (s.vpre[mid] - s.vpre[a]) + (s.lpre[mid] - s.lpre[a]) +
                                      (n + 7) / 8 <= kPageSize;
                    if (ok) lo = mid;
                    else hi = mid - 1;
                }
                np += 1;
                a = lo;
            }
            ++ns;
        }
        s.seg[ns] = nt;
        s.segpg[ns] = np;
        *s_nseg = ns;
    }
    __syncthreads();
    return *s_nseg;
}

__global__ void __launch_bounds__(kMatThreads)
    k_varchar_plan(ColView col, uint64_t rows, uint32_t TR, uint32_t *__restrict__ tile_pages) {
    extern __shared__ __align__(16) uint8_t dsm[];
    __shared__ uint32_t wbuf[kMatThreads / 32 + 1];
    __shared__ uint32_t s_nseg;
    VarSmem s = carve(dsm, TR);
    const uint64_t tiles = (rows + TR - 1) / TR;
    for (uint64_t t = blockIdx.x; t < tiles; t += gridDim.x) {
        const uint64_t r0 = t * TR;
        const uint32_t nt = (uint32_t)min((uint64_t)TR, rows - r0);
        uint32_t ns = plan_tile(col, r0, nt, TR, s, wbuf, &s_nseg);
        if (threadIdx.x == 0) tile_pages[t] = s.segpg[ns];
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kMatThreads)
    k_varchar_write(ColView col, uint64_t rows, uint32_t TR, const uint64_t *__restrict__ tile_base,
                    uint8_t *__restrict__ out) {
    extern __shared__ __align__(16) uint8_t dsm[];
    __shared__ uint4 s_page[kPageSize / 16];
    __shared__ uint32_t wbuf[kMatThreads / 32 + 1];
    __shared__ uint32_t s_nseg;
    VarSmem s = carve(dsm, TR);
    uint8_t *sp = reinterpret_cast<uint8_t *>(s_page);
    const uint32_t warp = threadIdx.x >> 5, lane = lane_id(), nwarps = blockDim.x >> 5;
    const uint64_t tiles = (rows + TR - 1) / TR;
    for (uint64_t t = blockIdx.x; t < tiles; t += gridDim.x) {
        const uint64_t r0 = t * TR;
        const uint32_t nt = (uint32_t)min((uint64_t)TR, rows - r0);
        const uint32_t ns = plan_tile(col, r0, nt, TR, s, wbuf, &s_nseg);
        const uint64_t base = tile_base[t];
        for (uint32_t g = 0; g < ns; ++g) {
            const uint32_t a = s.seg[g], b = s.seg[g + 1];
            const uint64_t opg = base + s.segpg[g];
            const uint64_t d0 = s.desc[a];
            if (d0 && desc_is_long(d0)) {
                const uint4 *src = reinterpret_cast<const uint4 *>(col.pages + desc_pos(d0) * kPageSize);
                uint4 *dst = reinterpret_cast<uint4 *>(out + opg * kPageSize);
                const uint64_t n16 = (uint64_t)desc_len(d0) * (kPageSize / 16);
                for (uint64_t k = threadIdx.x; k < n16; k += blockDim.x) dst[k] = __ldg(src + k);
                continue;
            }
            for (uint32_t k = threadIdx.x; k < kPageSize / 16; k += blockDim.x) s_page[k] = make_uint4(0, 0, 0, 0);
            __syncthreads();
            const uint32_t n = b - a, nv = s.vpre[b] - s.vpre[a];
            const uint32_t chars_at = 4u + 2u * nv;
            const uint32_t bm_bytes = (n + 7) / 8;
            uint8_t *bm = sp + kPageSize - bm_bytes;
            uint16_t *offs = reinterpret_cast<uint16_t *>(sp + 4);
            /* offsets, bitmap and short strings */
            for (uint32_t j0 = 0; j0 < n; j0 += blockDim.x) {
                const uint32_t j = j0 + threadIdx.x;
                bool v = false;
                if (j < n) {
                    const uint32_t r = a + j;
                    const uint64_t d = s.desc[r];
                    if (d) {
                        v = true;
                        const uint32_t k = s.vpre[r] - s.vpre[a];
                        const uint32_t beg = s.lpre[r] - s.lpre[a];
                        const uint32_t len = desc_len(d);
                        offs[k] = (uint16_t)(beg + len);
                        if (len <= 32) {
                            const uint8_t *src = col.pages + desc_pos(d);
                            uint8_t *dst = sp + chars_at + beg;
                            for (uint32_t q = 0; q < len; ++q) dst[q] = __ldg(src + q);
                        }
                    }
                }
                uint32_t ball = __ballot_sync(0xffffffffu, v);
                if (lane < 4) {
                    uint32_t byte = (j0 + warp * 32) / 8 + lane;
                    if (byte < bm_bytes) bm[byte] = (uint8_t)(ball >> (8 * lane));
                }
            }
            /* longer strings: one warp per string */
            for (uint32_t r = a + warp; r < b; r += nwarps) {
                const uint64_t d = s.desc[r];
                if (!d || desc_len(d) <= 32) continue;
                const uint8_t *src = col.pages + desc_pos(d);
                uint8_t *dst = sp + chars_at + (s.lpre[r] - s.lpre[a]);
                const uint32_t len = desc_len(d);
                for (uint32_t q = lane; q < len; q += 32) dst[q] = __ldg(src + q);
            }
            if (threadIdx.x == 0) {
                reinterpret_cast<uint16_t *>(sp)[0] = (uint16_t)n;
                reinterpret_cast<uint16_t *>(sp)[1] = (uint16_t)nv;
            }
            __syncthreads();
            uint4 *dst = reinterpret_cast<uint4 *>(out + opg * kPageSize);
            for (uint32_t k = threadIdx.x; k < kPageSize / 16; k += blockDim.x) dst[k] = s_page[k];
            __syncthreads();
        }
        __syncthreads();
    }
}

size_t var_dyn_smem(uint32_t TR) { return (size_t)TR * 8 + 5 * ((size_t)TR + 1) * 4; }

bool g_var_attrs = false;
void set_var_attrs() {
    if (g_var_attrs) return;
    cudaFuncSetAttribute(k_varchar_plan, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(k_varchar_write, cudaFuncAttributeMaxDynamicSharedMemorySize, 190 * 1024);
    g_var_attrs = true;
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

} // namespace

cudaError_t launch_gather_u32(const Launch &L, const uint32_t *src, const uint32_t *idx, uint64_t n,
                              uint32_t *out) {
    if (n == 0) return cudaSuccess;
    uint64_t g = (n + 255) / 256;
    uint64_t cap = (uint64_t)L.num_sms * 8;
    if (g > cap) g = cap;
    k_gather_u32<<<(unsigned)g, 256, 0, L.stream>>>(src, idx, n, out);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_write_fixed_grouped(const Launch &L, const PageTask *tasks_dev, uint32_t ntasks,
                                      uint64_t total_pages) {
    if (!total_pages) return cudaSuccess;
    uint64_t g = std::min<uint64_t>(total_pages, (uint64_t)L.num_sms * kMatMinBlocks);
    k_write_fixed_grouped<<<(unsigned)g, kMatThreads, 0, L.stream>>>(tasks_dev, ntasks, total_pages);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_gather_grouped(const Launch &L, const GatherTask *tasks_dev, uint32_t ntasks,
                                  uint64_t total_chunks) {
    if (!total_chunks) return cudaSuccess;
    uint64_t g = std::min<uint64_t>(total_chunks, (uint64_t)L.num_sms * 8);
    k_gather_grouped<<<(unsigned)g, 256, 0, L.stream>>>(tasks_dev, ntasks, total_chunks);
    count_launches(1);
    return cudaGetLastError();
}

uint32_t rows_per_page_fixed(int32_t type) {
    return type == CJ_INT32 ? kRowsPerPageInt32 : kRowsPerPage8B;
}

cudaError_t launch_write_fixed_pages(const Launch &L, const ColView &col, uint64_t rows,
                                     uint8_t *out, const unsigned long long *rows_dev) {
    if (rows == 0) return cudaSuccess;
    const uint32_t R = rows_per_page_fixed(col.type);
    const uint64_t np = (rows + R - 1) / R;
    uint64_t g = np, cap = (uint64_t)L.num_sms * kMatMinBlocks;
    if (g > cap) g = cap;
    if (col.type == CJ_INT32) {
        k_write_fixed<int32_t><<<(unsigned)g, kMatThreads, 0, L.stream>>>(col, rows, rows_dev, R, out);
        count_launches(1);
    } else {
        k_write_fixed<long long><<<(unsigned)g, kMatThreads, 0, L.stream>>>(col, rows, rows_dev, R, out);
        count_launches(1);
    }
    return cudaGetLastError();
}

cudaError_t launch_finish_dense_pages(const Launch &L, uint8_t *pages, uint64_t rows, int32_t type,
                                      const unsigned long long *rows_dev) {
    if (rows == 0) return cudaSuccess;
    const uint32_t R = rows_per_page_fixed(type);
    const uint64_t np = (rows + R - 1) / R;
    const unsigned g = (unsigned)std::min<uint64_t>(np, (uint64_t)L.num_sms * 8);
    if (type == CJ_INT32) k_finish_dense_pages<int32_t><<<g, 128, 0, L.stream>>>(pages, rows, rows_dev);
    else k_finish_dense_pages<long long><<<g, 128, 0, L.stream>>>(pages, rows, rows_dev);
    count_launches(1);
    return cudaGetLastError();
}

size_t varchar_temp_bytes(uint64_t rows, uint32_t TR) {
    uint64_t tiles = (rows + TR - 1) / TR;
    return align256(tiles * 4) + align256((tiles + 1) * 8) + scan_temp_bytes(tiles) + 256;
}

cudaError_t launch_varchar_plan(const Launch &L, const ColView &col, uint64_t rows, uint32_t TR,
                                void *temp, unsigned long long *total_pages_dev) {
    set_var_attrs();
    const uint64_t tiles = (rows + TR - 1) / TR;
    char *t = reinterpret_cast<char *>(temp);
    uint32_t *tile_pages = reinterpret_cast<uint32_t *>(t);
    uint64_t *tile_base = reinterpret_cast<uint64_t *>(t + align256(tiles * 4));
    void *scan_tmp = t + align256(tiles * 4) + align256((tiles + 1) * 8);
    if (tiles) {
        uint64_t g = tiles, cap = (uint64_t)L.num_sms * 2;
        if (g > cap) g = cap;
        k_varchar_plan<<<(unsigned)g, kMatThreads, var_dyn_smem(TR), L.stream>>>(col, rows, TR, tile_pages);
        count_launches(1);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    cudaError_t e = scan_u32_to_u64(L, tile_pages, tile_base, tiles, scan_tmp);
    if (e != cudaSuccess) return e;
    return cudaMemcpyAsync(total_pages_dev, tile_base + tiles, sizeof(unsigned long long),
                           cudaMemcpyDeviceToDevice, L.stream);
}

cudaError_t launch_varchar_write(const Launch &L, const ColView &col, uint64_t rows, uint32_t TR,
                                 void *temp, uint8_t *out) {
    set_var_attrs();
    const uint64_t tiles = (rows + TR - 1) / TR;
    if (!tiles) return cudaSuccess;
    const uint64_t *tile_base =
        reinterpret_cast<const uint64_t *>(reinterpret_cast<char *>(temp) + align256(tiles * 4));
    uint64_t g = tiles, cap = (uint64_t)L.num_sms * 2;
    if (g > cap) g = cap;
    k_varchar_write<<<(unsigned)g, kMatThreads, var_dyn_smem(TR), L.stream>>>(col, rows, TR, tile_base, out);
    count_launches(1);
    return cudaGetLastError();
}

} // namespace cj
