/*
 * k_decode.cu — page decode: 8 KiB pages in HBM -> dense device columns.
 *
 * Follows the page format of the reference (include/data_model/plan.h:
 * 75-142, 187-366; README.md "Data format") and its readers:
 *   - row counts per page, long-string pages counting as one row (0xffff)
 *     or none (0xfffe): PageIndex::build (include/data_access/
 *     columnar_reader.h:122-200)
 *   - dense pages (n_rows == n_values) read values in row order without
 *     the bitmap, sparse pages locate a value by popcount of the bitmap
 *     prefix: ColumnarReader::read_dense_int32 / read_sparse
 *     (columnar_reader.h:385-393, 452-474)
 *   - VARCHAR: n_values u16 end offsets at +4, characters after them
 *     (include/materialization/page_builders.h:26-37)
 *
 * One CTA decodes one page at a time (grid-stride over pages); the page's
 * bitmap and its popcount prefix live in shared memory. Value writes are
 * coalesced; the validity bitmap is written with plain stores except for
 * the (at most two) 32-row words a page shares with its neighbours, which
 * use atomicOr on a zeroed bitmap.
 */
#include <algorithm>

#include "cj_device.cuh"

namespace cj {
namespace {

constexpr int kDecodeThreads = 256;
constexpr uint32_t kMaxBitmapWords = 2048; /* 65535 rows */

CJ_DEV uint16_t rd16(const uint8_t *p) { return *reinterpret_cast<const uint16_t *>(p); }

/* Rows a page contributes (n_rows; 1 for a long-string start page, 0 for a
 * continuation) and header checks. */
CJ_DEV uint32_t page_rows_of(const uint8_t *pg, int32_t type, unsigned int *err) {
    uint32_t nr = rd16(pg), nv = rd16(pg + 2);
    uint32_t r = nr;
    if (type == CJ_VARCHAR) {
        if (nr == 0xffff) {
            r = 1;
            if (nv == 0 || nv > kLongChunk) atomicOr(err, DEV_ERR_PAGE_HEADER);
        } else if (nr == 0xfffe) {
            r = 0;
            if (nv == 0 || nv > kLongChunk) atomicOr(err, DEV_ERR_PAGE_HEADER);
        } else if (nv > nr || 4u + 2u * nv + (nr + 7) / 8 > kPageSize) {
            atomicOr(err, DEV_ERR_PAGE_HEADER);
        }
    } else {
        uint32_t w = type == CJ_INT32 ? 4u : 8u;
        if (nv > nr || w + w * nv + (nr + 7) / 8 > kPageSize) atomicOr(err, DEV_ERR_PAGE_HEADER);
    }
    return r;
}

/* COL_* flags of page p of np: COL_HAS_NULLS if a regular page stores
 * fewer values than rows (long-string pages hold one non-NULL row or none);
 * COL_NOT_DIRECT for VARCHAR, or unless every page but the last holds
 * exactly R rows and the last 1..R. */
CJ_DEV uint32_t page_flags(const uint8_t *pg, uint64_t p, uint64_t np, int32_t type) {
    const uint32_t nr = rd16(pg), nv = rd16(pg + 2);
    if (type == CJ_VARCHAR) return COL_NOT_DIRECT | ((nr < 0xfffe && nv < nr) ? COL_HAS_NULLS : 0u);
    const uint32_t R = type == CJ_INT32 ? kRowsPerPageInt32 : kRowsPerPage8B;
    uint32_t f = nv < nr ? COL_HAS_NULLS : 0u;
    if (p + 1 < np ? nr != R : (nr == 0 || nr > R)) f |= COL_NOT_DIRECT;
    return f;
}

/* Page index of one column in two launches. Block b of both kernels owns
 * pages [b * chunk, (b + 1) * chunk).
 * k_page_index: rows per page, the column's COL_* flags (ORed into
 * state[0]) and each block's row total (partials[b]); the last block to
 * finish (state[1] counts finished blocks) adds the totals, stores
 * row_start[np] and checks the row count against the table's (a mismatch
 * raises DEV_ERR_ROW_COUNT and makes the column NOT_DIRECT, so readers stay
 * inside its decoded arrays).
 * k_page_index_scan: row_start[p] = rows before page p; skipped for a
 * column read in place (state[0] == 0), which needs no row offsets. */
constexpr int kIndexThreads = 256;

__global__ void __launch_bounds__(kIndexThreads)
    k_page_index(const uint8_t *__restrict__ pages, uint64_t np, int32_t type, uint64_t chunk, uint64_t expected,
                 uint32_t *__restrict__ rows, uint64_t *__restrict__ partials, uint64_t *__restrict__ row_start,
                 uint32_t *state, unsigned int *err) {
    __shared__ uint64_t wsum[kIndexThreads / 32];
    __shared__ bool s_last;
    const uint64_t p0 = (uint64_t)blockIdx.x * chunk, p1 = min(np, p0 + chunk);
    uint64_t s = 0;
    uint32_t f = 0;
    for (uint64_t p = p0 + threadIdx.x; p < p1; p += blockDim.x) {
        const uint8_t *pg = pages + p * kPageSize;
        const uint32_t r = page_rows_of(pg, type, err);
        rows[p] = r;
        s += r;
        f |= page_flags(pg, p, np, type);
    }
    f = __reduce_or_sync(0xffffffffu, f);
    if (f && lane_id() == 0) atomicOr(state, f);
    s = warp_sum(s);
    if (lane_id() == 0) wsum[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint64_t t = 0;
        for (int w = 0; w < kIndexThreads / 32; ++w) t += wsum[w];
        partials[blockIdx.x] = t;
        __threadfence();
        s_last = atomicAdd(state + 1, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    uint64_t t = 0;
    for (uint32_t b = threadIdx.x; b < gridDim.x; b += blockDim.x) t += __ldcg(partials + b);
    t = warp_sum(t);
    __syncthreads();
    if (lane_id() == 0) wsum[threadIdx.x >> 5] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint64_t total = 0;
        for (int w = 0; w < kIndexThreads / 32; ++w) total += wsum[w];
        row_start[np] = total;
        if (total != expected) {
            atomicOr(err, DEV_ERR_ROW_COUNT);
            atomicOr(state, COL_NOT_DIRECT);
        }
    }
}

/* A column without pages: zero rows (any other count is an error). */
__global__ void k_page_index_empty(uint64_t expected, uint64_t *row_start, uint32_t *state, unsigned int *err) {
    row_start[0] = 0;
    if (expected != 0) {
        atomicOr(err, DEV_ERR_ROW_COUNT);
        atomicOr(state, COL_NOT_DIRECT);
    }
}

__global__ void __launch_bounds__(kIndexThreads)
    k_page_index_scan(const uint32_t *__restrict__ rows, uint64_t np, uint64_t chunk,
                      const uint64_t *__restrict__ partials, uint64_t *__restrict__ row_start,
                      const uint32_t *state) {
    __shared__ uint64_t wbuf[kIndexThreads / 32 + 1];
    if (*state == 0u) return; /* uniform: read in place */
    uint64_t o = 0;
    for (uint32_t b = threadIdx.x; b < blockIdx.x; b += blockDim.x) o += partials[b];
    uint64_t off;
    block_exclusive_scan<uint64_t>(o, wbuf, &off);
    const uint64_t p0 = (uint64_t)blockIdx.x * chunk, p1 = min(np, p0 + chunk);
    for (uint64_t base = p0; base < p1; base += blockDim.x) {
        const uint64_t p = base + threadIdx.x;
        const uint64_t v = p < p1 ? rows[p] : 0;
        uint64_t tot;
        const uint64_t pre = block_exclusive_scan<uint64_t>(v, wbuf, &tot);
        if (p < p1) row_start[p] = off + pre;
        off += tot;
    }
}

/* Loads a sparse page's bitmap into s_bm (bits past n_rows cleared) and the
 * exclusive popcount prefix per word into s_pre. Block-wide. */
CJ_DEV void load_page_bitmap(const uint8_t *pg, uint32_t nr, uint32_t *s_bm, uint32_t *s_pre,
                             uint32_t *wbuf) {
    const uint32_t nbytes = (nr + 7) / 8, nwords = (nr + 31) / 32;
    const uint8_t *bmb = pg + kPageSize - nbytes;
    for (uint32_t w = threadIdx.x; w < nwords; w += blockDim.x) {
        uint32_t v = 0;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            uint32_t bi = w * 4 + b;
            if (bi < nbytes) v |= (uint32_t)bmb[bi] << (8 * b);
        }
        uint32_t live = nr - w * 32;
        if (live < 32) v &= (1u << live) - 1u;
        s_bm[w] = v;
    }
    __syncthreads();
    const uint32_t per = (nwords + blockDim.x - 1) / blockDim.x;
    const uint32_t w0 = threadIdx.x * per;
    uint32_t s = 0;
    for (uint32_t k = 0; k < per; ++k)
        if (w0 + k < nwords) s += __popc(s_bm[w0 + k]);
    uint32_t tot;
    uint32_t pre = block_exclusive_scan<uint32_t>(s, wbuf, &tot);
    for (uint32_t k = 0; k < per; ++k)
        if (w0 + k < nwords) {
            s_pre[w0 + k] = pre;
            pre += __popc(s_bm[w0 + k]);
        }
    __syncthreads();
}

/* Value index of page row i of a sparse page, or -1 if the row is NULL. */
CJ_DEV int value_index(const uint32_t *s_bm, const uint32_t *s_pre, uint32_t i) {
    uint32_t w = i >> 5, b = i & 31;
    uint32_t word = s_bm[w];
    if (!((word >> b) & 1u)) return -1;
    return (int)(s_pre[w] + __popc(word & ((1u << b) - 1u)));
}

/* 32 validity bits of the output word whose first row is page row `off`
 * (off may be negative for the page's first word). */
CJ_DEV uint32_t page_bits(bool dense, const uint32_t *s_bm, uint32_t nr, int64_t off) {
    if (dense) {
        int64_t lo = off < 0 ? -off : 0;
        int64_t hi = (int64_t)nr - off;
        if (hi > 32) hi = 32;
        if (hi <= lo) return 0;
        uint32_t width = (uint32_t)(hi - lo);
        uint32_t m = width >= 32 ? 0xffffffffu : ((1u << width) - 1u);
        return m << lo;
    }
    if (off < 0) return s_bm[0] << (uint32_t)(-off);
    const uint32_t nwords = (nr + 31) / 32;
    uint32_t w0 = (uint32_t)(off >> 5), s = (uint32_t)(off & 31);
    uint32_t lo = w0 < nwords ? s_bm[w0] : 0u;
    uint32_t hi = w0 + 1 < nwords ? s_bm[w0 + 1] : 0u;
    return s ? (lo >> s) | (hi << (32 - s)) : lo;
}

CJ_DEV void write_validity(bool dense, const uint32_t *s_bm, uint32_t nr, uint64_t rs,
                           uint32_t *valid) {
    if (nr == 0) return;
    const uint64_t fw = rs >> 5, lw = (rs + nr - 1) >> 5;
    for (uint64_t ow = fw + threadIdx.x; ow <= lw; ow += blockDim.x) {
        int64_t off = (int64_t)(ow * 32) - (int64_t)rs;
        uint32_t bits = page_bits(dense, s_bm, nr, off);
        if (off >= 0 && off + 32 <= (int64_t)nr)
            valid[ow] = bits;
        else if (bits)
            atomicOr(valid + ow, bits);
    }
}

struct DecodeSmem {
    uint32_t bm[kMaxBitmapWords];
    uint32_t pre[kMaxBitmapWords];
    uint32_t wbuf[kDecodeThreads / 32 + 1];
};

/* Decodes fixed-width page p (of a column whose pages start at `pages`)
 * whose first row is rs. Block-wide. */
template <typename T>
CJ_DEV void decode_fixed_page(const uint8_t *__restrict__ pages, uint64_t p, uint64_t rs, uint64_t max_rows,
                              T *__restrict__ values, uint32_t *__restrict__ valid, unsigned int *err,
                              DecodeSmem &sm) {
    constexpr uint32_t DB = sizeof(T) == 4 ? 4u : 8u;
    const uint8_t *pg = pages + p * kPageSize;
    const uint32_t nr = rd16(pg), nv = rd16(pg + 2);
    if (nv > nr || DB + (uint32_t)sizeof(T) * nv + (nr + 7) / 8 > kPageSize) return;
    if (rs + nr > max_rows) {
        if (threadIdx.x == 0) atomicOr(err, DEV_ERR_ROW_COUNT);
        return;
    }
    const T *vals = reinterpret_cast<const T *>(pg + DB);
    const bool dense = nr == nv;
    if (!dense) {
        load_page_bitmap(pg, nr, sm.bm, sm.pre, sm.wbuf);
        /* Sparse page: a thread takes 4 consecutive rows, whose non-NULL
         * values are consecutive in the page (one bitmap word and its
         * prefix give the first index), and stores the 4 rows at once when
         * the page starts on a multiple of 4 rows. */
        const bool vec = sizeof(T) == 4 && (rs & 3u) == 0;
        for (uint32_t g = threadIdx.x; g * 4 < nr; g += blockDim.x) {
            const uint32_t r = g * 4, w = r >> 5, sh = r & 31u;
            const uint32_t word = sm.bm[w]; /* bits past n_rows are clear */
            uint32_t idx = sm.pre[w] + __popc(word & ((1u << sh) - 1u));
            const uint32_t nib = (word >> sh) & 0xFu;
            T v[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                v[k] = T(0);
                if ((nib >> k) & 1u) {
                    if (idx >= nv) atomicOr(err, DEV_ERR_PAGE_HEADER); /* bitmap holds > n_values bits */
                    else v[k] = __ldcs(vals + idx);
                    ++idx;
                }
            }
            bool done = false;
            if constexpr (sizeof(T) == 4) {
                if (vec && r + 4 <= nr) {
                    *reinterpret_cast<int4 *>(values + rs + r) = make_int4(v[0], v[1], v[2], v[3]);
                    done = true;
                }
            }
            if (!done) {
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    if (r + k < nr) values[rs + r + k] = v[k];
            }
        }
        write_validity(false, sm.bm, nr, rs, valid);
        __syncthreads();
        return;
    }
    /* All loads of a chunk are issued before any store: a full page (1984 /
     * 1007 rows) is one chunk, so it costs one DRAM round trip. */
    constexpr int kSlabs =
        (int)(((sizeof(T) == 4 ? kRowsPerPageInt32 : kRowsPerPage8B) + kDecodeThreads - 1) / kDecodeThreads);
    for (uint32_t base = 0; base < nr; base += kSlabs * kDecodeThreads) {
        T v[kSlabs];
#pragma unroll
        for (int k = 0; k < kSlabs; ++k) {
            const uint32_t i = base + k * kDecodeThreads + threadIdx.x;
            v[k] = T(0);
            if (i < nr) {
                const int idx = dense ? (int)i : value_index(sm.bm, sm.pre, i);
                if (idx >= (int)nv) atomicOr(err, DEV_ERR_PAGE_HEADER); /* bitmap holds > n_values bits */
                else if (idx >= 0) v[k] = __ldcs(vals + idx);
            }
        }
#pragma unroll
        for (int k = 0; k < kSlabs; ++k) {
            const uint32_t i = base + k * kDecodeThreads + threadIdx.x;
            if (i < nr) values[rs + i] = v[k];
        }
    }
    write_validity(dense, sm.bm, nr, rs, valid);
    __syncthreads();
}

CJ_DEV void decode_varchar_page(const uint8_t *__restrict__ pages, uint64_t p, uint64_t np, uint64_t rs,
                                uint64_t max_rows, uint64_t *__restrict__ desc, uint32_t *__restrict__ valid,
                                unsigned int *err, DecodeSmem &sm) {
    const uint8_t *pg = pages + p * kPageSize;
    const uint32_t nr = rd16(pg), nv = rd16(pg + 2);
    if (nr == 0xfffe) {
        if (threadIdx.x == 0) {
            uint32_t prev = p ? rd16(pg - kPageSize) : 0u;
            if (prev != 0xffff && prev != 0xfffe) atomicOr(err, DEV_ERR_LONG_CHAIN);
        }
        return;
    }
    if (nr == 0xffff) {
        if (threadIdx.x == 0 && rs >= max_rows) atomicOr(err, DEV_ERR_ROW_COUNT);
        if (threadIdx.x == 0 && rs < max_rows) {
            uint64_t q = p + 1;
            while (q < np && rd16(pages + q * kPageSize) == 0xfffe) ++q;
            uint64_t chain = q - p;
            if (chain > 0xFFFFFFull) {
                atomicOr(err, DEV_ERR_LONG_CHAIN);
                chain = 0xFFFFFF;
            }
            desc[rs] = desc_long(p, (uint32_t)chain);
            atomicOr(valid + (rs >> 5), 1u << (rs & 31));
        }
        return;
    }
    if (nv > nr || 4u + 2u * nv + (nr + 7) / 8 > kPageSize) return;
    if (rs + nr > max_rows) {
        if (threadIdx.x == 0) atomicOr(err, DEV_ERR_ROW_COUNT);
        return;
    }
    const bool dense = nr == nv;
    if (!dense) load_page_bitmap(pg, nr, sm.bm, sm.pre, sm.wbuf);
    const uint16_t *offs = reinterpret_cast<const uint16_t *>(pg + 4);
    const uint32_t chars_at = 4u + 2u * nv;
    const uint32_t chars_cap = kPageSize - (nr + 7) / 8 - chars_at;
    for (uint32_t i = threadIdx.x; i < nr; i += blockDim.x) {
        int k = dense ? (int)i : value_index(sm.bm, sm.pre, i);
        uint64_t d = 0;
        if (k >= (int)nv) {
            atomicOr(err, DEV_ERR_PAGE_HEADER); /* bitmap holds > n_values bits */
        } else if (k >= 0) {
            uint32_t start = k ? offs[k - 1] : 0u, end = offs[k];
            if (end < start || end > chars_cap) {
                atomicOr(err, DEV_ERR_VARCHAR_OFFSETS);
            } else {
                d = desc_short(p * kPageSize + chars_at + start, end - start);
            }
        }
        desc[rs + i] = d;
    }
    write_validity(dense, sm.bm, nr, rs, valid);
    __syncthreads();
}

template <typename T>
__global__ void __launch_bounds__(kDecodeThreads, 8)
    k_decode_fixed(const uint8_t *__restrict__ pages, uint64_t np, const uint64_t *__restrict__ row_start,
                   uint64_t max_rows, T *__restrict__ values, uint32_t *__restrict__ valid, unsigned int *err,
                   const uint32_t *__restrict__ col_flags) {
    __shared__ DecodeSmem sm;
    if (col_flags && *col_flags == 0u) return; /* read in place from the pages */
    for (uint64_t p = blockIdx.x; p < np; p += gridDim.x)
        decode_fixed_page<T>(pages, p, row_start[p], max_rows, values, valid, err, sm);
}

__global__ void __launch_bounds__(kDecodeThreads)
    k_decode_varchar(const uint8_t *__restrict__ pages, uint64_t np, const uint64_t *__restrict__ row_start,
                     uint64_t max_rows, uint64_t *__restrict__ desc, uint32_t *__restrict__ valid, unsigned int *err) {
    __shared__ DecodeSmem sm;
    for (uint64_t p = blockIdx.x; p < np; p += gridDim.x)
        decode_varchar_page(pages, p, np, row_start[p], max_rows, desc, valid, err, sm);
}

/* ---- grouped: every column a batch needs, one launch per pass ---- */
CJ_DEV uint32_t find_column(const DecodeTask *tasks, uint32_t ntasks, uint64_t gpage) {
    uint32_t lo = 0, hi = ntasks;
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (tasks[mid].page_base <= gpage) lo = mid;
        else hi = mid;
    }
    return lo;
}

__global__ void k_page_rows_grouped(const DecodeTask *__restrict__ tasks, uint32_t ntasks, uint64_t total_pages,
                                    uint32_t *__restrict__ rows, unsigned int *err) {
    for (uint64_t gp = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; gp < total_pages;
         gp += (uint64_t)gridDim.x * blockDim.x) {
        const DecodeTask &T = tasks[find_column(tasks, ntasks, gp)];
        const uint8_t *pg = T.pages + (gp - T.page_base) * kPageSize;
        rows[gp] = page_rows_of(pg, T.type, err);
    }
}

__global__ void k_check_rows_grouped(const DecodeTask *__restrict__ tasks, uint32_t ntasks,
                                     const uint64_t *__restrict__ row_start, unsigned int *err) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < ntasks; k += gridDim.x * blockDim.x) {
        const DecodeTask &T = tasks[k];
        if (row_start[T.page_base + T.num_pages] - row_start[T.page_base] != T.rows) atomicOr(err, DEV_ERR_ROW_COUNT);
    }
}

__global__ void __launch_bounds__(kDecodeThreads)
    k_decode_grouped(const DecodeTask *__restrict__ tasks, uint32_t ntasks, uint64_t total_pages,
                     const uint64_t *__restrict__ row_start, unsigned int *err) {
    __shared__ DecodeSmem sm;
    __shared__ uint32_t s_task;
    for (uint64_t gp = blockIdx.x; gp < total_pages; gp += gridDim.x) {
        if (threadIdx.x == 0) s_task = find_column(tasks, ntasks, gp);
        __syncthreads();
        const DecodeTask &T = tasks[s_task];
        const uint64_t p = gp - T.page_base;
        const uint64_t rs = row_start[gp] - row_start[T.page_base];
        if (T.type == CJ_VARCHAR)
            decode_varchar_page(T.pages, p, T.num_pages, rs, T.rows, T.desc, T.valid, err, sm);
        else if (T.type == CJ_INT32)
            decode_fixed_page<int32_t>(T.pages, p, rs, T.rows, reinterpret_cast<int32_t *>(T.values), T.valid, err, sm);
        else
            decode_fixed_page<long long>(T.pages, p, rs, T.rows, reinterpret_cast<long long *>(T.values), T.valid,
                                         err, sm);
        __syncthreads();
    }
}

unsigned grid_for(const Launch &L, uint64_t units, int per_sm) {
    uint64_t g = (uint64_t)L.num_sms * per_sm;
    if (units < g) g = units;
    return (unsigned)(g ? g : 1);
}

} // namespace

uint64_t page_index_blocks(const Launch &L, uint64_t np) {
    const uint64_t chunk = std::max<uint64_t>(kIndexThreads, (np + L.num_sms * 8 - 1) / (L.num_sms * 8));
    return std::max<uint64_t>((np + chunk - 1) / chunk, 1);
}

cudaError_t launch_page_index(const Launch &L, const uint8_t *pages, uint64_t np, int32_t type, uint64_t rows,
                              uint32_t *rows_pp, uint64_t *partials, uint64_t *row_start, uint32_t *state) {
    if (np == 0) {
        k_page_index_empty<<<1, 1, 0, L.stream>>>(rows, row_start, state, L.dev_errors);
        count_launches(1);
        return cudaGetLastError();
    }
    const unsigned g = (unsigned)page_index_blocks(L, np);
    const uint64_t chunk = (np + g - 1) / g;
    k_page_index<<<g, kIndexThreads, 0, L.stream>>>(pages, np, type, chunk, rows, rows_pp, partials, row_start,
                                                     state, L.dev_errors);
    k_page_index_scan<<<g, kIndexThreads, 0, L.stream>>>(rows_pp, np, chunk, partials, row_start, state);
    count_launches(2);
    return cudaGetLastError();
}

cudaError_t launch_decode_fixed(const Launch &L, const uint8_t *pages, uint64_t np, int32_t type,
                                const uint64_t *row_start, uint64_t max_rows, void *values,
                                uint32_t *valid, const uint32_t *col_flags) {
    if (np == 0) return cudaSuccess;
    unsigned g = grid_for(L, np, 8); /* 32 registers, 16 KB shared: 8 CTAs per SM */
    if (type == CJ_INT32) {
        k_decode_fixed<int32_t><<<g, kDecodeThreads, 0, L.stream>>>(
            pages, np, row_start, max_rows, reinterpret_cast<int32_t *>(values), valid, L.dev_errors, col_flags);
        count_launches(1);
    } else {
        k_decode_fixed<long long><<<g, kDecodeThreads, 0, L.stream>>>(
            pages, np, row_start, max_rows, reinterpret_cast<long long *>(values), valid, L.dev_errors,
            col_flags);
        count_launches(1);
    }
    return cudaGetLastError();
}

cudaError_t launch_decode_varchar(const Launch &L, const uint8_t *pages, uint64_t np,
                                  const uint64_t *row_start, uint64_t max_rows, uint64_t *desc,
                                  uint32_t *valid) {
    if (np == 0) return cudaSuccess;
    unsigned g = grid_for(L, np, 6);
    k_decode_varchar<<<g, kDecodeThreads, 0, L.stream>>>(pages, np, row_start, max_rows, desc, valid,
                                                          L.dev_errors);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_decode_grouped(const Launch &L, const DecodeTask *tasks_dev, uint32_t ntasks, uint64_t total_pages,
                                  uint32_t *rows_pp, uint64_t *row_start, void *scan_temp) {
    if (!ntasks) return cudaSuccess;
    if (total_pages) {
        unsigned g = (unsigned)std::min<uint64_t>((total_pages + 255) / 256, (uint64_t)L.num_sms * 8);
        k_page_rows_grouped<<<g, 256, 0, L.stream>>>(tasks_dev, ntasks, total_pages, rows_pp, L.dev_errors);
        count_launches(1);
    }
    cudaError_t e = scan_u32_to_u64(L, rows_pp, row_start, total_pages, scan_temp);
    if (e != cudaSuccess) return e;
    k_check_rows_grouped<<<(ntasks + 127) / 128, 128, 0, L.stream>>>(tasks_dev, ntasks, row_start, L.dev_errors);
    count_launches(1);
    if (total_pages) {
        unsigned g = grid_for(L, total_pages, 6);
        k_decode_grouped<<<g, kDecodeThreads, 0, L.stream>>>(tasks_dev, ntasks, total_pages, row_start, L.dev_errors);
        count_launches(1);
    }
    return cudaGetLastError();
}


} // namespace cj
