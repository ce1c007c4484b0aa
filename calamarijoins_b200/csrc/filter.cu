/*
 * filter.cu — scan-side filters on resident tables (cj_table_filter): the
 * GPU form of the predicate evaluation the reference runs while it loads a
 * table, before execute() (src/build_table.cpp:201-367; Comparison and
 * LogicalOperation, include/data_model/statement.h:54-260,
 * src/statement.cpp:47-241, InnerColumn<T>, include/data_model/
 * inner_column.h).
 *
 * The reference evaluates a predicate column-wise into byte bitmaps and
 * copies the selected rows into a new ColumnarTable. Here:
 *   1. each column the predicate or the projection needs is decoded from its
 *      resident pages (page index, then dense values / string descriptors
 *      and a validity bitmap, or read in place when its pages are full and
 *      NULL-free);
 *   2. every comparison node is one kernel writing a u32 word bitmap (one
 *      thread per row, a ballot per 32 rows); AND / OR / NOT nodes combine
 *      word bitmaps, NOT over the table's rows only;
 *   3. the selected rows' ids are compacted in row order (per-word
 *      popcounts, a scan, then each word's set bits written at its offset);
 *   4. each projected column's pages are written by the result page writers
 *      through those row ids, so the new table's pages are exactly
 *      ColumnInserter<T>'s.
 * Semantics kept from the reference: a comparison is false on NULL rows;
 * IS_NULL / IS_NOT_NULL read the validity bit; NOT flips every row (NULL
 * rows included); INT32 columns compare with the literal's low 32 bits
 * (static_cast<int32_t>); VARCHAR compares bytewise as std::string_view;
 * LIKE matches the whole string with '%' = any run of code points and '_' =
 * one code point, neither matching a newline (the RE2 pattern of
 * Comparison::like_match).
 */
#include <algorithm>
#include <functional>
#include <set>
#include <string>
#include <vector>

#include "cj_device.cuh"
#include "engine.h"
#include "exec_common.h"

namespace cj {
namespace {

constexpr int kFilterThreads = 256;

/* A VARCHAR value's bytes, short or spread over a long-string page chain. */
struct StrView {
    const uint8_t *pages;
    const uint8_t *p = nullptr; /* short string: its bytes */
    uint32_t len = 0;
    /* long string: chain walking cursor */
    uint64_t first = 0, chain = 0;
    uint64_t cur_page = 0, cur_start = 0;
    uint32_t cur_count = 0;
    bool is_long = false;

    CJ_DEV static uint32_t page_count(const uint8_t *page) { return *reinterpret_cast<const uint16_t *>(page + 2); }

    CJ_DEV void init(const uint8_t *pg, uint64_t desc) {
        pages = pg;
        if (!desc_is_long(desc)) {
            p = pg + desc_pos(desc);
            len = desc_len(desc);
            return;
        }
        is_long = true;
        first = desc_pos(desc);
        chain = desc_len(desc);
        uint64_t total = 0;
        for (uint64_t k = 0; k < chain; ++k) total += page_count(pg + (first + k) * kPageSize);
        len = (uint32_t)total;
        cur_page = 0;
        cur_start = 0;
        cur_count = page_count(pg + first * kPageSize);
    }
    CJ_DEV uint8_t at(uint32_t i) {
        if (!is_long) return p[i];
        while (i >= cur_start + cur_count && cur_page + 1 < chain) {
            cur_start += cur_count;
            ++cur_page;
            cur_count = page_count(pages + (first + cur_page) * kPageSize);
        }
        while (i < cur_start && cur_page > 0) {
            --cur_page;
            cur_count = page_count(pages + (first + cur_page) * kPageSize);
            cur_start -= cur_count;
        }
        return pages[(first + cur_page) * kPageSize + 4 + (i - cur_start)];
    }
};

/* Three-way bytewise comparison with the literal (std::string_view order). */
CJ_DEV int str_compare(StrView &s, const uint8_t *lit, uint32_t lit_len) {
    const uint32_t m = s.len < lit_len ? s.len : lit_len;
    for (uint32_t i = 0; i < m; ++i) {
        const uint8_t a = s.at(i), b = lit[i];
        if (a != b) return a < b ? -1 : 1;
    }
    return s.len < lit_len ? -1 : (s.len > lit_len ? 1 : 0);
}

/* Bytes of the UTF-8 code point that starts with byte b (1 for bytes that
 * cannot start one). */
CJ_DEV uint32_t cp_len(uint8_t b) {
    if (b < 0x80) return 1;
    if ((b & 0xE0) == 0xC0) return 2;
    if ((b & 0xF0) == 0xE0) return 3;
    if ((b & 0xF8) == 0xF0) return 4;
    return 1;
}

/* Whole-string LIKE: '%' matches any run of code points and '_' one code
 * point, neither a newline; other pattern bytes match themselves. Greedy
 * with backtracking to the last '%': each '%' extends one code point at a
 * time and never over a newline. */
CJ_DEV bool like_match(StrView &s, const uint8_t *pat, uint32_t m) {
    const uint32_t n = s.len;
    uint32_t i = 0, j = 0;
    int64_t star_j = -1;
    uint32_t star_i = 0;
    while (i < n) {
        if (j < m && pat[j] == '%') {
            star_j = j++;
            star_i = i;
            continue;
        }
        const uint8_t c = s.at(i);
        if (j < m && pat[j] == '_' && c != '\n') {
            i += cp_len(c);
            ++j;
            continue;
        }
        if (j < m && pat[j] != '_' && pat[j] == c) {
            ++i;
            ++j;
            continue;
        }
        if (star_j < 0) return false;
        const uint8_t sc = s.at(star_i);
        if (sc == '\n') return false;
        star_i += cp_len(sc);
        i = star_i;
        j = (uint32_t)star_j + 1;
    }
    while (j < m && pat[j] == '%') ++j;
    return j == m && i == n;
}

struct CmpArgs {
    ColView col;
    uint64_t rows;
    int32_t op;
    int64_t i64;
    double f64;
    const uint8_t *lit;
    uint32_t lit_len;
    uint32_t *out; /* word bitmap */
};

template <typename T> CJ_DEV bool cmp_num(int op, T a, T b) {
    switch (op) {
    case CJ_CMP_EQ: return a == b;
    case CJ_CMP_NEQ: return a != b;
    case CJ_CMP_LT: return a < b;
    case CJ_CMP_GT: return a > b;
    case CJ_CMP_LEQ: return a <= b;
    case CJ_CMP_GEQ: return a >= b;
    default: return false;
    }
}

/* Value of base row r of a fixed-width column and whether it is present. */
template <typename T> CJ_DEV bool fixed_value(const ColView &c, uint32_t r, T *v) {
    if (col_direct(c)) {
        *v = page_value<T>(c.pages, r);
        return true;
    }
    if (!valid_bit(c.valid, r)) return false;
    *v = __ldg(reinterpret_cast<const T *>(c.values) + r);
    return true;
}

CJ_DEV bool row_valid(const ColView &c, uint32_t r) { return col_direct(c) || valid_bit(c.valid, r); }

__global__ void __launch_bounds__(kFilterThreads) k_compare(CmpArgs a) {
    const ColView c = resolve_view(a.col);
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < a.rows; base += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t i = base + threadIdx.x;
        bool bit = false;
        if (i < a.rows) {
            const uint32_t r = (uint32_t)i;
            if (a.op == CJ_CMP_IS_NULL) {
                bit = !row_valid(c, r);
            } else if (a.op == CJ_CMP_IS_NOT_NULL) {
                bit = row_valid(c, r);
            } else if (c.type == CJ_INT32) {
                int32_t v;
                bit = fixed_value<int32_t>(c, r, &v) && cmp_num<int32_t>(a.op, v, (int32_t)a.i64);
            } else if (c.type == CJ_INT64) {
                long long v;
                bit = fixed_value<long long>(c, r, &v) && cmp_num<long long>(a.op, v, (long long)a.i64);
            } else if (c.type == CJ_FP64) {
                double v;
                bit = fixed_value<double>(c, r, &v) && cmp_num<double>(a.op, v, a.f64);
            } else if (valid_bit(c.valid, r)) { /* VARCHAR */
                StrView s;
                s.init(c.pages, __ldg(c.str_desc + r));
                if (a.op == CJ_CMP_LIKE) bit = like_match(s, a.lit, a.lit_len);
                else if (a.op == CJ_CMP_NOT_LIKE) bit = !like_match(s, a.lit, a.lit_len);
                else {
                    const int d = str_compare(s, a.lit, a.lit_len);
                    bit = cmp_num<int>(a.op, d, 0);
                }
            }
        }
        const uint32_t w = __ballot_sync(0xffffffffu, bit);
        if (lane_id() == 0 && base + threadIdx.x < a.rows) a.out[(base + threadIdx.x) >> 5] = w;
    }
}

/* out = a op b over `words` words; NOT (b null) keeps only rows < rows. */
__global__ void k_bitmap_logic(const uint32_t *a, const uint32_t *b, uint32_t *out, uint64_t words, uint64_t rows,
                               int kind) {
    for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < words; w += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t v;
        if (kind == CJ_PRED_AND) v = a[w] & b[w];
        else if (kind == CJ_PRED_OR) v = a[w] | b[w];
        else {
            v = ~a[w];
            const uint64_t lo = w * 32;
            if (lo + 32 > rows) v &= (rows > lo) ? ((1u << (rows - lo)) - 1u) : 0u;
        }
        out[w] = v;
    }
}

__global__ void k_word_popc(const uint32_t *words, uint64_t n, uint32_t *cnt) {
    for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < n; w += (uint64_t)gridDim.x * blockDim.x)
        cnt[w] = __popc(words[w]);
}

/* Row ids of the set bits, in row order: word w's rows go to off[w]... */
__global__ void k_word_emit(const uint32_t *words, const uint64_t *off, uint64_t n, uint32_t *rids) {
    for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < n; w += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t v = words[w];
        uint64_t o = off[w];
        while (v) {
            const int b = __ffs(v) - 1;
            rids[o++] = (uint32_t)(w * 32 + b);
            v &= v - 1;
        }
    }
}

unsigned grid_for(const Context &ctx, uint64_t n, unsigned threads) {
    return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + threads - 1) / threads, (uint64_t)ctx.num_sms * 8));
}

class Filter {
  public:
    Filter(Context &c, const cj_table &t, const cj_predicate *p) : ctx(c), in(t), pred(p), L(c.launch()) {}

    cj_table *run(uint64_t ncols, const uint64_t *cols, uint64_t *num_rows) {
        validate(ncols, cols);
        const uint64_t rows = in.num_rows;
        if (rows > 0xFFFFFFFFull) fail(CJ_ERR_LIMIT, "table exceeds 2^32-1 rows");
        const uint64_t words = std::max<uint64_t>((rows + 31) / 32, 1);
        DevPtr sel;
        uint64_t count = rows;
        if (pred && rows) {
            DevPtr bits = eval(pred->root, words, 0);
            DevPtr cnt = ctx.alloc(words * 4), off = ctx.alloc((words + 1) * 8);
            DevPtr tmp = ctx.alloc(scan_temp_bytes(words));
            k_word_popc<<<grid_for(ctx, words, 256), 256, 0, ctx.stream>>>(bits->as<uint32_t>(), words,
                                                                             cnt->as<uint32_t>());
            count_launches(1);
            check_cuda(cudaGetLastError(), "popc");
            check_cuda(scan_u32_to_u64(L, cnt->as<uint32_t>(), off->as<uint64_t>(), words, tmp->ptr), "scan");
            /* the count goes back with the status block (sync_status copies
             * all of it to the host) */
            check_cuda(cudaMemcpyAsync(&ctx.d_status->aux[7], off->as<uint64_t>() + words, 8,
                                       cudaMemcpyDeviceToDevice, ctx.stream),
                       "copy");
            ctx.sync_status();
            count = ctx.h_status->aux[7];
            sel = ctx.alloc(std::max<uint64_t>(count, 1) * 4);
            k_word_emit<<<grid_for(ctx, words, 256), 256, 0, ctx.stream>>>(bits->as<uint32_t>(), off->as<uint64_t>(),
                                                                             words, sel->as<uint32_t>());
            count_launches(1);
            check_cuda(cudaGetLastError(), "emit");
        }
        auto tab = std::make_unique<cj_table>();
        tab->ctx = &ctx;
        tab->num_rows = count;
        const uint32_t TR = 2048;
        for (uint64_t k = 0; k < ncols; ++k) {
            const uint64_t c = cols[k];
            ColumnPages cp;
            cp.type = in.cols[c].type;
            if (count) {
                ColView v = view(c);
                v.rid_a = sel ? sel->as<uint32_t>() : nullptr;
                if (cp.type != CJ_VARCHAR) {
                    const uint32_t R = rows_per_page_fixed(cp.type);
                    cp.num_pages = (count + R - 1) / R;
                    cp.owner = ctx.alloc(cp.num_pages * kPageSize);
                    check_cuda(launch_write_fixed_pages(L, v, count, cp.owner->as<uint8_t>()), "write_fixed");
                } else {
                    DevPtr temp = ctx.alloc(varchar_temp_bytes(count, TR));
                    check_cuda(launch_varchar_plan(L, v, count, TR, temp->ptr,
                                                   reinterpret_cast<unsigned long long *>(&ctx.d_status->aux[7])),
                               "varchar_plan");
                    ctx.sync_status(); /* brings the page count back in aux[7] */
                    cp.num_pages = ctx.h_status->aux[7];
                    cp.owner = ctx.alloc(cp.num_pages * kPageSize);
                    check_cuda(launch_varchar_write(L, v, count, TR, temp->ptr, cp.owner->as<uint8_t>()),
                               "varchar_write");
                }
                cp.dev = cp.owner->as<uint8_t>();
            }
            tab->cols.push_back(std::move(cp));
        }
        ctx.sync_status();
        if (num_rows) *num_rows = count;
        return tab.release();
    }

  private:
    Context &ctx;
    const cj_table &in;
    const cj_predicate *pred;
    Launch L;
    std::map<uint64_t, Decoded> decoded;
    std::vector<DevPtr> keep;

    void validate(uint64_t ncols, const uint64_t *cols) {
        if (ncols && !cols) fail(CJ_ERR_INVALID_ARGUMENT, "null column list");
        for (uint64_t k = 0; k < ncols; ++k)
            if (cols[k] >= in.cols.size()) fail(CJ_ERR_INVALID_PLAN, "projected column out of range");
        if (!pred) return;
        if (!pred->nodes || pred->root >= pred->num_nodes) fail(CJ_ERR_INVALID_PLAN, "bad predicate root");
        for (uint64_t i = 0; i < pred->num_nodes; ++i) {
            const cj_pred_node &n = pred->nodes[i];
            if (n.kind == CJ_PRED_CMP) {
                if (n.column >= in.cols.size()) fail(CJ_ERR_INVALID_PLAN, "predicate column out of range");
                if (n.op < CJ_CMP_EQ || n.op > CJ_CMP_IS_NOT_NULL) fail(CJ_ERR_INVALID_PLAN, "unknown comparison");
                if (n.op == CJ_CMP_IS_NULL || n.op == CJ_CMP_IS_NOT_NULL) continue;
                const int32_t t = in.cols[n.column].type;
                const bool like = n.op == CJ_CMP_LIKE || n.op == CJ_CMP_NOT_LIKE;
                if (t == CJ_VARCHAR) {
                    if (n.literal_type != CJ_VARCHAR || (n.str_len && !n.str))
                        fail(CJ_ERR_INVALID_PLAN, "VARCHAR column compared with a non-string literal");
                    if (n.str_len > 0xFFFFFFFFull) fail(CJ_ERR_LIMIT, "literal too long");
                } else if (like || n.literal_type == CJ_VARCHAR || (t != CJ_FP64 && n.literal_type != CJ_INT64)) {
                    fail(CJ_ERR_INVALID_PLAN, "comparison literal does not fit the column's type");
                }
            } else if (n.kind == CJ_PRED_AND || n.kind == CJ_PRED_OR) {
                if (n.left >= pred->num_nodes || n.right >= pred->num_nodes)
                    fail(CJ_ERR_INVALID_PLAN, "predicate child out of range");
            } else if (n.kind == CJ_PRED_NOT) {
                if (n.left >= pred->num_nodes) fail(CJ_ERR_INVALID_PLAN, "predicate child out of range");
            } else {
                fail(CJ_ERR_INVALID_PLAN, "unknown predicate node");
            }
        }
    }

    const Decoded &decode(uint64_t c) {
        auto it = decoded.find(c);
        if (it != decoded.end()) return it->second;
        Decoded d;
        d.type = in.cols[c].type;
        d.rows = in.num_rows;
        d.src = in.cols[c];
        const uint64_t np = d.src.num_pages;
        DevPtr rows_pp = ctx.alloc(std::max<uint64_t>(np, 1) * 4);
        DevPtr row_start = ctx.alloc((np + 1) * 8);
        DevPtr partials = ctx.alloc(page_index_blocks(L, np) * 8);
        keep.push_back(rows_pp);
        keep.push_back(row_start);
        keep.push_back(partials);
        d.col_flags = ctx.alloc(8);
        check_cuda(cudaMemsetAsync(d.col_flags->ptr, 0, 8, ctx.stream), "memset");
        check_cuda(launch_page_index(L, d.src.dev, np, d.type, d.rows, rows_pp->as<uint32_t>(),
                                     partials->as<uint64_t>(), row_start->as<uint64_t>(), d.col_flags->as<uint32_t>()),
                   "page_index");
        const uint64_t words = std::max<uint64_t>((d.rows + 31) / 32, 1);
        d.valid = ctx.alloc(words * 4);
        check_cuda(cudaMemsetAsync(d.valid->ptr, 0, words * 4, ctx.stream), "memset");
        if (d.type == CJ_VARCHAR) {
            d.desc = ctx.alloc(std::max<uint64_t>(d.rows, 1) * 8);
            check_cuda(launch_decode_varchar(L, d.src.dev, np, row_start->as<uint64_t>(), d.rows,
                                             d.desc->as<uint64_t>(), d.valid->as<uint32_t>()),
                       "decode_varchar");
        } else {
            d.values = ctx.alloc(std::max<uint64_t>(d.rows, 1) * (d.type == CJ_INT32 ? 4 : 8));
            check_cuda(launch_decode_fixed(L, d.src.dev, np, d.type, row_start->as<uint64_t>(), d.rows,
                                           d.values->ptr, d.valid->as<uint32_t>(), d.col_flags->as<uint32_t>()),
                       "decode_fixed");
        }
        return decoded.emplace(c, std::move(d)).first->second;
    }

    ColView view(uint64_t c) {
        const Decoded &d = decode(c);
        Relation R;
        RelCol rc{d.type, 0, c, -1, false};
        return make_view(d, R, rc, nullptr);
    }

    DevPtr eval(uint64_t node, uint64_t words, int depth) {
        if (depth > (int)pred->num_nodes) fail(CJ_ERR_INVALID_PLAN, "predicate has a cycle");
        const cj_pred_node &n = pred->nodes[node];
        DevPtr out = ctx.alloc(words * 4);
        if (n.kind == CJ_PRED_CMP) {
            CmpArgs a{};
            a.col = view(n.column);
            a.rows = in.num_rows;
            a.op = n.op;
            a.i64 = n.i64;
            a.f64 = n.literal_type == CJ_INT64 ? (double)n.i64 : n.f64;
            a.out = out->as<uint32_t>();
            if (in.cols[n.column].type == CJ_VARCHAR && n.op != CJ_CMP_IS_NULL && n.op != CJ_CMP_IS_NOT_NULL) {
                DevPtr lit = ctx.alloc(std::max<uint64_t>(n.str_len, 1));
                if (n.str_len)
                    check_cuda(cudaMemcpyAsync(lit->ptr, n.str, n.str_len, cudaMemcpyHostToDevice, ctx.stream),
                               "literal");
                a.lit = lit->as<uint8_t>();
                a.lit_len = (uint32_t)n.str_len;
                keep.push_back(lit);
            }
            const unsigned grid = grid_for(ctx, in.num_rows, kFilterThreads);
            k_compare<<<grid, kFilterThreads, 0, ctx.stream>>>(a);
            count_launches(1);
            check_cuda(cudaGetLastError(), "compare");
        } else {
            DevPtr l = eval(n.left, words, depth + 1);
            DevPtr r = n.kind == CJ_PRED_NOT ? nullptr : eval(n.right, words, depth + 1);
            k_bitmap_logic<<<grid_for(ctx, words, 256), 256, 0, ctx.stream>>>(
                l->as<uint32_t>(), r ? r->as<uint32_t>() : nullptr, out->as<uint32_t>(), words, in.num_rows, n.kind);
            count_launches(1);
            check_cuda(cudaGetLastError(), "bitmap logic");
        }
        return out;
    }
};

} // namespace

cj_table *filter_table(Context &ctx, const cj_table &in, const cj_predicate *pred, uint64_t ncols,
                       const uint64_t *cols, uint64_t *num_rows) {
    Filter f(ctx, in, pred);
    return f.run(ncols, cols, num_rows);
}

} // namespace cj

extern "C" int cj_table_filter(cj_context *ctx, const cj_table *in, const cj_predicate *pred, uint64_t num_columns,
                               const uint64_t *columns, cj_table **out, uint64_t *num_rows) {
    if (!ctx || !in || !out) return cj::set_last_error(CJ_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    if (in->ctx != ctx && in->ctx->device != ctx->device)
        return cj::set_last_error(CJ_ERR_INVALID_ARGUMENT, "table of another device");
    cudaSetDevice(ctx->device);
    try {
        *out = cj::filter_table(*ctx, *in, pred, num_columns, columns, num_rows);
    } catch (const cj::Error &e) {
        cudaStreamSynchronize(ctx->stream);
        cudaGetLastError();
        return cj::set_last_error(e.code, e.msg);
    } catch (const std::bad_alloc &) {
        return cj::set_last_error(CJ_ERR_OUT_OF_MEMORY, "host allocation failed");
    }
    cj::clear_last_error();
    return CJ_OK;
}
