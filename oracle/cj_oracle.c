/*
 * cj_oracle.c — CPU oracle (checker) for the B200 join pipeline.
 *
 * TEST INFRASTRUCTURE ONLY: loaded by tests/, __graft_entry__.smoke() and
 * the CPU-baseline leg of bench.py. The product library never uses it.
 *
 * A single-threaded restatement of CalamariJoins' execute() path. Each
 * function names the reference code it follows (paths relative to the
 * CalamariJoins tree). Where the reference is defective the restatement
 * follows the format contract instead, and says so:
 *   - INT64 / FP64 output columns: the reference routes them through its
 *     VARCHAR page builder (include/materialization/materialize.h:235-263)
 *     and produces garbage or aborts; here they are encoded exactly as
 *     ColumnInserter<int64_t/double> (include/data_model/plan.h:187-270).
 *   - NULL VARCHAR output rows: the reference's VarcharPageBuilder drops or
 *     misaligns them (include/materialization/page_builders.h:207-212,
 *     293-301); here they are encoded as ColumnInserter<std::string> does.
 *   - NULL build keys from an intermediate: the reference inserts the
 *     INT32_MIN NULL sentinel into the hash table
 *     (include/join_execution/hashtable.h:355-361); here NULL never matches,
 *     as in its nested-loop path (include/join_execution/nested_loop.h:80-86).
 *   - INT64 keys are accepted (the reference supports INT32 keys only,
 *     hashtable.h:66-69); keys compare as 64-bit integers.
 */
#define _GNU_SOURCE
#include "cj_oracle.h"

#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define PAGE ((uint64_t)CJ_PAGE_SIZE)

static inline uint16_t rd16(const uint8_t *p) {
    uint16_t v;
    memcpy(&v, p, 2);
    return v;
}
static inline void wr16(uint8_t *p, uint16_t v) { memcpy(p, &v, 2); }

static void fmt_msg(char *msg, uint64_t len, const char *f, ...) {
    if (!msg || !len) return;
    va_list ap;
    va_start(ap, f);
    vsnprintf(msg, (size_t)len, f, ap);
    va_end(ap);
}

static void *xcalloc(uint64_t n, uint64_t sz) {
    if (n == 0) n = 1;
    return calloc((size_t)n, (size_t)sz);
}

/* ======================================================================== */
/* Growable page buffer (pages are zero-initialised for determinism).        */
/* ======================================================================== */
typedef struct {
    uint8_t *data;
    uint64_t pages;
    uint64_t cap;
} pagebuf;

static uint8_t *pb_page(pagebuf *b, uint64_t idx) {
    while (idx >= b->cap) {
        uint64_t nc = b->cap ? b->cap * 2 : 16;
        uint8_t *nd = (uint8_t *)realloc(b->data, nc * PAGE);
        if (!nd) return NULL;
        memset(nd + b->cap * PAGE, 0, (nc - b->cap) * PAGE);
        b->data = nd;
        b->cap = nc;
    }
    if (idx + 1 > b->pages) b->pages = idx + 1;
    return b->data + idx * PAGE;
}

/* ======================================================================== */
/* ColumnInserter<T> restatement (include/data_model/plan.h:187-366).        */
/* ======================================================================== */
typedef struct {
    int32_t type;
    pagebuf *pb;
    uint64_t last_page_idx;
    uint16_t num_rows;
    uint64_t data_end;   /* fixed: byte offset of next value              */
    uint8_t bitmap[PAGE];
    /* VARCHAR state (plan.h:273-366) */
    uint16_t data_size;
    uint64_t offset_end;
    char data[PAGE];
    int oom;
} inserter;

static uint64_t elem_size(int32_t t) { return t == CJ_INT32 ? 4 : 8; }

/* plan.h:196-202: values start at max(4, sizeof(T)). */
static uint64_t data_begin(int32_t t) { return t == CJ_INT32 ? 4 : 8; }

static void ins_init(inserter *in, int32_t type, pagebuf *pb) {
    memset(in, 0, sizeof(*in));
    in->type = type;
    in->pb = pb;
    in->data_end = data_begin(type);
    in->offset_end = 4;
}

static uint8_t *ins_get_page(inserter *in) { /* plan.h:207-213 */
    uint8_t *p = pb_page(in->pb, in->last_page_idx);
    if (!p) in->oom = 1;
    return p;
}

static void ins_save_page_fixed(inserter *in) { /* plan.h:215-227 */
    uint8_t *page = ins_get_page(in);
    if (!page) return;
    uint64_t w = elem_size(in->type);
    wr16(page, in->num_rows);
    wr16(page + 2, (uint16_t)((in->data_end - data_begin(in->type)) / w));
    uint64_t bitmap_size = (in->num_rows + 7) / 8;
    memcpy(page + PAGE - bitmap_size, in->bitmap, bitmap_size);
    ++in->last_page_idx;
    in->num_rows = 0;
    in->data_end = data_begin(in->type);
}

static void set_bit(uint8_t *bm, uint64_t i) { bm[i / 8] |= (uint8_t)(1u << (i % 8)); }
static void unset_bit(uint8_t *bm, uint64_t i) { bm[i / 8] &= (uint8_t)~(1u << (i % 8)); }

/* plan.h:241-250, with one correction: ColumnInserter tests
 * data_end + 4 + num_rows/8 + 1, which for 8-byte values lets the last value
 * overlap the bitmap (whose copy then clobbers its top byte). The test here
 * reserves the value's real width, as Table::to_columnar does for INT64 /
 * FP64 (src/build_table.cpp:746-752); for INT32 both tests are the same. */
static void ins_insert_fixed(inserter *in, const void *value) {
    uint64_t w = elem_size(in->type);
    if (in->data_end + w + in->num_rows / 8 + 1 > PAGE) ins_save_page_fixed(in);
    uint8_t *page = ins_get_page(in);
    if (!page) return;
    memcpy(page + in->data_end, value, w);
    in->data_end += w;
    set_bit(in->bitmap, in->num_rows);
    ++in->num_rows;
}

static void ins_insert_null_fixed(inserter *in) { /* plan.h:252-258 */
    if (in->data_end + in->num_rows / 8 + 1 > PAGE) ins_save_page_fixed(in);
    unset_bit(in->bitmap, in->num_rows);
    ++in->num_rows;
}

static void ins_save_long_string(inserter *in, const char *s, uint64_t len) {
    /* plan.h:294-312 */
    uint64_t offset = 0;
    int first = 1;
    while (offset < len) {
        uint8_t *page = ins_get_page(in);
        if (!page) return;
        wr16(page, first ? 0xffff : 0xfffe);
        first = 0;
        uint64_t chunk = len - offset < PAGE - 4 ? len - offset : PAGE - 4;
        wr16(page + 2, (uint16_t)chunk);
        memcpy(page + 4, s + offset, chunk);
        offset += chunk;
        ++in->last_page_idx;
    }
}

static void ins_save_page_varchar(inserter *in) { /* plan.h:314-326 */
    uint8_t *page = ins_get_page(in);
    if (!page) return;
    wr16(page, in->num_rows);
    wr16(page + 2, (uint16_t)((in->offset_end - 4) / 2));
    uint64_t bitmap_size = (in->num_rows + 7) / 8;
    memcpy(page + in->offset_end, in->data, in->data_size);
    memcpy(page + PAGE - bitmap_size, in->bitmap, bitmap_size);
    ++in->last_page_idx;
    in->num_rows = 0;
    in->data_size = 0;
    in->offset_end = 4;
}

static void ins_insert_varchar(inserter *in, const char *s, uint64_t len) {
    /* plan.h:340-361 */
    if (len > PAGE - 7) {
        if (in->num_rows > 0) ins_save_page_varchar(in);
        ins_save_long_string(in, s, len);
        return;
    }
    if (in->offset_end + 2 + in->data_size + len + in->num_rows / 8 + 1 > PAGE)
        ins_save_page_varchar(in);
    memcpy(in->data + in->data_size, s, len);
    in->data_size = (uint16_t)(in->data_size + len);
    uint8_t *page = ins_get_page(in);
    if (!page) return;
    wr16(page + in->offset_end, in->data_size);
    in->offset_end += 2;
    set_bit(in->bitmap, in->num_rows);
    ++in->num_rows;
}

static void ins_insert_null_varchar(inserter *in) { /* plan.h:363-369 */
    if (in->offset_end + in->data_size + in->num_rows / 8 + 1 > PAGE)
        ins_save_page_varchar(in);
    unset_bit(in->bitmap, in->num_rows);
    ++in->num_rows;
}

static void ins_finalize(inserter *in) { /* plan.h:261-265, 371-375 */
    if (in->num_rows != 0) {
        if (in->type == CJ_VARCHAR)
            ins_save_page_varchar(in);
        else
            ins_save_page_fixed(in);
    }
}

int cjo_encode_column(int32_t type, const void *values, const uint64_t *offsets,
                      const uint8_t *valid, uint64_t n, void *out_pages,
                      uint64_t capacity, uint64_t *num_pages) {
    if (type < CJ_INT32 || type > CJ_VARCHAR || !num_pages) return CJ_ERR_INVALID_ARGUMENT;
    if (n && !values) return CJ_ERR_INVALID_ARGUMENT;
    if (type == CJ_VARCHAR && n && !offsets) return CJ_ERR_INVALID_ARGUMENT;
    pagebuf pb = {0};
    inserter *in = (inserter *)malloc(sizeof(inserter));
    if (!in) return CJ_ERR_OUT_OF_MEMORY;
    ins_init(in, type, &pb);
    for (uint64_t i = 0; i < n && !in->oom; ++i) {
        int v = valid ? valid[i] != 0 : 1;
        if (type == CJ_VARCHAR) {
            if (v)
                ins_insert_varchar(in, (const char *)values + offsets[i],
                                   offsets[i + 1] - offsets[i]);
            else
                ins_insert_null_varchar(in);
        } else {
            if (v)
                ins_insert_fixed(in, (const uint8_t *)values + i * elem_size(type));
            else
                ins_insert_null_fixed(in);
        }
    }
    ins_finalize(in);
    int oom = in->oom;
    uint64_t pages = in->last_page_idx;
    free(in);
    if (oom) {
        free(pb.data);
        return CJ_ERR_OUT_OF_MEMORY;
    }
    *num_pages = pages;
    int rc = CJ_OK;
    if (out_pages) {
        if (pages > capacity)
            rc = CJ_ERR_LIMIT;
        else if (pages)
            memcpy(out_pages, pb.data, pages * PAGE);
    }
    free(pb.data);
    return rc;
}

/* ======================================================================== */
/* Page decode: Table::from_columnar restatement (src/build_table.cpp:520-659)*/
/* ======================================================================== */
typedef struct {
    cjo_column *c;
    uint64_t cap;
    uint64_t char_cap;
} colbuilder;

static int cb_reserve(colbuilder *b, uint64_t rows) {
    cjo_column *c = b->c;
    if (rows <= b->cap) return 0;
    uint64_t nc = b->cap ? b->cap : 64;
    while (nc < rows) nc *= 2;
    uint8_t *nv = (uint8_t *)realloc(c->valid, nc);
    if (!nv) return -1;
    c->valid = nv;
    if (c->type == CJ_INT32) {
        int32_t *p = (int32_t *)realloc(c->i32, nc * 4);
        if (!p) return -1;
        c->i32 = p;
    } else if (c->type == CJ_INT64) {
        int64_t *p = (int64_t *)realloc(c->i64, nc * 8);
        if (!p) return -1;
        c->i64 = p;
    } else if (c->type == CJ_FP64) {
        double *p = (double *)realloc(c->f64, nc * 8);
        if (!p) return -1;
        c->f64 = p;
    } else {
        uint64_t *p = (uint64_t *)realloc(c->str_off, (nc + 1) * 8);
        if (!p) return -1;
        c->str_off = p;
    }
    b->cap = nc;
    return 0;
}

static int cb_chars(colbuilder *b, uint64_t need) {
    if (need <= b->char_cap) return 0;
    uint64_t nc = b->char_cap ? b->char_cap : 256;
    while (nc < need) nc *= 2;
    char *p = (char *)realloc(b->c->chars, nc);
    if (!p) return -1;
    b->c->chars = p;
    b->char_cap = nc;
    return 0;
}

static int get_bitmap(const uint8_t *bm, uint64_t i) { return (bm[i / 8] >> (i % 8)) & 1; }

int cjo_decode_column(int32_t type, const void *const *pages, uint64_t num_pages,
                      uint64_t expected_rows, cjo_column *out) {
    if (!out || type < CJ_INT32 || type > CJ_VARCHAR || (num_pages && !pages))
        return CJ_ERR_INVALID_ARGUMENT;
    memset(out, 0, sizeof(*out));
    out->type = type;
    colbuilder b = {out, 0, 0};
    if (cb_reserve(&b, 1)) return CJ_ERR_OUT_OF_MEMORY;
    uint64_t rows = 0, nchars = 0;
    if (type == CJ_VARCHAR) out->str_off[0] = 0;
    for (uint64_t p = 0; p < num_pages; ++p) {
        const uint8_t *page = (const uint8_t *)pages[p];
        uint16_t nr = rd16(page);
        if (type != CJ_VARCHAR) {
            /* INT32: values at +4; INT64/FP64 at +8 (build_table.cpp:533-592) */
            uint64_t w = elem_size(type), base = data_begin(type);
            const uint8_t *bm = page + PAGE - (nr + 7) / 8;
            uint16_t di = 0;
            if (cb_reserve(&b, rows + nr + 1)) return CJ_ERR_OUT_OF_MEMORY;
            for (uint16_t i = 0; i < nr; ++i) {
                if (get_bitmap(bm, i)) {
                    if (base + (uint64_t)(di + 1) * w > PAGE) {
                        cjo_column_free(out);
                        return CJ_ERR_MALFORMED_PAGE;
                    }
                    const uint8_t *src = page + base + (uint64_t)di * w;
                    out->valid[rows] = 1;
                    if (type == CJ_INT32) memcpy(&out->i32[rows], src, 4);
                    else if (type == CJ_INT64) memcpy(&out->i64[rows], src, 8);
                    else memcpy(&out->f64[rows], src, 8);
                    ++di;
                } else {
                    out->valid[rows] = 0;
                    if (type == CJ_INT32) out->i32[rows] = 0;
                    else if (type == CJ_INT64) out->i64[rows] = 0;
                    else out->f64[rows] = 0;
                }
                ++rows;
            }
        } else if (nr == 0xffff) { /* build_table.cpp:597-606 */
            uint16_t nch = rd16(page + 2);
            if (nch > PAGE - 4) { cjo_column_free(out); return CJ_ERR_MALFORMED_PAGE; }
            if (cb_reserve(&b, rows + 2) || cb_chars(&b, nchars + nch))
                return CJ_ERR_OUT_OF_MEMORY;
            memcpy(out->chars + nchars, page + 4, nch);
            nchars += nch;
            out->valid[rows] = 1;
            out->str_off[rows + 1] = nchars;
            ++rows;
        } else if (nr == 0xfffe) { /* build_table.cpp:607-621 */
            uint16_t nch = rd16(page + 2);
            if (rows == 0 || !out->valid[rows - 1] || nch > PAGE - 4) {
                cjo_column_free(out);
                return CJ_ERR_MALFORMED_PAGE; /* "must follow a string" */
            }
            if (cb_chars(&b, nchars + nch)) return CJ_ERR_OUT_OF_MEMORY;
            memcpy(out->chars + nchars, page + 4, nch);
            nchars += nch;
            out->str_off[rows] = nchars;
        } else { /* build_table.cpp:622-647 */
            uint16_t nv = rd16(page + 2);
            const uint8_t *offs = page + 4;
            const uint8_t *data = page + 4 + (uint64_t)nv * 2;
            const uint8_t *bm = page + PAGE - (nr + 7) / 8;
            if (4 + (uint64_t)nv * 2 > PAGE) { cjo_column_free(out); return CJ_ERR_MALFORMED_PAGE; }
            uint16_t di = 0;
            uint16_t prev = 0;
            if (cb_reserve(&b, rows + nr + 1)) return CJ_ERR_OUT_OF_MEMORY;
            for (uint16_t i = 0; i < nr; ++i) {
                if (get_bitmap(bm, i)) {
                    if (di >= nv) { cjo_column_free(out); return CJ_ERR_MALFORMED_PAGE; }
                    uint16_t end = rd16(offs + (uint64_t)di * 2);
                    if (end < prev || data + end > page + PAGE) {
                        cjo_column_free(out);
                        return CJ_ERR_MALFORMED_PAGE;
                    }
                    uint64_t len = (uint64_t)(end - prev);
                    if (cb_chars(&b, nchars + len)) return CJ_ERR_OUT_OF_MEMORY;
                    memcpy(out->chars + nchars, data + prev, len);
                    nchars += len;
                    prev = end;
                    ++di;
                    out->valid[rows] = 1;
                } else {
                    out->valid[rows] = 0;
                }
                out->str_off[rows + 1] = nchars;
                ++rows;
            }
        }
    }
    out->num_rows = rows;
    if (expected_rows != UINT64_MAX && rows != expected_rows) {
        cjo_column_free(out);
        return CJ_ERR_MALFORMED_PAGE;
    }
    return CJ_OK;
}

int cjo_decode_column_contig(int32_t type, const void *pages, uint64_t num_pages,
                             uint64_t expected_rows, cjo_column *out) {
    const void **ptrs = (const void **)xcalloc(num_pages, sizeof(void *));
    if (!ptrs) return CJ_ERR_OUT_OF_MEMORY;
    for (uint64_t i = 0; i < num_pages; ++i) ptrs[i] = (const uint8_t *)pages + i * PAGE;
    int rc = cjo_decode_column(type, ptrs, num_pages, expected_rows, out);
    free(ptrs);
    return rc;
}

void cjo_column_free(cjo_column *c) {
    if (!c) return;
    free(c->valid);
    free(c->i32);
    free(c->i64);
    free(c->f64);
    free(c->str_off);
    free(c->chars);
    memset(c, 0, sizeof(*c));
}

/* ======================================================================== */
/* Structural validation of a column's pages (format rules of plan.h and     */
/* README.md "Data format").                                                 */
/* ======================================================================== */
static int popcount_bits(const uint8_t *bm, uint64_t n) {
    int c = 0;
    for (uint64_t i = 0; i < n; ++i) c += get_bitmap(bm, i);
    return c;
}

int cjo_validate_column(int32_t type, const void *pages, uint64_t num_pages,
                        uint64_t expected_rows, char *msg, uint64_t msg_len) {
    uint64_t rows = 0;
    int in_long = 0;
    for (uint64_t p = 0; p < num_pages; ++p) {
        const uint8_t *page = (const uint8_t *)pages + p * PAGE;
        uint16_t nr = rd16(page), nv = rd16(page + 2);
        if (type == CJ_VARCHAR && (nr == 0xffff || nr == 0xfffe)) {
            if (nr == 0xfffe && !in_long) {
                fmt_msg(msg, msg_len, "page %llu: continuation without start", (unsigned long long)p);
                return CJ_ERR_MALFORMED_PAGE;
            }
            if (nv == 0 || nv > PAGE - 4) {
                fmt_msg(msg, msg_len, "page %llu: long-string chunk %u", (unsigned long long)p, nv);
                return CJ_ERR_MALFORMED_PAGE;
            }
            in_long = 1;
            if (nr == 0xffff) rows += 1;
            continue;
        }
        in_long = 0;
        if (nr == 0) {
            fmt_msg(msg, msg_len, "page %llu: empty page", (unsigned long long)p);
            return CJ_ERR_MALFORMED_PAGE;
        }
        uint64_t bms = (nr + 7) / 8;
        const uint8_t *bm = page + PAGE - bms;
        int pc = popcount_bits(bm, nr);
        if (pc != nv) {
            fmt_msg(msg, msg_len, "page %llu: popcount %d != n_values %u", (unsigned long long)p, pc, nv);
            return CJ_ERR_MALFORMED_PAGE;
        }
        if (type != CJ_VARCHAR) {
            uint64_t end = data_begin(type) + (uint64_t)nv * elem_size(type);
            if (end > PAGE - bms) {
                fmt_msg(msg, msg_len, "page %llu: values overlap bitmap", (unsigned long long)p);
                return CJ_ERR_MALFORMED_PAGE;
            }
        } else {
            uint64_t cb = 4 + (uint64_t)nv * 2;
            uint16_t prev = 0;
            for (uint16_t k = 0; k < nv; ++k) {
                uint16_t e = rd16(page + 4 + (uint64_t)k * 2);
                if (e < prev) {
                    fmt_msg(msg, msg_len, "page %llu: offsets not monotone", (unsigned long long)p);
                    return CJ_ERR_MALFORMED_PAGE;
                }
                prev = e;
            }
            if (cb + prev > PAGE - bms) {
                fmt_msg(msg, msg_len, "page %llu: chars overlap bitmap", (unsigned long long)p);
                return CJ_ERR_MALFORMED_PAGE;
            }
        }
        rows += nr;
    }
    if (expected_rows != UINT64_MAX && rows != expected_rows) {
        fmt_msg(msg, msg_len, "rows %llu != expected %llu", (unsigned long long)rows,
                (unsigned long long)expected_rows);
        return CJ_ERR_MALFORMED_PAGE;
    }
    return CJ_OK;
}

/* ======================================================================== */
/* Hash table restatement (include/join_execution/hashtable.h, bloom_tags.h) */
/* ======================================================================== */

/* CRC32C update of one 32-bit word with initial value `crc`, as
 * _mm_crc32_u32 / __crc32w compute it (hashtable.h:146-154): reflected
 * Castagnoli polynomial 0x82F63B78, no pre/post inversion. */
static uint32_t crc32c_u32(uint32_t crc, uint32_t v) {
    for (int b = 0; b < 4; ++b) {
        crc ^= (v >> (8 * b)) & 0xffu;
        for (int k = 0; k < 8; ++k) crc = (crc >> 1) ^ (0x82F63B78u & (0u - (crc & 1u)));
    }
    return crc;
}

/* hash_key (hashtable.h:146-154). 64-bit keys that do not fit in 32 bits
 * (an extension) fold both halves through the CRC. */
static uint64_t hash_key(int64_t key) {
    const uint64_t k = 0x8648DBDBull;
    uint32_t crc;
    if (key >= INT32_MIN && key <= INT32_MAX)
        crc = crc32c_u32(0, (uint32_t)(int32_t)key);
    else
        crc = crc32c_u32(crc32c_u32(0, (uint32_t)key), (uint32_t)((uint64_t)key >> 32));
    return (uint64_t)crc * ((k << 32) + 1);
}

/* BLOOM_TAGS (bloom_tags.h:35-263) is the ascending list of the 2048
 * smallest 16-bit values with exactly five bits set; regenerated here. */
static uint16_t BLOOM[2048];
static int bloom_ready = 0;
static void bloom_init(void) {
    if (bloom_ready) return;
    int n = 0;
    for (uint32_t v = 0; v < 65536 && n < 2048; ++v)
        if (__builtin_popcount(v) == 5) BLOOM[n++] = (uint16_t)v;
    bloom_ready = 1;
}
static uint16_t bloom_tag(uint64_t h) { return BLOOM[(h >> 32) & 0x7FF]; } /* :163-165 */

typedef struct {
    uint64_t *directory; /* (end << 16) | tags                          */
    int64_t *keys;
    uint32_t *row_ids;
    uint64_t num_slots;
    int shift;           /* log2(num_slots)                             */
    uint64_t size;
} uht;

/* Constructor (hashtable.h:255-264): directory = pow2 >= max(2048, n). */
static int uht_init(uht *t, uint64_t build_size) {
    memset(t, 0, sizeof(*t));
    uint64_t pow2 = 2048;
    while (pow2 < build_size) pow2 <<= 1;
    t->directory = (uint64_t *)xcalloc(pow2, 8);
    if (!t->directory) return -1;
    t->num_slots = pow2;
    t->shift = __builtin_ctzll(pow2);
    return 0;
}
static void uht_free(uht *t) {
    free(t->directory);
    free(t->keys);
    free(t->row_ids);
}
static uint64_t slot_for(const uht *t, uint64_t h) { return h >> (64 - t->shift); } /* :167-169 */

/* Build from (key, row id) tuples: the per-slot counting sort of
 * build_partition (hashtable.h:197-246) applied to the whole directory
 * (partitioning only splits this work among threads). */
static int uht_build(uht *t, const int64_t *keys, const uint32_t *rids, uint64_t n) {
    if (n == 0) return 0;
    uint32_t *counts = (uint32_t *)xcalloc(t->num_slots, 4);
    t->keys = (int64_t *)xcalloc(n, 8);
    t->row_ids = (uint32_t *)xcalloc(n, 4);
    if (!counts || !t->keys || !t->row_ids) { free(counts); return -1; }
    for (uint64_t i = 0; i < n; ++i) counts[slot_for(t, hash_key(keys[i]))]++;
    uint64_t running = 0;
    uint64_t *offsets = (uint64_t *)xcalloc(t->num_slots, 8);
    if (!offsets) { free(counts); return -1; }
    for (uint64_t s = 0; s < t->num_slots; ++s) {
        offsets[s] = running;
        running += counts[s];
        counts[s] = 0;
    }
    for (uint64_t i = 0; i < n; ++i) {
        uint64_t h = hash_key(keys[i]);
        uint64_t s = slot_for(t, h);
        uint64_t idx = offsets[s] + counts[s]++;
        t->keys[idx] = keys[i];
        t->row_ids[idx] = rids[i];
        t->directory[s] |= bloom_tag(h);
    }
    for (uint64_t s = 0; s < t->num_slots; ++s) {
        uint64_t end = offsets[s] + counts[s];
        t->directory[s] = (end << 16) | (t->directory[s] & 0xFFFF);
    }
    t->size = n;
    free(counts);
    free(offsets);
    return 0;
}

/* find_indices (hashtable.h:298-313). */
static void uht_find(const uht *t, int64_t key, uint64_t *start, uint64_t *end) {
    *start = *end = 0;
    if (t->size == 0) return;
    uint64_t h = hash_key(key);
    uint64_t s = slot_for(t, h);
    uint64_t entry = t->directory[s];
    uint16_t tag = bloom_tag(h);
    if ((entry & tag) != tag) return;
    *end = entry >> 16;
    *start = s == 0 ? 0 : (t->directory[s - 1] >> 16);
}

/* ======================================================================== */
/* Join execution restatement (src/execute.cpp).                             */
/* ======================================================================== */

/* An intermediate column (mema::column_t, include/data_model/intermediate.h:
 * 82-162). INT32 values carry the INT32_MIN NULL sentinel of value_t
 * (intermediate.h:40-63); VARCHAR values refer to a base-table row (the
 * page/offset reference of value_t); INT64 / FP64 (not representable in the
 * reference) carry a value plus a validity byte. */
typedef struct {
    int32_t type;
    uint8_t *valid;
    int32_t *i32;
    int64_t *i64;
    double *f64;
    uint64_t src_table, src_col; /* VARCHAR provenance                    */
    uint32_t *src_row;
} icol;

/* JoinInput (include/join_execution/join_setup.h:39-67). */
typedef struct {
    int is_columnar;
    uint64_t table_id;
    const cj_plan_node *node;
    uint64_t num_rows;
    uint64_t ncols;
    icol *cols; /* intermediate only */
} joininput;

typedef struct {
    const cj_plan_desc *plan;
    cjo_column **decoded; /* [input][column], lazily decoded              */
    int depth;
} octx;

static void icol_free(icol *c) {
    free(c->valid);
    free(c->i32);
    free(c->i64);
    free(c->f64);
    free(c->src_row);
}
static void ji_free(joininput *j) {
    if (!j->is_columnar) {
        for (uint64_t i = 0; i < j->ncols; ++i) icol_free(&j->cols[i]);
        free(j->cols);
    }
    memset(j, 0, sizeof(*j));
}

static const cjo_column *base_column(octx *o, uint64_t table, uint64_t col, int *rc) {
    const cj_plan_desc *p = o->plan;
    if (table >= p->num_inputs || !p->inputs || col >= p->inputs[table].num_columns) {
        *rc = CJ_ERR_INVALID_PLAN;
        return NULL;
    }
    if (!o->decoded[table]) {
        o->decoded[table] = (cjo_column *)xcalloc(p->inputs[table].num_columns, sizeof(cjo_column));
        if (!o->decoded[table]) { *rc = CJ_ERR_OUT_OF_MEMORY; return NULL; }
    }
    cjo_column *c = &o->decoded[table][col];
    if (!c->valid) {
        const cj_column_desc *cd = &p->inputs[table].columns[col];
        int r = cjo_decode_column(cd->type, cd->pages, cd->num_pages, p->inputs[table].num_rows, c);
        if (r) { *rc = r; return NULL; }
    }
    return c;
}

/* A value read from a JoinInput column at row `rid`: ColumnarReader::
 * read_value for base tables (include/data_access/columnar_reader.h:300-356)
 * or column_t::operator[] for intermediates. */
typedef struct {
    int valid;
    int64_t i;  /* INT32 / INT64 */
    double f;
    const char *s;
    uint64_t len;
} value;

typedef struct {
    int32_t type;
    const cjo_column *base; /* columnar source, or VARCHAR provenance     */
    const icol *ic;         /* intermediate source                        */
} colsrc;

static int resolve_col(octx *o, const joininput *in, uint64_t local, colsrc *cs) {
    int rc = CJ_OK;
    memset(cs, 0, sizeof(*cs));
    if (local >= in->ncols) return CJ_ERR_INVALID_PLAN;
    if (in->is_columnar) {
        const cj_attr *a = &in->node->output_attrs[local];
        cs->base = base_column(o, in->table_id, a->index, &rc);
        if (!cs->base) return rc;
        cs->type = cs->base->type;
    } else {
        cs->ic = &in->cols[local];
        cs->type = cs->ic->type;
        if (cs->type == CJ_VARCHAR) {
            cs->base = base_column(o, cs->ic->src_table, cs->ic->src_col, &rc);
            if (!cs->base) return rc;
        }
    }
    return CJ_OK;
}

static value read_value(const colsrc *cs, uint64_t rid) {
    value v = {0};
    if (cs->ic) {
        const icol *c = cs->ic;
        switch (c->type) {
        case CJ_INT32:
            v.valid = c->i32[rid] != INT32_MIN; /* value_t::is_null */
            v.i = c->i32[rid];
            break;
        case CJ_INT64: v.valid = c->valid[rid]; v.i = c->i64[rid]; break;
        case CJ_FP64: v.valid = c->valid[rid]; v.f = c->f64[rid]; break;
        default:
            v.valid = c->valid[rid];
            if (v.valid) {
                uint32_t r = c->src_row[rid];
                v.s = cs->base->chars + cs->base->str_off[r];
                v.len = cs->base->str_off[r + 1] - cs->base->str_off[r];
            }
        }
        return v;
    }
    const cjo_column *b = cs->base;
    v.valid = b->valid[rid];
    switch (b->type) {
    case CJ_INT32: v.i = b->i32[rid]; break;
    case CJ_INT64: v.i = b->i64[rid]; break;
    case CJ_FP64: v.f = b->f64[rid]; break;
    default:
        v.s = b->chars + b->str_off[rid];
        v.len = b->str_off[rid + 1] - b->str_off[rid];
    }
    return v;
}

/* Match buffer (ThreadLocalMatchBuffer, match_collector.h:66-221), one
 * thread. */
typedef struct {
    uint32_t *left, *right; /* build row ids, probe row ids */
    uint64_t n, cap;
} matches;

static int add_match(matches *m, uint32_t l, uint32_t r) {
    if (m->n == m->cap) {
        uint64_t nc = m->cap ? m->cap * 2 : 1024;
        uint32_t *a = (uint32_t *)realloc(m->left, nc * 4);
        if (!a) return -1;
        m->left = a;
        uint32_t *b = (uint32_t *)realloc(m->right, nc * 4);
        if (!b) return -1;
        m->right = b;
        m->cap = nc;
    }
    m->left[m->n] = l;
    m->right[m->n] = r;
    m->n++;
    return 0;
}

static int exec_node(octx *o, uint64_t node_idx, int is_root, joininput *out_inter,
                     cjo_result **out_root);

/* resolve_join_input (src/execute.cpp:84-99). */
static int resolve_input(octx *o, uint64_t node_idx, joininput *in) {
    const cj_plan_desc *p = o->plan;
    if (node_idx >= p->num_nodes) return CJ_ERR_INVALID_PLAN;
    const cj_plan_node *n = &p->nodes[node_idx];
    memset(in, 0, sizeof(*in));
    in->node = n;
    in->ncols = n->num_output_attrs;
    if (n->node_type == CJ_NODE_SCAN) {
        if (n->base_table_id >= p->num_inputs || !p->inputs) return CJ_ERR_INVALID_PLAN;
        in->is_columnar = 1;
        in->table_id = n->base_table_id;
        in->num_rows = p->inputs[n->base_table_id].num_rows;
        for (uint64_t i = 0; i < n->num_output_attrs; ++i) {
            const cj_attr *a = &n->output_attrs[i];
            if (a->index >= p->inputs[in->table_id].num_columns) return CJ_ERR_INVALID_PLAN;
            if (p->inputs[in->table_id].columns[a->index].type != a->type) return CJ_ERR_INVALID_PLAN;
        }
        return CJ_OK;
    }
    if (n->node_type != CJ_NODE_HASH_JOIN) return CJ_ERR_INVALID_PLAN;
    return exec_node(o, node_idx, 0, in, NULL);
}

/* ColumnarTable result with ColumnInserter-encoded columns. */
struct cjo_result {
    uint64_t num_rows;
    uint64_t ncols;
    int32_t *types;
    pagebuf *cols;
};

void cjo_result_free(cjo_result *r) {
    if (!r) return;
    for (uint64_t c = 0; c < r->ncols; ++c) free(r->cols[c].data);
    free(r->cols);
    free(r->types);
    free(r);
}
uint64_t cjo_result_num_rows(const cjo_result *r) { return r ? r->num_rows : 0; }
uint64_t cjo_result_num_columns(const cjo_result *r) { return r ? r->ncols : 0; }
int cjo_result_column(const cjo_result *r, uint64_t c, int32_t *type, uint64_t *num_pages,
                      const void **pages) {
    if (!r || c >= r->ncols) return CJ_ERR_INVALID_ARGUMENT;
    if (type) *type = r->types[c];
    if (num_pages) *num_pages = r->cols[c].pages;
    if (pages) *pages = r->cols[c].data;
    return CJ_OK;
}

static cjo_result *new_result(uint64_t ncols) {
    cjo_result *r = (cjo_result *)calloc(1, sizeof(cjo_result));
    if (!r) return NULL;
    r->ncols = ncols;
    r->types = (int32_t *)xcalloc(ncols, 4);
    r->cols = (pagebuf *)xcalloc(ncols, sizeof(pagebuf));
    if (!r->types || !r->cols) { cjo_result_free(r); return NULL; }
    return r;
}

/* Encode one output column from a value source over a row-id list (the
 * materialize_column_from_buffers loop, materialize.h:111-171, writing
 * through ColumnInserter<T>). */
static int encode_output(const colsrc *cs, const uint32_t *rids, uint64_t n, pagebuf *pb) {
    inserter *in = (inserter *)malloc(sizeof(inserter));
    if (!in) return CJ_ERR_OUT_OF_MEMORY;
    ins_init(in, cs->type, pb);
    for (uint64_t i = 0; i < n && !in->oom; ++i) {
        uint64_t rid = rids ? rids[i] : i;
        value v = read_value(cs, rid);
        if (cs->type == CJ_VARCHAR) {
            if (v.valid) ins_insert_varchar(in, v.s, v.len);
            else ins_insert_null_varchar(in);
        } else if (!v.valid) {
            ins_insert_null_fixed(in);
        } else if (cs->type == CJ_INT32) {
            int32_t x = (int32_t)v.i;
            ins_insert_fixed(in, &x);
        } else if (cs->type == CJ_INT64) {
            ins_insert_fixed(in, &v.i);
        } else {
            ins_insert_fixed(in, &v.f);
        }
    }
    ins_finalize(in);
    int oom = in->oom;
    free(in);
    return oom ? CJ_ERR_OUT_OF_MEMORY : CJ_OK;
}

/* Build an intermediate column from a source over row ids
 * (construct_intermediate_from_buffers, construct_intermediate.h:121-220). */
static int make_icol(octx *o, const joininput *in, uint64_t local, const colsrc *cs,
                     const uint32_t *rids, uint64_t n, icol *out) {
    memset(out, 0, sizeof(*out));
    out->type = cs->type;
    out->valid = (uint8_t *)xcalloc(n, 1);
    if (!out->valid) return CJ_ERR_OUT_OF_MEMORY;
    if (cs->type == CJ_INT32) out->i32 = (int32_t *)xcalloc(n, 4);
    else if (cs->type == CJ_INT64) out->i64 = (int64_t *)xcalloc(n, 8);
    else if (cs->type == CJ_FP64) out->f64 = (double *)xcalloc(n, 8);
    else out->src_row = (uint32_t *)xcalloc(n, 4);
    if (!out->i32 && !out->i64 && !out->f64 && !out->src_row) return CJ_ERR_OUT_OF_MEMORY;
    if (cs->type == CJ_VARCHAR) {
        /* provenance: initialize_output_columns (join_setup.h:180-213) */
        if (in->is_columnar) {
            out->src_table = in->table_id;
            out->src_col = in->node->output_attrs[local].index;
        } else {
            out->src_table = cs->ic->src_table;
            out->src_col = cs->ic->src_col;
        }
    }
    (void)o;
    for (uint64_t i = 0; i < n; ++i) {
        uint32_t rid = rids[i];
        value v = read_value(cs, rid);
        out->valid[i] = (uint8_t)v.valid;
        switch (cs->type) {
        case CJ_INT32:
            /* value_t: NULL is stored as INT32_MIN (intermediate.h:56-62) */
            out->i32[i] = v.valid ? (int32_t)v.i : INT32_MIN;
            break;
        case CJ_INT64: out->i64[i] = v.valid ? v.i : 0; break;
        case CJ_FP64: out->f64[i] = v.valid ? v.f : 0.0; break;
        default:
            out->src_row[i] = v.valid ? (cs->ic ? cs->ic->src_row[rid] : rid) : 0;
        }
    }
    return CJ_OK;
}

/* Key of a JoinInput row: NULL via bitmap (columnar) or value_t sentinel
 * (intermediate). */
static int read_key(const colsrc *cs, uint64_t rid, int64_t *key) {
    value v = read_value(cs, rid);
    *key = v.i;
    return v.valid;
}

/* execute_impl (src/execute.cpp:207-300) with execute_join_with_mode
 * (src/execute.cpp:112-194). */
static int exec_node(octx *o, uint64_t node_idx, int is_root, joininput *out_inter,
                     cjo_result **out_root) {
    const cj_plan_desc *p = o->plan;
    if (++o->depth > (int)p->num_nodes + 1) return CJ_ERR_INVALID_PLAN;
    const cj_plan_node *node = &p->nodes[node_idx];
    int rc = CJ_OK;

    if (node->node_type == CJ_NODE_SCAN) {
        /* Root scan (the reference requires a join root; a scan root is
         * answered with the projected table). */
        joininput in;
        rc = resolve_input(o, node_idx, &in);
        if (rc) return rc;
        cjo_result *r = new_result(node->num_output_attrs);
        if (!r) return CJ_ERR_OUT_OF_MEMORY;
        r->num_rows = in.num_rows;
        for (uint64_t c = 0; c < node->num_output_attrs && !rc; ++c) {
            colsrc cs;
            rc = resolve_col(o, &in, c, &cs);
            if (!rc) {
                r->types[c] = cs.type;
                rc = encode_output(&cs, NULL, in.num_rows, &r->cols[c]);
            }
        }
        if (rc) { cjo_result_free(r); return rc; }
        *out_root = r;
        return CJ_OK;
    }

    joininput left, right;
    rc = resolve_input(o, node->left, &left);
    if (rc) return rc;
    rc = resolve_input(o, node->right, &right);
    if (rc) { ji_free(&left); return rc; }

    /* select_build_probe_side (join_setup.h:108-136): smaller row count is
     * the build side, left wins ties; build_left of the plan is ignored. */
    int build_left = left.num_rows <= right.num_rows;
    joininput *build = build_left ? &left : &right;
    joininput *probe = build_left ? &right : &left;
    uint64_t build_attr = build_left ? node->left_attr : node->right_attr;
    uint64_t probe_attr = build_left ? node->right_attr : node->left_attr;

    colsrc bkey, pkey;
    if ((rc = resolve_col(o, build, build_attr, &bkey)) ||
        (rc = resolve_col(o, probe, probe_attr, &pkey))) {
        ji_free(&left);
        ji_free(&right);
        return rc;
    }
    if ((bkey.type != CJ_INT32 && bkey.type != CJ_INT64) ||
        (pkey.type != CJ_INT32 && pkey.type != CJ_INT64)) {
        ji_free(&left);
        ji_free(&right);
        return CJ_ERR_UNSUPPORTED;
    }
    /* Output attributes: declared type must equal the source type. */
    uint64_t lsz = left.ncols;
    for (uint64_t i = 0; i < node->num_output_attrs; ++i) {
        uint64_t idx = node->output_attrs[i].index;
        if (idx >= left.ncols + right.ncols) { rc = CJ_ERR_INVALID_PLAN; break; }
        colsrc cs;
        rc = idx < lsz ? resolve_col(o, &left, idx, &cs) : resolve_col(o, &right, idx - lsz, &cs);
        if (rc) break;
        if (cs.type != node->output_attrs[i].type) { rc = CJ_ERR_INVALID_PLAN; break; }
    }
    if (rc) { ji_free(&left); ji_free(&right); return rc; }

    matches m = {0};
    uint64_t build_rows = build->num_rows;
    if (build_rows > 0 && probe->num_rows > 0) {
        if (build_rows < 8) {
            /* nested_loop_join (nested_loop.h:107-244): collect non-NULL
             * build keys (visit_rows, 50-90), compare every probe row. */
            int64_t bv[8];
            uint32_t bid[8];
            int bc = 0;
            for (uint64_t r = 0; r < build_rows; ++r) {
                int64_t k;
                if (read_key(&bkey, r, &k) && bc < 8) { bv[bc] = k; bid[bc] = (uint32_t)r; ++bc; }
            }
            for (uint64_t r = 0; r < probe->num_rows && !rc; ++r) {
                int64_t k;
                if (!read_key(&pkey, r, &k)) continue;
                for (int j = 0; j < bc; ++j)
                    if (bv[j] == k && add_match(&m, bid[j], (uint32_t)r)) { rc = CJ_ERR_OUT_OF_MEMORY; break; }
            }
        } else {
            /* build_from_columnar / build_from_intermediate (hash_join.h:48-74) */
            uht t;
            int64_t *keys = (int64_t *)xcalloc(build_rows, 8);
            uint32_t *rids = (uint32_t *)xcalloc(build_rows, 4);
            if (!keys || !rids || uht_init(&t, build_rows)) rc = CJ_ERR_OUT_OF_MEMORY;
            uint64_t nt = 0;
            for (uint64_t r = 0; r < build_rows && !rc; ++r) {
                int64_t k;
                if (read_key(&bkey, r, &k)) { keys[nt] = k; rids[nt] = (uint32_t)r; ++nt; }
            }
            if (!rc && uht_build(&t, keys, rids, nt)) rc = CJ_ERR_OUT_OF_MEMORY;
            free(keys);
            free(rids);
            /* probe_columnar / probe_intermediate (hash_join.h:87-244) */
            for (uint64_t r = 0; r < probe->num_rows && !rc; ++r) {
                int64_t k;
                if (!read_key(&pkey, r, &k)) continue;
                uint64_t s, e;
                uht_find(&t, k, &s, &e);
                for (uint64_t j = s; j < e; ++j)
                    if (t.keys[j] == k && add_match(&m, t.row_ids[j], (uint32_t)r)) { rc = CJ_ERR_OUT_OF_MEMORY; break; }
            }
            uht_free(&t);
        }
    }
    if (rc) { free(m.left); free(m.right); ji_free(&left); ji_free(&right); return rc; }

    /* Output columns in output_attrs order; index space left ++ right. */
    if (is_root) {
        cjo_result *r = new_result(node->num_output_attrs);
        if (!r) rc = CJ_ERR_OUT_OF_MEMORY;
        else r->num_rows = m.n;
        for (uint64_t i = 0; i < node->num_output_attrs && !rc; ++i) {
            uint64_t idx = node->output_attrs[i].index;
            joininput *side = idx < lsz ? &left : &right;
            uint64_t local = idx < lsz ? idx : idx - lsz;
            colsrc cs;
            rc = resolve_col(o, side, local, &cs);
            if (rc) break;
            r->types[i] = cs.type;
            if (m.n) /* create_empty_result (materialize.h:61-69) otherwise */
                rc = encode_output(&cs, side == build ? m.left : m.right, m.n, &r->cols[i]);
        }
        if (rc) cjo_result_free(r);
        else *out_root = r;
    } else {
        out_inter->is_columnar = 0;
        out_inter->node = node;
        out_inter->num_rows = m.n;
        out_inter->ncols = node->num_output_attrs;
        out_inter->cols = (icol *)xcalloc(node->num_output_attrs, sizeof(icol));
        if (!out_inter->cols) rc = CJ_ERR_OUT_OF_MEMORY;
        for (uint64_t i = 0; i < node->num_output_attrs && !rc; ++i) {
            uint64_t idx = node->output_attrs[i].index;
            joininput *side = idx < lsz ? &left : &right;
            uint64_t local = idx < lsz ? idx : idx - lsz;
            colsrc cs;
            rc = resolve_col(o, side, local, &cs);
            if (!rc)
                rc = make_icol(o, side, local, &cs, side == build ? m.left : m.right, m.n,
                               &out_inter->cols[i]);
        }
        if (rc) ji_free(out_inter);
    }
    free(m.left);
    free(m.right);
    ji_free(&left);
    ji_free(&right);
    o->depth--;
    return rc;
}

int cjo_execute(const cj_plan_desc *plan, cjo_result **out) {
    if (!plan || !out || plan->root >= plan->num_nodes || (plan->num_nodes && !plan->nodes))
        return CJ_ERR_INVALID_ARGUMENT;
    bloom_init();
    octx o = {0};
    o.plan = plan;
    o.decoded = (cjo_column **)xcalloc(plan->num_inputs, sizeof(cjo_column *));
    if (!o.decoded) return CJ_ERR_OUT_OF_MEMORY;
    *out = NULL;
    int rc = exec_node(&o, plan->root, 1, NULL, out);
    for (uint64_t t = 0; t < plan->num_inputs; ++t) {
        if (!o.decoded[t]) continue;
        for (uint64_t c = 0; c < plan->inputs[t].num_columns; ++c) cjo_column_free(&o.decoded[t][c]);
        free(o.decoded[t]);
    }
    free(o.decoded);
    return rc;
}

/* ======================================================================== */
/* Row-multiset comparison (read_sql.cpp:1325-1360 compares sorted rows).    */
/* ======================================================================== */
typedef struct {
    const cjo_table *t;
} cmpctx;

static int cmp_cell(const cjo_column *c, uint64_t a, uint64_t b) {
    int va = c->valid[a], vb = c->valid[b];
    if (va != vb) return va < vb ? -1 : 1;
    if (!va) return 0;
    switch (c->type) {
    case CJ_INT32: return c->i32[a] < c->i32[b] ? -1 : c->i32[a] > c->i32[b];
    case CJ_INT64: return c->i64[a] < c->i64[b] ? -1 : c->i64[a] > c->i64[b];
    case CJ_FP64: {
        uint64_t x, y;
        memcpy(&x, &c->f64[a], 8);
        memcpy(&y, &c->f64[b], 8);
        return x < y ? -1 : x > y;
    }
    default: {
        uint64_t la = c->str_off[a + 1] - c->str_off[a], lb = c->str_off[b + 1] - c->str_off[b];
        uint64_t l = la < lb ? la : lb;
        int r = memcmp(c->chars + c->str_off[a], c->chars + c->str_off[b], l);
        if (r) return r < 0 ? -1 : 1;
        return la < lb ? -1 : la > lb;
    }
    }
}

static int cmp_rows(const void *x, const void *y, void *arg) {
    const cmpctx *cc = (const cmpctx *)arg;
    uint64_t a = *(const uint64_t *)x, b = *(const uint64_t *)y;
    for (uint64_t c = 0; c < cc->t->num_columns; ++c) {
        int r = cmp_cell(&cc->t->columns[c], a, b);
        if (r) return r;
    }
    return 0;
}

static int cmp_cross(const cjo_column *ca, uint64_t a, const cjo_column *cb, uint64_t b) {
    int va = ca->valid[a], vb = cb->valid[b];
    if (va != vb) return 1;
    if (!va) return 0;
    switch (ca->type) {
    case CJ_INT32: return ca->i32[a] != cb->i32[b];
    case CJ_INT64: return ca->i64[a] != cb->i64[b];
    case CJ_FP64: return memcmp(&ca->f64[a], &cb->f64[b], 8) != 0;
    default: {
        uint64_t la = ca->str_off[a + 1] - ca->str_off[a], lb = cb->str_off[b + 1] - cb->str_off[b];
        if (la != lb) return 1;
        return memcmp(ca->chars + ca->str_off[a], cb->chars + cb->str_off[b], la) != 0;
    }
    }
}

static uint64_t *sorted_index(const cjo_table *t) {
    uint64_t *idx = (uint64_t *)xcalloc(t->num_rows, 8);
    if (!idx) return NULL;
    for (uint64_t i = 0; i < t->num_rows; ++i) idx[i] = i;
    cmpctx cc = {t};
    qsort_r(idx, (size_t)t->num_rows, 8, cmp_rows, &cc);
    return idx;
}

int cjo_tables_equal(const cjo_table *a, const cjo_table *b, char *msg, uint64_t msg_len) {
    if (a->num_columns != b->num_columns) {
        fmt_msg(msg, msg_len, "column count %llu vs %llu", (unsigned long long)a->num_columns,
                (unsigned long long)b->num_columns);
        return 0;
    }
    if (a->num_rows != b->num_rows) {
        fmt_msg(msg, msg_len, "row count %llu vs %llu", (unsigned long long)a->num_rows,
                (unsigned long long)b->num_rows);
        return 0;
    }
    for (uint64_t c = 0; c < a->num_columns; ++c)
        if (a->columns[c].type != b->columns[c].type) {
            fmt_msg(msg, msg_len, "column %llu type %d vs %d", (unsigned long long)c,
                    a->columns[c].type, b->columns[c].type);
            return 0;
        }
    uint64_t *ia = sorted_index(a), *ib = sorted_index(b);
    if (!ia || !ib) {
        free(ia);
        free(ib);
        fmt_msg(msg, msg_len, "out of memory");
        return 0;
    }
    int eq = 1;
    for (uint64_t r = 0; r < a->num_rows && eq; ++r)
        for (uint64_t c = 0; c < a->num_columns; ++c)
            if (cmp_cross(&a->columns[c], ia[r], &b->columns[c], ib[r])) {
                fmt_msg(msg, msg_len, "sorted row %llu differs in column %llu (rows %llu / %llu)",
                        (unsigned long long)r, (unsigned long long)c, (unsigned long long)ia[r],
                        (unsigned long long)ib[r]);
                eq = 0;
                break;
            }
    free(ia);
    free(ib);
    return eq;
}

static int decode_table(uint64_t ncols, const int32_t *types, uint64_t rows, const uint64_t *np,
                        const void *const *pages, cjo_table *t) {
    t->num_rows = rows;
    t->num_columns = ncols;
    t->columns = (cjo_column *)xcalloc(ncols, sizeof(cjo_column));
    if (!t->columns) return CJ_ERR_OUT_OF_MEMORY;
    for (uint64_t c = 0; c < ncols; ++c) {
        int rc = cjo_decode_column_contig(types[c], pages[c], np[c], rows, &t->columns[c]);
        if (rc) return rc;
    }
    return CJ_OK;
}

static void free_table(cjo_table *t) {
    if (!t->columns) return;
    for (uint64_t c = 0; c < t->num_columns; ++c) cjo_column_free(&t->columns[c]);
    free(t->columns);
    t->columns = NULL;
}

int cjo_paged_tables_equal(uint64_t ncols, const int32_t *types, uint64_t rows_a,
                           const uint64_t *num_pages_a, const void *const *pages_a,
                           uint64_t rows_b, const uint64_t *num_pages_b,
                           const void *const *pages_b, char *msg, uint64_t msg_len) {
    cjo_table a = {0}, b = {0};
    int rc = decode_table(ncols, types, rows_a, num_pages_a, pages_a, &a);
    if (rc) {
        fmt_msg(msg, msg_len, "table A does not decode (status %d)", rc);
        free_table(&a);
        return 0;
    }
    rc = decode_table(ncols, types, rows_b, num_pages_b, pages_b, &b);
    if (rc) {
        fmt_msg(msg, msg_len, "table B does not decode (status %d)", rc);
        free_table(&a);
        free_table(&b);
        return 0;
    }
    int eq = cjo_tables_equal(&a, &b, msg, msg_len);
    free_table(&a);
    free_table(&b);
    return eq;
}

static uint64_t mix64(uint64_t x) {
    x ^= x >> 30;
    x *= 0xbf58476d1ce4e5b9ull;
    x ^= x >> 27;
    x *= 0x94d049bb133111ebull;
    x ^= x >> 31;
    return x;
}

int cjo_paged_table_fingerprint(uint64_t ncols, const int32_t *types, uint64_t rows,
                                const uint64_t *num_pages, const void *const *pages, uint64_t *fp) {
    uint64_t *rowh = (uint64_t *)xcalloc(rows, 8);
    if (!rowh) return CJ_ERR_OUT_OF_MEMORY;
    for (uint64_t c = 0; c < ncols; ++c) {
        cjo_column col;
        int rc = cjo_decode_column_contig(types[c], pages[c], num_pages[c], rows, &col);
        if (rc) { free(rowh); return rc; }
        for (uint64_t r = 0; r < rows; ++r) {
            uint64_t h;
            if (!col.valid[r]) h = 0x9e3779b97f4a7c15ull;
            else if (col.type == CJ_INT32) h = (uint64_t)(int64_t)col.i32[r];
            else if (col.type == CJ_INT64) h = (uint64_t)col.i64[r];
            else if (col.type == CJ_FP64) memcpy(&h, &col.f64[r], 8);
            else {
                h = 1469598103934665603ull; /* FNV-1a over the bytes */
                for (uint64_t k = col.str_off[r]; k < col.str_off[r + 1]; ++k)
                    h = (h ^ (uint8_t)col.chars[k]) * 1099511628211ull;
            }
            rowh[r] = mix64(rowh[r] * 31 + mix64(h + c));
        }
        cjo_column_free(&col);
    }
    uint64_t s = 0;
    for (uint64_t r = 0; r < rows; ++r) s += mix64(rowh[r]);
    free(rowh);
    *fp = s + rows;
    return CJ_OK;
}


/* ------------------------------------------------------------------------ */
/* Scan-side filters (the loader's predicate pass, src/build_table.cpp:      */
/* 318-366; src/statement.cpp:47-241; include/data_model/inner_column.h)     */
/* ------------------------------------------------------------------------ */

static uint64_t cp_len_o(uint8_t b) {
    if (b < 0x80) return 1;
    if ((b & 0xE0) == 0xC0) return 2;
    if ((b & 0xF0) == 0xE0) return 3;
    if ((b & 0xF8) == 0xF0) return 4;
    return 1;
}

/* Exact matcher by dynamic programming over (text byte, pattern byte):
 * ok[i][j] = pattern[j..] matches text[i..]. The translated RE2 pattern
 * (statement.h:125-147) is '%' -> ".*", '_' -> ".", every other byte
 * literal; RE2's '.' is one UTF-8 code point other than a newline. */
int cjo_like(const char *s, uint64_t n, const char *pat, uint64_t m) {
    const uint8_t *t = (const uint8_t *)s;
    const uint8_t *p = (const uint8_t *)pat;
    uint8_t *ok = (uint8_t *)calloc((n + 1) * (m + 1), 1);
    if (!ok) return -1;
#define OK(i, j) ok[(uint64_t)(i) * (m + 1) + (j)]
    OK(n, m) = 1;
    for (uint64_t ii = n + 1; ii-- > 0;) {
        for (uint64_t jj = m + 1; jj-- > 0;) {
            if (jj == m) { OK(ii, jj) = ii == n; continue; }
            uint8_t r = 0;
            if (p[jj] == '%') {
                r = OK(ii, jj + 1);
                if (!r && ii < n && t[ii] != '\n') {
                    uint64_t nx = ii + cp_len_o(t[ii]);
                    r = nx <= n && OK(nx, jj);
                }
            } else if (p[jj] == '_') {
                if (ii < n && t[ii] != '\n') {
                    uint64_t nx = ii + cp_len_o(t[ii]);
                    r = nx <= n && OK(nx, jj + 1);
                }
            } else {
                r = ii < n && t[ii] == p[jj] && OK(ii + 1, jj + 1);
            }
            OK(ii, jj) = r;
        }
    }
    int res = OK(0, 0);
#undef OK
    free(ok);
    return res;
}

static int cmp_i(int op, int64_t a, int64_t b) {
    switch (op) {
    case CJ_CMP_EQ: return a == b;
    case CJ_CMP_NEQ: return a != b;
    case CJ_CMP_LT: return a < b;
    case CJ_CMP_GT: return a > b;
    case CJ_CMP_LEQ: return a <= b;
    case CJ_CMP_GEQ: return a >= b;
    default: return 0;
    }
}

static int cmp_f(int op, double a, double b) {
    switch (op) {
    case CJ_CMP_EQ: return a == b;
    case CJ_CMP_NEQ: return a != b;
    case CJ_CMP_LT: return a < b;
    case CJ_CMP_GT: return a > b;
    case CJ_CMP_LEQ: return a <= b;
    case CJ_CMP_GEQ: return a >= b;
    default: return 0;
    }
}

/* std::string_view ordering: bytes as unsigned char, then length. */
static int str_cmp3(const char *a, uint64_t la, const char *b, uint64_t lb) {
    uint64_t m = la < lb ? la : lb;
    int c = m ? memcmp(a, b, m) : 0;
    if (c) return c < 0 ? -1 : 1;
    return la < lb ? -1 : (la > lb ? 1 : 0);
}

/* One row of one comparison, as InnerColumn<T>::equal / less / ... /
 * like / not_like write it: false on a NULL row (inner_column.h:240-313,
 * 387-588); IS_NULL / IS_NOT_NULL read the bitmap (statement.cpp:49-53). */
static int eval_cmp_row(const cj_pred_node *nd, const cjo_column *c, uint64_t r) {
    int valid = c->valid[r] != 0;
    if (nd->op == CJ_CMP_IS_NULL) return !valid;
    if (nd->op == CJ_CMP_IS_NOT_NULL) return valid;
    if (!valid) return 0;
    switch (c->type) {
    case CJ_INT32: /* static_cast<int32_t>(std::get<int64_t>(value)), statement.cpp:54 */
        return cmp_i(nd->op, c->i32[r], (int32_t)nd->i64);
    case CJ_INT64: return cmp_i(nd->op, c->i64[r], nd->i64);
    case CJ_FP64: return cmp_f(nd->op, c->f64[r], nd->literal_type == CJ_INT64 ? (double)nd->i64 : nd->f64);
    default: {
        const char *sv = c->chars + c->str_off[r];
        uint64_t len = c->str_off[r + 1] - c->str_off[r];
        if (nd->op == CJ_CMP_LIKE) return cjo_like(sv, len, nd->str, nd->str_len) == 1;
        if (nd->op == CJ_CMP_NOT_LIKE) return cjo_like(sv, len, nd->str, nd->str_len) == 0;
        int d = str_cmp3(sv, len, nd->str, nd->str_len);
        return cmp_i(nd->op, d, 0);
    }
    }
}

/* LogicalOperation: AND / OR of the children's bitmaps, NOT flips every
 * row's bit (statement.cpp:222-241). */
static int eval_pred_row(const cj_predicate *pr, uint64_t node, const cjo_column *cols, uint64_t r, int depth) {
    const cj_pred_node *nd = &pr->nodes[node];
    if (depth > (int)pr->num_nodes) return 0;
    switch (nd->kind) {
    case CJ_PRED_CMP: return eval_cmp_row(nd, &cols[nd->column], r);
    case CJ_PRED_AND:
        return eval_pred_row(pr, nd->left, cols, r, depth + 1) & eval_pred_row(pr, nd->right, cols, r, depth + 1);
    case CJ_PRED_OR:
        return eval_pred_row(pr, nd->left, cols, r, depth + 1) | eval_pred_row(pr, nd->right, cols, r, depth + 1);
    default: return !eval_pred_row(pr, nd->left, cols, r, depth + 1);
    }
}

int cjo_filter(const cj_table_desc *table, const cj_predicate *pred, uint64_t ncols, const uint64_t *cols,
               cjo_result **out, uint8_t *selected) {
    *out = NULL;
    uint64_t nc = table->num_columns, rows = table->num_rows;
    cjo_column *dec = (cjo_column *)xcalloc(nc ? nc : 1, sizeof(cjo_column));
    if (!dec) return CJ_ERR_OUT_OF_MEMORY;
    int rc = CJ_OK;
    for (uint64_t c = 0; c < nc && rc == CJ_OK; ++c) {
        const cj_column_desc *cd = &table->columns[c];
        rc = cjo_decode_column(cd->type, cd->pages, cd->num_pages, rows, &dec[c]);
    }
    uint32_t *sel = rc == CJ_OK ? (uint32_t *)xcalloc(rows ? rows : 1, 4) : NULL;
    uint64_t n = 0;
    if (rc == CJ_OK && !sel) rc = CJ_ERR_OUT_OF_MEMORY;
    for (uint64_t r = 0; rc == CJ_OK && r < rows; ++r) {
        int keep = pred ? eval_pred_row(pred, pred->root, dec, r, 0) : 1;
        if (selected) selected[r] = (uint8_t)keep;
        if (keep) sel[n++] = (uint32_t)r;
    }
    cjo_result *res = rc == CJ_OK ? new_result(ncols) : NULL;
    if (rc == CJ_OK && !res) rc = CJ_ERR_OUT_OF_MEMORY;
    if (res) res->num_rows = n;
    for (uint64_t k = 0; rc == CJ_OK && k < ncols; ++k) {
        const cjo_column *c = &dec[cols[k]];
        res->types[k] = c->type;
        inserter *in = (inserter *)malloc(sizeof(inserter));
        if (!in) { rc = CJ_ERR_OUT_OF_MEMORY; break; }
        ins_init(in, c->type, &res->cols[k]);
        for (uint64_t i = 0; i < n && !in->oom; ++i) {
            uint64_t r = sel[i];
            if (!c->valid[r]) {
                if (c->type == CJ_VARCHAR) ins_insert_null_varchar(in);
                else ins_insert_null_fixed(in);
            } else if (c->type == CJ_INT32) {
                ins_insert_fixed(in, &c->i32[r]);
            } else if (c->type == CJ_INT64) {
                ins_insert_fixed(in, &c->i64[r]);
            } else if (c->type == CJ_FP64) {
                ins_insert_fixed(in, &c->f64[r]);
            } else {
                ins_insert_varchar(in, c->chars + c->str_off[r], c->str_off[r + 1] - c->str_off[r]);
            }
        }
        ins_finalize(in);
        if (in->oom) rc = CJ_ERR_OUT_OF_MEMORY;
        free(in);
    }
    for (uint64_t c = 0; c < nc; ++c) cjo_column_free(&dec[c]);
    free(dec);
    free(sel);
    if (rc != CJ_OK) {
        cjo_result_free(res);
        return rc;
    }
    *out = res;
    return CJ_OK;
}
