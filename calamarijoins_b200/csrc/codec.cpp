/*
 * codec.cpp — host page encoder with the packing of the reference's
 * ColumnInserter<T> (include/data_model/plan.h:187-366): the canonical
 * writer of the 8 KiB page format, used by callers and the benchmark to
 * build input tables.
 *
 * Fixed width: values from max(4, sizeof(T)) on, one bitmap bit per row
 * at the page end; a value is appended while
 *   data_begin + (n_values + 1) * sizeof(T) + n_rows/8 + 1 <= 8192,
 * a NULL while data_begin + n_values * sizeof(T) + n_rows/8 + 1 <= 8192.
 * For INT32 this is ColumnInserter's test (plan.h:241-258). For 8-byte
 * types ColumnInserter reserves only 4 bytes for the next value, so some
 * NULL patterns let the last value overlap the bitmap, which then
 * overwrites its top byte; the test above is the one the reference's
 * Table::to_columnar uses for INT64 / FP64 (src/build_table.cpp:746-752),
 * which keeps every page well formed.
 * VARCHAR: n_values u16 end offsets at +4, characters after them; strings
 * longer than 8185 bytes go to long-string pages (0xffff first, 0xfffe
 * continuations, u16 chunk length at +2, up to 8188 bytes at +4)
 * (plan.h:294-369). Pages are zero-filled so the output is deterministic.
 */
#include <algorithm>
#include <cstring>
#include <vector>

#include "../../include/cj_b200.h"

namespace {

constexpr uint64_t P = CJ_PAGE_SIZE;

inline void wr16(uint8_t *p, uint32_t v) {
    uint16_t x = (uint16_t)v;
    std::memcpy(p, &x, 2);
}

class Sink {
  public:
    Sink(uint8_t *out, uint64_t cap) : out_(out), cap_(cap) {}
    /* Returns the next page (zeroed) or nullptr when only counting. */
    uint8_t *next() {
        uint8_t *p = nullptr;
        if (out_) {
            if (pages_ >= cap_) {
                overflow_ = true;
            } else {
                p = out_ + pages_ * P;
                std::memset(p, 0, P);
            }
        }
        ++pages_;
        return p;
    }
    uint64_t pages() const { return pages_; }
    bool overflow() const { return overflow_; }

  private:
    uint8_t *out_;
    uint64_t cap_;
    uint64_t pages_ = 0;
    bool overflow_ = false;
};

void encode_fixed(int32_t type, const uint8_t *vals, const uint8_t *valid, uint64_t n, Sink &sink) {
    const uint64_t w = type == CJ_INT32 ? 4 : 8, db = w; /* values start at max(4, sizeof(T)) */
    uint8_t bitmap[P];
    uint32_t nr = 0, nv = 0;
    uint8_t *page = nullptr;
    bool open = false;
    auto close = [&]() {
        if (page) {
            wr16(page, nr);
            wr16(page + 2, nv);
            uint64_t bs = (nr + 7) / 8;
            std::memcpy(page + P - bs, bitmap, bs);
        }
        nr = nv = 0;
        open = false;
    };
    auto ensure = [&]() {
        if (!open) {
            page = sink.next();
            std::memset(bitmap, 0, sizeof(bitmap));
            open = true;
        }
    };
    for (uint64_t i = 0; i < n; ++i) {
        const bool v = valid ? valid[i] != 0 : true;
        ensure();
        if (v) {
            if (db + (nv + 1) * w + nr / 8 + 1 > P) {
                close();
                ensure();
            }
            if (page) std::memcpy(page + db + nv * w, vals + i * w, w);
            bitmap[nr / 8] |= (uint8_t)(1u << (nr % 8));
            ++nv;
        } else {
            if (db + nv * w + nr / 8 + 1 > P) {
                close();
                ensure();
            }
        }
        ++nr;
    }
    if (open && nr) close();
}

void encode_varchar(const char *chars, const uint64_t *offs, const uint8_t *valid, uint64_t n, Sink &sink) {
    uint8_t bitmap[P];
    uint8_t data[P];
    uint16_t ends[P / 2];
    uint32_t nr = 0, nv = 0, bytes = 0;
    auto flush = [&]() {
        uint8_t *page = sink.next();
        if (page) {
            wr16(page, nr);
            wr16(page + 2, nv);
            std::memcpy(page + 4, ends, (size_t)nv * 2);
            std::memcpy(page + 4 + (size_t)nv * 2, data, bytes);
            uint64_t bs = (nr + 7) / 8;
            std::memcpy(page + P - bs, bitmap, bs);
        }
        nr = nv = bytes = 0;
        std::memset(bitmap, 0, sizeof(bitmap));
    };
    std::memset(bitmap, 0, sizeof(bitmap));
    for (uint64_t i = 0; i < n; ++i) {
        const bool v = valid ? valid[i] != 0 : true;
        if (!v) {
            if (4 + 2ull * nv + bytes + nr / 8 + 1 > P) flush();
            ++nr;
            continue;
        }
        const char *s = chars + offs[i];
        const uint64_t len = offs[i + 1] - offs[i];
        if (len > P - 7) {
            if (nr > 0) flush();
            uint64_t off = 0;
            bool first = true;
            while (off < len) {
                uint8_t *page = sink.next();
                const uint64_t chunk = std::min<uint64_t>(len - off, P - 4);
                if (page) {
                    wr16(page, first ? 0xffff : 0xfffe);
                    wr16(page + 2, (uint32_t)chunk);
                    std::memcpy(page + 4, s + off, chunk);
                }
                first = false;
                off += chunk;
            }
            continue;
        }
        if (4 + 2ull * nv + 2 + bytes + len + nr / 8 + 1 > P) flush();
        std::memcpy(data + bytes, s, len);
        bytes += (uint32_t)len;
        ends[nv++] = (uint16_t)bytes;
        bitmap[nr / 8] |= (uint8_t)(1u << (nr % 8));
        ++nr;
    }
    if (nr) flush();
}

int encode(int32_t type, const void *values, const uint64_t *offsets, const uint8_t *valid, uint64_t n,
           uint8_t *out, uint64_t cap, uint64_t *num_pages) {
    if (type < CJ_INT32 || type > CJ_VARCHAR || !num_pages) return CJ_ERR_INVALID_ARGUMENT;
    if (n && !values) return CJ_ERR_INVALID_ARGUMENT;
    if (type == CJ_VARCHAR && n && !offsets) return CJ_ERR_INVALID_ARGUMENT;
    Sink sink(out, cap);
    if (type == CJ_VARCHAR)
        encode_varchar(static_cast<const char *>(values), offsets, valid, n, sink);
    else
        encode_fixed(type, static_cast<const uint8_t *>(values), valid, n, sink);
    *num_pages = sink.pages();
    return sink.overflow() ? CJ_ERR_LIMIT : CJ_OK;
}

} // namespace

extern "C" {

int cj_encode_num_pages(int32_t type, const void *values, const uint64_t *offsets, const uint8_t *valid,
                        uint64_t n, uint64_t *num_pages) {
    return encode(type, values, offsets, valid, n, nullptr, 0, num_pages);
}

int cj_encode_column(int32_t type, const void *values, const uint64_t *offsets, const uint8_t *valid,
                     uint64_t n, void *out_pages, uint64_t capacity, uint64_t *num_pages) {
    if (!out_pages && capacity) return CJ_ERR_INVALID_ARGUMENT;
    return encode(type, values, offsets, valid, n, static_cast<uint8_t *>(out_pages), capacity, num_pages);
}

} /* extern "C" */
