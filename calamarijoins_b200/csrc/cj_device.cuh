/*
 * cj_device.cuh — device helpers shared by the sm_100a kernels: hashing,
 * Bloom tags, warp/block scans and column accessors.
 */
#pragma once

#include <cstdint>

#include "cj_internal.h"

namespace cj {

#define CJ_DEV __device__ __forceinline__

/* Key hash for the unchained table, a function of the key's 64-bit value
 * (INT32 and INT64 keys of equal value hash alike). The 64-bit value is
 * folded to 32 bits (a bijection on INT32 values), then two 32-bit
 * multiplicative hashes (Knuth's method: the product's top bits are the
 * well-mixed ones) give the high word, whose top bits are the radix
 * partition and the directory slot, and the low word, whose top 11 bits
 * index the Bloom tag table. The reference hashes with the x86/ARM CRC32C
 * instruction times a multiplier (include/join_execution/hashtable.h:
 * 146-154); the GPU has no CRC instruction, and the hash changes no result,
 * only where a key lands. Three 32-bit multiplies; the slot bits and the
 * Bloom bits come from different products, so a slot's keys still differ
 * in their tags for every directory size. */
__host__ __device__ __forceinline__ uint64_t hash_key(int64_t key) {
    const uint64_t x = (uint64_t)key;
    const uint32_t m = (uint32_t)x ^ ((uint32_t)(x >> 32) * 0x2545F491u);
    const uint32_t hi = m * 0x9E3779B1u;
    const uint32_t lo = (m ^ (m >> 15)) * 0x85EBCA77u;
    return ((uint64_t)hi << 32) | lo;
}

/* Slot = top log2_slots bits (as slot_for, hashtable.h:167-169);
 * log2_slots <= 32. */
CJ_DEV uint32_t slot_of(uint64_t h, int log2_slots) {
    return (uint32_t)(h >> (64 - log2_slots));
}

CJ_DEV uint32_t bloom_index(uint64_t h) { return (uint32_t)h >> 21; }

/* First slot of an INT32 key in an open-addressing table of nslots (< 2^32)
 * slots: Knuth's multiplicative hashing (the key times 2^32 / golden ratio,
 * mod 2^32), whose top bits are scaled to [0, nslots). Two instructions. */
CJ_DEV uint32_t open_slot(int64_t key, uint32_t nslots) {
    return __umulhi((uint32_t)key * 0x9E3779B9u, nslots);
}

/* Loads the 2048-entry Bloom tag table into shared memory. */
CJ_DEV void load_bloom(uint16_t *s_bloom, const uint16_t *g_bloom) {
    const uint32_t *src = reinterpret_cast<const uint32_t *>(g_bloom);
    uint32_t *dst = reinterpret_cast<uint32_t *>(s_bloom);
    for (int i = threadIdx.x; i < 1024; i += blockDim.x) dst[i] = src[i];
}

CJ_DEV uint32_t lane_id() { return threadIdx.x & 31u; }
CJ_DEV uint32_t lanemask_lt() { return (1u << lane_id()) - 1u; }

template <typename T> CJ_DEV T warp_inclusive_scan(T v) {
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        T o = __shfl_up_sync(0xffffffffu, v, d);
        if ((int)lane_id() >= d) v += o;
    }
    return v;
}

template <typename T> CJ_DEV T warp_sum(T v) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
    return v;
}

/* Exclusive scan over the block; `warp_buf` needs blockDim.x/32 + 1
 * entries. Returns the exclusive prefix and the block total in *total.
 * Contains __syncthreads(): every thread of the block must call it. */
template <typename T> CJ_DEV T block_exclusive_scan(T v, T *warp_buf, T *total) {
    const int warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    T incl = warp_inclusive_scan(v);
    if (lane_id() == 31) warp_buf[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        T w = (int)lane_id() < nwarps ? warp_buf[lane_id()] : T(0);
        T wi = warp_inclusive_scan(w);
        if ((int)lane_id() < nwarps) warp_buf[lane_id()] = wi - w;
        if (lane_id() == 31) warp_buf[nwarps] = wi;
    }
    __syncthreads();
    T res = warp_buf[warp] + incl - v;
    *total = warp_buf[nwarps];
    __syncthreads();
    return res;
}

/* Relation row -> base row through the view's indirections. */
CJ_DEV uint32_t base_row(const ColView &c, uint32_t i) {
    if (c.rid_a) i = __ldg(c.rid_a + i);
    if (c.rid_b) i = __ldg(c.rid_b + i);
    return i;
}

CJ_DEV bool valid_bit(const uint32_t *valid, uint32_t r) {
    return (__ldg(valid + (r >> 5)) >> (r & 31)) & 1u;
}

/* A fixed-width column read in place from its pages (no NULL, full
 * pages; COL_* flags word 0). */
CJ_DEV bool col_direct(const ColView &c) { return c.col_flags && __ldg(c.col_flags) == 0u; }
/* A column without NULLs: validity need not be read. */
CJ_DEV bool col_all_valid(const ColView &c) { return c.col_flags && (__ldg(c.col_flags) & COL_HAS_NULLS) == 0u; }

/* Base row r of a direct column: value r % R of page r / R (R constant per
 * width, so the division is a multiply). */
template <typename T> CJ_DEV T page_value(const uint8_t *pages, uint32_t r) {
    constexpr uint32_t R = sizeof(T) == 4 ? kRowsPerPageInt32 : kRowsPerPage8B;
    constexpr uint32_t DB = sizeof(T) == 4 ? 4u : 8u;
    const uint32_t p = r / R, k = r - p * R;
    return __ldg(reinterpret_cast<const T *>(pages + (uint64_t)p * kPageSize + DB) + k);
}

/* Join key of relation row i as a 64-bit integer; false if NULL. */
CJ_DEV bool load_key(const ColView &c, uint32_t i, int64_t *key) {
    uint32_t r = base_row(c, i);
    if (col_direct(c)) {
        if (c.type == CJ_INT32) {
            const int32_t v = page_value<int32_t>(c.pages, r);
            if (c.null_sentinel && v == INT32_MIN) return false;
            *key = v;
        } else {
            *key = page_value<long long>(c.pages, r);
        }
        return true;
    }
    if (!valid_bit(c.valid, r)) return false;
    if (c.type == CJ_INT32) {
        int32_t v = __ldg(reinterpret_cast<const int32_t *>(c.values) + r);
        if (c.null_sentinel && v == INT32_MIN) return false;
        *key = v;
    } else {
        *key = __ldg(reinterpret_cast<const long long *>(c.values) + r);
    }
    return true;
}

/* A copy of `c` whose col_flags pointer is kept only when the column is
 * read in place (col_direct): with it, per-row loaders test a kernel
 * argument instead of loading the flag word for every row. */
CJ_DEV ColView resolve_view(const ColView &c) {
    ColView v = c;
    if (!col_direct(c)) v.col_flags = nullptr;
    return v;
}

/* Streaming variant for a dense key column read once in row order: the
 * loads are marked evict-first so the hash table stays in L2. */
CJ_DEV bool load_key_stream(const ColView &c, uint32_t i, int64_t *key) {
    if (c.rid_a || c.rid_b || col_direct(c)) return load_key(c, i, key);
    if (!((__ldcs(c.valid + (i >> 5)) >> (i & 31)) & 1u)) return false;
    if (c.type == CJ_INT32) {
        int32_t v = __ldcs(reinterpret_cast<const int32_t *>(c.values) + i);
        if (c.null_sentinel && v == INT32_MIN) return false;
        *key = v;
    } else {
        *key = __ldcs(reinterpret_cast<const long long *>(c.values) + i);
    }
    return true;
}

} // namespace cj
