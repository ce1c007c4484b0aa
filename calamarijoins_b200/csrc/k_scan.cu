/*
 * k_scan.cu — device-wide exclusive prefix sum (u32 or u64 in, u64 out):
 * tile reduce -> scan of tile totals (recursive) -> tile scan with offsets.
 * Used for page row offsets, radix partition offsets and VARCHAR page
 * counts; none of these is on the per-row hot path.
 */
#include "cj_device.cuh"

namespace cj {
namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr size_t kScanTile = (size_t)kScanThreads * kScanItems;

template <typename TIn>
__global__ void __launch_bounds__(kScanThreads)
    k_tile_reduce(const TIn *__restrict__ in, size_t n, uint64_t *__restrict__ partials) {
    __shared__ uint64_t wbuf[kScanThreads / 32 + 1];
    size_t base = (size_t)blockIdx.x * kScanTile;
    uint64_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        size_t i = base + (size_t)k * kScanThreads + threadIdx.x;
        if (i < n) s += (uint64_t)in[i];
    }
    uint64_t tot;
    block_exclusive_scan<uint64_t>(s, wbuf, &tot);
    if (threadIdx.x == 0) partials[blockIdx.x] = tot;
}

/* out[i] = offset(tile) + exclusive prefix within the tile; the last tile
 * also writes out[n] = grand total. */
template <typename TIn>
__global__ void __launch_bounds__(kScanThreads)
    k_tile_scan(const TIn *__restrict__ in, size_t n, const uint64_t *__restrict__ tile_off,
                uint64_t *__restrict__ out) {
    __shared__ uint64_t tile[kScanTile];
    __shared__ uint64_t wbuf[kScanThreads / 32 + 1];
    size_t base = (size_t)blockIdx.x * kScanTile;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        size_t li = (size_t)k * kScanThreads + threadIdx.x;
        size_t i = base + li;
        tile[li] = i < n ? (uint64_t)in[i] : 0;
    }
    __syncthreads();
    uint64_t local[kScanItems];
    uint64_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        local[k] = tile[threadIdx.x * kScanItems + k];
        s += local[k];
    }
    uint64_t tot;
    uint64_t pre = block_exclusive_scan<uint64_t>(s, wbuf, &tot);
    uint64_t off = tile_off ? tile_off[blockIdx.x] : 0;
    pre += off;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        tile[threadIdx.x * kScanItems + k] = pre;
        pre += local[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        size_t li = (size_t)k * kScanThreads + threadIdx.x;
        size_t i = base + li;
        if (i < n) out[i] = tile[li];
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[n] = off + tot;
}

size_t align_elems(size_t x) { return (x + 31) & ~size_t(31); }

template <typename TIn>
cudaError_t scan_impl(const Launch &L, const TIn *in, uint64_t *out, size_t n, void *temp) {
    if (n == 0) {
        return cudaMemsetAsync(out, 0, sizeof(uint64_t), L.stream);
    }
    size_t tiles = (n + kScanTile - 1) / kScanTile;
    if (tiles == 1) {
        k_tile_scan<TIn><<<1, kScanThreads, 0, L.stream>>>(in, n, nullptr, out);
        count_launches(1);
        return cudaGetLastError();
    }
    uint64_t *partials = reinterpret_cast<uint64_t *>(temp);
    uint64_t *offs = partials + align_elems(tiles);
    void *next = offs + align_elems(tiles + 1);
    k_tile_reduce<TIn><<<(unsigned)tiles, kScanThreads, 0, L.stream>>>(in, n, partials);
    count_launches(1);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    e = scan_impl<uint64_t>(L, partials, offs, tiles, next);
    if (e != cudaSuccess) return e;
    k_tile_scan<TIn><<<(unsigned)tiles, kScanThreads, 0, L.stream>>>(in, n, offs, out);
    count_launches(1);
    return cudaGetLastError();
}

} // namespace

size_t scan_temp_bytes(size_t n) {
    size_t tiles = (n + kScanTile - 1) / kScanTile;
    if (tiles <= 1) return 256;
    return (align_elems(tiles) + align_elems(tiles + 1)) * sizeof(uint64_t) + scan_temp_bytes(tiles);
}

cudaError_t scan_u32_to_u64(const Launch &L, const uint32_t *in, uint64_t *out, size_t n,
                            void *temp) {
    return scan_impl<uint32_t>(L, in, out, n, temp);
}

} // namespace cj
