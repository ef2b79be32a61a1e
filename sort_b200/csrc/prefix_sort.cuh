// Device-wide exclusive prefix sums and a stable least-significant-digit radix
// sort of (key, int32 value) pairs, written for this library's own passes:
// the sorted traversal schedule (trace.cu), the SAH builder's partition
// (builder_gpu.cu) and the LBVH builder's Morton order (builder_lbvh.cu).
//
// Scan: tiles of kScanTile values, one block of 1,024 threads per tile
// (warp shuffles, then the warps' totals); the tiles' totals are scanned the
// same way, level by level, and added back.
//
// Sort: passes of kDigitBits-bit digits from the least significant, over tiles
// of kSortTile keys per block of kSortThreads threads. Per pass:
//   k_digit_count    the tile's digit counts in shared memory, written
//                    digit-major (count[d * tiles + tile]);
//   a scan of those counts, so each (digit, tile) knows where its run starts;
//   k_digit_scatter  each warp owns a contiguous kWarpChunk-key chunk of its
//                    tile, counts its digits, the block turns the counts into
//                    per-warp starting places, and each warp writes its keys
//                    in order, ranking the lanes of one digit with
//                    __match_any_sync: equal digits keep their order, so the
//                    sort is stable and the passes compose into a full sort.
// Everything here is stream-ordered and allocates nothing; callers provide
// the scratch (scan_scratch_words, sort_count_words).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace sg {
namespace psort {
namespace {  // each translation unit that includes this gets its own kernels

constexpr int kDigitBits = 10;
constexpr int kDigits = 1 << kDigitBits;
constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 16;                         // keys per thread
constexpr int kSortTile = kSortThreads * kSortItems;  // 4,096 keys per block
constexpr int kWarpChunk = kSortTile / kSortWarps;    // 512 keys per warp
constexpr int kScanTile = 2048;                       // values per scan block (1,024 threads x 2)

// ---- Exclusive prefix sums ---------------------------------------------------

// out[i] = sum of in[tile start .. i) inside each tile of kScanTile values
// (in may equal out); the tile's total goes to tile_sum[tile]. Values past
// `count` read as 0 and are not written.
__global__ void __launch_bounds__(1024) k_scan_tiles(const uint32_t* in, uint32_t* out, size_t count,
                                                     uint32_t* __restrict__ tile_sum) {
    __shared__ uint32_t warp_sum[32];
    const size_t base = (size_t)blockIdx.x * kScanTile + 2 * threadIdx.x;
    const uint32_t a = base < count ? in[base] : 0u, b = base + 1 < count ? in[base + 1] : 0u;
    const uint32_t mine = a + b;
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t x = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= (unsigned)o) x += y;
    }
    if (lane == 31) warp_sum[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = warp_sum[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= (unsigned)o) w += y;
        }
        warp_sum[lane] = w;  // inclusive over warps
    }
    __syncthreads();
    const uint32_t before = (warp > 0 ? warp_sum[warp - 1] : 0u) + x - mine;
    if (base < count) out[base] = before;
    if (base + 1 < count) out[base + 1] = before + a;
    if (threadIdx.x == 1023) tile_sum[blockIdx.x] = warp_sum[31];
}

// v[i] += tile_start[i / kScanTile].
__global__ void __launch_bounds__(256) k_add_tile_start(uint32_t* __restrict__ v, size_t count,
                                                        const uint32_t* __restrict__ tile_start) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) v[i] += __ldg(tile_start + i / kScanTile);
}

// Large arrays: reduce, then scan, over tiles of kBigTile values (8 per thread
// of a 1,024-thread block, staged through shared memory so the global loads
// and stores stay coalesced): the tiles' totals, their prefix sums, then each
// tile scanned from its start. 1.5 passes of traffic and three launches.
constexpr int kBigItems = 8;
constexpr int kBigTile = 1024 * kBigItems;

__device__ __forceinline__ uint32_t block_exclusive_1024(uint32_t mine, uint32_t* warp_sum, uint32_t* total) {
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t x = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= (unsigned)o) x += y;
    }
    if (lane == 31) warp_sum[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = warp_sum[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= (unsigned)o) w += y;
        }
        warp_sum[lane] = w;
    }
    __syncthreads();
    *total = warp_sum[31];
    return (warp > 0 ? warp_sum[warp - 1] : 0u) + x - mine;
}

// tile_sum[b] = sum of in[b * kBigTile ..) (values past count read as 0).
__global__ void __launch_bounds__(1024) k_big_tile_sums(const uint32_t* __restrict__ in, size_t count,
                                                        uint32_t* __restrict__ tile_sum) {
    __shared__ uint32_t warp_sum[32];
    const size_t base = (size_t)blockIdx.x * kBigTile;
    uint32_t mine = 0;
#pragma unroll
    for (int j = 0; j < kBigItems; ++j) {
        const size_t i = base + (size_t)j * 1024 + threadIdx.x;
        if (i < count) mine += in[i];
    }
    uint32_t total;
    block_exclusive_1024(mine, warp_sum, &total);
    if (threadIdx.x == 0) tile_sum[blockIdx.x] = total;
}

// Exclusive prefix sums of up to kBigTile values in place, one block.
__global__ void __launch_bounds__(1024) k_scan_one_block(uint32_t* __restrict__ v, int count) {
    __shared__ uint32_t stage[kBigTile];
    __shared__ uint32_t warp_sum[32];
#pragma unroll
    for (int j = 0; j < kBigItems; ++j) {
        const int i = j * 1024 + threadIdx.x;
        stage[i] = i < count ? v[i] : 0u;
    }
    __syncthreads();
    uint32_t run = 0, own[kBigItems];
#pragma unroll
    for (int j = 0; j < kBigItems; ++j) {
        own[j] = run;
        run += stage[threadIdx.x * kBigItems + j];
    }
    uint32_t total;
    const uint32_t before = block_exclusive_1024(run, warp_sum, &total);
#pragma unroll
    for (int j = 0; j < kBigItems; ++j) stage[threadIdx.x * kBigItems + j] = before + own[j];
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kBigItems; ++j) {
        const int i = j * 1024 + threadIdx.x;
        if (i < count) v[i] = stage[i];
    }
}

// out = exclusive prefix sums inside each kBigTile tile of in, plus the
// tile's start tile_start[b] (in may equal out).
__global__ void __launch_bounds__(1024) k_big_scan(const uint32_t* in, uint32_t* out, size_t count,
                                                   const uint32_t* __restrict__ tile_start) {
    __shared__ uint32_t stage[kBigTile];
    __shared__ uint32_t warp_sum[32];
    const size_t base = (size_t)blockIdx.x * kBigTile;
#pragma unroll
    for (int j = 0; j < kBigItems; ++j) {
        const size_t i = base + (size_t)j * 1024 + threadIdx.x;
        stage[j * 1024 + threadIdx.x] = i < count ? in[i] : 0u;
    }
    __syncthreads();
    uint32_t run = 0, own[kBigItems];
#pragma unroll
    for (int j = 0; j < kBigItems; ++j) {
        own[j] = run;
        run += stage[threadIdx.x * kBigItems + j];
    }
    uint32_t total;
    const uint32_t before = block_exclusive_1024(run, warp_sum, &total) + __ldg(tile_start + blockIdx.x);
#pragma unroll
    for (int j = 0; j < kBigItems; ++j) stage[threadIdx.x * kBigItems + j] = before + own[j];
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kBigItems; ++j) {
        const size_t i = base + (size_t)j * 1024 + threadIdx.x;
        if (i < count) out[i] = stage[j * 1024 + threadIdx.x];
    }
}

// Words of scratch scan_exclusive needs for `count` values.
inline size_t scan_scratch_words(size_t count) {
    const size_t big = (count + kBigTile - 1) / kBigTile;
    if (big > 1 && big <= (size_t)kBigTile) return big;
    const size_t tiles = (count + kScanTile - 1) / kScanTile;
    return tiles <= 1 ? 1 : tiles + scan_scratch_words(tiles);
}

// out = exclusive prefix sums of in[0 .. count) (in may equal out).
inline cudaError_t scan_exclusive(const uint32_t* in, uint32_t* out, size_t count, uint32_t* scratch,
                                  cudaStream_t s) {
    if (count == 0) return cudaSuccess;
    const size_t big = (count + kBigTile - 1) / kBigTile;
    if (big > 1 && big <= (size_t)kBigTile) {  // up to 67M values: reduce, scan the totals, scan
        k_big_tile_sums<<<(unsigned)big, 1024, 0, s>>>(in, count, scratch);
        k_scan_one_block<<<1, 1024, 0, s>>>(scratch, (int)big);
        k_big_scan<<<(unsigned)big, 1024, 0, s>>>(in, out, count, scratch);
        return cudaGetLastError();
    }
    const size_t tiles = (count + kScanTile - 1) / kScanTile;
    k_scan_tiles<<<(unsigned)tiles, 1024, 0, s>>>(in, out, count, scratch);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || tiles == 1) return e;
    if ((e = scan_exclusive(scratch, scratch, tiles, scratch + tiles, s)) != cudaSuccess) return e;
    k_add_tile_start<<<(unsigned)((count + 255) / 256), 256, 0, s>>>(out, count, scratch);
    return cudaGetLastError();
}

// Exclusive prefix sums of the tile totals written by k_scan_tiles, in place
// (one block; tiles <= 1024).
__global__ void __launch_bounds__(1024) k_scan_tile_sums(uint32_t* __restrict__ tile_sum, int tiles) {
    __shared__ uint32_t warp_sum[32];
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t mine = (int)threadIdx.x < tiles ? tile_sum[threadIdx.x] : 0u;
    uint32_t x = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= (unsigned)o) x += y;
    }
    if (lane == 31) warp_sum[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = warp_sum[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= (unsigned)o) w += y;
        }
        warp_sum[lane] = w;
    }
    __syncthreads();
    if ((int)threadIdx.x < tiles) tile_sum[threadIdx.x] = (warp > 0 ? warp_sum[warp - 1] : 0u) + x - mine;
}

// ---- Stable LSD radix sort of (key, int32 value) pairs --------------------------

template <class K>
__device__ __forceinline__ uint32_t digit_of(K key, int shift) {
    return (uint32_t)(key >> shift) & (kDigits - 1);
}

// Digit counts of a tile of kSortTile keys, digit-major: count[d * tiles + tile].
template <class K>
__global__ void __launch_bounds__(kSortThreads) k_digit_count(const K* __restrict__ keys, int64_t n, int shift,
                                                              int tiles, uint32_t* __restrict__ count) {
    __shared__ uint32_t hist[kDigits];
    for (int d = threadIdx.x; d < kDigits; d += kSortThreads) hist[d] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kSortTile;
#pragma unroll 4
    for (int j = 0; j < kSortItems; ++j) {
        const int64_t p = base + j * kSortThreads + threadIdx.x;
        if (p < n) atomicAdd(&hist[digit_of(__ldg(keys + p), shift)], 1u);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < kDigits; d += kSortThreads) count[(size_t)d * tiles + blockIdx.x] = hist[d];
}

// One stable pass: keys and values of each tile to their digit's run, whose
// start for (digit, tile) is start[c] (+ start_tile[c / kScanTile] when set),
// c = digit * tiles + tile.
template <class K>
__global__ void __launch_bounds__(kSortThreads) k_digit_scatter(const K* __restrict__ keys_in,
                                                                const int32_t* __restrict__ idx_in, int64_t n,
                                                                int shift, int tiles,
                                                                const uint32_t* __restrict__ start,
                                                                const uint32_t* __restrict__ start_tile,
                                                                K* __restrict__ keys_out,
                                                                int32_t* __restrict__ idx_out) {
    __shared__ uint32_t wcount[kSortWarps][kDigits];  // per warp: keys of each digit, then its starting place
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    for (int k = threadIdx.x; k < kSortWarps * kDigits; k += kSortThreads) (&wcount[0][0])[k] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kSortTile + (int64_t)warp * kWarpChunk;
    K key[kSortItems];
    int32_t idx[kSortItems];
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        const int64_t p = base + j * 32 + lane;
        const bool ok = p < n;
        key[j] = ok ? __ldg(keys_in + p) : K(0);
        idx[j] = ok ? __ldg(idx_in + p) : 0;
        const uint32_t d = ok ? digit_of(key[j], shift) : 0xffffffffu;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        if (ok && (peers & lt) == 0) wcount[warp][d] += (uint32_t)__popc(peers);
        __syncwarp();
    }
    __syncthreads();
    for (int d = threadIdx.x; d < kDigits; d += kSortThreads) {
        const size_t c = (size_t)d * tiles + blockIdx.x;
        uint32_t run = __ldg(start + c) + (start_tile ? __ldg(start_tile + c / kScanTile) : 0u);
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w) {
            const uint32_t cnt = wcount[w][d];
            wcount[w][d] = run;
            run += cnt;
        }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        const int64_t p = base + j * 32 + lane;
        const bool ok = p < n;
        const uint32_t d = ok ? digit_of(key[j], shift) : 0xffffffffu;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        uint32_t q = 0;
        if (ok) q = wcount[warp][d] + (uint32_t)__popc(peers & lt);
        __syncwarp();
        if (ok && (peers & lt) == 0) wcount[warp][d] += (uint32_t)__popc(peers);
        __syncwarp();
        if (ok) {
            keys_out[q] = key[j];
            idx_out[q] = idx[j];
        }
    }
}

inline int sort_tiles(int64_t n) { return (int)((n + kSortTile - 1) / kSortTile); }
// Words of count scratch a sort of n keys needs (digit-major counts).
inline size_t sort_count_words(int64_t n) { return (size_t)kDigits * (size_t)sort_tiles(n); }
// Words of scan scratch a sort of n keys needs.
inline size_t sort_scan_words(int64_t n) { return scan_scratch_words(sort_count_words(n)); }

// Sorts n (key, value) pairs by key bits [begin_bit, end_bit), stably, in
// passes of kDigitBits (the last may be narrower; the digit mask reads any
// higher bits as 0 only if the keys have none). The pairs start in buffer 0
// (keys[0], vals[0]); *result is the buffer they end in. When first_counted,
// `count` already holds the first pass's digit counts. n < 2^31.
template <class K>
cudaError_t sort_pairs(K* keys[2], int32_t* vals[2], int64_t n, int begin_bit, int end_bit, uint32_t* count,
                       uint32_t* scan, bool first_counted, int* result, cudaStream_t s) {
    *result = 0;
    if (n <= 0) return cudaSuccess;
    const int tiles = sort_tiles(n);
    const size_t counts = sort_count_words(n);
    const size_t scan_tiles = (counts + kScanTile - 1) / kScanTile;
    cudaError_t e = cudaSuccess;
    int cur = 0;
    for (int shift = begin_bit; shift < end_bit && e == cudaSuccess; shift += kDigitBits) {
        if (!(first_counted && shift == begin_bit)) {
            k_digit_count<K><<<tiles, kSortThreads, 0, s>>>(keys[cur], n, shift, tiles, count);
            if ((e = cudaGetLastError()) != cudaSuccess) break;
        }
        const uint32_t* tile_start = nullptr;
        if (scan_tiles <= 1024) {  // two levels; the scatter adds the tile's start itself
            k_scan_tiles<<<(unsigned)scan_tiles, 1024, 0, s>>>(count, count, counts, scan);
            k_scan_tile_sums<<<1, 1024, 0, s>>>(scan, (int)scan_tiles);
            tile_start = scan;
            e = cudaGetLastError();
        } else {
            e = scan_exclusive(count, count, counts, scan, s);
        }
        if (e != cudaSuccess) break;
        k_digit_scatter<K><<<tiles, kSortThreads, 0, s>>>(keys[cur], vals[cur], n, shift, tiles, count, tile_start,
                                                          keys[cur ^ 1], vals[cur ^ 1]);
        e = cudaGetLastError();
        cur ^= 1;
    }
    *result = cur;
    return e;
}

}  // namespace
}  // namespace psort
}  // namespace sg
