// Closest-hit and any-hit traversal of SORT-topology wide BVHs on sm_100a.
//
// The per-ray traversal restates Fbvh::GetIntersect
// (accel/fast_bvh.hpp:305-504, SIMD branch):
//   * root slab test against the enlarged scene box (scalar Intersect);
//   * a stack of (node, entry distance) pairs; a popped entry is skipped when
//     the current hit is nearer than its entry distance (strict <, line 343);
//   * a leaf tests its triangles in SIMD-lane packing order and keeps a hit only
//     when strictly nearer (simd/simd_triangle.h:359-369), so the first of equal
//     distances wins;
//   * an interior node's hit children are visited nearest first; equal distances
//     visit the higher child slot first (the 1-, 2- and >=3-hit cases of lines
//     416-455 all reduce to that order);
//   * any-hit returns at the first triangle hit (opaque early exit, 362-373).
// With FP32 child boxes and the same rounding, hits, distances and barycentrics
// are bit-identical to SORT's.
//
// GPU-side choices that leave that order intact:
//   * the entry SORT would pop right after pushing a node's children (the
//     nearest) stays in registers and is descended into directly;
//   * leaf triangles are fetched two at a time (the triangle array carries one
//     padding slot), so the second's loads overlap the first's test;
//   * schedules: one ray per thread for the whole launch; persistent warps in
//     which a lane whose ray finished takes the next ray of the batch, so warps
//     stay full instead of idling on their slowest ray; while-while and its
//     speculative form; and one ray per thread with the rays taken in the order
//     of a coherence key (direction octant, origin cell, coarse direction), so
//     a warp's rays visit similar nodes (fewer idle lanes), which the automatic
//     default uses for large closest-hit batches.
#include <cuda_runtime.h>

#include <mutex>
#include <vector>

#include "prefix_sort.cuh"
#include "trace_kernels.h"
#include "traversal.cuh"

namespace sg {

// One ray per thread for the whole launch. With n_dev set, the batch size is
// min(n, *n_dev), read on the device (queues whose length only the GPU knows).
// Q8 reads 8-bit nodes.
// With `order` set, thread k traces ray order[k] (the sorted schedule).
template <int W, bool ANY, int STACK, bool STATS, bool Q8>
__device__ __forceinline__ void trace_one_ray(const DevTree& tr, const DevRays& rays, int64_t n,
                                              int32_t* __restrict__ prim_out, float* __restrict__ t_out,
                                              float* __restrict__ u_out, float* __restrict__ v_out,
                                              uint8_t* __restrict__ occ_out, int* __restrict__ err,
                                              unsigned long long* __restrict__ stats, const int* __restrict__ n_dev,
                                              const int32_t* __restrict__ order) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n_dev && k >= (int64_t)*n_dev) return;
    if (k >= n) return;
    const int64_t i = order ? (int64_t)__ldg(order + k) : k;
    Traversal<W, ANY, STACK, STATS, Q8, true> tv;
    uint2 stk_mem[STACK];
    tv.stk = stk_mem;
    if (tv.start(tr, rays, i))
        while (!tv.step(tr, err)) {
        }
    tv.finish(i, prim_out, t_out, u_out, v_out, occ_out, stats);
}

// Launch bounds: registers limit the occupancy of these kernels. Left alone,
// the compiler gives the width-8 any-hit kernel 61 registers (8 blocks of 128
// per SM); held to 9 blocks it fits 56 with 8 bytes spilled and runs 5.8%
// faster on 4M shadow rays. The others already fit their bound (width 8
// closest 56, width 4 closest 55, width 4 any-hit 48 at 10 blocks).
template <int W, bool ANY, int STACK, bool STATS, bool Q8 = false>
__global__ void __launch_bounds__(128, (W == 4 && ANY) ? 10 : 9) k_trace_fp32(DevTree tr, DevRays rays, int64_t n, int32_t* __restrict__ prim_out,
                                                    float* __restrict__ t_out, float* __restrict__ u_out,
                                                    float* __restrict__ v_out, uint8_t* __restrict__ occ_out,
                                                    int* __restrict__ err, unsigned long long* __restrict__ stats,
                                                    const int* __restrict__ n_dev,
                                                    const int32_t* __restrict__ order = nullptr) {
    trace_one_ray<W, ANY, STACK, STATS, Q8>(tr, rays, n, prim_out, t_out, u_out, v_out, occ_out, err, stats, n_dev,
                                           order);
}

// One ray per thread with RayWalk, the hot path for FP32 and 8-bit nodes. With
// n_dev set the batch is min(n, *n_dev); with `order` set, thread k traces ray
// order[k]. Held to 9 blocks of 128 per SM (56 registers): left alone the
// compiler takes 94 registers (every node and triangle load in flight at
// once); 8 blocks ran at 994 Mrays/s, 9 at 1,031, and 10 (48 registers)
// spills inside the traversal loop and fell to 968 (one triangle per
// iteration) or to about 240 (two).
template <int W, bool ANY, int STACK, bool Q8>
__global__ void __launch_bounds__(128, 9)
    k_trace_walk(DevTree tr, DevRays rays, int64_t n, int32_t* __restrict__ prim_out, float* __restrict__ t_out,
                 float* __restrict__ u_out, float* __restrict__ v_out, uint8_t* __restrict__ occ_out,
                 int* __restrict__ err, const int* __restrict__ n_dev, const int32_t* __restrict__ order) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n_dev && k >= (int64_t)*n_dev) return;
    if (k >= n) return;
    const int64_t i = order ? (int64_t)__ldg(order + k) : k;
    uint2 stk[STACK];
    RayWalk<W, ANY, STACK, Q8> w;
    if (w.start(tr, rays, i))
        while (!w.step(tr, stk, err)) {
        }
    w.finish(tr, i, prim_out, t_out, u_out, v_out, occ_out);
}

// The same for 8-bit nodes, held to 9 blocks of 128 per SM: the decode leaves
// the compiler at 72-80 registers (7 blocks); at 56 it spills 64 bytes and is
// still 4.6% faster on 4M incoherent rays (more warps hide the node loads).
template <int W, bool ANY, int STACK, bool STATS>
__global__ void __launch_bounds__(128, 9) k_trace_q8(DevTree tr, DevRays rays, int64_t n, int32_t* __restrict__ prim_out,
                                                     float* __restrict__ t_out, float* __restrict__ u_out,
                                                     float* __restrict__ v_out, uint8_t* __restrict__ occ_out,
                                                     int* __restrict__ err, unsigned long long* __restrict__ stats,
                                                     const int* __restrict__ n_dev,
                                                     const int32_t* __restrict__ order = nullptr) {
    trace_one_ray<W, ANY, STACK, STATS, true>(tr, rays, n, prim_out, t_out, u_out, v_out, occ_out, err, stats, n_dev,
                                             order);
}

// Persistent warps: a lane whose ray finished takes the next ray in batch order
// once at least `refill` lanes of its warp are idle; the warp's leader claims
// those rays from a launch-wide counter, so the whole GPU still advances
// through the batch in order (neighbouring rays share tree nodes in L1/L2).
template <int W, bool ANY, int STACK, bool STATS>
__global__ void __launch_bounds__(128) k_trace_fp32_persistent(DevTree tr, DevRays rays, int64_t n,
                                                               unsigned long long* __restrict__ counter, int refill,
                                                               int32_t* __restrict__ prim_out, float* __restrict__ t_out,
                                                               float* __restrict__ u_out, float* __restrict__ v_out,
                                                               uint8_t* __restrict__ occ_out, int* __restrict__ err,
                                                               unsigned long long* __restrict__ stats) {
    const unsigned lane = threadIdx.x & 31u;
    const unsigned lt_mask = (1u << lane) - 1u;
    Traversal<W, ANY, STACK, STATS, false, true> tv;
    uint2 stk_mem[STACK];
    tv.stk = stk_mem;
    bool alive = false;
    bool drained = false;  // warp-uniform: the counter has passed n
    int64_t ray = -1;
    for (;;) {
        const unsigned idle = __ballot_sync(0xffffffffu, !alive);
        if (idle != 0 && !drained) {
            unsigned long long base = 0;
            if (lane == 0) base = atomicAdd(counter, (unsigned long long)__popc(idle));
            base = __shfl_sync(0xffffffffu, base, 0);
            if ((int64_t)base >= n) drained = true;
            if (!alive) {
                const int64_t idx = (int64_t)base + __popc(idle & lt_mask);
                if (idx < n) {
                    ray = idx;
                    alive = tv.start(tr, rays, idx);
                    if (!alive) tv.finish(idx, prim_out, t_out, u_out, v_out, occ_out, stats);
                }
            }
        }
        const unsigned busy0 = __ballot_sync(0xffffffffu, alive);
        if (busy0 == 0) {
            if (drained) break;
            continue;
        }
        // Traverse until enough lanes are idle to be worth refilling.
        for (;;) {
            if (alive && tv.step(tr, err)) {
                tv.finish(ray, prim_out, t_out, u_out, v_out, occ_out, stats);
                alive = false;
            }
            const unsigned busy = __ballot_sync(0xffffffffu, alive);
            if (busy == 0) break;
            if (!drained && 32 - __popc(busy) >= refill) break;
        }
    }
}

// Persistent warps over RayWalk (the persistent schedule without counters): a
// lane whose ray finished takes the next ray once at least `refill` lanes of
// its warp are idle; the warp's leader claims those rays from a launch-wide
// counter, in batch order or, with `order` set, in the order it lists.
template <int W, bool ANY, int STACK, bool Q8>
__global__ void __launch_bounds__(128, 9)
    k_trace_walk_persistent(DevTree tr, DevRays rays, int64_t n, unsigned long long* __restrict__ counter, int refill,
                            const int32_t* __restrict__ order, int32_t* __restrict__ prim_out,
                            float* __restrict__ t_out, float* __restrict__ u_out, float* __restrict__ v_out,
                            uint8_t* __restrict__ occ_out, int* __restrict__ err) {
    const unsigned lane = threadIdx.x & 31u;
    const unsigned lt_mask = (1u << lane) - 1u;
    uint2 stk[STACK];
    RayWalk<W, ANY, STACK, Q8> w;
    bool alive = false;
    bool drained = false;  // warp-uniform: the counter has passed n
    int64_t ray = -1;
    for (;;) {
        const unsigned idle = __ballot_sync(0xffffffffu, !alive);
        if (idle != 0 && !drained) {
            unsigned long long base = 0;
            if (lane == 0) base = atomicAdd(counter, (unsigned long long)__popc(idle));
            base = __shfl_sync(0xffffffffu, base, 0);
            if ((int64_t)base >= n) drained = true;
            if (!alive) {
                const int64_t k = (int64_t)base + __popc(idle & lt_mask);
                if (k < n) {
                    ray = order ? (int64_t)__ldg(order + k) : k;
                    alive = w.start(tr, rays, ray);
                    if (!alive) w.finish(tr, ray, prim_out, t_out, u_out, v_out, occ_out);
                }
            }
        }
        const unsigned busy0 = __ballot_sync(0xffffffffu, alive);
        if (busy0 == 0) {
            if (drained) break;
            continue;
        }
        for (;;) {  // traverse until enough lanes are idle to be worth refilling
            if (alive && w.step(tr, stk, err)) {
                w.finish(tr, ray, prim_out, t_out, u_out, v_out, occ_out);
                alive = false;
            }
            const unsigned busy = __ballot_sync(0xffffffffu, alive);
            if (busy == 0) break;
            if (!drained && 32 - __popc(busy) >= refill) break;
        }
    }
}

// While-while traversal over RayWalk, one ray per thread: the warp alternates
// an interior phase (each lane pops / descends until it holds an un-culled
// leaf; with SPEC a lane that holds one keeps descending while others lack
// one) and a leaf phase. Leaves are tested in SORT's order and culled with the
// hit found so far, so results are SORT's: a speculative visit only sees
// interior nodes SORT visits too, or that SORT culls -- and then every leaf
// below is culled here as well, because a child's entry distance is never
// below its parent's (each slab bound of a child lies inside the parent's, and
// the rounded t = -o/d + b/d is monotonic in b). With `order` set, thread k
// traces ray order[k]. Measured on 4,194,304 incoherent rays: 850 (plain) and
// 902 (speculative) Mrays/s against 969 for one ray per thread, and 900 / 960
// against 1,036 in sorted order: the phase bookkeeping costs more issue slots
// than the split saves.
template <int W, bool ANY, int STACK, bool SPEC>
__global__ void __launch_bounds__(128, 9)
    k_trace_walk_ww(DevTree tr, DevRays rays, int64_t n, const int32_t* __restrict__ order,
                    int32_t* __restrict__ prim_out, float* __restrict__ t_out, float* __restrict__ u_out,
                    float* __restrict__ v_out, uint8_t* __restrict__ occ_out, int* __restrict__ err) {
    const int64_t k0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = k0 < n;
    const int64_t k = valid ? k0 : n - 1;  // lanes past the batch end idle through the loop
    const int64_t i = order ? (int64_t)__ldg(order + k) : k;
    uint2 stk[STACK];
    RayWalk<W, ANY, STACK, false> w;
    const bool started = w.start(tr, rays, i);
    bool have = valid && started;
    bool pend = false;
    int32_t lf = 0;
    float lf_d = 0.0f;
    while (__any_sync(0xffffffffu, have || pend)) {
        for (;;) {
            const bool needs = have && !pend;
            const bool spec = SPEC && have && pend;
            if (!__any_sync(0xffffffffu, needs)) break;
            if (needs || spec) {
                bool descend = false;
                bool blocked = false;
                if (!(w.best_t < w.cur_d)) {
                    if (w.cur < 0) {
                        if (w.cur == kEmpty) {
                        } else if (!pend) {
                            lf = w.cur;
                            lf_d = w.cur_d;
                            pend = true;
                        } else {
                            blocked = true;  // second leaf: wait for the leaf phase
                        }
                    } else if (w.si + W > STACK) {  // cannot happen when STACK >= depth*(W-1)+1
                        atomicOr(err, 1);
                        have = false;
                        blocked = true;
                    } else {
                        descend = w.interior(tr, stk);
                    }
                }
                if (!descend && !blocked) {
                    if (w.si == 0) {
                        have = false;
                    } else {
                        const uint2 e = stk[--w.si];
                        w.cur = (int32_t)e.x;
                        w.cur_d = __uint_as_float(e.y);
                    }
                }
            }
        }
        if (pend) {
            pend = false;
            if (!(w.best_t < lf_d) && w.leaf(tr, lf)) have = false;  // any-hit: done
        }
    }
    if (valid) w.finish(tr, i, prim_out, t_out, u_out, v_out, occ_out);
}

// Stream-ordered scratch for the sorted schedule: one pool per device that
// keeps up to 1 GiB mapped between launches (NULL if it cannot be made).
static cudaMemPool_t trace_scratch_pool(int device) {
    static std::mutex lock;
    static std::vector<cudaMemPool_t> pools;
    std::lock_guard<std::mutex> g(lock);
    if (device < 0) return nullptr;
    if (pools.size() <= size_t(device)) pools.resize(size_t(device) + 1, nullptr);
    if (!pools[size_t(device)]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        cudaMemPool_t pool = nullptr;
        if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) return nullptr;
        uint64_t keep = uint64_t(1) << 30;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        pools[size_t(device)] = pool;
    }
    return pools[size_t(device)];
}

// ---------------------------------------------------------------------------
// Sorted schedule (SG_SCHEDULE_SORTED, and the automatic choice for large
// closest-hit batches): rays are put in the order of a 30-bit coherence key
// before the thread-per-ray traversal, so that a warp holds rays that start
// near one another and head the same way and take more of the same branches.
// The key: direction octant (3 bits), the Morton code of the origin's cell on a
// 128^3 grid over the scene box (21 bits), then 2 bits per axis of direction.
//
// The order is a stable sort of the keys (equal keys keep batch order, which
// carries the input's own coherence: neighbouring pixels, neighbouring hit
// points), made by least-significant-digit radix passes of 10 bits over the
// whole key (three passes):
//  * k_sort_keys: key and batch index per ray (coalesced SoA reads);
//  * per pass, k_digit_count: a tile of 4,096 keys per block counts its digits
//    in shared memory and writes them digit-major (count[d * tiles + tile]);
//    scan_exclusive: prefix sums over those counts, so each (digit, tile)
//    knows where its run starts; k_digit_scatter: each warp owns a contiguous
//    512-key chunk of its tile, counts its digits, the block turns the counts
//    into per-warp starting places, and each warp writes its keys in order
//    (lanes of one digit ranked by __match_any_sync), which keeps the sort
//    stable;
//  * k_trace_walk with `order`: thread k traces ray order[k] and writes its
//    answer at that ray's own index, so results do not depend on the order.
// Measured on 4,194,304 incoherent rays (21M triangles): 1,034.5 Mrays/s
// including the sort, against 1,031.1 with CUB's radix sort of the same keys
// (same order) and 968.7 unsorted. Sorting only the key's top 10 or 20 bits
// (one or two passes, batch order inside each group) gave 936 and 974, and
// single-pass bucketing whose order inside a bucket followed warp timing gave
// 902-954: the order inside a group matters.
constexpr int kKeyBits = 30;
constexpr int kSortBits = 30;  // top bits of the key that are sorted
using psort::kDigits;
using psort::kSortTile;
using psort::kSortThreads;
using psort::kSortItems;
static_assert(kSortBits % psort::kDigitBits == 0 && kSortBits <= kKeyBits, "whole digits of the key");

struct KeyGrid {
    float lo[3];
    float scale[3];  // 128 cells over the scene box's extent on each axis
};

__device__ __forceinline__ uint32_t spread7(uint32_t v) {  // bit b of v to bit 3b
    uint32_t r = 0;
#pragma unroll
    for (int b = 0; b < 7; ++b) r |= ((v >> b) & 1u) << (3 * b);
    return r;
}

// Key and batch index of every ray of a tile of kSortTile rays, and the tile's
// counts of the first pass's digit (as k_digit_count).
__global__ void __launch_bounds__(kSortThreads) k_sort_keys(DevRays rays, int64_t n, KeyGrid g, int shift, int tiles,
                                                            uint32_t* __restrict__ keys, int32_t* __restrict__ index,
                                                            uint32_t* __restrict__ count) {
    __shared__ uint32_t hist[kDigits];
    for (int d = threadIdx.x; d < kDigits; d += kSortThreads) hist[d] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kSortTile;
#pragma unroll 4
    for (int j = 0; j < kSortItems; ++j) {
        const int64_t i = base + j * kSortThreads + threadIdx.x;
        if (i >= n) continue;
        const float o[3] = {rays.ox[i], rays.oy[i], rays.oz[i]}, d[3] = {rays.dx[i], rays.dy[i], rays.dz[i]};
        uint32_t oct = 0, cell = 0, dir = 0;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            oct |= (d[a] < 0.0f ? 1u : 0u) << (2 - a);
            const float q = fminf(fmaxf((o[a] - g.lo[a]) * g.scale[a], 0.0f), 127.0f);  // NaN -> 0
            cell |= spread7((uint32_t)q) << (2 - a);
            const float e = fminf(fmaxf((d[a] + 1.0f) * 2.0f, 0.0f), 3.0f);
            dir |= ((uint32_t)e & 1u) << (2 - a) | (((uint32_t)e >> 1) & 1u) << (5 - a);
        }
        const uint32_t key = (oct << 27) | (cell << 6) | dir;
        keys[i] = key;
        index[i] = (int32_t)i;
        atomicAdd(&hist[(key >> shift) & (kDigits - 1)], 1u);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < kDigits; d += kSortThreads) count[(size_t)d * tiles + blockIdx.x] = hist[d];
}

// The sorted schedule. Scratch (16 bytes per ray, 4 per (digit, tile) and the
// scan's) comes from the library's stream-ordered pool and is freed in stream
// order.
template <int W, bool ANY, int STACK, bool Q8>
static cudaError_t launch_sorted(const TraceLaunch& L, const DevTree& tr, const DevRays& rays, int64_t n,
                                 cudaStream_t s) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    cudaMemPool_t pool = trace_scratch_pool(dev);
    if (!pool) return cudaErrorMemoryAllocation;
    const int tiles = psort::sort_tiles(n);
    const size_t al = 256;
    auto up = [al](size_t b) { return ((b + al - 1) / al) * al; };
    const size_t b_ray = up(size_t(n) * 4), b_count = up(psort::sort_count_words(n) * 4),
                 b_scan = up(psort::sort_scan_words(n) * 4);
    char* base = nullptr;
    e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&base), 4 * b_ray + b_count + b_scan, pool, s);
    if (e != cudaSuccess) return e;
    uint32_t* keys[2] = {reinterpret_cast<uint32_t*>(base), reinterpret_cast<uint32_t*>(base + b_ray)};
    int32_t* idx[2] = {reinterpret_cast<int32_t*>(base + 2 * b_ray), reinterpret_cast<int32_t*>(base + 3 * b_ray)};
    uint32_t* count = reinterpret_cast<uint32_t*>(base + 4 * b_ray);
    uint32_t* scan = reinterpret_cast<uint32_t*>(base + 4 * b_ray + b_count);
    KeyGrid g;
    for (int a = 0; a < 3; ++a) {
        const float ext = tr.box_hi[a] - tr.box_lo[a];
        g.lo[a] = tr.box_lo[a];
        g.scale[a] = ext > 0.0f ? 128.0f / ext : 0.0f;
    }
    const int first = kKeyBits - kSortBits;
    k_sort_keys<<<tiles, kSortThreads, 0, s>>>(rays, n, g, first, tiles, keys[0], idx[0], count);
    int cur = 0;
    if ((e = cudaGetLastError()) == cudaSuccess)
        e = psort::sort_pairs<uint32_t>(keys, idx, n, first, kKeyBits, count, scan, true, &cur, s);
    if (e == cudaSuccess) {
        k_trace_walk<W, ANY, STACK, Q8><<<(unsigned)((n + 127) / 128), 128, 0, s>>>(
            tr, rays, n, L.prim, L.t, L.u, L.v, L.occ, L.err, nullptr, idx[cur]);
        e = cudaGetLastError();
    }
    const cudaError_t f = cudaFreeAsync(base, s);
    return e != cudaSuccess ? e : f;
}

template <int W, bool ANY, int STACK, bool STATS>
static cudaError_t launch_stack(const TraceLaunch& L, const DevTree& tr, const DevRays& rays, int64_t n,
                                cudaStream_t s) {
    const int threads = 128;
    // Batches large enough for reordering to pay (and within a 32-bit sort);
    // the automatic choice sorts large closest-hit batches only (any-hit rays
    // end early, and measured no faster sorted).
    const bool sorted = L.tuning.schedule == kScheduleSorted ? n >= (int64_t(1) << 16)
                        : L.tuning.schedule == kScheduleAuto  ? !ANY && n >= (int64_t(1) << 21)
                                                              : false;
    if (!STATS && !L.n_dev && sorted && n < (int64_t(1) << 31))
        return L.q8 ? launch_sorted<W, ANY, STACK, true>(L, tr, rays, n, s)
                    : launch_sorted<W, ANY, STACK, false>(L, tr, rays, n, s);
    // Counting launches keep the one-entry-per-step loop, whose interior-node
    // visits are exactly SORT's (speculation visits extra ones).
    // 8-bit nodes are read by the one-ray-per-thread kernels.
    if (L.q8) {
        const int64_t blocks = (n + threads - 1) / threads;
        if (STATS)
            k_trace_q8<W, ANY, STACK, STATS><<<(unsigned)blocks, threads, 0, s>>>(
                tr, rays, n, L.prim, L.t, L.u, L.v, L.occ, L.err, L.stats, L.n_dev);
        else
            k_trace_walk<W, ANY, STACK, true><<<(unsigned)blocks, threads, 0, s>>>(
                tr, rays, n, L.prim, L.t, L.u, L.v, L.occ, L.err, L.n_dev, nullptr);
        return cudaGetLastError();
    }
    // A device-side batch size is only read by the one-ray-per-thread kernel.
    if (!STATS && !L.n_dev &&
        (L.tuning.schedule == kScheduleWhileWhile || L.tuning.schedule == kScheduleSpeculative)) {
        const int64_t blocks = (n + threads - 1) / threads;
        if (L.tuning.schedule == kScheduleSpeculative)
            k_trace_walk_ww<W, ANY, STACK, true><<<(unsigned)blocks, threads, 0, s>>>(tr, rays, n, nullptr, L.prim,
                                                                                      L.t, L.u, L.v, L.occ, L.err);
        else
            k_trace_walk_ww<W, ANY, STACK, false><<<(unsigned)blocks, threads, 0, s>>>(tr, rays, n, nullptr, L.prim,
                                                                                       L.t, L.u, L.v, L.occ, L.err);
        return cudaGetLastError();
    }
    if (L.tuning.schedule == kSchedulePersistent && !L.n_dev && !STATS) {
        int dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        int64_t blocks = (int64_t)(sms < 1 ? 1 : sms) * 9;  // 9 resident blocks of 128 per SM
        const int64_t needed = (n + threads - 1) / threads;
        if (blocks > needed) blocks = needed;
        const int refill = L.tuning.refill_threshold < 1 ? 1 : (L.tuning.refill_threshold > 32 ? 32 : L.tuning.refill_threshold);
        cudaError_t e = cudaMemsetAsync(L.counter, 0, sizeof(unsigned long long), s);
        if (e != cudaSuccess) return e;
        k_trace_walk_persistent<W, ANY, STACK, false><<<(unsigned)blocks, threads, 0, s>>>(
            tr, rays, n, L.counter, refill, nullptr, L.prim, L.t, L.u, L.v, L.occ, L.err);
        return cudaGetLastError();
    }
    if (L.tuning.schedule == kSchedulePersistent && !L.n_dev) {
        int dev = 0, sms = 0, blocks_per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, k_trace_fp32_persistent<W, ANY, STACK, STATS>,
                                                      threads, 0);
        if (blocks_per_sm < 1) blocks_per_sm = 1;
        if (sms < 1) sms = 1;
        int64_t blocks = (int64_t)sms * blocks_per_sm;
        const int64_t needed = (n + threads - 1) / threads;
        if (blocks > needed) blocks = needed;
        const int refill = L.tuning.refill_threshold < 1 ? 1 : (L.tuning.refill_threshold > 32 ? 32 : L.tuning.refill_threshold);
        cudaError_t e = cudaMemsetAsync(L.counter, 0, sizeof(unsigned long long), s);
        if (e != cudaSuccess) return e;
        k_trace_fp32_persistent<W, ANY, STACK, STATS><<<(unsigned)blocks, threads, 0, s>>>(
            tr, rays, n, L.counter, refill, L.prim, L.t, L.u, L.v, L.occ, L.err, L.stats);
    } else if (STATS) {
        const int64_t blocks = (n + threads - 1) / threads;
        k_trace_fp32<W, ANY, STACK, STATS><<<(unsigned)blocks, threads, 0, s>>>(tr, rays, n, L.prim, L.t, L.u, L.v,
                                                                                L.occ, L.err, L.stats, L.n_dev);
    } else {
        const int64_t blocks = (n + threads - 1) / threads;
        k_trace_walk<W, ANY, STACK, false><<<(unsigned)blocks, threads, 0, s>>>(tr, rays, n, L.prim, L.t, L.u, L.v,
                                                                               L.occ, L.err, L.n_dev, nullptr);
    }
    return cudaGetLastError();
}

template <int W, bool ANY, bool STATS>
static cudaError_t launch_w(const TraceLaunch& L, const DevTree& tr, const DevRays& rays, int64_t n, cudaStream_t s) {
    if (L.stack_need <= 64) return launch_stack<W, ANY, 64, STATS>(L, tr, rays, n, s);
    if (L.stack_need <= 128) return launch_stack<W, ANY, 128, STATS>(L, tr, rays, n, s);
    if (L.stack_need <= 256) return launch_stack<W, ANY, 256, STATS>(L, tr, rays, n, s);
    return cudaErrorInvalidValue;
}

template <bool STATS>
static cudaError_t launch_any_width(const TraceLaunch& L, const DevTree& tr, const DevRays& rays, int64_t n,
                                    cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    if (L.width == 8)
        return L.any ? launch_w<8, true, STATS>(L, tr, rays, n, s) : launch_w<8, false, STATS>(L, tr, rays, n, s);
    return L.any ? launch_w<4, true, STATS>(L, tr, rays, n, s) : launch_w<4, false, STATS>(L, tr, rays, n, s);
}

cudaError_t launch_trace_fp32(const TraceLaunch& L, const DevTree& tr, const DevRays& rays, int64_t n,
                              cudaStream_t s) {
    return L.stats ? launch_any_width<true>(L, tr, rays, n, s) : launch_any_width<false>(L, tr, rays, n, s);
}

}  // namespace sg
