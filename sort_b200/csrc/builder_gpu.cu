// build_tree_gpu: SORT's Fbvh::Build split rules (the tree build_tree makes),
// computed on the GPU.
//
// SORT splits a node breadth-first: the node's range list starts as its whole
// primitive range; the front range is split (16-bin SAH on the longest axis of
// its centroid bounds, normalised by the node's box, then std::partition) into
// two ranges appended to the list, or set aside as a child when the split does
// not pay, until the node has W children (accel/fast_bvh.hpp:138-211,
// accel/bvh_utils.h:69-118). Each split only permutes its own range, so the
// splits of different nodes are independent, and the ones of one node depend
// only on their order. Here every node under construction takes the split of
// its front range in the same round, and a round is a few data-parallel passes
// over the primitives of the ranges being split:
//   * centroid bounds and bins (counts, primitive boxes) per range: lanes of a
//     warp with the same key combine their values (match + warp reductions),
//     blocks inside one range combine in shared memory, and one lane per group
//     applies atomics on order-preserving integer images of the floats;
//   * the SAH sweep, one thread per range, in SORT's arithmetic order;
//   * the boxes of both halves of every split range, reduced in the pass that
//     counts the left half: they are the child boxes and the children's SAH
//     normalisers, so no pass computes child boxes afterwards;
//   * std::partition as libstdc++ performs it on random-access iterators: the
//     k-th element of the left part that fails the predicate is swapped with
//     the k-th element from the right end of the right part that passes it,
//     so the result is found with two prefix sums and one swap per pair.
// Centroids and primitive boxes travel with the primitives (slot order), so
// every pass reads them coalesced. The nodes under construction live on the
// GPU too, in primitive-range order: after the passes, one thread per node
// applies its split to the node's range lists, a finished node writes its
// children as shape nodes, and prefix sums place the continuing nodes and the
// new ones in the next round's list. A round costs one 16-byte download (the
// sizes of the next round). The host only flattens the finished shape tree.
// The tree, the leaf order and every box value are build_tree's; a box bound
// that is zero may carry the other sign, which no comparison sees.
#include <cuda_runtime.h>


#include <algorithm>
#include <cfloat>
#include <cstdint>
#include <cstring>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "builder.h"
#include "gpu_build_common.cuh"
#include "staged_upload.h"
#include "layout.h"
#include "prefix_sort.cuh"

namespace sg {
namespace gpub {

void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string("GPU build: ") + what + ": " + cudaGetErrorString(e));
}

cudaMemPool_t scratch_pool(int device) {
    static std::mutex lock;
    static std::vector<cudaMemPool_t> pools;
    std::lock_guard<std::mutex> g(lock);
    if (device < 0) throw std::invalid_argument("device out of range");
    if (pools.size() <= size_t(device)) pools.resize(size_t(device) + 1, nullptr);
    if (!pools[size_t(device)]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        cudaMemPool_t pool = nullptr;
        check(cudaMemPoolCreate(&pool, &props), "cudaMemPoolCreate");
        uint64_t keep = UINT64_MAX;  // release only when a build ends (trim below)
        check(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep), "pool threshold");
        pools[size_t(device)] = pool;
    }
    return pools[size_t(device)];
}

thread_local Scratch scratch;

namespace {

// Pinned host memory the GPU builds of a device read their results into,
// kept between builds (pinning 130 MB anew costs about 200 ms); one build at
// a time per device holds it.
struct Staging {
    std::mutex lock;
    void* p = nullptr;
    size_t bytes = 0;
};

Staging& staging(int device) {
    static std::mutex lock;
    static std::vector<std::unique_ptr<Staging>> all;
    std::lock_guard<std::mutex> g(lock);
    if (all.size() <= size_t(device)) all.resize(size_t(device) + 1);
    if (!all[size_t(device)]) all[size_t(device)] = std::make_unique<Staging>();
    return *all[size_t(device)];
}

}  // namespace

}  // namespace gpub
namespace {

using namespace gpub;

constexpr int kBins = 16;

// Per range being split this round.
struct RangeTask {
    int64_t s, e;
    float node_area;  // half_area of the node's box (SAH normaliser)
    int inner[6];     // centroid bounds: min xyz, max xyz (order images)
    unsigned bin_cnt[kBins];
    int bin_box[kBins][6];
    // decision
    int axis;
    float split_pos;
    int split;           // 1 = partition this range
    unsigned left;       // primitives passing the predicate
    int half_box[2][6];  // primitive boxes of the left (passing) and right halves
};

// Device-resident build state: the rounds need no host round trip.
struct BuildState {
    int na;         // nodes under construction this round (= ranges split)
    int shapes;     // shape nodes written so far
    int depth_max;  // Fbvh::m_depth
    int rounds;     // rounds that split something
    int next;       // this round's results, consumed by k_advance
    int new_shapes;
};

__device__ __forceinline__ int find_range(const int64_t* __restrict__ starts, const int64_t* __restrict__ ends,
                                          int nr, int64_t i) {
    int lo = 0, hi = nr - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (starts[mid] <= i)
            lo = mid;
        else
            hi = mid - 1;
    }
    return (nr > 0 && starts[lo] <= i && i < ends[lo]) ? lo : -1;
}

__device__ __forceinline__ bool leads(unsigned peers) { return int(__ffs(peers)) - 1 == int(threadIdx.x & 31); }

// Lanes with the same key combine: min over v[0..K), max over v[K..2K).
// Every lane of the warp calls it; returns the lanes sharing the caller's key.
template <int K>
__device__ __forceinline__ unsigned group_minmax(long long key, int (&v)[2 * K]) {
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    for (int a = 0; a < K; ++a) {
        v[a] = __reduce_min_sync(peers, v[a]);
        v[K + a] = __reduce_max_sync(peers, v[K + a]);
    }
    return peers;
}

// Blocks whose primitives all belong to one range (the common case while
// ranges are large) reduce in shared memory first and touch the range's
// global accumulators once; other blocks update them per warp group.
__device__ __forceinline__ bool block_in_one_range(int r, int& shared_r) {
    if (threadIdx.x == 0) shared_r = r;
    __syncthreads();
    return __syncthreads_and(r == shared_r && r >= 0) != 0;
}

// Range id of every primitive (-1 outside the round's ranges) and centroid bounds.
__global__ void __launch_bounds__(256) k_bounds(int64_t n, const int64_t* __restrict__ starts,
                                                const int64_t* __restrict__ ends, const BuildState* __restrict__ bs,
                                                const float* __restrict__ cx,
                                                const float* __restrict__ cy, const float* __restrict__ cz,
                                                int* __restrict__ rid, RangeTask* __restrict__ rt) {
    __shared__ int sr, sbox[6];
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = i < n;
    const int r = in ? find_range(starts, ends, bs->na, i) : -1;
    if (in) rid[i] = r;
    if (threadIdx.x == 0) empty_box(sbox);
    const bool one = block_in_one_range(r, sr);
    int v[6];
    if (r >= 0) {
        v[0] = v[3] = f2o(cx[i]);
        v[1] = v[4] = f2o(cy[i]);
        v[2] = v[5] = f2o(cz[i]);
    } else {
        empty_box(v);
    }
    const unsigned peers = group_minmax<3>(r, v);
    const bool lead = r >= 0 && leads(peers);
    if (one) {
        if (lead) atomic_box(sbox, v);
        __syncthreads();
        if (threadIdx.x < 3) {
            atomicMin(&rt[r].inner[threadIdx.x], sbox[threadIdx.x]);
            atomicMax(&rt[r].inner[3 + threadIdx.x], sbox[3 + threadIdx.x]);
        }
        return;
    }
    if (lead) atomic_box(rt[r].inner, v);
}

__device__ __forceinline__ float half_area(const float* mn, const float* mx) {
    const float ox = __fsub_rn(mx[0], mn[0]), oy = __fsub_rn(mx[1], mn[1]), oz = __fsub_rn(mx[2], mn[2]);
    const float a = __fmul_rn(ox, oy), c = __fmul_rn(oy, oz), e = __fmul_rn(oz, ox);
    return __fadd_rn(__fadd_rn(a, c), e);
}

// Axis and bin geometry of a range (pick_best_split's first half).
__device__ __forceinline__ bool bin_geometry(const RangeTask& t, int& axis, float& start, float& delta, float& inv) {
    float mn[3], mx[3];
    for (int a = 0; a < 3; ++a) {
        mn[a] = o2f(t.inner[a]);
        mx[a] = o2f(t.inner[3 + a]);
    }
    const float ox = __fsub_rn(mx[0], mn[0]), oy = __fsub_rn(mx[1], mn[1]), oz = __fsub_rn(mx[2], mn[2]);
    axis = (ox > oy && ox > oz) ? 0 : ((oy > ox && oy > oz) ? 1 : 2);
    start = mn[axis];
    delta = __fmul_rn(__fsub_rn(mx[axis], mn[axis]), 1.0f / float(kBins));
    if (delta == 0.0f) return false;
    inv = __fdiv_rn(1.0f, delta);
    return true;
}

// Bin counts and bin boxes (primitive boxes, slot order).
__global__ void __launch_bounds__(256) k_bin(int64_t n, const int* __restrict__ rid, const float* __restrict__ cx,
                                             const float* __restrict__ cy, const float* __restrict__ cz,
                                             const float* __restrict__ pb, RangeTask* __restrict__ rt) {
    __shared__ int sr;
    __shared__ unsigned scnt[kBins];
    __shared__ int sbox[kBins][6];
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int r = i < n ? rid[i] : -1;
    if (threadIdx.x < kBins) {
        scnt[threadIdx.x] = 0;
        empty_box(sbox[threadIdx.x]);
    }
    const bool one = block_in_one_range(r, sr);
    int axis = 0;
    float start = 0.0f, delta = 0.0f, inv = 0.0f;
    const bool binned = r >= 0 && bin_geometry(rt[r], axis, start, delta, inv);
    int b = 0;
    int v[6];
    if (binned) {
        const float c = axis == 0 ? cx[i] : (axis == 1 ? cy[i] : cz[i]);
        b = __float2int_rz(__fmul_rn(__fsub_rn(c, start), inv));
        b = max(0, min(b, kBins - 1));  // c >= start, so b >= 0 for finite input; the clamp guards the bins
        for (int a = 0; a < 6; ++a) v[a] = f2o(pb[a * n + i]);
    } else {
        empty_box(v);
    }
    const unsigned peers = group_minmax<3>(binned ? ((long long)r << 4) | b : -1, v);
    const bool lead = binned && leads(peers);
    if (one) {  // every thread of the block is in range r (binned or not, uniformly)
        if (lead) {
            atomicAdd(&scnt[b], (unsigned)__popc(peers));
            atomic_box(sbox[b], v);
        }
        __syncthreads();
        if (binned && threadIdx.x < kBins && scnt[threadIdx.x]) {
            const int k = threadIdx.x;
            atomicAdd(&rt[r].bin_cnt[k], scnt[k]);
            for (int a = 0; a < 3; ++a) {
                atomicMin(&rt[r].bin_box[k][a], sbox[k][a]);
                atomicMax(&rt[r].bin_box[k][3 + a], sbox[k][3 + a]);
            }
        }
        return;
    }
    if (!lead) return;
    atomicAdd(&rt[r].bin_cnt[b], (unsigned)__popc(peers));
    atomic_box(rt[r].bin_box[b], v);
}

// The SAH sweep of pick_best_split and splitNode's decision, one thread per range.
__global__ void k_sweep(const BuildState* __restrict__ bs, RangeTask* __restrict__ rt, int max_leaf) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= bs->na) return;
    RangeTask& t = rt[r];
    const unsigned n = (unsigned)(t.e - t.s);
    t.split = 0;
    int axis;
    float start, delta, inv;
    float min_sah = FLT_MAX, split_pos = 0.0f;
    if (bin_geometry(t, axis, start, delta, inv)) {
        float bmn[kBins][3], bmx[kBins][3];
        for (int b = 0; b < kBins; ++b)
            for (int a = 0; a < 3; ++a) {
                bmn[b][a] = o2f(t.bin_box[b][a]);
                bmx[b][a] = o2f(t.bin_box[b][3 + a]);
            }
        // right boxes: rbox[i] = union of bins i+1 .. 15 (BBox::Union order is immaterial to the values)
        float rmn[kBins - 1][3], rmx[kBins - 1][3];
        for (int a = 0; a < 3; ++a) {
            rmn[kBins - 2][a] = bmn[kBins - 1][a];
            rmx[kBins - 2][a] = bmx[kBins - 1][a];
        }
        for (int i = kBins - 3; i >= 0; --i)
            for (int a = 0; a < 3; ++a) {
                rmn[i][a] = fminf(rmn[i + 1][a], bmn[i + 1][a]);
                rmx[i][a] = fmaxf(rmx[i + 1][a], bmx[i + 1][a]);
            }
        unsigned left = t.bin_cnt[0];
        float lmn[3] = {bmn[0][0], bmn[0][1], bmn[0][2]}, lmx[3] = {bmx[0][0], bmx[0][1], bmx[0][2]};
        float pos = __fadd_rn(delta, start);
        for (int i = 0; i < kBins - 1; ++i) {
            const float l = __fmul_rn(__uint2float_rn(left), half_area(lmn, lmx));
            const float rr = __fmul_rn(__uint2float_rn(n - left), half_area(rmn[i], rmx[i]));
            const float sah = __fdiv_rn(__fadd_rn(l, rr), t.node_area);
            if (sah < min_sah) {
                min_sah = sah;
                split_pos = pos;
            }
            left += t.bin_cnt[i + 1];
            for (int a = 0; a < 3; ++a) {
                lmn[a] = fminf(lmn[a], bmn[i + 1][a]);
                lmx[a] = fmaxf(lmx[a], bmx[i + 1][a]);
            }
            pos = __fadd_rn(pos, delta);
        }
    }
    t.axis = axis;
    t.split_pos = split_pos;
    t.split = !(min_sah >= __uint2float_rn(n) || n <= (unsigned)max_leaf);
    t.left = 0;
}

__device__ __forceinline__ bool passes(const RangeTask& t, float x, float y, float z) {
    const float c = t.axis == 0 ? x : (t.axis == 1 ? y : z);
    return c < t.split_pos;
}

// Size and box of both halves of every range being split.
__global__ void __launch_bounds__(256) k_count_left(int64_t n, const int* __restrict__ rid,
                                                    const float* __restrict__ cx, const float* __restrict__ cy,
                                                    const float* __restrict__ cz, const float* __restrict__ pb,
                                                    RangeTask* __restrict__ rt) {
    __shared__ int sr;
    __shared__ unsigned sleft;
    __shared__ int sbox[2][6];
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int r = i < n ? rid[i] : -1;
    if (threadIdx.x == 0) {
        sleft = 0;
        empty_box(sbox[0]);
        empty_box(sbox[1]);
    }
    const bool one = block_in_one_range(r, sr);
    const bool act = r >= 0 && rt[r].split;
    bool pass = false;
    int v[6];
    if (act) {
        pass = passes(rt[r], cx[i], cy[i], cz[i]);
        for (int a = 0; a < 6; ++a) v[a] = f2o(pb[a * n + i]);
    } else {
        empty_box(v);
    }
    const unsigned peers = group_minmax<3>(act ? ((long long)r << 1) | (pass ? 0 : 1) : -1, v);
    const bool lead = act && leads(peers);
    const int side = pass ? 0 : 1;
    if (one) {  // `act` is uniform here
        if (lead) {
            if (pass) atomicAdd(&sleft, (unsigned)__popc(peers));
            atomic_box(sbox[side], v);
        }
        __syncthreads();
        if (act && threadIdx.x < 12) {
            const int h = threadIdx.x / 6, a = threadIdx.x % 6;
            if (a < 3)
                atomicMin(&rt[r].half_box[h][a], sbox[h][a]);
            else
                atomicMax(&rt[r].half_box[h][a], sbox[h][a]);
        }
        if (act && threadIdx.x == 0 && sleft) atomicAdd(&rt[r].left, sleft);
        return;
    }
    if (!lead) return;
    if (pass) atomicAdd(&rt[r].left, (unsigned)__popc(peers));
    atomic_box(rt[r].half_box[side], v);
}

// Misplaced elements: failing the predicate left of the cut (ml), passing it right of it (mr).
__global__ void k_misplaced(int64_t n, const int* __restrict__ rid, const float* __restrict__ cx,
                            const float* __restrict__ cy, const float* __restrict__ cz,
                            const RangeTask* __restrict__ rt, int* __restrict__ ml, int* __restrict__ mr) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int r = rid[i];
    int a = 0, b = 0;
    if (r >= 0 && rt[r].split) {
        const RangeTask& t = rt[r];
        const int64_t mid = t.s + t.left;
        const bool p = passes(t, cx[i], cy[i], cz[i]);
        a = (i < mid && !p) ? 1 : 0;
        b = (i >= mid && p) ? 1 : 0;
    }
    ml[i] = a;
    mr[i] = b;
}

// Pair k of a range: k-th misplaced from the left with k-th misplaced from the right.
__global__ void k_pairs(int64_t n, const int* __restrict__ rid, const RangeTask* __restrict__ rt,
                        const int* __restrict__ ml, const int* __restrict__ mr, const int* __restrict__ sl,
                        const int* __restrict__ sr, int64_t* __restrict__ pl, int64_t* __restrict__ pr) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int r = rid[i];
    if (r < 0 || !rt[r].split) return;
    const int64_t s = rt[r].s, e = rt[r].e;
    const int base = sl[s];  // pairs before this range (misplaced counts match per range)
    if (ml[i]) pl[base + (sl[i] - sl[s])] = i;
    if (mr[i]) {
        const int total = (e < n ? sr[e] : sr[n - 1] + mr[n - 1]) - sr[s];
        pr[base + (total - 1 - (sr[i] - sr[s]))] = i;
    }
}

template <class T>
__device__ __forceinline__ void swap_at(T* __restrict__ p, int64_t a, int64_t b) {
    const T t = p[a];
    p[a] = p[b];
    p[b] = t;
}

// One thread per pair; the pair count is the total of the left misplaced flags.
__global__ void k_swap(int64_t n, const int* __restrict__ sl, const int* __restrict__ ml,
                       const int64_t* __restrict__ pl, const int64_t* __restrict__ pr, float* __restrict__ cx,
                       float* __restrict__ cy, float* __restrict__ cz, float* __restrict__ pb,
                       int32_t* __restrict__ idx) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t pairs = int64_t(sl[n - 1]) + ml[n - 1];
    if (k >= pairs) return;
    const int64_t a = pl[k], b = pr[k];
    swap_at(cx, a, b);
    swap_at(cy, a, b);
    swap_at(cz, a, b);
    swap_at(idx, a, b);
    for (int q = 0; q < 6; ++q) swap_at(pb + q * n, a, b);
}

// A primitive range of a node under construction and the union of its primitive boxes.
struct DRange {
    int32_t s, e;
    float mn[3], mx[3];
};

// A node under construction: SORT's to_split list (fifo) and done list. The
// list holds at most W ranges at a time (fewer than W before a split, one
// more after it), so the fifo is a ring of 8 indexed by running counters.
struct DNode {
    int32_t id;  // shape index
    int32_t depth;
    float area;  // half_area of the node's box (SAH normaliser)
    int32_t head, tail, ndone;
    DRange fifo[8];
    DRange done[8];
};

// The tree before flattening: a node's children are consecutive shape ids.
struct DShape {
    int32_t off, cnt, first_kid, nkids;
    float mn[3], mx[3];  // box of the primitive range (the parent's child box)
};

__device__ __forceinline__ bool starts_node(const DRange& x, int depth, int max_leaf, int max_depth) {
    return (x.e - x.s) > max_leaf && depth != max_depth;  // else splitNode returns at once
}

__device__ __forceinline__ DRange make_range(int32_t s, int32_t e, const int (&img)[6]) {
    DRange x;
    x.s = s;
    x.e = e;
    for (int a = 0; a < 3; ++a) {
        x.mn[a] = o2f(img[a]);
        x.mx[a] = o2f(img[3 + a]);
    }
    return x;
}

// The front range of every node is split this round (range r belongs to node r).
__global__ void k_node_ranges(const BuildState* __restrict__ bs, const DNode* __restrict__ nodes,
                              RangeTask* __restrict__ rt, int64_t* __restrict__ starts, int64_t* __restrict__ ends) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= bs->na) return;
    const DNode& nd = nodes[r];
    const DRange& x = nd.fifo[nd.head & 7];
    RangeTask& t = rt[r];
    t.s = starts[r] = x.s;
    t.e = ends[r] = x.e;
    t.node_area = nd.area;
    empty_box(t.inner);
    for (int b = 0; b < kBins; ++b) {
        t.bin_cnt[b] = 0;
        empty_box(t.bin_box[b]);
    }
    t.axis = 0;
    t.split_pos = 0.0f;
    t.split = 0;
    t.left = 0;
    empty_box(t.half_box[0]);
    empty_box(t.half_box[1]);
}

// Applies the round's split to every node (SORT's loop body) and counts what
// the node hands to the next round: itself, or its children that are nodes.
__global__ void k_node_apply(BuildState* __restrict__ bs, DNode* __restrict__ nodes, const RangeTask* __restrict__ rt,
                             int W, int max_leaf, int max_depth, int* __restrict__ cnt_next,
                             int* __restrict__ cnt_shape) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= bs->na) return;
    DNode& nd = nodes[r];
    const RangeTask& t = rt[r];
    const DRange x = nd.fifo[nd.head & 7];
    const int32_t mid = x.s + int32_t(t.left);
    int head = nd.head + 1, tail = nd.tail, ndone = nd.ndone;
    if (!t.split || mid == x.s || mid == x.e) {
        nd.done[ndone++] = x;
    } else {
        nd.fifo[tail++ & 7] = make_range(x.s, mid, t.half_box[0]);
        nd.fifo[tail++ & 7] = make_range(mid, x.e, t.half_box[1]);
    }
    nd.head = head;
    nd.tail = tail;
    nd.ndone = ndone;
    const int total = (tail - head) + ndone;
    int next = 0, shapes = 0;
    if (head != tail && total < W) {
        next = 1;
    } else if (total == 1) {
        atomicMax(&bs->depth_max, nd.depth);
    } else {
        shapes = total;
        int kid_max = 0;
        for (int q = head; q < tail; ++q) {
            if (starts_node(nd.fifo[q & 7], nd.depth + 1, max_leaf, max_depth))
                ++next;
            else
                kid_max = nd.depth + 1;
        }
        for (int q = 0; q < ndone; ++q) {
            if (starts_node(nd.done[q], nd.depth + 1, max_leaf, max_depth))
                ++next;
            else
                kid_max = nd.depth + 1;
        }
        if (kid_max) atomicMax(&bs->depth_max, kid_max);
    }
    cnt_next[r] = next;
    cnt_shape[r] = shapes;
}

__global__ void k_summary(BuildState* __restrict__ bs, const int* __restrict__ cnt_next,
                          const int* __restrict__ off_next, const int* __restrict__ cnt_shape,
                          const int* __restrict__ off_shape) {
    const int na = bs->na;
    bs->next = na > 0 ? off_next[na - 1] + cnt_next[na - 1] : 0;
    bs->new_shapes = na > 0 ? off_shape[na - 1] + cnt_shape[na - 1] : 0;
}

// Finished nodes write their children (SORT's child order: the remaining list,
// then the done list) as shape nodes; the next round's nodes are the
// continuing ones and the new children, in primitive-range order.
__global__ void k_node_commit(const BuildState* __restrict__ bs, const DNode* __restrict__ cur,
                              const int* __restrict__ off_next, const int* __restrict__ off_shape,
                              const int* __restrict__ cnt_shape, int W, int max_leaf, int max_depth,
                              DShape* __restrict__ shapes, DNode* __restrict__ next) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= bs->na) return;
    const DNode& nd = cur[r];
    const int total = (nd.tail - nd.head) + nd.ndone;
    int o = off_next[r];
    if (nd.head != nd.tail && total < W) {
        next[o] = nd;
        return;
    }
    const int m = cnt_shape[r];
    if (m == 0) return;  // a single range: the node is a leaf
    const int first = bs->shapes + off_shape[r];
    shapes[nd.id].first_kid = first;
    shapes[nd.id].nkids = m;
    DRange ks[8];
    int k = 0;
    for (int q = nd.head; q < nd.tail; ++q) ks[k++] = nd.fifo[q & 7];
    for (int q = 0; q < nd.ndone; ++q) ks[k++] = nd.done[q];
    int ord[8];
    for (int q = 0; q < m; ++q) {
        DShape& sh = shapes[first + q];
        sh.off = ks[q].s;
        sh.cnt = ks[q].e - ks[q].s;
        sh.first_kid = -1;
        sh.nkids = 0;
        for (int a = 0; a < 3; ++a) {
            sh.mn[a] = ks[q].mn[a];
            sh.mx[a] = ks[q].mx[a];
        }
        int j = q;  // insertion by range start
        while (j > 0 && ks[ord[j - 1]].s > ks[q].s) {
            ord[j] = ord[j - 1];
            --j;
        }
        ord[j] = q;
    }
    const int depth = nd.depth + 1;
    for (int j = 0; j < m; ++j) {
        const DRange& x = ks[ord[j]];
        if (!starts_node(x, depth, max_leaf, max_depth)) continue;
        DNode& c = next[o++];
        c.id = first + ord[j];
        c.depth = depth;
        c.area = half_area(x.mn, x.mx);
        c.head = 0;
        c.tail = 1;
        c.ndone = 0;
        c.fifo[0] = x;
    }
}

// Interior node k of the flattened tree in the device layout (layout.h, FP32
// boxes), from its shape: children in shape order, a leaf child as its first
// leaf slot, an interior child as base[k] plus its rank among the interior
// children (the host's numbering), empty slots with SORT's empty box.
template <int W>
__global__ void k_write_nodes(int64_t nodes, const DShape* __restrict__ shapes, const int32_t* __restrict__ shape_of,
                              const int32_t* __restrict__ base, float4* __restrict__ out) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nodes) return;
    constexpr int Q = W / 4;
    constexpr int F4 = W == 8 ? NodeShape<8>::kF4 : NodeShape<4>::kF4;
    const DShape sn = shapes[shape_of[k]];
    float* node = reinterpret_cast<float*>(out + k * F4);
    int32_t* ch = reinterpret_cast<int32_t*>(node + 6 * Q * 4);
    int inner = 0;
    for (int j = 0; j < W; ++j) {
        if (j >= sn.nkids) {
            for (int a = 0; a < 3; ++a) {
                node[(2 * a) * Q * 4 + j] = FLT_MAX;
                node[(2 * a + 1) * Q * 4 + j] = -FLT_MAX;
            }
            ch[j] = kEmptyRef;
            continue;
        }
        const DShape kid = shapes[sn.first_kid + j];
        for (int a = 0; a < 3; ++a) {
            node[(2 * a) * Q * 4 + j] = kid.mn[a];
            node[(2 * a + 1) * Q * 4 + j] = kid.mx[a];
        }
        ch[j] = kid.nkids == 0 ? int32_t(uint32_t(kid.off) | 0x80000000u) : base[k] + inner++;
    }
    if (W == 4)  // the layout's padding
        for (int x = 28; x < 32; ++x) node[x] = 0.0f;
}

// The last-in-leaf flag of every leaf shape's last slot (flags zeroed first).
__global__ void k_leaf_flags(int shapes, const DShape* __restrict__ shape, uint8_t* __restrict__ last) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= shapes) return;
    const DShape sn = shape[i];
    if (sn.nkids == 0) last[sn.off + sn.cnt - 1] = 1;
}

__global__ void k_advance(BuildState* __restrict__ bs) {
    if (bs->na > 0) ++bs->rounds;
    bs->shapes += bs->new_shapes;
    bs->na = bs->next;
    bs->next = bs->new_shapes = 0;
}

}  // namespace

BuiltTree build_tree_gpu(const float* tri, int64_t ntri, const BuildParams& p, int device) {
    if (p.width != 4 && p.width != 8) throw std::invalid_argument("width must be 4 or 8");
    if (p.max_leaf < 1 || p.max_depth < 1) throw std::invalid_argument("max_leaf and max_depth must be >= 1");
    if (ntri < 0 || ntri >= int64_t(0x7fffffff)) throw std::invalid_argument("triangle count out of range");
    const int W = p.width;
    if (p.nextra < 0 || (p.nextra > 0 && !p.extra_boxes)) throw std::invalid_argument("bad extra primitive boxes");
    const int64_t nt = ntri;           // triangles
    const int64_t n = ntri + p.nextra;  // every primitive
    if (n >= int64_t(0x7fffffff)) throw std::invalid_argument("primitive count out of range");
    BuiltTree t;
    t.width = W;
    int prev = -1;
    cudaGetDevice(&prev);
    check(cudaSetDevice(device), "cudaSetDevice");
    struct Restore {
        int d;
        ~Restore() {
            if (d >= 0) cudaSetDevice(d);
        }
    } restore{prev};
    Stream stream;
    const cudaStream_t st = stream.s;
    ScratchScope scope(scratch_pool(device), st);  // declared before every DevBuf: outlives them

    DevBuf<float> d_tri, d_cx, d_cy, d_cz, d_pb;
    DevBuf<int32_t> d_idx;
    DevBuf<int> d_rid, d_ml, d_mr, d_sl, d_sr, d_scene;
    DevBuf<int64_t> d_pl, d_pr, d_starts, d_ends;
    DevBuf<RangeTask> d_rt;
    DevBuf<DNode> d_cur, d_next;
    DevBuf<DShape> d_shapes;
    DevBuf<int> d_cnt_next, d_off_next, d_cnt_shape, d_off_shape;
    DevBuf<BuildState> d_state;
    DevBuf<unsigned char> d_temp;
    PinnedBuf<int> h_scene;
    PinnedBuf<BuildState> h_state;
    const int64_t nn = std::max<int64_t>(n, 1);
    d_tri.alloc(size_t(std::max<int64_t>(nt, 1)) * 9);
    DevBuf<float> d_extra;
    d_cx.alloc(size_t(nn));
    d_cy.alloc(size_t(nn));
    d_cz.alloc(size_t(nn));
    d_pb.alloc(size_t(nn) * 6);
    d_idx.alloc(size_t(nn));
    d_rid.alloc(size_t(nn));
    d_ml.alloc(size_t(nn));
    d_mr.alloc(size_t(nn));
    d_sl.alloc(size_t(nn));
    d_sr.alloc(size_t(nn));
    d_pl.alloc(size_t(nn));
    d_pr.alloc(size_t(nn));
    d_scene.alloc(6);
    d_state.alloc(1);
    h_scene.alloc(6);
    h_state.alloc(1);

    // Scene box (core/scene.cpp:146-154): union of the primitive boxes, enlarged by 0.1%.
    Box scene;
    {
        empty_box(h_scene.p);
        if (n > 0) {
            if (nt > 0) {
                check(upload_host(d_tri.p, tri, size_t(nt) * 9 * sizeof(float), st), "upload");
                k_prim_setup<<<grid(nt), 256, 0, st>>>(d_tri.p, nt, n, d_cx.p, d_cy.p, d_cz.p, d_idx.p, d_pb.p);
            }
            if (p.nextra > 0) {
                d_extra.alloc(size_t(p.nextra) * 6);
                check(cudaMemcpyAsync(d_extra.p, p.extra_boxes, size_t(p.nextra) * 6 * sizeof(float),
                                      cudaMemcpyHostToDevice, st),
                      "upload boxes");
                k_box_setup<<<grid(p.nextra), 256, 0, st>>>(d_extra.p, nt, p.nextra, n, d_cx.p, d_cy.p, d_cz.p,
                                                            d_idx.p, d_pb.p);
            }
            check(cudaMemcpyAsync(d_scene.p, h_scene.p, 6 * sizeof(int), cudaMemcpyHostToDevice, st), "scene box");
            k_scene_box<<<std::min<unsigned>(grid(n), 148 * 8), 256, 0, st>>>(n, d_pb.p, d_scene.p);
            check(cudaGetLastError(), "primitive setup");
            check(cudaMemcpyAsync(h_scene.p, d_scene.p, 6 * sizeof(int), cudaMemcpyDeviceToHost, st), "scene box");
            check(cudaStreamSynchronize(st), "primitive setup");
        }
        scene = box_from_images(h_scene.p);
        const float threshold = 0.001f;
        float delta[3];
        for (int k = 0; k < 3; ++k) delta[k] = (scene.mx[k] - scene.mn[k]) * threshold;
        for (int k = 0; k < 3; ++k) {
            scene.mn[k] -= delta[k];
            scene.mx[k] += delta[k];
        }
    }
    t.scene = scene;
    if (p.nextra > 0) t.first_extra = nt;
    if (n == 0) return t;

    // Node-sized buffers at their bounds: nodes under construction own disjoint
    // ranges of more than max_leaf primitives; the tree has fewer than 2n nodes.
    const int64_t cap = std::min<int64_t>(n, n / (int64_t(p.max_leaf) + 1) + 1);
    d_cur.alloc(size_t(cap));
    d_next.alloc(size_t(cap));
    d_rt.alloc(size_t(cap));
    d_starts.alloc(size_t(cap));
    d_ends.alloc(size_t(cap));
    d_cnt_next.alloc(size_t(cap));
    d_off_next.alloc(size_t(cap));
    d_cnt_shape.alloc(size_t(cap));
    d_off_shape.alloc(size_t(cap));
    d_shapes.alloc(size_t(2 * n));
    // The node prefix sums run over all cap entries: the ones past a round's
    // node count must hold small values (zero, or counts of earlier rounds).
    check(cudaMemsetAsync(d_cnt_next.p, 0, size_t(cap) * sizeof(int), st), "clear counts");
    check(cudaMemsetAsync(d_cnt_shape.p, 0, size_t(cap) * sizeof(int), st), "clear counts");

    // Scan scratch for the prefix sums over primitives and over nodes.
    const size_t scan_words = std::max(psort::scan_scratch_words(size_t(n)), psort::scan_scratch_words(size_t(cap)));
    d_temp.alloc(scan_words * sizeof(uint32_t));
    uint32_t* scan_tmp = reinterpret_cast<uint32_t*>(d_temp.p);
    auto scan = [&](const int* in, int* out, int64_t count) {
        check(psort::scan_exclusive(reinterpret_cast<const uint32_t*>(in), reinterpret_cast<uint32_t*>(out),
                                    size_t(count), scan_tmp, st),
              "scan");
    };

    // The root shape, and the root node unless splitNode returns at once.
    {
        DShape root{0, int32_t(n), -1, 0, {scene.mn[0], scene.mn[1], scene.mn[2]},
                    {scene.mx[0], scene.mx[1], scene.mx[2]}};
        check(cudaMemcpyAsync(d_shapes.p, &root, sizeof(root), cudaMemcpyHostToDevice, st), "root");
    }
    const bool root_node = n > p.max_leaf && p.max_depth != 1;
    *h_state.p = BuildState{root_node ? 1 : 0, 1, root_node ? 0 : 1, 0, 0, 0};
    check(cudaMemcpyAsync(d_state.p, h_state.p, sizeof(BuildState), cudaMemcpyHostToDevice, st), "state");
    if (root_node) {
        DNode root{};
        root.id = 0;
        root.depth = 1;
        root.area = host_half_area(scene);
        root.tail = 1;
        root.fifo[0] = DRange{0, int32_t(n), {scene.mn[0], scene.mn[1], scene.mn[2]},
                              {scene.mx[0], scene.mx[1], scene.mx[2]}};
        check(cudaMemcpyAsync(d_cur.p, &root, sizeof(root), cudaMemcpyHostToDevice, st), "root");
    }
    check(cudaStreamSynchronize(st), "root");

    // Rounds are queued in groups without a host round trip (a round with no
    // node left does no work); the host reads the state after each group. A
    // node splits at most W - 1 times and the depth is capped, which bounds
    // the rounds.
    constexpr int kGroup = 8;
    const int64_t max_rounds = int64_t(W - 1) * p.max_depth + 1;
    const unsigned ng = grid(cap, 128);
    int64_t queued = 0;
    while (root_node) {
        for (int g = 0; g < kGroup; ++g) {
            k_node_ranges<<<ng, 128, 0, st>>>(d_state.p, d_cur.p, d_rt.p, d_starts.p, d_ends.p);
            k_bounds<<<grid(n), 256, 0, st>>>(n, d_starts.p, d_ends.p, d_state.p, d_cx.p, d_cy.p, d_cz.p, d_rid.p,
                                              d_rt.p);
            k_bin<<<grid(n), 256, 0, st>>>(n, d_rid.p, d_cx.p, d_cy.p, d_cz.p, d_pb.p, d_rt.p);
            k_sweep<<<ng, 128, 0, st>>>(d_state.p, d_rt.p, p.max_leaf);
            k_count_left<<<grid(n), 256, 0, st>>>(n, d_rid.p, d_cx.p, d_cy.p, d_cz.p, d_pb.p, d_rt.p);
            k_misplaced<<<grid(n), 256, 0, st>>>(n, d_rid.p, d_cx.p, d_cy.p, d_cz.p, d_rt.p, d_ml.p, d_mr.p);
            check(cudaGetLastError(), "split kernels");
            scan(d_ml.p, d_sl.p, n);
            scan(d_mr.p, d_sr.p, n);
            k_pairs<<<grid(n), 256, 0, st>>>(n, d_rid.p, d_rt.p, d_ml.p, d_mr.p, d_sl.p, d_sr.p, d_pl.p, d_pr.p);
            k_swap<<<grid((n + 1) / 2), 256, 0, st>>>(n, d_sl.p, d_ml.p, d_pl.p, d_pr.p, d_cx.p, d_cy.p, d_cz.p,
                                                      d_pb.p, d_idx.p);
            k_node_apply<<<ng, 128, 0, st>>>(d_state.p, d_cur.p, d_rt.p, W, p.max_leaf, p.max_depth, d_cnt_next.p,
                                             d_cnt_shape.p);
            check(cudaGetLastError(), "partition kernels");
            scan(d_cnt_next.p, d_off_next.p, cap);
            scan(d_cnt_shape.p, d_off_shape.p, cap);
            k_summary<<<1, 1, 0, st>>>(d_state.p, d_cnt_next.p, d_off_next.p, d_cnt_shape.p, d_off_shape.p);
            k_node_commit<<<ng, 128, 0, st>>>(d_state.p, d_cur.p, d_off_next.p, d_off_shape.p, d_cnt_shape.p, W,
                                              p.max_leaf, p.max_depth, d_shapes.p, d_next.p);
            k_advance<<<1, 1, 0, st>>>(d_state.p);
            check(cudaGetLastError(), "node commit");
            swap_bufs(d_cur, d_next);
        }
        queued += kGroup;
        check(cudaMemcpyAsync(h_state.p, d_state.p, sizeof(BuildState), cudaMemcpyDeviceToHost, st), "state");
        check(cudaStreamSynchronize(st), "split rounds");
        if (h_state.p->na == 0) break;
        if (queued > max_rounds) throw std::runtime_error("GPU build: the split rounds did not finish");
    }
    const BuildState fin = *h_state.p;
    const int shape_count = fin.shapes;
    t.depth = fin.depth_max;

    // Shapes and the final permutation (leaf order) to the host, through the
    // device's pinned staging memory (pageable copies of these 130 MB cost
    // about 100 ms).
    Staging& stage = staging(device);
    std::lock_guard<std::mutex> stage_lock(stage.lock);
    // Host arrays (child references, leaf order and flags) only where the scene
    // reads them: 8-bit nodes and mixed primitives. A triangle scene with FP32
    // nodes takes its nodes and records from the device (its topology export
    // reads them back from there).
    const bool host = p.host_boxes || p.nextra > 0;
    const size_t shape_bytes = (size_t(shape_count) * sizeof(DShape) + 255) & ~size_t(255);
    const size_t stage_bytes = shape_bytes + (host ? size_t(n) * 4 : 0);
    if (stage.bytes < stage_bytes) {
        if (stage.p) cudaFreeHost(stage.p);
        stage.p = nullptr;
        stage.bytes = 0;
        check(cudaMallocHost(&stage.p, stage_bytes), "cudaMallocHost(staging)");
        stage.bytes = stage_bytes;
    }
    const DShape* shape = static_cast<const DShape*>(stage.p);
    const int32_t* h_order = reinterpret_cast<const int32_t*>(static_cast<const char*>(stage.p) + shape_bytes);
    check(cudaMemcpyAsync(stage.p, d_shapes.p, size_t(shape_count) * sizeof(DShape), cudaMemcpyDeviceToHost, st),
          "shapes");
    if (host)
        check(cudaMemcpyAsync(const_cast<int32_t*>(h_order), d_idx.p, size_t(n) * 4, cudaMemcpyDeviceToHost, st),
              "order");
    check(cudaStreamSynchronize(st), "download");
    if (host) {
        t.order.assign(h_order, h_order + n);
        t.leaf_last.assign(size_t(n), 0);
    }
    // Flatten exactly as build_tree numbers nodes: a node allocates its interior
    // children consecutively when it is filled, then fills them in order. The
    // arrays are sized once (the interior count is known), then filled.
    size_t interior_total = 0;
    for (int s_ = 0; s_ < shape_count; ++s_) interior_total += shape[s_].nkids ? 1 : 0;
    if (host) {
        t.first_interior.assign(interior_total, -1);
        t.child.assign(interior_total * W, kEmptyRef);
    } else {
        t.n_interior = int64_t(interior_total);
        t.n_tri = n;
    }
    if (p.host_boxes) {  // only a scene with 8-bit nodes reads the boxes on the host
        t.lo.assign(interior_total * 3 * W, FLT_MAX);
        t.hi.assign(interior_total * 3 * W, -FLT_MAX);
    }
    std::vector<int32_t> shape_of(interior_total);  // the shape each interior node came from
    std::vector<int32_t> base_of(interior_total);   // and its first interior child
    int32_t allocated = 0;
    auto leaf = [&](const DShape& sn) {
        t.leaves++;
        if (host) t.leaf_last[size_t(sn.off + sn.cnt - 1)] = 1;
    };
    std::vector<std::pair<int, int32_t>> stack;  // (shape id, node index), filled depth-first in order
    stack.reserve(64 * 8);
    if (shape[0].nkids == 0) {
        t.root = leaf_ref(0);
        leaf(shape[0]);
    } else {
        t.root = allocated++;
        stack.push_back({0, t.root});
    }
    while (!stack.empty()) {
        const auto [sid, idx] = stack.back();
        stack.pop_back();
        const DShape& sn = shape[sid];
        shape_of[size_t(idx)] = sid;
        int interior = 0;
        for (int j = 0; j < sn.nkids; ++j) interior += shape[sn.first_kid + j].nkids ? 1 : 0;
        const int32_t base = interior ? allocated : -1;
        allocated += interior;
        base_of[size_t(idx)] = base;
        if (host) t.first_interior[size_t(idx)] = base;
        int k = 0;
        std::pair<int, int32_t> sub[8];
        int nsub = 0;
        for (int j = 0; j < sn.nkids; ++j) {
            const int kid_id = sn.first_kid + j;
            const DShape& kid = shape[kid_id];
            int32_t ref;
            if (kid.nkids == 0) {
                ref = leaf_ref(kid.off);
                leaf(kid);
            } else {
                ref = base + k++;
                sub[nsub++] = {kid_id, ref};
            }
            if (host) t.child[size_t(idx) * W + j] = ref;
            if (p.host_boxes)
                for (int a = 0; a < 3; ++a) {
                    t.lo[(size_t(idx) * 3 + a) * W + j] = kid.mn[a];
                    t.hi[(size_t(idx) * 3 + a) * W + j] = kid.mx[a];
                }
        }
        for (int q = nsub - 1; q >= 0; --q) stack.push_back(sub[q]);  // first child filled next
    }

    // The interior nodes in the device layout, written where the shapes are
    // (FP32 boxes; a scene with 8-bit nodes converts the host arrays instead).
    // Owned here until the tree is returned.
    struct Owned {
        float4* p = nullptr;
        ~Owned() {
            if (p) cudaFree(p);
        }
    } nodes_owned;
    if (interior_total > 0) {
        DevBuf<int32_t> d_map;
        d_map.alloc(2 * interior_total);
        check(upload_host(d_map.p, shape_of.data(), interior_total * 4, st), "node map");
        check(upload_host(d_map.p + interior_total, base_of.data(), interior_total * 4, st), "node map");
        const int F4 = W == 8 ? NodeShape<8>::kF4 : NodeShape<4>::kF4;
        check(cudaMalloc(&nodes_owned.p, interior_total * F4 * sizeof(float4)), "cudaMalloc(nodes)");
        if (W == 8)
            k_write_nodes<8><<<grid(int64_t(interior_total)), 256, 0, st>>>(
                int64_t(interior_total), d_shapes.p, d_map.p, d_map.p + interior_total, nodes_owned.p);
        else
            k_write_nodes<4><<<grid(int64_t(interior_total)), 256, 0, st>>>(
                int64_t(interior_total), d_shapes.p, d_map.p, d_map.p + interior_total, nodes_owned.p);
        check(cudaGetLastError(), "write nodes");
        check(cudaStreamSynchronize(st), "write nodes");
    }

    // This file's kernels: setup and scene box, 13 per queued round, the node
    // writer, the triangle records (the prefix sums are counted apart, four per round).
    t.rounds = int(fin.rounds);
    t.launches = int(4 + 13 * queued + (host ? 0 : 1));
    if (p.nextra > 0) {  // mixed primitives: the scene writes its slot records on the host
        t.d_nodes = nodes_owned.p;
        nodes_owned.p = nullptr;
        return t;
    }
    // The triangle records in leaf order, built where the triangles already are.
    uint8_t* d_last = reinterpret_cast<uint8_t*>(d_rid.p);  // n bytes fit in the n-int buffer
    if (host) {
        check(cudaMemcpyAsync(d_last, t.leaf_last.data(), size_t(n), cudaMemcpyHostToDevice, st), "leaf flags");
    } else {
        check(cudaMemsetAsync(d_last, 0, size_t(n), st), "leaf flags");
        k_leaf_flags<<<grid(shape_count), 256, 0, st>>>(shape_count, d_shapes.p, d_last);
        check(cudaGetLastError(), "leaf flags");
    }
    const size_t tris_bytes = size_t(n + kPadSlots) * 3 * sizeof(float4);
    float4* d_tris = nullptr;
    check(cudaMalloc(&d_tris, tris_bytes), "cudaMalloc(triangles)");
    cudaError_t e = cudaMemsetAsync(d_tris + size_t(n) * 3, 0, size_t(kPadSlots) * 3 * sizeof(float4), st);
    if (e == cudaSuccess) {
        k_leaf_tris<<<grid(n), 256, 0, st>>>(n, d_tri.p, d_idx.p, d_last, d_tris);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        cudaFree(d_tris);
        check(e, "triangle records");
    }
    t.d_tris = d_tris;
    t.d_nodes = nodes_owned.p;
    nodes_owned.p = nullptr;
    return t;
}

}  // namespace sg
