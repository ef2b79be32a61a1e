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
//   * centroid bounds and bins (counts, primitive boxes) per range with
//     atomics on order-preserving integer images of the floats;
//   * the SAH sweep, one thread per range, in SORT's arithmetic order;
//   * std::partition as libstdc++ performs it on random-access iterators: the
//     k-th element of the left part that fails the predicate is swapped with
//     the k-th element from the right end of the right part that passes it,
//     so the result is found with two prefix sums and one swap per pair.
// The host keeps each node's range list and finishes a node when SORT's loop
// would; a finished node's ranges become its children, whose boxes (for their
// own SAH normalisation and for the stored child boxes) are reduced on the
// GPU. The tree, the leaf order and every box value are build_tree's; a box
// bound that is zero may carry the other sign, which no comparison sees.
#include <cuda_runtime.h>

#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cfloat>
#include <cstring>
#include <deque>
#include <stdexcept>
#include <string>
#include <vector>

#include "builder.h"

namespace sg {
namespace {

constexpr int kBins = 16;

// Order-preserving int image of a float (for atomicMin / atomicMax).
__host__ __device__ __forceinline__ int f2o(float f) {
    int i;
    std::memcpy(&i, &f, 4);
    return i >= 0 ? i : i ^ 0x7fffffff;
}
__host__ __device__ __forceinline__ float o2f(int i) {
    const int b = i >= 0 ? i : i ^ 0x7fffffff;
    float f;
    std::memcpy(&f, &b, 4);
    return f;
}

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
    int split;       // 1 = partition this range
    unsigned left;   // primitives passing the predicate
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

__global__ void k_prim_setup(const float* __restrict__ tri, int64_t n, float* __restrict__ cx, float* __restrict__ cy,
                             float* __restrict__ cz, int32_t* __restrict__ idx, float* __restrict__ pb) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, mx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int k = 0; k < 3; ++k)  // BBox::Union(const Point&) per vertex (math/bbox.cpp:106-113)
        for (int a = 0; a < 3; ++a) {
            const float p = tri[i * 9 + 3 * k + a];
            if (p < mn[a]) mn[a] = p;
            if (p > mx[a]) mx[a] = p;
        }
    for (int a = 0; a < 3; ++a) {
        pb[a * n + i] = mn[a];
        pb[(3 + a) * n + i] = mx[a];
    }
    cx[i] = __fmul_rn(__fadd_rn(mx[0], mn[0]), 0.5f);
    cy[i] = __fmul_rn(__fadd_rn(mx[1], mn[1]), 0.5f);
    cz[i] = __fmul_rn(__fadd_rn(mx[2], mn[2]), 0.5f);
    idx[i] = (int32_t)i;
}

// Range id of every primitive (-1 outside the round's ranges) and centroid bounds.
__global__ void k_bounds(int64_t n, const int64_t* __restrict__ starts, const int64_t* __restrict__ ends, int nr,
                         const float* __restrict__ cx, const float* __restrict__ cy, const float* __restrict__ cz,
                         int* __restrict__ rid, RangeTask* __restrict__ rt) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int r = find_range(starts, ends, nr, i);
    rid[i] = r;
    if (r < 0) return;
    const float c[3] = {cx[i], cy[i], cz[i]};
    for (int a = 0; a < 3; ++a) {
        atomicMin(&rt[r].inner[a], f2o(c[a]));
        atomicMax(&rt[r].inner[3 + a], f2o(c[a]));
    }
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

__global__ void k_bin(int64_t n, const int* __restrict__ rid, const float* __restrict__ cx, const float* __restrict__ cy,
                      const float* __restrict__ cz, const int32_t* __restrict__ idx, const float* __restrict__ pb,
                      int64_t np, RangeTask* __restrict__ rt) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int r = rid[i];
    if (r < 0) return;
    int axis;
    float start, delta, inv;
    if (!bin_geometry(rt[r], axis, start, delta, inv)) return;
    const float c = axis == 0 ? cx[i] : (axis == 1 ? cy[i] : cz[i]);
    int b = __float2int_rz(__fmul_rn(__fsub_rn(c, start), inv));
    b = max(0, min(b, kBins - 1));  // c >= start, so b >= 0 for finite input; the clamp guards the bins
    atomicAdd(&rt[r].bin_cnt[b], 1u);
    const int32_t p = idx[i];
    for (int a = 0; a < 6; ++a) {
        const int v = f2o(pb[a * np + p]);
        if (a < 3)
            atomicMin(&rt[r].bin_box[b][a], v);
        else
            atomicMax(&rt[r].bin_box[b][a], v);
    }
}

// The SAH sweep of pick_best_split and splitNode's decision, one thread per range.
__global__ void k_sweep(int nr, RangeTask* __restrict__ rt, int max_leaf) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nr) return;
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

__global__ void k_count_left(int64_t n, const int* __restrict__ rid, const float* __restrict__ cx,
                             const float* __restrict__ cy, const float* __restrict__ cz, RangeTask* __restrict__ rt) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int r = rid[i];
    if (r < 0 || !rt[r].split) return;
    if (passes(rt[r], cx[i], cy[i], cz[i])) atomicAdd(&rt[r].left, 1u);
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

__global__ void k_swap(int64_t pairs, const int64_t* __restrict__ pl, const int64_t* __restrict__ pr,
                       float* __restrict__ cx, float* __restrict__ cy, float* __restrict__ cz,
                       int32_t* __restrict__ idx) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= pairs) return;
    const int64_t a = pl[k], b = pr[k];
    float t = cx[a];
    cx[a] = cx[b];
    cx[b] = t;
    t = cy[a];
    cy[a] = cy[b];
    cy[b] = t;
    t = cz[a];
    cz[a] = cz[b];
    cz[b] = t;
    const int32_t q = idx[a];
    idx[a] = idx[b];
    idx[b] = q;
}

// Boxes of ranges (children of finished nodes): union of primitive boxes.
__global__ void k_range_boxes(int64_t n, const int64_t* __restrict__ starts, const int64_t* __restrict__ ends, int nr,
                              const int32_t* __restrict__ idx, const float* __restrict__ pb, int64_t np,
                              int* __restrict__ boxes) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int r = find_range(starts, ends, nr, i);
    if (r < 0) return;
    const int32_t p = idx[i];
    for (int a = 0; a < 3; ++a) {
        atomicMin(&boxes[6 * r + a], f2o(pb[a * np + p]));
        atomicMax(&boxes[6 * r + 3 + a], f2o(pb[(3 + a) * np + p]));
    }
}

void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string("GPU build: ") + what + ": " + cudaGetErrorString(e));
}

template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    void alloc(size_t count) {
        if (count <= n) return;
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        check(cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)), "cudaMalloc");
        n = count;
    }
    ~DevBuf() {
        if (p) cudaFree(p);
    }
};

// Compact per-range input (host -> device) and decision (device -> host).
struct RangeIn {
    int64_t s, e;
    float area;
    int pad;
};
struct RangeOut {
    int split;
    unsigned left;
};

__global__ void k_range_init(int nr, const RangeIn* __restrict__ in, RangeTask* __restrict__ rt) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nr) return;
    RangeTask& t = rt[r];
    t.s = in[r].s;
    t.e = in[r].e;
    t.node_area = in[r].area;
    for (int a = 0; a < 3; ++a) {
        t.inner[a] = f2o(FLT_MAX);
        t.inner[3 + a] = f2o(-FLT_MAX);
    }
    for (int b = 0; b < kBins; ++b) {
        t.bin_cnt[b] = 0;
        for (int a = 0; a < 3; ++a) {
            t.bin_box[b][a] = f2o(FLT_MAX);
            t.bin_box[b][3 + a] = f2o(-FLT_MAX);
        }
    }
    t.axis = 0;
    t.split_pos = 0.0f;
    t.split = 0;
    t.left = 0;
}

__global__ void k_range_out(int nr, const RangeTask* __restrict__ rt, RangeOut* __restrict__ out) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nr) return;
    out[r].split = rt[r].split;
    out[r].left = rt[r].left;
}

struct Range {
    int64_t s, e;
};

// A node under construction: SORT's to_split list (fifo) and done list.
struct NodeTask {
    int id;  // index into the shape array
    int depth;
    float area;
    int head = 0, tail = 0, ndone = 0;
    Range fifo[16];  // 1 + 2 * (W - 1) entries at most
    Range done[8];
    int total() const { return (tail - head) + ndone; }
};

struct ShapeNode {
    int64_t off = 0, cnt = 0;
    int nkids = 0;
    int kid[8];
    Box kid_box[8];
};

unsigned grid(int64_t n, int t = 256) { return (unsigned)std::max<int64_t>(1, (n + t - 1) / t); }

Box box_from_images(const int* o) {
    Box b;
    for (int a = 0; a < 3; ++a) {
        b.mn[a] = o2f(o[a]);
        b.mx[a] = o2f(o[3 + a]);
    }
    return b;
}

float host_half_area(const Box& b) {
    const float ox = b.mx[0] - b.mn[0], oy = b.mx[1] - b.mn[1], oz = b.mx[2] - b.mn[2];
    const float a = ox * oy;
    const float c = oy * oz;
    const float e = oz * ox;
    return (a + c) + e;
}

}  // namespace

BuiltTree build_tree_gpu(const float* tri, int64_t ntri, const BuildParams& p, int device) {
    if (p.width != 4 && p.width != 8) throw std::invalid_argument("width must be 4 or 8");
    if (p.max_leaf < 1 || p.max_depth < 1) throw std::invalid_argument("max_leaf and max_depth must be >= 1");
    if (ntri < 0 || ntri >= int64_t(0x7fffffff)) throw std::invalid_argument("triangle count out of range");
    const int W = p.width;
    const int64_t n = ntri;
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

    DevBuf<float> d_tri, d_cx, d_cy, d_cz, d_pb;
    DevBuf<int32_t> d_idx;
    DevBuf<int> d_rid, d_ml, d_mr, d_sl, d_sr, d_boxes;
    DevBuf<int64_t> d_pl, d_pr, d_starts, d_ends;
    DevBuf<RangeTask> d_rt;
    DevBuf<RangeIn> d_in;
    DevBuf<RangeOut> d_out;
    DevBuf<unsigned char> d_temp;
    const int64_t nn = std::max<int64_t>(n, 1);
    d_tri.alloc(size_t(nn) * 9);
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
    if (n > 0) check(cudaMemcpy(d_tri.p, tri, size_t(n) * 9 * sizeof(float), cudaMemcpyHostToDevice), "upload");
    if (n > 0) k_prim_setup<<<grid(n), 256>>>(d_tri.p, n, d_cx.p, d_cy.p, d_cz.p, d_idx.p, d_pb.p);
    check(cudaGetLastError(), "primitive setup");

    // Scene box (core/scene.cpp:146-154): union of the primitive boxes, enlarged by 0.1%.
    std::vector<float> pb(size_t(nn) * 6);
    if (n > 0) check(cudaMemcpy(pb.data(), d_pb.p, size_t(n) * 6 * sizeof(float), cudaMemcpyDeviceToHost), "boxes");
    Box scene;
    for (int a = 0; a < 3; ++a) {
        scene.mn[a] = FLT_MAX;
        scene.mx[a] = -FLT_MAX;
    }
    for (int64_t i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) {
            const float lo = pb[size_t(a) * n + i], hi = pb[size_t(3 + a) * n + i];
            scene.mn[a] = (lo < scene.mn[a]) ? lo : scene.mn[a];
            scene.mx[a] = (scene.mx[a] < hi) ? hi : scene.mx[a];
        }
    {
        const float threshold = 0.001f;
        float delta[3];
        for (int k = 0; k < 3; ++k) delta[k] = (scene.mx[k] - scene.mn[k]) * threshold;
        for (int k = 0; k < 3; ++k) {
            scene.mn[k] -= delta[k];
            scene.mx[k] += delta[k];
        }
    }
    t.scene = scene;
    if (n == 0) return t;

    size_t temp_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, temp_bytes, d_ml.p, d_sl.p, (int)n);
    d_temp.alloc(temp_bytes);

    std::vector<ShapeNode> shape(1);
    shape[0].off = 0;
    shape[0].cnt = n;
    int depth_max = 0;
    // Nodes under construction, in order of their primitive ranges (disjoint), so
    // the ranges split in a round come out sorted for the per-primitive lookup.
    std::vector<NodeTask> active, next;
    auto start_node = [&](std::vector<NodeTask>& into, int id, int depth, const Box& box) {
        const ShapeNode& sn = shape[size_t(id)];
        if (sn.cnt <= p.max_leaf || depth == p.max_depth) {  // splitNode's early return
            depth_max = std::max(depth_max, depth);
            return;
        }
        NodeTask nt;
        nt.id = id;
        nt.depth = depth;
        nt.area = host_half_area(box);
        nt.fifo[nt.tail++] = {sn.off, sn.off + sn.cnt};
        into.push_back(nt);
    };
    start_node(active, 0, 1, scene);

    std::vector<RangeIn> rin;
    std::vector<RangeOut> rout;
    std::vector<int> owner;
    std::vector<int64_t> starts, ends;
    while (!active.empty()) {
        // One split per node: the front of its list, while SORT's loop would go on.
        rin.clear();
        owner.clear();
        for (size_t k = 0; k < active.size(); ++k) {
            NodeTask& nt = active[k];
            if (nt.head == nt.tail || nt.total() >= W) continue;
            const Range r = nt.fifo[nt.head++];
            rin.push_back({r.s, r.e, nt.area, 0});
            owner.push_back(int(k));
        }
        const int nr = int(rin.size());
        if (nr > 0) {
            starts.resize(size_t(nr));
            ends.resize(size_t(nr));
            for (int k = 0; k < nr; ++k) {
                starts[size_t(k)] = rin[size_t(k)].s;
                ends[size_t(k)] = rin[size_t(k)].e;
            }
            d_rt.alloc(size_t(nr));
            d_in.alloc(size_t(nr));
            d_out.alloc(size_t(nr));
            d_starts.alloc(size_t(nr));
            d_ends.alloc(size_t(nr));
            check(cudaMemcpy(d_in.p, rin.data(), size_t(nr) * sizeof(RangeIn), cudaMemcpyHostToDevice), "ranges");
            check(cudaMemcpy(d_starts.p, starts.data(), size_t(nr) * 8, cudaMemcpyHostToDevice), "ranges");
            check(cudaMemcpy(d_ends.p, ends.data(), size_t(nr) * 8, cudaMemcpyHostToDevice), "ranges");
            k_range_init<<<grid(nr, 128), 128>>>(nr, d_in.p, d_rt.p);
            k_bounds<<<grid(n), 256>>>(n, d_starts.p, d_ends.p, nr, d_cx.p, d_cy.p, d_cz.p, d_rid.p, d_rt.p);
            k_bin<<<grid(n), 256>>>(n, d_rid.p, d_cx.p, d_cy.p, d_cz.p, d_idx.p, d_pb.p, n, d_rt.p);
            k_sweep<<<grid(nr, 128), 128>>>(nr, d_rt.p, p.max_leaf);
            k_count_left<<<grid(n), 256>>>(n, d_rid.p, d_cx.p, d_cy.p, d_cz.p, d_rt.p);
            k_misplaced<<<grid(n), 256>>>(n, d_rid.p, d_cx.p, d_cy.p, d_cz.p, d_rt.p, d_ml.p, d_mr.p);
            check(cudaGetLastError(), "split kernels");
            check(cub::DeviceScan::ExclusiveSum(d_temp.p, temp_bytes, d_ml.p, d_sl.p, (int)n), "scan");
            check(cub::DeviceScan::ExclusiveSum(d_temp.p, temp_bytes, d_mr.p, d_sr.p, (int)n), "scan");
            k_pairs<<<grid(n), 256>>>(n, d_rid.p, d_rt.p, d_ml.p, d_mr.p, d_sl.p, d_sr.p, d_pl.p, d_pr.p);
            k_range_out<<<grid(nr, 128), 128>>>(nr, d_rt.p, d_out.p);
            int last_sl = 0, last_ml = 0;
            check(cudaMemcpy(&last_sl, d_sl.p + (n - 1), 4, cudaMemcpyDeviceToHost), "pairs");
            check(cudaMemcpy(&last_ml, d_ml.p + (n - 1), 4, cudaMemcpyDeviceToHost), "pairs");
            const int64_t pairs = int64_t(last_sl) + last_ml;
            if (pairs > 0) k_swap<<<grid(pairs), 256>>>(pairs, d_pl.p, d_pr.p, d_cx.p, d_cy.p, d_cz.p, d_idx.p);
            check(cudaGetLastError(), "partition kernels");
            rout.resize(size_t(nr));
            check(cudaMemcpy(rout.data(), d_out.p, size_t(nr) * sizeof(RangeOut), cudaMemcpyDeviceToHost), "results");
            for (int k = 0; k < nr; ++k) {
                NodeTask& nt = active[size_t(owner[size_t(k)])];
                const RangeIn& x = rin[size_t(k)];
                const int64_t mid = x.s + rout[size_t(k)].left;
                if (!rout[size_t(k)].split || mid == x.s || mid == x.e) {
                    nt.done[nt.ndone++] = {x.s, x.e};
                } else {
                    nt.fifo[nt.tail++] = {x.s, mid};
                    nt.fifo[nt.tail++] = {mid, x.e};
                }
            }
        }
        // Nodes whose loop has ended become leaves, or hand their ranges on as
        // children (SORT's child order: the remaining list, then the done list).
        struct Kid {
            int id, depth, parent, j;  // j: position among the parent's children
        };
        std::vector<Kid> kids;
        next.clear();
        for (NodeTask& nt : active) {
            if (nt.head != nt.tail && nt.total() < W) {
                next.push_back(nt);
                continue;
            }
            if (nt.total() == 1) {
                depth_max = std::max(depth_max, nt.depth);
                continue;
            }
            Range rs[8];
            int m = 0;
            for (int q = nt.head; q < nt.tail; ++q) rs[m++] = nt.fifo[q];
            for (int q = 0; q < nt.ndone; ++q) rs[m++] = nt.done[q];
            const int first_kid = int(shape.size());
            for (int q = 0; q < m; ++q) {
                ShapeNode sn;
                sn.off = rs[q].s;
                sn.cnt = rs[q].e - rs[q].s;
                shape[size_t(nt.id)].kid[shape[size_t(nt.id)].nkids++] = int(shape.size());
                shape.push_back(sn);
            }
            // in range order for the sorted active list
            int ord[8];
            for (int q = 0; q < m; ++q) ord[q] = q;
            std::sort(ord, ord + m, [&](int a, int b) { return rs[a].s < rs[b].s; });
            for (int q = 0; q < m; ++q) {
                kids.push_back({first_kid + ord[q], nt.depth + 1, nt.id, ord[q]});
                next.emplace_back();  // placeholder
                next.back().id = -1;
            }
        }
        if (!kids.empty()) {
            // Boxes of the new children (kids are in range order): their own SAH
            // normaliser, and their parent's child boxes.
            const int nk = int(kids.size());
            starts.resize(size_t(nk));
            ends.resize(size_t(nk));
            for (int k = 0; k < nk; ++k) {
                const ShapeNode& sn = shape[size_t(kids[size_t(k)].id)];
                starts[size_t(k)] = sn.off;
                ends[size_t(k)] = sn.off + sn.cnt;
            }
            std::vector<int> boxes(size_t(nk) * 6);
            for (int k = 0; k < nk; ++k)
                for (int a = 0; a < 3; ++a) {
                    boxes[size_t(k) * 6 + a] = f2o(FLT_MAX);
                    boxes[size_t(k) * 6 + 3 + a] = f2o(-FLT_MAX);
                }
            d_starts.alloc(size_t(nk));
            d_ends.alloc(size_t(nk));
            d_boxes.alloc(size_t(nk) * 6);
            check(cudaMemcpy(d_starts.p, starts.data(), size_t(nk) * 8, cudaMemcpyHostToDevice), "kids");
            check(cudaMemcpy(d_ends.p, ends.data(), size_t(nk) * 8, cudaMemcpyHostToDevice), "kids");
            check(cudaMemcpy(d_boxes.p, boxes.data(), boxes.size() * 4, cudaMemcpyHostToDevice), "kids");
            k_range_boxes<<<grid(n), 256>>>(n, d_starts.p, d_ends.p, nk, d_idx.p, d_pb.p, n, d_boxes.p);
            check(cudaGetLastError(), "child boxes");
            check(cudaMemcpy(boxes.data(), d_boxes.p, boxes.size() * 4, cudaMemcpyDeviceToHost), "kids");
            std::vector<NodeTask> filled;
            filled.reserve(next.size());
            size_t kk = 0;
            for (size_t q = 0; q < next.size(); ++q) {
                if (next[q].id >= 0) {
                    filled.push_back(next[q]);
                    continue;
                }
                const Kid& kd = kids[kk];
                const Box b = box_from_images(&boxes[kk * 6]);
                ++kk;
                shape[size_t(kd.parent)].kid_box[kd.j] = b;
                start_node(filled, kd.id, kd.depth, b);
            }
            next.swap(filled);
        }
        active.swap(next);
    }
    t.depth = depth_max;

    // Final permutation -> leaf order.
    std::vector<int32_t> order(static_cast<size_t>(n));
    check(cudaMemcpy(order.data(), d_idx.p, size_t(n) * 4, cudaMemcpyDeviceToHost), "order");
    t.order = order;
    t.slot_box.resize(size_t(n));
    t.leaf_last.assign(size_t(n), 0);
    for (int64_t i = 0; i < n; ++i) {
        const int32_t q = order[size_t(i)];
        Box& b = t.slot_box[size_t(i)];
        for (int a = 0; a < 3; ++a) {
            b.mn[a] = pb[size_t(a) * n + q];
            b.mx[a] = pb[size_t(3 + a) * n + q];
        }
    }
    // Flatten exactly as build_tree numbers nodes: a node allocates its interior
    // children consecutively when it is filled, then fills them in order.
    auto alloc = [&](int cnt) {
        const int32_t base = int32_t(t.first_interior.size());
        t.first_interior.resize(t.first_interior.size() + size_t(cnt), -1);
        t.child.resize(t.child.size() + size_t(cnt) * W, kEmptyRef);
        t.lo.resize(t.lo.size() + size_t(cnt) * 3 * W, FLT_MAX);
        t.hi.resize(t.hi.size() + size_t(cnt) * 3 * W, -FLT_MAX);
        return base;
    };
    auto leaf = [&](const ShapeNode& sn) {
        t.leaves++;
        t.leaf_last[size_t(sn.off + sn.cnt - 1)] = 1;
    };
    std::vector<std::pair<int, int32_t>> stack;  // (shape id, node index), filled depth-first in order
    if (shape[0].nkids == 0) {
        t.root = leaf_ref(0);
        leaf(shape[0]);
    } else {
        t.root = alloc(1);
        stack.push_back({0, t.root});
    }
    while (!stack.empty()) {
        const auto [sid, idx] = stack.back();
        stack.pop_back();
        const ShapeNode sn = shape[size_t(sid)];
        int interior = 0;
        for (int j = 0; j < sn.nkids; ++j) interior += shape[size_t(sn.kid[j])].nkids ? 1 : 0;
        const int32_t base = interior ? alloc(interior) : -1;
        t.first_interior[size_t(idx)] = base;
        int k = 0;
        std::pair<int, int32_t> sub[8];
        int nsub = 0;
        for (int j = 0; j < sn.nkids; ++j) {
            const ShapeNode& kid = shape[size_t(sn.kid[j])];
            int32_t ref;
            if (kid.nkids == 0) {
                ref = leaf_ref(kid.off);
                leaf(kid);
            } else {
                ref = base + k++;
                sub[nsub++] = {sn.kid[j], ref};
            }
            t.child[size_t(idx) * W + j] = ref;
            for (int a = 0; a < 3; ++a) {
                t.lo[(size_t(idx) * 3 + a) * W + j] = sn.kid_box[j].mn[a];
                t.hi[(size_t(idx) * 3 + a) * W + j] = sn.kid_box[j].mx[a];
            }
        }
        for (int q = nsub - 1; q >= 0; --q) stack.push_back(sub[q]);  // first child filled next
    }
    return t;
}

}  // namespace sg
