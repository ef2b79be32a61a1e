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
    b = min(b, kBins - 1);
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

struct Range {
    int64_t s, e;
};

struct NodeTask {  // a node under construction
    int id;        // index into shape
    int depth;
    float area;
    std::deque<Range> fifo;
    std::vector<Range> done;
};

struct ShapeNode {
    int64_t off = 0, cnt = 0;
    std::vector<int> kids;  // indices into the shape array
    std::vector<Box> kid_box;
};

unsigned grid(int64_t n, int t = 256) { return (unsigned)std::max<int64_t>(1, (n + t - 1) / t); }

Box host_half_area_box(const int* o) {
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

    // Scan scratch for n ints.
    size_t temp_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, temp_bytes, d_ml.p, d_sl.p, (int)n);
    d_temp.alloc(temp_bytes);

    std::vector<ShapeNode> shape(1);
    shape[0].off = 0;
    shape[0].cnt = n;
    int depth_max = 0;
    std::vector<NodeTask> active;
    auto start_node = [&](int id, int depth, const Box& box) {
        const ShapeNode& sn = shape[size_t(id)];
        if (sn.cnt <= p.max_leaf || depth == p.max_depth) {  // splitNode's early return
            depth_max = std::max(depth_max, depth);
            return;
        }
        NodeTask nt;
        nt.id = id;
        nt.depth = depth;
        nt.area = host_half_area(box);
        nt.fifo.push_back({sn.off, sn.off + sn.cnt});
        active.push_back(std::move(nt));
    };
    start_node(0, 1, scene);

    std::vector<RangeTask> rt;
    std::vector<int64_t> starts, ends;
    std::vector<int> owner;
    while (!active.empty()) {
        // One split per node: the front of its list, while SORT's loop would go on.
        rt.clear();
        starts.clear();
        ends.clear();
        owner.clear();
        for (size_t k = 0; k < active.size(); ++k) {
            NodeTask& nt = active[k];
            if (nt.fifo.empty() || int(nt.fifo.size() + nt.done.size()) >= W) continue;
            const Range r = nt.fifo.front();
            nt.fifo.pop_front();
            RangeTask x;
            std::memset(&x, 0, sizeof(x));
            x.s = r.s;
            x.e = r.e;
            x.node_area = nt.area;
            for (int a = 0; a < 3; ++a) {
                x.inner[a] = f2o(FLT_MAX);
                x.inner[3 + a] = f2o(-FLT_MAX);
            }
            for (int b = 0; b < kBins; ++b)
                for (int a = 0; a < 3; ++a) {
                    x.bin_box[b][a] = f2o(FLT_MAX);
                    x.bin_box[b][3 + a] = f2o(-FLT_MAX);
                }
            rt.push_back(x);
            owner.push_back(int(k));
        }
        if (!rt.empty()) {
            // ranges sorted by start for the per-primitive lookup (they are disjoint)
            std::vector<int> ord(rt.size());
            for (size_t k = 0; k < ord.size(); ++k) ord[k] = int(k);
            std::sort(ord.begin(), ord.end(), [&](int a, int b) { return rt[size_t(a)].s < rt[size_t(b)].s; });
            std::vector<RangeTask> rs(rt.size());
            std::vector<int> os(rt.size());
            for (size_t k = 0; k < ord.size(); ++k) {
                rs[k] = rt[size_t(ord[k])];
                os[k] = owner[size_t(ord[k])];
                starts.push_back(rs[k].s);
                ends.push_back(rs[k].e);
            }
            rt.swap(rs);
            owner.swap(os);
            const int nr = int(rt.size());
            d_rt.alloc(size_t(nr));
            d_starts.alloc(size_t(nr));
            d_ends.alloc(size_t(nr));
            check(cudaMemcpy(d_rt.p, rt.data(), size_t(nr) * sizeof(RangeTask), cudaMemcpyHostToDevice), "ranges");
            check(cudaMemcpy(d_starts.p, starts.data(), size_t(nr) * 8, cudaMemcpyHostToDevice), "ranges");
            check(cudaMemcpy(d_ends.p, ends.data(), size_t(nr) * 8, cudaMemcpyHostToDevice), "ranges");
            k_bounds<<<grid(n), 256>>>(n, d_starts.p, d_ends.p, nr, d_cx.p, d_cy.p, d_cz.p, d_rid.p, d_rt.p);
            k_bin<<<grid(n), 256>>>(n, d_rid.p, d_cx.p, d_cy.p, d_cz.p, d_idx.p, d_pb.p, n, d_rt.p);
            k_sweep<<<grid(nr, 128), 128>>>(nr, d_rt.p, p.max_leaf);
            k_count_left<<<grid(n), 256>>>(n, d_rid.p, d_cx.p, d_cy.p, d_cz.p, d_rt.p);
            k_misplaced<<<grid(n), 256>>>(n, d_rid.p, d_cx.p, d_cy.p, d_cz.p, d_rt.p, d_ml.p, d_mr.p);
            check(cudaGetLastError(), "split kernels");
            check(cub::DeviceScan::ExclusiveSum(d_temp.p, temp_bytes, d_ml.p, d_sl.p, (int)n), "scan");
            check(cub::DeviceScan::ExclusiveSum(d_temp.p, temp_bytes, d_mr.p, d_sr.p, (int)n), "scan");
            k_pairs<<<grid(n), 256>>>(n, d_rid.p, d_rt.p, d_ml.p, d_mr.p, d_sl.p, d_sr.p, d_pl.p, d_pr.p);
            int last_sl = 0, last_ml = 0;
            check(cudaMemcpy(&last_sl, d_sl.p + (n - 1), 4, cudaMemcpyDeviceToHost), "pairs");
            check(cudaMemcpy(&last_ml, d_ml.p + (n - 1), 4, cudaMemcpyDeviceToHost), "pairs");
            const int64_t pairs = int64_t(last_sl) + last_ml;
            if (pairs > 0) k_swap<<<grid(pairs), 256>>>(pairs, d_pl.p, d_pr.p, d_cx.p, d_cy.p, d_cz.p, d_idx.p);
            check(cudaGetLastError(), "partition kernels");
            check(cudaMemcpy(rt.data(), d_rt.p, size_t(nr) * sizeof(RangeTask), cudaMemcpyDeviceToHost), "results");
            for (int k = 0; k < nr; ++k) {
                NodeTask& nt = active[size_t(owner[size_t(k)])];
                const RangeTask& x = rt[size_t(k)];
                const int64_t mid = x.s + x.left;
                if (!x.split || mid == x.s || mid == x.e) {
                    nt.done.push_back({x.s, x.e});
                } else {
                    nt.fifo.push_back({x.s, mid});
                    nt.fifo.push_back({mid, x.e});
                }
            }
        }
        // Nodes whose loop has ended: leaves, or children from their ranges.
        std::vector<NodeTask> still;
        std::vector<std::pair<int, int>> new_kids;  // (shape id, depth)
        std::vector<int> new_parent;                // shape id of each new kid's parent
        for (NodeTask& nt : active) {
            const int total = int(nt.fifo.size() + nt.done.size());
            if (!nt.fifo.empty() && total < W) {
                still.push_back(std::move(nt));
                continue;
            }
            if (total == 1) {
                depth_max = std::max(depth_max, nt.depth);
                continue;
            }
            std::vector<Range> kids(nt.fifo.begin(), nt.fifo.end());
            kids.insert(kids.end(), nt.done.begin(), nt.done.end());
            for (const Range& r : kids) {
                ShapeNode sn;
                sn.off = r.s;
                sn.cnt = r.e - r.s;
                shape.push_back(std::move(sn));
                shape[size_t(nt.id)].kids.push_back(int(shape.size()) - 1);
                new_kids.push_back({int(shape.size()) - 1, nt.depth + 1});
                new_parent.push_back(nt.id);
            }
        }
        active.swap(still);
        if (!new_kids.empty()) {
            // Boxes of the new children (their own SAH normaliser, and their parent's child boxes).
            std::vector<int> ord(new_kids.size());
            for (size_t k = 0; k < ord.size(); ++k) ord[k] = int(k);
            std::sort(ord.begin(), ord.end(), [&](int a, int b) {
                return shape[size_t(new_kids[size_t(a)].first)].off < shape[size_t(new_kids[size_t(b)].first)].off;
            });
            const int nk = int(ord.size());
            starts.assign(size_t(nk), 0);
            ends.assign(size_t(nk), 0);
            for (int k = 0; k < nk; ++k) {
                const ShapeNode& sn = shape[size_t(new_kids[size_t(ord[size_t(k)])].first)];
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
            std::vector<Box> kb(static_cast<size_t>(nk));
            for (int k = 0; k < nk; ++k) kb[size_t(ord[size_t(k)])] = host_half_area_box(&boxes[size_t(k) * 6]);
            // parents' child boxes, in child order (a parent's kids are consecutive in new_kids)
            for (size_t j = 0; j < new_kids.size(); ++j)
                shape[size_t(new_parent[j])].kid_box.push_back(kb[j]);
            for (size_t j = 0; j < new_kids.size(); ++j) start_node(new_kids[j].first, new_kids[j].second, kb[j]);
        }
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
    if (shape[0].kids.empty()) {
        t.root = leaf_ref(0);
        leaf(shape[0]);
    } else {
        t.root = alloc(1);
        stack.push_back({0, t.root});
    }
    while (!stack.empty()) {
        const auto [sid, idx] = stack.back();
        stack.pop_back();
        const ShapeNode& sn = shape[size_t(sid)];
        int interior = 0;
        for (int k : sn.kids) interior += shape[size_t(k)].kids.empty() ? 0 : 1;
        const int32_t base = interior ? alloc(interior) : -1;
        t.first_interior[size_t(idx)] = base;
        int k = 0;
        std::vector<std::pair<int, int32_t>> sub;
        for (size_t j = 0; j < sn.kids.size(); ++j) {
            const ShapeNode& kid = shape[size_t(sn.kids[j])];
            int32_t ref;
            if (kid.kids.empty()) {
                ref = leaf_ref(kid.off);
                leaf(kid);
            } else {
                ref = base + k++;
                sub.push_back({sn.kids[j], ref});
            }
            t.child[size_t(idx) * W + j] = ref;
            for (int a = 0; a < 3; ++a) {
                t.lo[(size_t(idx) * 3 + a) * W + j] = sn.kid_box[j].mn[a];
                t.hi[(size_t(idx) * 3 + a) * W + j] = sn.kid_box[j].mx[a];
            }
        }
        for (auto it = sub.rbegin(); it != sub.rend(); ++it) stack.push_back(*it);  // first child filled next
    }
    return t;
}

}  // namespace sg
