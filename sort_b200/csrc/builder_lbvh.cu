// build_tree_lbvh: a wide BVH in Morton order, built entirely on the GPU.
//
// The fast builder for scenes that must be admitted quickly. Its tree is not
// SORT's (build_tree / build_tree_gpu build that one): hits and distances equal
// SORT's, because the box and triangle tests are the same, except near-ties
// (two triangles hit within 1e-6 of each other: a rounded box entry distance
// decides which one a traversal keeps), and where SORT's slab test
// (with its 1e-5 clamp of direction components) misses a hit triangle's own box
// by rounding: such a triangle is found only through a larger leaf box, which
// depends on the tree.
//
//   1. primitive boxes and centroids, the scene box (SORT's, enlarged by 0.1%,
//      core/scene.cpp:146-154) and the centroid bounds;
//   2. 63-bit Morton codes of the centroids (21 bits per axis over the
//      centroid bounds), sorted with their primitive indices (CUB radix sort);
//   3. the binary radix tree over the sorted codes, one thread per internal
//      node (the split is where the common prefix of the codes ends; equal
//      codes are told apart by their positions);
//   4. node boxes bottom-up: one thread per primitive climbs towards the root,
//      and of the two threads that reach a node the second one (by an atomic
//      counter) writes its box, so no thread ever waits;
//   5. the W-wide tree top-down, one thread per wide node per level: a wide
//      node starts from a binary node's two children and keeps opening the
//      child of largest surface area until it has W children; a child that
//      covers at most max_leaf primitives is a leaf (its primitives are
//      contiguous in Morton order, which is the leaf order). Nodes are written
//      straight into the device layout (layout.h);
//   6. the leaf-order triangle records.
// The host reads one count per level of the wide tree; nothing else crosses
// to the host. max_depth does not apply (it is part of SORT's split rules).
#include <cuda_runtime.h>


#include <algorithm>
#include <cfloat>
#include <cstdint>
#include <stdexcept>
#include <string>

#include "builder.h"
#include "gpu_build_common.cuh"
#include "staged_upload.h"
#include "layout.h"
#include "prefix_sort.cuh"

namespace sg {
namespace {

using namespace gpub;

constexpr int kMortonBits = 21;

// Centroid bounds (order images of the floats).
__global__ void __launch_bounds__(256) k_centroid_box(int64_t n, const float* __restrict__ cx,
                                                      const float* __restrict__ cy, const float* __restrict__ cz,
                                                      int* __restrict__ out) {
    __shared__ int sbox[6];
    if (threadIdx.x == 0) empty_box(sbox);
    __syncthreads();
    int v[6];
    empty_box(v);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int c[3] = {f2o(cx[i]), f2o(cy[i]), f2o(cz[i])};
        for (int a = 0; a < 3; ++a) {
            v[a] = min(v[a], c[a]);
            v[3 + a] = max(v[3 + a], c[a]);
        }
    }
    for (int a = 0; a < 3; ++a) {
        v[a] = __reduce_min_sync(0xffffffffu, v[a]);
        v[3 + a] = __reduce_max_sync(0xffffffffu, v[3 + a]);
    }
    if ((threadIdx.x & 31) == 0) atomic_box(sbox, v);
    __syncthreads();
    if (threadIdx.x < 3) {
        atomicMin(&out[threadIdx.x], sbox[threadIdx.x]);
        atomicMax(&out[3 + threadIdx.x], sbox[3 + threadIdx.x]);
    }
}

// Spreads the low 21 bits of v to every third bit.
__device__ __forceinline__ uint64_t spread3(uint64_t v) {
    v &= 0x1fffffull;
    v = (v | (v << 32)) & 0x1f00000000ffffull;
    v = (v | (v << 16)) & 0x1f0000ff0000ffull;
    v = (v | (v << 8)) & 0x100f00f00f00f00full;
    v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

__device__ __forceinline__ uint64_t quantise(float c, float lo, float scale) {
    const float q = (c - lo) * scale;
    const float top = float((1 << kMortonBits) - 1);
    return (uint64_t)fminf(fmaxf(q, 0.0f), top);
}

__global__ void k_morton(int64_t n, const float* __restrict__ cx, const float* __restrict__ cy,
                         const float* __restrict__ cz, const int* __restrict__ cbox, uint64_t* __restrict__ keys,
                         int32_t* __restrict__ vals) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float lo[3], scale[3];
    for (int a = 0; a < 3; ++a) {
        lo[a] = o2f(cbox[a]);
        const float ext = o2f(cbox[3 + a]) - lo[a];
        scale[a] = ext > 0.0f ? float((1 << kMortonBits) - 1) / ext : 0.0f;
    }
    const uint64_t x = quantise(cx[i], lo[0], scale[0]), y = quantise(cy[i], lo[1], scale[1]),
                   z = quantise(cz[i], lo[2], scale[2]);
    keys[i] = (spread3(x) << 2) | (spread3(y) << 1) | spread3(z);
    vals[i] = (int32_t)i;
}

// Length of the common prefix of sorted keys i and j; equal keys compare
// their positions. -1 outside [0, n).
__device__ __forceinline__ int prefix(const uint64_t* __restrict__ k, int64_t n, int64_t i, int64_t j) {
    if (j < 0 || j >= n) return -1;
    const uint64_t a = k[i], b = k[j];
    if (a != b) return __clzll((long long)(a ^ b));
    return 64 + __clzll((long long)((uint64_t)i ^ (uint64_t)j));
}

// Child reference of the binary tree: >= 0 internal node, < 0 leaf ~j.
__global__ void k_radix_tree(int64_t n, const uint64_t* __restrict__ keys, int32_t* __restrict__ left,
                             int32_t* __restrict__ right, int32_t* __restrict__ parent_int,
                             int32_t* __restrict__ parent_leaf, int32_t* __restrict__ lo_of,
                             int32_t* __restrict__ hi_of) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    const int64_t d = prefix(keys, n, i, i + 1) > prefix(keys, n, i, i - 1) ? 1 : -1;
    const int dmin = prefix(keys, n, i, i - d);
    int64_t lmax = 2;
    while (prefix(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
    int64_t l = 0;
    for (int64_t t = lmax >> 1; t >= 1; t >>= 1)
        if (prefix(keys, n, i, i + (l + t) * d) > dmin) l += t;
    const int64_t j = i + l * d;
    const int dnode = prefix(keys, n, i, j);
    int64_t s = 0;
    for (int64_t div = 2;; div <<= 1) {
        const int64_t t = (l + div - 1) / div;
        if (prefix(keys, n, i, i + (s + t) * d) > dnode) s += t;
        if (t <= 1) break;
    }
    const int64_t g = i + s * d + (d < 0 ? -1 : 0);
    const int64_t lo = min(i, j), hi = max(i, j);
    const int32_t lc = (lo == g) ? ~int32_t(g) : int32_t(g);
    const int32_t rc = (hi == g + 1) ? ~int32_t(g + 1) : int32_t(g + 1);
    left[i] = lc;
    right[i] = rc;
    lo_of[i] = int32_t(lo);
    hi_of[i] = int32_t(hi);
    if (lc < 0)
        parent_leaf[~lc] = int32_t(i);
    else
        parent_int[lc] = int32_t(i);
    if (rc < 0)
        parent_leaf[~rc] = int32_t(i);
    else
        parent_int[rc] = int32_t(i);
}

__device__ __forceinline__ void load_box(int32_t c, const float* __restrict__ ibox, const int32_t* __restrict__ idx,
                                         const float* __restrict__ pb, int64_t n, float (&b)[6]) {
    if (c >= 0) {
        for (int a = 0; a < 6; ++a) b[a] = __ldcg(ibox + int64_t(c) * 6 + a);
    } else {
        const int32_t p = idx[~c];
        for (int a = 0; a < 6; ++a) b[a] = pb[a * n + p];
    }
}

// Boxes of the internal nodes, bottom-up (the second thread to reach a node
// writes it; visits must start at zero).
__global__ void k_boxes_up(int64_t n, const int32_t* __restrict__ idx, const float* __restrict__ pb,
                           const int32_t* __restrict__ left, const int32_t* __restrict__ right,
                           const int32_t* __restrict__ parent_int, const int32_t* __restrict__ parent_leaf,
                           int* __restrict__ visits, float* __restrict__ ibox) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    int32_t p = parent_leaf[j];
    for (;;) {
        __threadfence();
        if (atomicAdd(&visits[p], 1) == 0) return;  // the sibling's box is not written yet
        float a[6], b[6];
        load_box(left[p], ibox, idx, pb, n, a);
        load_box(right[p], ibox, idx, pb, n, b);
        for (int k = 0; k < 3; ++k) {
            __stcg(ibox + int64_t(p) * 6 + k, fminf(a[k], b[k]));
            __stcg(ibox + int64_t(p) * 6 + 3 + k, fmaxf(a[3 + k], b[3 + k]));
        }
        if (p == 0) return;
        p = parent_int[p];
    }
}

struct CollapseState {
    int nodes;      // wide nodes allocated
    int depth;      // Fbvh::m_depth convention: root at 1, leaves included
    int leaves;
    int pad;
};

__device__ __forceinline__ float box_area(const float (&b)[6]) {
    const float x = b[3] - b[0], y = b[4] - b[1], z = b[5] - b[2];
    return x * y + y * z + z * x;
}

// One wide node per work item (binary node, wide index). Children of at most
// max_leaf primitives become leaves; the others get consecutive wide indices
// and go to the next level's queue at (index - next_base).
template <int W>
__global__ void k_collapse(int nq, const int2* __restrict__ q_in, int2* __restrict__ q_out, int next_base, int level,
                           int64_t n, int max_leaf, const int32_t* __restrict__ idx, const float* __restrict__ pb,
                           const float* __restrict__ ibox, const int32_t* __restrict__ left,
                           const int32_t* __restrict__ right, const int32_t* __restrict__ lo_of,
                           const int32_t* __restrict__ hi_of, uint8_t* __restrict__ last,
                           CollapseState* __restrict__ cs, float4* __restrict__ nodes) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nq) return;
    const int2 item = q_in[q];
    const int32_t b = item.x;
    int32_t kid[W];
    int m = 2;
    kid[0] = left[b];
    kid[1] = right[b];
    auto opens = [&](int32_t c) { return c >= 0 && hi_of[c] - lo_of[c] + 1 > max_leaf; };
    while (m < W) {
        int best = -1;
        float best_area = -1.0f;
        for (int k = 0; k < m; ++k) {
            if (!opens(kid[k])) continue;
            float bx[6];
            load_box(kid[k], ibox, idx, pb, n, bx);
            const float ar = box_area(bx);
            if (ar > best_area) {
                best_area = ar;
                best = k;
            }
        }
        if (best < 0) break;
        const int32_t c = kid[best];
        kid[best] = left[c];
        kid[m++] = right[c];
    }
    int inner = 0;
    for (int k = 0; k < m; ++k) inner += opens(kid[k]) ? 1 : 0;
    const int base = inner ? atomicAdd(&cs->nodes, inner) : 0;
    constexpr int Q = W / 4;
    constexpr int F4 = W == 8 ? NodeShape<8>::kF4 : NodeShape<4>::kF4;
    float* node = reinterpret_cast<float*>(nodes + int64_t(item.y) * F4);
    int32_t* ch = reinterpret_cast<int32_t*>(node + 6 * Q * 4);
    int k_in = 0, n_leaf = 0;
    for (int j = 0; j < W; ++j) {
        if (j >= m) {
            for (int a = 0; a < 3; ++a) {
                node[(2 * a) * Q * 4 + j] = FLT_MAX;
                node[(2 * a + 1) * Q * 4 + j] = -FLT_MAX;
            }
            ch[j] = kEmptyRef;
            continue;
        }
        const int32_t c = kid[j];
        float bx[6];
        load_box(c, ibox, idx, pb, n, bx);
        for (int a = 0; a < 3; ++a) {
            node[(2 * a) * Q * 4 + j] = bx[a];
            node[(2 * a + 1) * Q * 4 + j] = bx[3 + a];
        }
        if (opens(c)) {
            const int w = base + k_in++;
            ch[j] = w;
            q_out[w - next_base] = make_int2(c, w);
        } else {
            const int32_t s = c >= 0 ? lo_of[c] : ~c;
            const int32_t e = c >= 0 ? hi_of[c] : ~c;
            ch[j] = int32_t(uint32_t(s) | 0x80000000u);
            last[e] = 1;
            ++n_leaf;
        }
    }
    if (W == 4) {  // the layout's padding
        for (int k = 28; k < 32; ++k) node[k] = 0.0f;
    }
    if (n_leaf) {
        atomicAdd(&cs->leaves, n_leaf);
        atomicMax(&cs->depth, level + 2);
    }
}

}  // namespace

BuiltTree build_tree_lbvh(const float* tri, int64_t ntri, const BuildParams& p, int device) {
    if (p.width != 4 && p.width != 8) throw std::invalid_argument("width must be 4 or 8");
    if (p.max_leaf < 1) throw std::invalid_argument("max_leaf must be >= 1");
    if (ntri < 0 || ntri >= int64_t(0x7fffffff)) throw std::invalid_argument("triangle count out of range");
    if (p.nextra != 0) throw std::invalid_argument("the LBVH builder takes triangles only");
    const int W = p.width;
    const int F4 = W == 8 ? NodeShape<8>::kF4 : NodeShape<4>::kF4;
    const int64_t n = ntri;
    BuiltTree t;
    t.width = W;
    t.n_tri = n;
    t.n_interior = 0;
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

    const int64_t nn = std::max<int64_t>(n, 1);
    DevBuf<float> d_tri, d_cx, d_cy, d_cz, d_pb, d_ibox;
    DevBuf<int32_t> d_idx, d_sorted, d_left, d_right, d_pint, d_pleaf, d_lo, d_hi;
    DevBuf<uint64_t> d_keys, d_keys_sorted;
    DevBuf<int> d_box, d_visits;
    DevBuf<uint8_t> d_last;
    DevBuf<int2> d_qa, d_qb;
    DevBuf<CollapseState> d_cs;
    DevBuf<float4> d_wide;
    DevBuf<unsigned char> d_temp;
    PinnedBuf<int> h_box;
    PinnedBuf<CollapseState> h_cs;
    d_tri.alloc(size_t(nn) * 9);
    d_cx.alloc(size_t(nn));
    d_cy.alloc(size_t(nn));
    d_cz.alloc(size_t(nn));
    d_pb.alloc(size_t(nn) * 6);
    d_idx.alloc(size_t(nn));
    d_box.alloc(12);
    h_box.alloc(12);
    h_cs.alloc(1);

    // Scene box (core/scene.cpp:146-154) and centroid bounds.
    empty_box(h_box.p);
    empty_box(h_box.p + 6);
    if (n > 0) {
        check(upload_host(d_tri.p, tri, size_t(n) * 9 * sizeof(float), st), "upload");
        k_prim_setup<<<grid(n), 256, 0, st>>>(d_tri.p, n, n, d_cx.p, d_cy.p, d_cz.p, d_idx.p, d_pb.p);
        check(cudaMemcpyAsync(d_box.p, h_box.p, 12 * sizeof(int), cudaMemcpyHostToDevice, st), "boxes");
        const unsigned gb = std::min<unsigned>(grid(n), 148 * 8);
        k_scene_box<<<gb, 256, 0, st>>>(n, d_pb.p, d_box.p);
        k_centroid_box<<<gb, 256, 0, st>>>(n, d_cx.p, d_cy.p, d_cz.p, d_box.p + 6);
        check(cudaGetLastError(), "primitive setup");
        check(cudaMemcpyAsync(h_box.p, d_box.p, 12 * sizeof(int), cudaMemcpyDeviceToHost, st), "boxes");
        check(cudaStreamSynchronize(st), "primitive setup");
    }
    Box scene = box_from_images(h_box.p);
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

    // Morton codes, sorted with their primitive indices.
    d_keys.alloc(size_t(n));
    d_keys_sorted.alloc(size_t(n));
    d_sorted.alloc(size_t(n));
    k_morton<<<grid(n), 256, 0, st>>>(n, d_cx.p, d_cy.p, d_cz.p, d_box.p + 6, d_keys.p, d_idx.p);
    check(cudaGetLastError(), "morton codes");
    // Stable radix sort of (code, primitive) over the code's 63 bits
    // (prefix_sort.cuh: seven passes of 10-bit digits).
    const size_t count_words = psort::sort_count_words(n), scan_words = psort::sort_scan_words(n);
    d_temp.alloc((count_words + scan_words) * sizeof(uint32_t));
    {
        uint64_t* keys[2] = {d_keys.p, d_keys_sorted.p};
        int32_t* vals[2] = {d_idx.p, d_sorted.p};
        uint32_t* cnt = reinterpret_cast<uint32_t*>(d_temp.p);
        int in = 0;
        check(psort::sort_pairs<uint64_t>(keys, vals, n, 0, 3 * kMortonBits, cnt, cnt + count_words, false, &in, st),
              "sort");
        if (in == 0) {  // an even pass count leaves the result where it started
            check(cudaMemcpyAsync(d_keys_sorted.p, d_keys.p, size_t(n) * 8, cudaMemcpyDeviceToDevice, st), "sort");
            check(cudaMemcpyAsync(d_sorted.p, d_idx.p, size_t(n) * 4, cudaMemcpyDeviceToDevice, st), "sort");
        }
    }
    int launches = 4;  // setup, scene box, centroid box, codes

    d_last.alloc(size_t(n));
    check(cudaMemsetAsync(d_last.p, 0, size_t(n), st), "leaf flags");
    int levels = 0;
    if (n <= p.max_leaf) {  // one leaf holds everything
        t.root = leaf_ref(0);
        t.depth = 1;
        t.leaves = 1;
        const uint8_t one = 1;
        check(cudaMemcpyAsync(d_last.p + (n - 1), &one, 1, cudaMemcpyHostToDevice, st), "leaf flags");
        check(cudaStreamSynchronize(st), "leaf flags");
    } else {
        const int64_t ni = n - 1;  // internal nodes of the binary tree
        d_left.alloc(size_t(ni));
        d_right.alloc(size_t(ni));
        d_pint.alloc(size_t(ni));
        d_pleaf.alloc(size_t(n));
        d_lo.alloc(size_t(ni));
        d_hi.alloc(size_t(ni));
        d_ibox.alloc(size_t(ni) * 6);
        d_visits.alloc(size_t(ni));
        check(cudaMemsetAsync(d_visits.p, 0, size_t(ni) * sizeof(int), st), "visits");
        k_radix_tree<<<grid(ni), 256, 0, st>>>(n, d_keys_sorted.p, d_left.p, d_right.p, d_pint.p, d_pleaf.p, d_lo.p,
                                               d_hi.p);
        k_boxes_up<<<grid(n), 256, 0, st>>>(n, d_sorted.p, d_pb.p, d_left.p, d_right.p, d_pint.p, d_pleaf.p,
                                            d_visits.p, d_ibox.p);
        check(cudaGetLastError(), "radix tree");
        launches += 2;

        // Wide nodes, level by level.
        *h_cs.p = CollapseState{1, 1, 0, 0};
        d_cs.alloc(1);
        check(cudaMemcpyAsync(d_cs.p, h_cs.p, sizeof(CollapseState), cudaMemcpyHostToDevice, st), "collapse state");
        size_t wide_cap = size_t(std::max<int64_t>(64, n / 16));
        d_wide.alloc(wide_cap * F4);
        d_qa.alloc(64);
        d_qb.alloc(64);
        const int2 root_item = make_int2(0, 0);
        check(cudaMemcpyAsync(d_qa.p, &root_item, sizeof(int2), cudaMemcpyHostToDevice, st), "root");
        int nq = 1, allocated = 1;
        while (nq > 0) {
            // A level adds at most W wide nodes per item.
            const size_t need = size_t(allocated) + size_t(nq) * W;
            if (need > wide_cap) {
                DevBuf<float4> bigger;
                const size_t cap2 = std::max(need, 2 * wide_cap);
                bigger.alloc(cap2 * F4);
                check(cudaMemcpyAsync(bigger.p, d_wide.p, size_t(allocated) * F4 * sizeof(float4),
                                      cudaMemcpyDeviceToDevice, st),
                      "grow nodes");
                swap_bufs(d_wide, bigger);
                wide_cap = cap2;
            }
            d_qb.alloc(size_t(nq) * W);
            const int next_base = allocated;
            if (W == 8)
                k_collapse<8><<<grid(nq, 128), 128, 0, st>>>(nq, d_qa.p, d_qb.p, next_base, levels, n, p.max_leaf,
                                                            d_sorted.p, d_pb.p, d_ibox.p, d_left.p, d_right.p, d_lo.p,
                                                            d_hi.p, d_last.p, d_cs.p, d_wide.p);
            else
                k_collapse<4><<<grid(nq, 128), 128, 0, st>>>(nq, d_qa.p, d_qb.p, next_base, levels, n, p.max_leaf,
                                                            d_sorted.p, d_pb.p, d_ibox.p, d_left.p, d_right.p, d_lo.p,
                                                            d_hi.p, d_last.p, d_cs.p, d_wide.p);
            check(cudaGetLastError(), "collapse");
            ++launches;
            check(cudaMemcpyAsync(h_cs.p, d_cs.p, sizeof(CollapseState), cudaMemcpyDeviceToHost, st), "level");
            check(cudaStreamSynchronize(st), "level");
            ++levels;
            nq = h_cs.p->nodes - next_base;
            allocated = h_cs.p->nodes;
            swap_bufs(d_qa, d_qb);
        }
        t.root = 0;
        t.depth = h_cs.p->depth;
        t.leaves = h_cs.p->leaves;
        t.n_interior = allocated;
        // The scene owns its nodes: an exact-size copy outside the scratch pool.
        float4* nodes = nullptr;
        check(cudaMalloc(&nodes, size_t(allocated) * F4 * sizeof(float4)), "cudaMalloc(nodes)");
        cudaError_t e = cudaMemcpyAsync(nodes, d_wide.p, size_t(allocated) * F4 * sizeof(float4),
                                        cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            cudaFree(nodes);
            check(e, "copy nodes");
        }
        t.d_nodes = nodes;
    }

    // The triangle records in leaf (Morton) order.
    const size_t tris_bytes = size_t(n + kPadSlots) * 3 * sizeof(float4);
    float4* d_tris = nullptr;
    cudaError_t e = cudaMalloc(&d_tris, tris_bytes);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_tris + size_t(n) * 3, 0, size_t(kPadSlots) * 3 * sizeof(float4), st);
    if (e == cudaSuccess) {
        k_leaf_tris<<<grid(n), 256, 0, st>>>(n, d_tri.p, d_sorted.p, d_last.p, d_tris);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        if (d_tris) cudaFree(d_tris);
        if (t.d_nodes) cudaFree(t.d_nodes);
        t.d_nodes = nullptr;
        check(e, "triangle records");
    }
    t.d_tris = d_tris;
    t.rounds = levels;
    t.launches = launches + 1;
    return t;
}

}  // namespace sg
