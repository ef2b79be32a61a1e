// Stages shared by the two builders that start from Morton order
// (builder_lbvh.cu: the binary radix tree; builder_ploc.cu: parallel
// locally-ordered clustering):
//
//   * primitive boxes and centroids, the scene box (SORT's, enlarged by 0.1%,
//     core/scene.cpp:146-154), the centroid bounds, and the primitives sorted
//     by the 63-bit Morton code of their centroids (21 bits per axis);
//   * the collapse of a binary tree into the W-wide device layout, top-down,
//     one thread per wide node per level: a wide node starts from a binary
//     node's two children and keeps opening, of the children holding more than
//     max_leaf primitives, the one of largest surface area until it has W
//     children; when none is left and slots are still free, it goes on opening
//     the largest of the other internal children (each would be a leaf) into
//     them. A child holding at most max_leaf primitives is a leaf, whose
//     primitives take consecutive leaf slots in the binary tree's
//     left-to-right order. Filling the slots costs no node test (every slot's
//     box is tested anyway) and makes leaves smaller: on a 21M-triangle sphere
//     field it cut triangle tests per ray by 37% at the same node tests;
//   * the leaf-order triangle records.
//
// A binary tree here: internal nodes 0 .. n-2 with left / right child
// references (>= 0 internal node, < 0 leaf ~j, j a position in Morton order),
// the primitive count under each internal node and its box (6 floats).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cstdint>

#include "builder.h"
#include "gpu_build_common.cuh"
#include "layout.h"
#include "prefix_sort.cuh"
#include "staged_upload.h"

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

// The binary tree the collapse reads (see the file comment).
struct BinaryTree {
    const int32_t* left;
    const int32_t* right;
    const int32_t* count;  // primitives under each internal node
    const float* ibox;     // 6 floats per internal node: min xyz, max xyz
    const int32_t* idx;    // primitive at each Morton position
    const float* pb;       // primitive boxes, 6 planes of n
    int64_t n;
};

__device__ __forceinline__ int32_t ref_count(const BinaryTree& bt, int32_t c) { return c >= 0 ? bt.count[c] : 1; }

__device__ __forceinline__ void load_box(const BinaryTree& bt, int32_t c, float (&b)[6]) {
    if (c >= 0) {
        for (int a = 0; a < 6; ++a) b[a] = __ldcg(bt.ibox + int64_t(c) * 6 + a);
    } else {
        const int32_t p = bt.idx[~c];
        for (int a = 0; a < 6; ++a) b[a] = bt.pb[a * bt.n + p];
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

// The primitives under binary reference c, left to right, into slots
// s .. s + k - 1 of perm: the k-th is found by descending from c with the
// counts (each step shrinks the subtree, so at most k - 1 steps).
__device__ __forceinline__ void leaf_slots(const BinaryTree& bt, int32_t c, int32_t s, int32_t k,
                                           int32_t* __restrict__ perm) {
    for (int32_t r = 0; r < k; ++r) {
        int32_t node = c, rank = r;
        while (node >= 0) {
            const int32_t l = bt.left[node];
            const int32_t cl = ref_count(bt, l);
            if (rank < cl) {
                node = l;
            } else {
                rank -= cl;
                node = bt.right[node];
            }
        }
        perm[s + r] = bt.idx[~node];
    }
}

// One wide node per work item (x: binary node, y: wide index, z: first leaf
// slot of the binary node's primitives). Children of at most max_leaf
// primitives become leaves (free slots are first filled by opening such
// children that are internal, largest area first); the others get consecutive
// wide indices and go to the next level's queue at (index - next_base).
template <int W>
__global__ void k_collapse(int nq, const int4* __restrict__ q_in, int4* __restrict__ q_out, int next_base, int level,
                           int max_leaf, BinaryTree bt, uint8_t* __restrict__ last, int32_t* __restrict__ perm,
                           CollapseState* __restrict__ cs, float4* __restrict__ nodes) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nq) return;
    const int4 item = q_in[q];
    const int32_t b = item.x;
    int32_t kid[W], start[W];
    int m = 2;
    kid[0] = bt.left[b];
    kid[1] = bt.right[b];
    start[0] = item.z;
    start[1] = item.z + ref_count(bt, kid[0]);
    auto opens = [&](int32_t c) { return c >= 0 && bt.count[c] > max_leaf; };
    bool fill = false;  // every child fits a leaf: open leaf-sized internal children into the free slots
    while (m < W) {
        int best = -1;
        float best_area = -1.0f;
        for (int k = 0; k < m; ++k) {
            if (!(fill ? kid[k] >= 0 : opens(kid[k]))) continue;
            float bx[6];
            load_box(bt, kid[k], bx);
            const float ar = box_area(bx);
            if (ar > best_area) {
                best_area = ar;
                best = k;
            }
        }
        if (best < 0) {
            if (fill) break;
            fill = true;
            continue;
        }
        const int32_t c = kid[best];
        const int32_t s = start[best];
        kid[best] = bt.left[c];
        kid[m] = bt.right[c];
        start[m] = s + ref_count(bt, kid[best]);
        ++m;
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
        load_box(bt, c, bx);
        for (int a = 0; a < 3; ++a) {
            node[(2 * a) * Q * 4 + j] = bx[a];
            node[(2 * a + 1) * Q * 4 + j] = bx[3 + a];
        }
        if (opens(c)) {
            const int w = base + k_in++;
            ch[j] = w;
            q_out[w - next_base] = make_int4(c, w, start[j], 0);
        } else {
            const int32_t s = start[j], k = ref_count(bt, c);
            ch[j] = int32_t(uint32_t(s) | 0x80000000u);
            leaf_slots(bt, c, s, k, perm);
            last[s + k - 1] = 1;
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

// Device buffers of the Morton stage. Declare after the build's ScratchScope.
struct MortonPrims {
    DevBuf<float> tri, cx, cy, cz, pb;
    DevBuf<int32_t> idx, sorted;
    DevBuf<uint64_t> keys, keys_sorted;
    DevBuf<int> box;
    DevBuf<unsigned char> temp;
    PinnedBuf<int> h_box;
    Box scene{};
    int launches = 0;
};

// Uploads the triangles; primitive boxes (6 planes of n in m.pb), centroids,
// the enlarged scene box (m.scene) and, when n > 0, the Morton-sorted
// primitive order (m.sorted, codes in m.keys_sorted).
inline void morton_prims(MortonPrims& m, const float* tri, int64_t n, cudaStream_t st) {
    const int64_t nn = std::max<int64_t>(n, 1);
    m.tri.alloc(size_t(nn) * 9);
    m.cx.alloc(size_t(nn));
    m.cy.alloc(size_t(nn));
    m.cz.alloc(size_t(nn));
    m.pb.alloc(size_t(nn) * 6);
    m.idx.alloc(size_t(nn));
    m.box.alloc(12);
    m.h_box.alloc(12);
    empty_box(m.h_box.p);
    empty_box(m.h_box.p + 6);
    if (n > 0) {
        check(upload_host(m.tri.p, tri, size_t(n) * 9 * sizeof(float), st), "upload");
        k_prim_setup<<<grid(n), 256, 0, st>>>(m.tri.p, n, n, m.cx.p, m.cy.p, m.cz.p, m.idx.p, m.pb.p);
        check(cudaMemcpyAsync(m.box.p, m.h_box.p, 12 * sizeof(int), cudaMemcpyHostToDevice, st), "boxes");
        const unsigned gb = std::min<unsigned>(grid(n), 148 * 8);
        k_scene_box<<<gb, 256, 0, st>>>(n, m.pb.p, m.box.p);
        k_centroid_box<<<gb, 256, 0, st>>>(n, m.cx.p, m.cy.p, m.cz.p, m.box.p + 6);
        check(cudaGetLastError(), "primitive setup");
        check(cudaMemcpyAsync(m.h_box.p, m.box.p, 12 * sizeof(int), cudaMemcpyDeviceToHost, st), "boxes");
        check(cudaStreamSynchronize(st), "primitive setup");
    }
    Box scene = box_from_images(m.h_box.p);
    const float threshold = 0.001f;
    float delta[3];
    for (int k = 0; k < 3; ++k) delta[k] = (scene.mx[k] - scene.mn[k]) * threshold;
    for (int k = 0; k < 3; ++k) {
        scene.mn[k] -= delta[k];
        scene.mx[k] += delta[k];
    }
    m.scene = scene;
    if (n == 0) return;

    m.keys.alloc(size_t(n));
    m.keys_sorted.alloc(size_t(n));
    m.sorted.alloc(size_t(n));
    k_morton<<<grid(n), 256, 0, st>>>(n, m.cx.p, m.cy.p, m.cz.p, m.box.p + 6, m.keys.p, m.idx.p);
    check(cudaGetLastError(), "morton codes");
    // Stable radix sort of (code, primitive) over the code's 63 bits
    // (prefix_sort.cuh: seven passes of 10-bit digits).
    const size_t count_words = psort::sort_count_words(n), scan_words = psort::sort_scan_words(n);
    m.temp.alloc((count_words + scan_words) * sizeof(uint32_t));
    uint64_t* keys[2] = {m.keys.p, m.keys_sorted.p};
    int32_t* vals[2] = {m.idx.p, m.sorted.p};
    uint32_t* cnt = reinterpret_cast<uint32_t*>(m.temp.p);
    int in = 0;
    check(psort::sort_pairs<uint64_t>(keys, vals, n, 0, 3 * kMortonBits, cnt, cnt + count_words, false, &in, st),
          "sort");
    if (in == 0) {  // an even pass count leaves the result where it started
        check(cudaMemcpyAsync(m.keys_sorted.p, m.keys.p, size_t(n) * 8, cudaMemcpyDeviceToDevice, st), "sort");
        check(cudaMemcpyAsync(m.sorted.p, m.idx.p, size_t(n) * 4, cudaMemcpyDeviceToDevice, st), "sort");
    }
    m.launches = 4;  // setup, scene box, centroid box, codes
}

// Collapses the binary tree rooted at internal node `root` (n > max_leaf) into
// t's W-wide device nodes; fills perm (leaf slot -> primitive) and last.
// Returns the number of levels (one launch each).
inline int collapse_wide(BuiltTree& t, const BinaryTree& bt, int32_t root, int W, int max_leaf, int32_t* perm,
                         uint8_t* last, cudaStream_t st) {
    const int F4 = W == 8 ? NodeShape<8>::kF4 : NodeShape<4>::kF4;
    PinnedBuf<CollapseState> h_cs;
    h_cs.alloc(1);
    *h_cs.p = CollapseState{1, 1, 0, 0};
    DevBuf<CollapseState> d_cs;
    DevBuf<int4> d_qa, d_qb;
    DevBuf<float4> d_wide;
    d_cs.alloc(1);
    check(cudaMemcpyAsync(d_cs.p, h_cs.p, sizeof(CollapseState), cudaMemcpyHostToDevice, st), "collapse state");
    size_t wide_cap = size_t(std::max<int64_t>(64, bt.n / 16));
    d_wide.alloc(wide_cap * F4);
    d_qa.alloc(64);
    d_qb.alloc(64);
    const int4 root_item = make_int4(root, 0, 0, 0);
    check(cudaMemcpyAsync(d_qa.p, &root_item, sizeof(int4), cudaMemcpyHostToDevice, st), "root");
    int nq = 1, allocated = 1, levels = 0;
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
            k_collapse<8><<<grid(nq, 128), 128, 0, st>>>(nq, d_qa.p, d_qb.p, next_base, levels, max_leaf, bt, last,
                                                        perm, d_cs.p, d_wide.p);
        else
            k_collapse<4><<<grid(nq, 128), 128, 0, st>>>(nq, d_qa.p, d_qb.p, next_base, levels, max_leaf, bt, last,
                                                        perm, d_cs.p, d_wide.p);
        check(cudaGetLastError(), "collapse");
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
    cudaError_t e =
        cudaMemcpyAsync(nodes, d_wide.p, size_t(allocated) * F4 * sizeof(float4), cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        cudaFree(nodes);
        check(e, "copy nodes");
    }
    t.d_nodes = nodes;
    return levels;
}

// A tree of one leaf holding all n primitives (n <= max_leaf), in Morton order.
inline void single_leaf(BuiltTree& t, int64_t n, uint8_t* last, cudaStream_t st) {
    t.root = leaf_ref(0);
    t.depth = 1;
    t.leaves = 1;
    const uint8_t one = 1;
    check(cudaMemcpyAsync(last + (n - 1), &one, 1, cudaMemcpyHostToDevice, st), "leaf flags");
    check(cudaStreamSynchronize(st), "leaf flags");
}

// The triangle records in leaf order (perm: leaf slot -> primitive), owned by t.
inline void leaf_records(BuiltTree& t, const float* d_tri, int64_t n, const int32_t* perm, const uint8_t* last,
                         cudaStream_t st) {
    const size_t tris_bytes = size_t(n + kPadSlots) * 3 * sizeof(float4);
    float4* d_tris = nullptr;
    cudaError_t e = cudaMalloc(&d_tris, tris_bytes);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_tris + size_t(n) * 3, 0, size_t(kPadSlots) * 3 * sizeof(float4), st);
    if (e == cudaSuccess) {
        k_leaf_tris<<<grid(n), 256, 0, st>>>(n, d_tri, perm, last, d_tris);
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
}

}  // namespace
}  // namespace sg
