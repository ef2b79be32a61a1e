// build_tree_lbvh: a wide BVH in Morton order, built entirely on the GPU.
//
// The fast builder for scenes that must be admitted quickly. Its tree is not
// SORT's (build_tree / build_tree_gpu build that one): hits and distances equal
// SORT's, because the box and triangle tests are the same, except near-ties
// (two triangles hit within rounding of each other, 1e-6 of the distance or
// more when the ray starts close to large triangles: a rounded box entry
// distance decides which one a traversal keeps), and where SORT's slab test
// (with its 1e-5 clamp of direction components) misses a hit triangle's own box
// by rounding: such a triangle is found only through a larger leaf box, which
// depends on the tree.
//
//   1. primitive boxes and centroids, the scene box (SORT's, enlarged by 0.1%,
//      core/scene.cpp:146-154) and the centroid bounds;
//   2. 63-bit Morton codes of the centroids (21 bits per axis over the
//      centroid bounds), sorted with their primitive indices (the stable
//      radix sort of prefix_sort.cuh);
//   3. the binary radix tree over the sorted codes, one thread per internal
//      node (the split is where the common prefix of the codes ends; equal
//      codes are told apart by their positions);
//   4. node boxes bottom-up: one thread per primitive climbs towards the root,
//      and of the two threads that reach a node the second one (by an atomic
//      counter) writes its box, so no thread ever waits;
//   5. the W-wide tree top-down (morton_tree.cuh, shared with the PLOC
//      builder): a child that covers at most max_leaf primitives is a leaf;
//      a subtree's primitives are contiguous in Morton order, so the leaf
//      order is Morton order. Nodes are written straight into the device
//      layout (layout.h);
//   6. the leaf-order triangle records.
// Steps 1, 2, 5 and 6 live in morton_tree.cuh.
// The host reads one count per level of the wide tree; nothing else crosses
// to the host. max_depth does not apply (it is part of SORT's split rules).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <stdexcept>

#include "morton_tree.cuh"

namespace sg {
namespace {

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
                             int32_t* __restrict__ parent_leaf, int32_t* __restrict__ count) {
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
    count[i] = int32_t(hi - lo + 1);
    if (lc < 0)
        parent_leaf[~lc] = int32_t(i);
    else
        parent_int[lc] = int32_t(i);
    if (rc < 0)
        parent_leaf[~rc] = int32_t(i);
    else
        parent_int[rc] = int32_t(i);
}

// Boxes of the internal nodes, bottom-up (the second thread to reach a node
// writes it; visits must start at zero).
__global__ void k_boxes_up(BinaryTree bt, const int32_t* __restrict__ parent_int,
                           const int32_t* __restrict__ parent_leaf, int* __restrict__ visits,
                           float* __restrict__ ibox) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= bt.n) return;
    int32_t p = parent_leaf[j];
    for (;;) {
        __threadfence();
        if (atomicAdd(&visits[p], 1) == 0) return;  // the sibling's box is not written yet
        float a[6], b[6];
        load_box(bt, bt.left[p], a);
        load_box(bt, bt.right[p], b);
        for (int k = 0; k < 3; ++k) {
            __stcg(ibox + int64_t(p) * 6 + k, fminf(a[k], b[k]));
            __stcg(ibox + int64_t(p) * 6 + 3 + k, fmaxf(a[3 + k], b[3 + k]));
        }
        if (p == 0) return;
        p = parent_int[p];
    }
}

}  // namespace

BuiltTree build_tree_lbvh(const float* tri, int64_t ntri, const BuildParams& p, int device) {
    if (p.width != 4 && p.width != 8) throw std::invalid_argument("width must be 4 or 8");
    if (p.max_leaf < 1) throw std::invalid_argument("max_leaf must be >= 1");
    if (ntri < 0 || ntri >= int64_t(0x7fffffff)) throw std::invalid_argument("triangle count out of range");
    if (p.nextra != 0) throw std::invalid_argument("the LBVH builder takes triangles only");
    const int W = p.width;
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

    MortonPrims m;
    morton_prims(m, tri, n, st);
    t.scene = m.scene;
    if (n == 0) return t;
    int launches = m.launches;

    DevBuf<int32_t> d_left, d_right, d_pint, d_pleaf, d_count, d_perm;
    DevBuf<float> d_ibox;
    DevBuf<int> d_visits;
    DevBuf<uint8_t> d_last;
    d_last.alloc(size_t(n));
    check(cudaMemsetAsync(d_last.p, 0, size_t(n), st), "leaf flags");
    int levels = 0;
    const int32_t* perm = m.sorted.p;  // one leaf: Morton order
    if (n <= p.max_leaf) {
        single_leaf(t, n, d_last.p, st);
    } else {
        const int64_t ni = n - 1;  // internal nodes of the binary tree
        d_left.alloc(size_t(ni));
        d_right.alloc(size_t(ni));
        d_pint.alloc(size_t(ni));
        d_pleaf.alloc(size_t(n));
        d_count.alloc(size_t(ni));
        d_ibox.alloc(size_t(ni) * 6);
        d_visits.alloc(size_t(ni));
        d_perm.alloc(size_t(n));
        check(cudaMemsetAsync(d_visits.p, 0, size_t(ni) * sizeof(int), st), "visits");
        const BinaryTree bt{d_left.p, d_right.p, d_count.p, d_ibox.p, m.sorted.p, m.pb.p, n};
        k_radix_tree<<<grid(ni), 256, 0, st>>>(n, m.keys_sorted.p, d_left.p, d_right.p, d_pint.p, d_pleaf.p,
                                               d_count.p);
        k_boxes_up<<<grid(n), 256, 0, st>>>(bt, d_pint.p, d_pleaf.p, d_visits.p, d_ibox.p);
        check(cudaGetLastError(), "radix tree");
        launches += 2;
        levels = collapse_wide(t, bt, 0, W, p.max_leaf, d_perm.p, d_last.p, st);
        launches += levels;
        perm = d_perm.p;
    }
    leaf_records(t, m.tri.p, n, perm, d_last.p, st);
    t.rounds = levels;
    t.launches = launches + 1;
    return t;
}

}  // namespace sg
