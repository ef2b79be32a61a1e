// Host-side wide-BVH builder producing the same tree as SORT's Fbvh::Build.
//
// The tree is split exactly as accel/fast_bvh.hpp:109-270 and
// accel/bvh_utils.h:27-118 do (16-bin SAH on the centroid bounds' longest
// axis, normalised by the parent box; breadth-first W-way split of each node;
// std::partition of the primitive list; leaves of <= max_leaf primitives or at
// max_depth), so leaf membership, leaf order and child order are identical to
// SORT's. That identity is what makes closest-hit IDs match SORT even when two
// triangles are hit at exactly the same distance.
//
// Differences from SORT, none of which change the tree:
//   * subtrees are built concurrently (each only permutes its own range);
//   * the result is a flat array form (BuiltTree) instead of unique_ptr nodes.
#pragma once

#include <vector_types.h>

#include <cstdint>
#include <vector>

namespace sg {

struct Box {
    float mn[3], mx[3];
};

constexpr int32_t kLeafBit = int32_t(0x80000000u);
constexpr int32_t kEmptyRef = -1;  // all bits set: never a valid node or leaf start

inline bool ref_is_leaf(int32_t r) { return r < 0 && r != kEmptyRef; }
inline int32_t leaf_ref(int64_t begin) { return int32_t(uint32_t(begin) | 0x80000000u); }
inline int64_t leaf_begin(int32_t r) { return int64_t(uint32_t(r) & 0x7fffffffu); }

struct BuildParams {
    int width = 8;
    int max_depth = 16;
    int max_leaf = 8;
    int threads = 0;  // 0 = hardware_concurrency
    // Primitives after the triangles (hair lines): their boxes, 6 floats each
    // (min xyz, max xyz), primitive indices ntri .. ntri + nextra - 1. SORT's
    // split rules see every primitive as its box and the box centre.
    const float* extra_boxes = nullptr;
    int64_t nextra = 0;
    // build_tree_gpu: also fill the host arrays lo / hi (the FP32 nodes are
    // written on the device either way; 8-bit nodes are made from lo / hi).
    bool host_boxes = true;
};

// Flat tree. Interior node k owns child[k*W + j] and, for child j on axis a,
// lo[(k*3 + a)*W + j] / hi[(k*3 + a)*W + j]. Interior children of a node are
// numbered consecutively (a node's first interior child is node
// first_interior[k]). Empty child slots hold kEmptyRef and the empty box
// (+FLT_MAX .. -FLT_MAX) SORT leaves in unused SIMD lanes.
struct BuiltTree {
    int width = 8;
    int depth = 0;  // Fbvh::m_depth
    Box scene{};    // enlarged scene box (core/scene.cpp:150-154)
    int32_t root = kEmptyRef;
    std::vector<int32_t> child;
    std::vector<float> lo, hi;
    std::vector<int32_t> first_interior;  // per node, -1 if none
    std::vector<int32_t> order;           // primitive index of each leaf slot (leaf order)
    std::vector<uint8_t> leaf_last;       // 1 on the last slot of every leaf
    // Set by build_tree_gpu only: the triangle records of the device layout
    // (layout.h), leaf order plus the zero pad slots, already on the build's
    // device. The receiver owns it (cudaFree).
    float4* d_tris = nullptr;
    // The interior nodes already in the device layout (layout.h, FP32 boxes),
    // owned like d_tris. Set by build_tree_lbvh and build_tree_ploc, whose host
    // arrays (child, lo, hi, first_interior, order, leaf_last) stay empty
    // (n_tri and n_interior give the sizes), and by build_tree_gpu beside its
    // host arrays (a scene with 8-bit nodes converts those instead).
    float4* d_nodes = nullptr;
    int64_t n_interior = -1, n_tri = -1;
    // Primitives from first_extra on are not triangles (hair lines, then from
    // first_shape on area shapes); -1: none. A leaf tests its triangles, then
    // its lines, then its shapes, as SORT's leaf tests its triangle packs, its
    // line packs, then its other_list.
    int64_t first_extra = -1;
    int64_t first_shape = -1;
    int rounds = 0, launches = 0;  // GPU builders: rounds (levels) and their own kernel launches
    int64_t leaves = 0;
    int64_t interior() const { return n_interior >= 0 ? n_interior : (width ? int64_t(child.size()) / width : 0); }
    int64_t triangles() const { return n_tri >= 0 ? n_tri : int64_t(order.size()); }
    bool host_arrays() const { return n_interior < 0; }
};

// Builds over ntri triangles, 9 floats each (v0, v1, v2). Throws
// std::invalid_argument / std::bad_alloc on bad input / memory exhaustion.
BuiltTree build_tree(const float* tri, int64_t ntri, const BuildParams& p);

// The same tree, built with data-parallel passes on CUDA device `device`
// (builder_gpu.cu). Throws std::invalid_argument on bad input and
// std::runtime_error on a CUDA error.
BuiltTree build_tree_gpu(const float* tri, int64_t ntri, const BuildParams& p, int device);

// A wide BVH in Morton order (LBVH), built entirely on the GPU: not SORT's
// tree (same hits except near-ties and rays whose slab test misses the hit
// triangle's own box by rounding), for fast scene admission.
// max_depth does not apply. The result has no host arrays (host_arrays()).
BuiltTree build_tree_lbvh(const float* tri, int64_t ntri, const BuildParams& p, int device);

// A wide BVH by parallel locally-ordered clustering (PLOC) over the Morton
// order, built entirely on the GPU (builder_ploc.cu): tighter boxes than the
// LBVH, the same promises and limits.
BuiltTree build_tree_ploc(const float* tri, int64_t ntri, const BuildParams& p, int device);

// 8-bit node format (quantize.cpp): one record per interior node in the layout
// layout.h describes; every decoded child box contains the FP32 box.
void quantize_nodes(const BuiltTree& t, std::vector<float4>& out);

// Pre-order topology in the oracle's comparison format:
//   interior node: [child_cnt, child0 ..., child_{n-1} ...]
//   leaf:          [0, pri_cnt, primitive indices in leaf order]
void tree_topology(const BuiltTree& t, std::vector<int32_t>& out);

}  // namespace sg
