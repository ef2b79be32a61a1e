// build_tree_ploc: a wide BVH by parallel locally-ordered clustering (PLOC;
// D. Meister and J. Bittner, "Parallel Locally-Ordered Clustering for Bounding
// Volume Hierarchy Construction", IEEE TVCG 24(3), 2018), built entirely on
// the GPU. Like the LBVH builder its tree is not SORT's (same hits and
// distances except near-ties and box-grazing rays, as build_tree_lbvh
// documents); it is built bottom-up by merging nearby clusters of small
// union area, so its boxes are tighter than the radix tree's.
//
//   1. primitive boxes, the scene box and the Morton order of the primitives
//      (morton_tree.cuh);
//   2. one cluster per primitive, in Morton order. Each iteration, until one
//      cluster remains:
//      a. every cluster picks, among the clusters at most kRadius positions
//         away in the current order, the one whose union box has the smallest
//         surface area (equal areas: the lower position). A block reads its
//         clusters and kRadius more on each side into shared memory once;
//      b. two clusters that pick each other merge into a new internal node:
//         the one at the lower position takes the node, the other leaves.
//         Each position is read only by its own thread and by its partner, so
//         the merge updates the cluster array in place;
//      c. the remaining clusters are compacted in order (prefix sum of the
//         keep flags, prefix_sort.cuh).
//      The pair that is closest over all (area, then positions) always picks
//      each other, so every iteration merges at least one pair;
//   3. the W-wide tree top-down and the leaf-order triangle records
//      (morton_tree.cuh): leaf slots follow the binary tree left to right.
// The host reads the cluster count once per iteration and one count per
// level of the wide tree. max_depth does not apply (it is part of SORT's
// split rules).
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cstdint>
#include <stdexcept>

#include "morton_tree.cuh"

namespace sg {
namespace {

constexpr int kRadius = 16;        // neighbours searched on each side
constexpr int kNearThreads = 256;  // clusters per block in the search

// Cluster i: rec[2i] = {min x, y, z (float bits), binary reference},
// rec[2i + 1] = {max x, y, z (float bits), primitive count}.
__global__ void k_ploc_init(int64_t n, const int32_t* __restrict__ sorted, const float* __restrict__ pb,
                            int4* __restrict__ rec) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t p = sorted[i];
    rec[2 * i] = make_int4(__float_as_int(pb[p]), __float_as_int(pb[n + p]), __float_as_int(pb[2 * n + p]),
                           ~int32_t(i));
    rec[2 * i + 1] = make_int4(__float_as_int(pb[3 * n + p]), __float_as_int(pb[4 * n + p]),
                               __float_as_int(pb[5 * n + p]), 1);
}

__device__ __forceinline__ float union_area(const float4& alo, const float4& ahi, const float4& blo,
                                            const float4& bhi) {
    const float x = fmaxf(ahi.x, bhi.x) - fminf(alo.x, blo.x);
    const float y = fmaxf(ahi.y, bhi.y) - fminf(alo.y, blo.y);
    const float z = fmaxf(ahi.z, bhi.z) - fminf(alo.z, blo.z);
    const float a = x * y + y * z + z * x;
    return a == a ? a : FLT_MAX * 2.0f;  // NaN (infinite extents) orders as +inf
}

__device__ __forceinline__ float4 planes(const int4& r) {
    return make_float4(__int_as_float(r.x), __int_as_float(r.y), __int_as_float(r.z), 0.0f);
}

// nn[i] = the position cluster i picks (step 2a).
__global__ void __launch_bounds__(kNearThreads) k_ploc_nearest(int nc, const int4* __restrict__ rec,
                                                              int32_t* __restrict__ nn) {
    __shared__ float4 s_lo[kNearThreads + 2 * kRadius], s_hi[kNearThreads + 2 * kRadius];
    const int base = blockIdx.x * kNearThreads;
    for (int k = threadIdx.x; k < kNearThreads + 2 * kRadius; k += kNearThreads) {
        const int g = base - kRadius + k;
        if (g >= 0 && g < nc) {
            s_lo[k] = planes(rec[2 * g]);
            s_hi[k] = planes(rec[2 * g + 1]);
        }
    }
    __syncthreads();
    const int i = base + threadIdx.x;
    if (i >= nc) return;
    const float4 lo = s_lo[threadIdx.x + kRadius], hi = s_hi[threadIdx.x + kRadius];
    const int j0 = max(0, i - kRadius), j1 = min(nc - 1, i + kRadius);
    float best = 0.0f;
    int bj = -1;
    for (int j = j0; j <= j1; ++j) {
        if (j == i) continue;
        const int k = j - base + kRadius;
        const float a = union_area(lo, hi, s_lo[k], s_hi[k]);
        if (bj < 0 || a < best) {  // ascending j: equal areas keep the lower position
            best = a;
            bj = j;
        }
    }
    nn[i] = bj;
}

// Step 2b: a mutual pair merges into a new internal node at the lower
// position; keep[i] = 0 for the position that leaves.
__global__ void __launch_bounds__(256) k_ploc_merge(int nc, int4* __restrict__ rec, const int32_t* __restrict__ nn,
                                                    uint32_t* __restrict__ keep, int32_t* __restrict__ left,
                                                    int32_t* __restrict__ right, int32_t* __restrict__ count,
                                                    float* __restrict__ ibox, int* __restrict__ nodes) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    bool host = false, gone = false;
    int j = -1;
    if (i < nc) {
        j = nn[i];
        const bool mutual = nn[j] == i;
        host = mutual && i < j;
        gone = mutual && j < i;
    }
    const unsigned lane = threadIdx.x & 31u;
    const unsigned hosts = __ballot_sync(0xffffffffu, host);
    int first = 0;
    if (lane == 0 && hosts) first = atomicAdd(nodes, __popc(hosts));
    first = __shfl_sync(0xffffffffu, first, 0);
    if (i >= nc) return;
    keep[i] = gone ? 0u : 1u;
    if (!host) return;
    const int id = first + __popc(hosts & ((1u << lane) - 1u));
    const int4 alo = rec[2 * i], ahi = rec[2 * i + 1], blo = rec[2 * j], bhi = rec[2 * j + 1];
    float u[6];
    u[0] = fminf(__int_as_float(alo.x), __int_as_float(blo.x));
    u[1] = fminf(__int_as_float(alo.y), __int_as_float(blo.y));
    u[2] = fminf(__int_as_float(alo.z), __int_as_float(blo.z));
    u[3] = fmaxf(__int_as_float(ahi.x), __int_as_float(bhi.x));
    u[4] = fmaxf(__int_as_float(ahi.y), __int_as_float(bhi.y));
    u[5] = fmaxf(__int_as_float(ahi.z), __int_as_float(bhi.z));
    const int32_t cnt = ahi.w + bhi.w;
    left[id] = alo.w;
    right[id] = blo.w;
    count[id] = cnt;
    for (int a = 0; a < 6; ++a) ibox[int64_t(id) * 6 + a] = u[a];
    rec[2 * i] = make_int4(__float_as_int(u[0]), __float_as_int(u[1]), __float_as_int(u[2]), id);
    rec[2 * i + 1] = make_int4(__float_as_int(u[3]), __float_as_int(u[4]), __float_as_int(u[5]), cnt);
}

// Step 2c: kept clusters to their prefix-sum positions; the new count.
__global__ void k_ploc_compact(int nc, const int4* __restrict__ rec, const uint32_t* __restrict__ keep,
                               const uint32_t* __restrict__ pos, int4* __restrict__ out, int* __restrict__ nc_out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nc) return;
    const uint32_t k = keep[i], p = pos[i];
    if (k) {
        out[2 * p] = rec[2 * i];
        out[2 * p + 1] = rec[2 * i + 1];
    }
    if (i == nc - 1) *nc_out = int(p + k);
}

}  // namespace

BuiltTree build_tree_ploc(const float* tri, int64_t ntri, const BuildParams& p, int device) {
    if (p.width != 4 && p.width != 8) throw std::invalid_argument("width must be 4 or 8");
    if (p.max_leaf < 1) throw std::invalid_argument("max_leaf must be >= 1");
    if (ntri < 0 || ntri >= int64_t(0x7fffffff)) throw std::invalid_argument("triangle count out of range");
    if (p.nextra != 0) throw std::invalid_argument("the PLOC builder takes triangles only");
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

    DevBuf<uint8_t> d_last;
    d_last.alloc(size_t(n));
    check(cudaMemsetAsync(d_last.p, 0, size_t(n), st), "leaf flags");
    int levels = 0, iterations = 0;
    DevBuf<int32_t> d_left, d_right, d_count, d_nn, d_perm;
    DevBuf<float> d_ibox;
    DevBuf<int4> d_rec[2];
    DevBuf<uint32_t> d_keep, d_pos, d_scan;
    DevBuf<int> d_ctr;
    PinnedBuf<int> h_ctr;
    const int32_t* perm = m.sorted.p;  // one leaf: Morton order
    if (n <= p.max_leaf) {
        single_leaf(t, n, d_last.p, st);
    } else {
        const int64_t ni = n - 1;  // internal nodes of the binary tree
        d_left.alloc(size_t(ni));
        d_right.alloc(size_t(ni));
        d_count.alloc(size_t(ni));
        d_ibox.alloc(size_t(ni) * 6);
        d_nn.alloc(size_t(n));
        d_rec[0].alloc(size_t(n) * 2);
        d_rec[1].alloc(size_t(n) * 2);
        d_keep.alloc(size_t(n));
        d_pos.alloc(size_t(n));
        d_scan.alloc(std::max<size_t>(psort::scan_scratch_words(size_t(n)), 8));  // covers every smaller count too
        d_ctr.alloc(2);  // [0] internal nodes made, [1] clusters left
        h_ctr.alloc(4);
        d_perm.alloc(size_t(n));
        check(cudaMemsetAsync(d_ctr.p, 0, 2 * sizeof(int), st), "counters");
        k_ploc_init<<<grid(n), 256, 0, st>>>(n, m.sorted.p, m.pb.p, d_rec[0].p);
        check(cudaGetLastError(), "clusters");
        ++launches;
        int nc = int(n), cur = 0;
        while (nc > 1) {
            k_ploc_nearest<<<grid(nc, kNearThreads), kNearThreads, 0, st>>>(nc, d_rec[cur].p, d_nn.p);
            k_ploc_merge<<<grid(nc), 256, 0, st>>>(nc, d_rec[cur].p, d_nn.p, d_keep.p, d_left.p, d_right.p,
                                                   d_count.p, d_ibox.p, d_ctr.p);
            check(cudaGetLastError(), "cluster merge");
            check(psort::scan_exclusive(d_keep.p, d_pos.p, size_t(nc), d_scan.p, st), "cluster scan");
            k_ploc_compact<<<grid(nc), 256, 0, st>>>(nc, d_rec[cur].p, d_keep.p, d_pos.p, d_rec[1 - cur].p,
                                                     d_ctr.p + 1);
            check(cudaGetLastError(), "cluster compaction");
            check(cudaMemcpyAsync(h_ctr.p, d_ctr.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, st), "cluster count");
            check(cudaStreamSynchronize(st), "cluster count");
            launches += 4 + (nc > psort::kScanTile ? 3 : 1);  // search, merge, scan, compaction
            ++iterations;
            if (h_ctr.p[1] >= nc || h_ctr.p[1] < 1)
                throw std::runtime_error("PLOC iteration merged no clusters");
            nc = h_ctr.p[1];
            cur = 1 - cur;
        }
        if (h_ctr.p[0] != ni) throw std::runtime_error("PLOC made a wrong number of internal nodes");
        int4 root_rec;
        check(cudaMemcpyAsync(&root_rec, d_rec[cur].p, sizeof(int4), cudaMemcpyDeviceToHost, st), "root");
        check(cudaStreamSynchronize(st), "root");
        const BinaryTree bt{d_left.p, d_right.p, d_count.p, d_ibox.p, m.sorted.p, m.pb.p, n};
        levels = collapse_wide(t, bt, root_rec.w, W, p.max_leaf, d_perm.p, d_last.p, st);
        launches += levels;
        perm = d_perm.p;
    }
    leaf_records(t, m.tri.p, n, perm, d_last.p, st);
    t.rounds = iterations + levels;
    t.launches = launches + 1;
    return t;
}

}  // namespace sg
