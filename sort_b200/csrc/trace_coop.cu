// Cooperative traversal: W lanes trace one ray together, the GPU analogue of
// SORT's SIMD-across-children design (simd/simd_bbox.h:62-85 tests 4/8 child
// boxes per instruction, simd/simd_triangle.h:212-300 tests 4/8 triangles).
//
// Lane j of a group box-tests child slot j of the current node and, in a leaf,
// triangle slot j of the current chunk of W slots. The visit order and tie
// rules are SORT's, computed across the group with shuffles:
//   * pop order of the hit children: ascending entry distance, equal distances
//     higher slot first; with three or more hits only distances > -1 take part
//     (accel/fast_bvh.hpp:416-455); the first in that order is descended into,
//     the rest go to the group's stack in shared memory;
//   * a leaf keeps the nearest hit of a chunk, lowest slot on equal distances,
//     and only if strictly nearer than the current hit — the same result as
//     SORT's lane-ordered min-reduce per 4/8-pack (simd_triangle.h:359-369).
// Hits, distances and barycentrics are therefore bit-identical to SORT's.
#include <cuda_runtime.h>

#include "trace_common.cuh"
#include "trace_kernels.h"

namespace sg {

template <int W, bool ANY, int STACK, bool STATS>
__global__ void __launch_bounds__(128) k_trace_fp32_coop(DevTree tr, DevRays rays, int64_t n,
                                                         int32_t* __restrict__ prim_out, float* __restrict__ t_out,
                                                         float* __restrict__ u_out, float* __restrict__ v_out,
                                                         uint8_t* __restrict__ occ_out, int* __restrict__ err,
                                                         unsigned long long* __restrict__ stats) {
    constexpr int G = W;                // lanes per ray
    constexpr int kGroups = 128 / G;    // rays per block
    constexpr unsigned kLow = (1u << G) - 1u;
    extern __shared__ uint2 smem_stack[];

    const int lane = threadIdx.x & 31;
    const int j = lane & (G - 1);
    const int shift = lane & ~(G - 1);  // first lane of this group in the warp
    const unsigned gmask = kLow << shift;
    const int group = threadIdx.x / G;
    uint2* stk = smem_stack + group * STACK;
    const int64_t i = (int64_t)blockIdx.x * kGroups + group;
    if (i >= n) return;  // whole group leaves together

    RayState r;
    r.o[0] = rays.ox[i];
    r.o[1] = rays.oy[i];
    r.o[2] = rays.oz[i];
    r.d[0] = rays.dx[i];
    r.d[1] = rays.dy[i];
    r.d[2] = rays.dz[i];
    r.tmin = rays.tmin[i];
    r.tmax = rays.tmax[i];
    ray_setup(r);

    float best_t = FLT_MAX, best_u = 0.0f, best_v = 0.0f;
    int32_t best_prim = -1;
    unsigned node_tests = 0, prim_tests = 0;

    const float f0 = root_intersect(r, tr.box_lo, tr.box_hi);
    if (f0 >= 0.0f && tr.root != kEmpty) {
        int si = 0;
        int32_t cur = tr.root;
        float cur_d = f0;
        bool finished = false;
        for (;;) {
            bool descend = false;
            if (!(best_t < cur_d)) {  // fast_bvh.hpp:343: skip when the hit is nearer than the entry
                if (cur < 0) {
                    // Leaf: chunks of G slots, lane j takes slot s + j.
                    int64_t s = (int64_t)((uint32_t)cur & 0x7fffffffu);
                    for (;;) {
                        const float4* q = tr.tris + 3 * (s + j);
                        const float4 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2);
                        const unsigned lastm = (__ballot_sync(gmask, __float_as_int(b.w) != 0) >> shift) & kLow;
                        const int e = lastm ? __ffs(lastm) - 1 : G - 1;  // last slot of the leaf in this chunk
                        float t = FLT_MAX, u = 0.0f, v = 0.0f;
                        const bool hit = j <= e && tri_test(r, a, b, c, t, u, v) && t < best_t;
                        if (STATS) prim_tests += (unsigned)(e + 1);
                        if (ANY) {
                            if (__ballot_sync(gmask, hit)) {
                                best_prim = 0;
                                finished = true;
                                if (STATS && !lastm) {  // SORT counts the whole leaf
                                    for (int64_t s2 = s + G;; s2 += G) {
                                        const float4 b2 = __ldg(tr.tris + 3 * (s2 + j) + 1);
                                        const unsigned l2 = (__ballot_sync(gmask, __float_as_int(b2.w) != 0) >> shift) & kLow;
                                        prim_tests += l2 ? (unsigned)__ffs(l2) : (unsigned)G;
                                        if (l2) break;
                                    }
                                }
                                break;
                            }
                        } else {
                            // nearest hit of the chunk, lowest slot on ties
                            float kt = hit ? t : __int_as_float(0x7f800000);
                            int kj = j;
#pragma unroll
                            for (int off = G / 2; off > 0; off >>= 1) {
                                const float ot = __shfl_xor_sync(gmask, kt, off, G);
                                const int oj = __shfl_xor_sync(gmask, kj, off, G);
                                if (ot < kt || (ot == kt && oj < kj)) {
                                    kt = ot;
                                    kj = oj;
                                }
                            }
                            const float bu = __shfl_sync(gmask, u, kj, G);
                            const float bv = __shfl_sync(gmask, v, kj, G);
                            const int bp = __shfl_sync(gmask, __float_as_int(a.w), kj, G);
                            if (kt < best_t) {
                                best_t = kt;
                                best_u = bu;
                                best_v = bv;
                                best_prim = bp;
                            }
                        }
                        if (lastm) break;
                        s += G;
                    }
                    if (ANY && finished) break;
                } else {
                    if (si + W > STACK) {  // cannot happen when STACK >= depth*(W-1)+1; reported, never overrun
                        if (j == 0) atomicOr(err, 1);
                        break;
                    }
                    if (STATS) ++node_tests;
                    const float4* p = tr.nodes + (size_t)cur * NodeShape<W>::kF4 + 2 * j;
                    const float4 lo = __ldg(p), hi = __ldg(p + 1);
                    const int32_t ref = __float_as_int(lo.w);
                    float d;
                    const bool hit = slab(r, lo.x, hi.x, lo.y, hi.y, lo.z, hi.z, d) && ref != kEmpty;
                    const unsigned m = (__ballot_sync(gmask, hit) >> shift) & kLow;
                    const int cnt = __popc(m);
                    if (cnt > 0) {
                        const unsigned P = cnt > 2 ? ((__ballot_sync(gmask, hit && d > -1.0f) >> shift) & kLow) : m;
                        const int count = __popc(P);
                        if (count > 0) {
                            const bool part = (P >> j) & 1u;
                            int pos = 0;  // entries that pop before this one
#pragma unroll
                            for (int k = 0; k < G; ++k) {
                                const float dk = __shfl_sync(gmask, d, k, G);
                                pos += (((P >> k) & 1u) && (dk < d || (dk == d && k > j))) ? 1 : 0;
                            }
                            if (part && pos > 0) stk[si + count - 1 - pos] = make_uint2((uint32_t)ref, __float_as_uint(d));
                            const unsigned nm = (__ballot_sync(gmask, part && pos == 0) >> shift) & kLow;
                            const int src = __ffs(nm) - 1;
                            cur = __shfl_sync(gmask, ref, src, G);
                            cur_d = __shfl_sync(gmask, d, src, G);
                            si += count - 1;
                            descend = true;
                            __syncwarp(gmask);
                        }
                    }
                }
            }
            if (!descend) {
                if (si == 0) break;
                const uint2 e = stk[--si];
                cur = (int32_t)e.x;
                cur_d = __uint_as_float(e.y);
            }
        }
    }

    if (j == 0) {
        if (STATS) {
            atomicAdd(stats, (unsigned long long)node_tests);
            atomicAdd(stats + 1, (unsigned long long)prim_tests);
        }
        if (ANY) {
            occ_out[i] = best_prim >= 0 ? 1 : 0;
        } else {
            prim_out[i] = best_prim;
            t_out[i] = best_prim >= 0 ? best_t : FLT_MAX;
            if (u_out) u_out[i] = best_prim >= 0 ? best_u : 0.0f;
            if (v_out) v_out[i] = best_prim >= 0 ? best_v : 0.0f;
        }
    }
}

template <int W, bool ANY, int STACK, bool STATS>
static cudaError_t launch_coop_stack(const TraceLaunch& L, const DevTree& tr, const DevRays& rays, int64_t n,
                                     cudaStream_t s) {
    constexpr int kThreads = 128;
    constexpr int kGroups = kThreads / W;
    const size_t smem = sizeof(uint2) * kGroups * STACK;
    auto kernel = k_trace_fp32_coop<W, ANY, STACK, STATS>;
    if (smem > 48 * 1024) {
        const cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    const int64_t blocks = (n + kGroups - 1) / kGroups;
    kernel<<<(unsigned)blocks, kThreads, smem, s>>>(tr, rays, n, L.prim, L.t, L.u, L.v, L.occ, L.err, L.stats);
    return cudaGetLastError();
}

template <int W, bool ANY, bool STATS>
static cudaError_t launch_coop_w(const TraceLaunch& L, const DevTree& tr, const DevRays& rays, int64_t n,
                                 cudaStream_t s) {
    if (L.stack_need <= 64) return launch_coop_stack<W, ANY, 64, STATS>(L, tr, rays, n, s);
    if (L.stack_need <= 128) return launch_coop_stack<W, ANY, 128, STATS>(L, tr, rays, n, s);
    if (L.stack_need <= 256) return launch_coop_stack<W, ANY, 256, STATS>(L, tr, rays, n, s);
    return cudaErrorInvalidValue;
}

template <bool STATS>
static cudaError_t launch_coop_any(const TraceLaunch& L, const DevTree& tr, const DevRays& rays, int64_t n,
                                   cudaStream_t s) {
    if (L.width == 8)
        return L.any ? launch_coop_w<8, true, STATS>(L, tr, rays, n, s) : launch_coop_w<8, false, STATS>(L, tr, rays, n, s);
    return L.any ? launch_coop_w<4, true, STATS>(L, tr, rays, n, s) : launch_coop_w<4, false, STATS>(L, tr, rays, n, s);
}

cudaError_t launch_trace_fp32_coop(const TraceLaunch& L, const DevTree& tr, const DevRays& rays, int64_t n,
                                   cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    return L.stats ? launch_coop_any<true>(L, tr, rays, n, s) : launch_coop_any<false>(L, tr, rays, n, s);
}

}  // namespace sg
