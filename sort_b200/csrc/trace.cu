// Closest-hit and any-hit traversal of SORT-topology wide BVHs on sm_100a.
//
// One ray per thread. The traversal restates Fbvh::GetIntersect
// (accel/fast_bvh.hpp:305-504, SIMD branch):
//   * root slab test against the enlarged scene box (scalar Intersect);
//   * a stack of (node, entry distance) pairs; a popped entry is skipped when
//     the current hit is nearer than its entry distance (strict <, line 343);
//   * a leaf tests its triangles in SIMD-lane packing order and keeps a hit only
//     when strictly nearer (simd/simd_triangle.h:359-369), so the first of equal
//     distances wins;
//   * an interior node's hit children are pushed so the nearest pops first; equal
//     distances pop the higher child slot first (the 1-, 2- and >=3-hit cases of
//     lines 416-455 all reduce to that order);
//   * any-hit returns at the first triangle hit (opaque early exit, 362-373).
// With FP32 child boxes and the same rounding, hits, distances and barycentrics
// are bit-identical to SORT's.
#include <cuda_runtime.h>

#include "trace_common.cuh"
#include "trace_kernels.h"

namespace sg {

template <int W>
struct NodeData {
    float lo[3][W], hi[3][W];
    int32_t ch[W];
};

template <int W>
__device__ __forceinline__ void load_node(const float4* __restrict__ nodes, int32_t ref, NodeData<W>& nd) {
    const float4* p = nodes + (size_t)ref * NodeShape<W>::kF4;
    constexpr int Q = W / 4;  // float4 per plane
#pragma unroll
    for (int a = 0; a < 3; ++a) {
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const float4 l = __ldg(p + (2 * a) * Q + q);
            const float4 h = __ldg(p + (2 * a + 1) * Q + q);
            nd.lo[a][4 * q + 0] = l.x;
            nd.lo[a][4 * q + 1] = l.y;
            nd.lo[a][4 * q + 2] = l.z;
            nd.lo[a][4 * q + 3] = l.w;
            nd.hi[a][4 * q + 0] = h.x;
            nd.hi[a][4 * q + 1] = h.y;
            nd.hi[a][4 * q + 2] = h.z;
            nd.hi[a][4 * q + 3] = h.w;
        }
    }
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int4 c = __ldg(reinterpret_cast<const int4*>(p + 6 * Q + q));
        nd.ch[4 * q + 0] = c.x;
        nd.ch[4 * q + 1] = c.y;
        nd.ch[4 * q + 2] = c.z;
        nd.ch[4 * q + 3] = c.w;
    }
}

// STATS adds SORT's traversal counters (accel/fast_bvh.hpp:50-96): interior
// nodes box-tested, and primitives tested counted per leaf entered
// (sIntersectionTest += pri_cnt), accumulated into stats[0] / stats[1].
//
// Two GPU-side changes leave SORT's visit order intact:
//   * the entry SORT would pop right after pushing an interior node's children
//     (the nearest one) is kept in registers and descended into directly; only
//     the others go to the stack, so a descent costs no stack round trip;
//   * leaf triangles are fetched two at a time (the triangle array carries one
//     padding slot), so the loads of the second overlap the test of the first.
template <int W, bool ANY, int STACK, bool STATS>
__global__ void __launch_bounds__(128) k_trace_fp32(DevTree tr, DevRays rays, int64_t n, int32_t* __restrict__ prim_out,
                                                    float* __restrict__ t_out, float* __restrict__ u_out,
                                                    float* __restrict__ v_out, uint8_t* __restrict__ occ_out,
                                                    int* __restrict__ err, unsigned long long* __restrict__ stats) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;

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
        uint2 stk[STACK];
        int si = 0;
        int32_t cur = tr.root;
        float cur_d = f0;
        bool done = false;
        for (;;) {
            bool descend = false;
            if (!(best_t < cur_d)) {  // fast_bvh.hpp:343: skip when the hit is nearer than the entry
                if (cur < 0) {
                    int64_t s = (int64_t)((uint32_t)cur & 0x7fffffffu);
                    unsigned tested = 0;
                    for (;;) {
                        const float4* q = tr.tris + 3 * s;
                        const float4 a0 = __ldg(q), b0 = __ldg(q + 1), c0 = __ldg(q + 2);
                        const float4 a1 = __ldg(q + 3), b1 = __ldg(q + 4), c1 = __ldg(q + 5);
                        float t, u, v;
                        ++tested;
                        if (tri_test(r, a0, b0, c0, t, u, v) && t < best_t) {
                            best_t = t;
                            best_u = u;
                            best_v = v;
                            best_prim = __float_as_int(a0.w);
                            if (ANY) {
                                done = true;
                                break;
                            }
                        }
                        if (__float_as_int(b0.w)) break;
                        ++tested;
                        if (tri_test(r, a1, b1, c1, t, u, v) && t < best_t) {
                            best_t = t;
                            best_u = u;
                            best_v = v;
                            best_prim = __float_as_int(a1.w);
                            if (ANY) {
                                ++s;
                                done = true;
                                break;
                            }
                        }
                        if (__float_as_int(b1.w)) break;
                        s += 2;
                    }
                    if (STATS) {
                        if (ANY && done)  // whole leaf, as SORT counts it
                            for (int64_t q = s; !__float_as_int(__ldg(tr.tris + 3 * q + 1).w); ++q) ++tested;
                        prim_tests += tested;
                    }
                    if (ANY && done) break;
                } else {
                    if (si + W > STACK) {  // cannot happen when STACK >= depth*(W-1)+1; reported, never overrun
                        atomicOr(err, 1);
                        break;
                    }
                    NodeData<W> nd;
                    load_node<W>(tr.nodes, cur, nd);
                    if (STATS) ++node_tests;
                    float d[W];
                    unsigned mask = 0;
#pragma unroll
                    for (int j = 0; j < W; ++j) {
                        const bool hit =
                            slab(r, nd.lo[0][j], nd.hi[0][j], nd.lo[1][j], nd.hi[1][j], nd.lo[2][j], nd.hi[2][j], d[j]);
                        if (hit && nd.ch[j] != kEmpty) mask |= 1u << j;
                    }
                    const int cnt = __popc(mask);
                    if (cnt == 1) {
#pragma unroll
                        for (int j = 0; j < W; ++j)
                            if (mask & (1u << j)) {
                                cur = nd.ch[j];
                                cur_d = d[j];
                            }
                        descend = true;
                    } else if (cnt == 2) {
                        // SORT pushes the far one first (t0 < t1) or the second slot last
                        // (otherwise); the one it would pop next is descended into.
                        int32_t c0 = 0, c1 = 0;
                        float t0 = 0.0f, t1 = 0.0f;
                        bool first = true;
#pragma unroll
                        for (int j = 0; j < W; ++j) {
                            if (mask & (1u << j)) {
                                if (first) {
                                    c0 = nd.ch[j];
                                    t0 = d[j];
                                    first = false;
                                } else {
                                    c1 = nd.ch[j];
                                    t1 = d[j];
                                }
                            }
                        }
                        if (t0 < t1) {
                            stk[si++] = make_uint2((uint32_t)c1, __float_as_uint(t1));
                            cur = c0;
                            cur_d = t0;
                        } else {
                            stk[si++] = make_uint2((uint32_t)c0, __float_as_uint(t0));
                            cur = c1;
                            cur_d = t1;
                        }
                        descend = true;
                    } else if (cnt > 2) {
                        // Selection by decreasing distance, ties lowest slot first; only
                        // entries with distance > -1 take part (fast_bvh.hpp:438-453).
                        int count = 0;
#pragma unroll
                        for (int j = 0; j < W; ++j) count += ((mask & (1u << j)) && d[j] > -1.0f) ? 1 : 0;
#pragma unroll
                        for (int j = 0; j < W; ++j) {
                            const bool hj = (mask & (1u << j)) && d[j] > -1.0f;
                            int rank = 0;
#pragma unroll
                            for (int k = 0; k < W; ++k) {
                                const bool hk = (mask & (1u << k)) && d[k] > -1.0f;
                                rank += (hk && (d[k] > d[j] || (d[k] == d[j] && k < j))) ? 1 : 0;
                            }
                            if (hj) {
                                if (rank == count - 1) {
                                    cur = nd.ch[j];
                                    cur_d = d[j];
                                } else {
                                    stk[si + rank] = make_uint2((uint32_t)nd.ch[j], __float_as_uint(d[j]));
                                }
                            }
                        }
                        if (count > 0) {
                            si += count - 1;
                            descend = true;
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

template <int W, bool ANY, bool STATS>
static cudaError_t launch_w(const DevTree& tr, const DevRays& rays, int64_t n, int stack_need, int32_t* prim, float* t,
                            float* u, float* v, uint8_t* occ, int* err, unsigned long long* stats, cudaStream_t s) {
    const int threads = 128;
    const int64_t blocks = (n + threads - 1) / threads;
    if (stack_need <= 64)
        k_trace_fp32<W, ANY, 64, STATS><<<(unsigned)blocks, threads, 0, s>>>(tr, rays, n, prim, t, u, v, occ, err, stats);
    else if (stack_need <= 128)
        k_trace_fp32<W, ANY, 128, STATS><<<(unsigned)blocks, threads, 0, s>>>(tr, rays, n, prim, t, u, v, occ, err, stats);
    else if (stack_need <= 256)
        k_trace_fp32<W, ANY, 256, STATS><<<(unsigned)blocks, threads, 0, s>>>(tr, rays, n, prim, t, u, v, occ, err, stats);
    else
        return cudaErrorInvalidValue;
    return cudaGetLastError();
}

template <bool STATS>
static cudaError_t launch_any_width(int width, bool any, const DevTree& tr, const DevRays& rays, int64_t n,
                                    int stack_need, int32_t* prim, float* t, float* u, float* v, uint8_t* occ, int* err,
                                    unsigned long long* stats, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    if (width == 8)
        return any ? launch_w<8, true, STATS>(tr, rays, n, stack_need, prim, t, u, v, occ, err, stats, s)
                   : launch_w<8, false, STATS>(tr, rays, n, stack_need, prim, t, u, v, occ, err, stats, s);
    return any ? launch_w<4, true, STATS>(tr, rays, n, stack_need, prim, t, u, v, occ, err, stats, s)
               : launch_w<4, false, STATS>(tr, rays, n, stack_need, prim, t, u, v, occ, err, stats, s);
}

cudaError_t launch_trace_fp32(int width, bool any, const DevTree& tr, const DevRays& rays, int64_t n, int stack_need,
                              int32_t* prim, float* t, float* u, float* v, uint8_t* occ, int* err, cudaStream_t s) {
    return launch_any_width<false>(width, any, tr, rays, n, stack_need, prim, t, u, v, occ, err, nullptr, s);
}

cudaError_t launch_trace_fp32_stats(int width, bool any, const DevTree& tr, const DevRays& rays, int64_t n,
                                    int stack_need, int32_t* prim, float* t, float* u, float* v, uint8_t* occ,
                                    int* err, unsigned long long* stats, cudaStream_t s) {
    return launch_any_width<true>(width, any, tr, rays, n, stack_need, prim, t, u, v, occ, err, stats, s);
}

}  // namespace sg
