// sg_trace_multi: SORT's BSSRDF probe query, batched.
//
// Restates Fbvh::GetIntersect(const Ray&, BSSRDFIntersections&, RenderContext&,
// StringID) (accel/fast_bvh.hpp:656-819, SIMD branch) with
// intersectTriangleMulti_SIMD (simd/simd_triangle.h:412-455): the traversal
// of the closest-hit query (same near-first order), culling an entry when the
// farthest kept hit is nearer than it (intersect.maxt < fmin), and at a leaf,
// one pack of W triangles at a time (SORT's Triangle4/8, leaf order):
//   * the pack's hits with t < maxt (maxt as it stood when the pack began) are
//     taken in lane order, skipping primitives of other materials;
//   * while fewer than 4 are kept, a hit is appended;
//   * after that it overwrites the kept hit of largest t (the first such slot),
//     and maxt becomes the largest kept t. maxt stays FLT_MAX until the first
//     overwrite, as in SORT (BSSRDFIntersections::ResolveMaxDepth,
//     scatteringevent/bssrdf/bssrdf.h:50-55, runs only on that path).
// Hits and distances are bit-identical to SORT's with FP32 nodes.
#include <cuda_runtime.h>

#include <cfloat>
#include <string>

#include "scene_access.h"
#include "sortgpu.h"
#include "trace_kernels.h"
#include "traversal.cuh"

namespace sg {
namespace {

constexpr int kMultiHits = 4;  // TOTAL_SSS_INTERSECTION_CNT (scatteringevent/bssrdf/bssrdf.h:32)

struct MultiHits {
    int cnt = 0;
    int32_t p[kMultiHits];
    float t[kMultiHits], u[kMultiHits], v[kMultiHits];

    __device__ __forceinline__ void put(int k, int32_t prim, float tt, float uu, float vv) {
#pragma unroll
        for (int j = 0; j < kMultiHits; ++j)
            if (j == k) {
                p[j] = prim;
                t[j] = tt;
                u[j] = uu;
                v[j] = vv;
            }
    }

    // Returns the new maxt when a hit was overwritten, else maxt unchanged.
    __device__ __forceinline__ float add(int32_t prim, float tt, float uu, float vv, float maxt) {
        if (cnt < kMultiHits) {
            put(cnt++, prim, tt, uu, vv);
            return maxt;
        }
        int picked = -1;
        float far = 0.0f;
#pragma unroll
        for (int j = 0; j < kMultiHits; ++j)
            if (far < t[j]) {
                far = t[j];
                picked = j;
            }
        if (picked >= 0) put(picked, prim, tt, uu, vv);
        // std::max(a, b) = a < b ? b : a, applied as ResolveMaxDepth applies it.
        float m = t[0] < t[1] ? t[1] : t[0];
        m = m < t[2] ? t[2] : m;
        return m < t[3] ? t[3] : m;
    }
};

template <int W, int STACK, bool Q8>
__global__ void __launch_bounds__(128) k_trace_multi(DevTree tr, DevRays rays, int64_t n,
                                                     const int32_t* __restrict__ prim_mat,
                                                     const int32_t* __restrict__ ray_mat, int32_t* __restrict__ count,
                                                     int32_t* __restrict__ prim_out, float* __restrict__ t_out,
                                                     float* __restrict__ u_out, float* __restrict__ v_out,
                                                     int* __restrict__ err) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Traversal<W, false, STACK, false, Q8> tv;  // best_t plays SORT's intersect.maxt
    uint2 stk_mem[STACK];
    tv.stk = stk_mem;
    MultiHits h;
    if (tv.start(tr, rays, i)) {
        const int32_t mat = ray_mat[i];
        for (;;) {
            bool descend = false;
            if (!(tv.best_t < tv.cur_d)) {
                if (tv.cur < 0) {
                    int64_t s = (int64_t)((uint32_t)tv.cur & 0x7fffffffu);
                    bool last = false;
                    while (!last) {  // one SIMD pack of W leaf slots per pass
                        const float maxt = tv.best_t;
                        for (int lane = 0; lane < W && !last; ++lane, ++s) {
                            const float4* q = tr.tris + 3 * s;
                            const float4 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2);
                            last = __float_as_int(b.w) != 0;
                            float t, u, v;
                            if (!tri_test(tv.r, a, b, c, t, u, v) || !(t < maxt)) continue;
                            const int32_t p = __float_as_int(a.w);
                            if (__ldg(prim_mat + p) != mat) continue;
                            tv.best_t = h.add(p, t, u, v, tv.best_t);
                        }
                    }
                } else if (tv.si + W > STACK) {  // cannot happen when STACK >= depth*(W-1)+1
                    atomicOr(err, 1);
                    break;
                } else {
                    descend = tv.interior(tr);
                }
            }
            if (!descend) {
                if (tv.si == 0) break;
                const uint2 e = tv.stk[--tv.si];
                tv.cur = (int32_t)e.x;
                tv.cur_d = __uint_as_float(e.y);
            }
        }
    }
    count[i] = h.cnt;
#pragma unroll
    for (int k = 0; k < kMultiHits; ++k) {
        const bool kept = k < h.cnt;
        prim_out[kMultiHits * i + k] = kept ? h.p[k] : -1;
        t_out[kMultiHits * i + k] = kept ? h.t[k] : FLT_MAX;
        if (u_out) u_out[kMultiHits * i + k] = kept ? h.u[k] : 0.0f;
        if (v_out) v_out[kMultiHits * i + k] = kept ? h.v[k] : 0.0f;
    }
}

template <int W, bool Q8>
cudaError_t launch_w(const TraceLaunch& L, const DevTree& tr, const DevRays& r, int64_t n, const int32_t* pm,
                     const int32_t* rm, const sg_multi_hits& h, cudaStream_t s) {
    const int64_t blocks = (n + 127) / 128;
#define SG_MULTI_LAUNCH(ST)                                                                                         \
    k_trace_multi<W, ST, Q8><<<(unsigned)blocks, 128, 0, s>>>(tr, r, n, pm, rm, h.count, h.prim, h.t, h.u, h.v, \
                                                              L.err)
    if (L.stack_need <= 64)
        SG_MULTI_LAUNCH(64);
    else if (L.stack_need <= 128)
        SG_MULTI_LAUNCH(128);
    else if (L.stack_need <= 256)
        SG_MULTI_LAUNCH(256);
    else
        return cudaErrorInvalidValue;
#undef SG_MULTI_LAUNCH
    return cudaGetLastError();
}

}  // namespace
}  // namespace sg

extern "C" sg_status sg_trace_multi(const sg_scene* scene, const sg_rays* rays, int64_t n, const int32_t* prim_material,
                                    const int32_t* ray_material, const sg_multi_hits* hits, void* stream) {
    if (!scene || !rays || !hits) return sg::set_error(SG_ERR_INVALID_ARGUMENT, "NULL argument");
    if (n < 0) return sg::set_error(SG_ERR_INVALID_ARGUMENT, "negative ray count");
    if (n == 0) return SG_OK;
    if (!rays->ox || !rays->oy || !rays->oz || !rays->dx || !rays->dy || !rays->dz || !rays->tmin || !rays->tmax)
        return sg::set_error(SG_ERR_INVALID_ARGUMENT, "NULL ray array");
    if (!prim_material || !ray_material || !hits->count || !hits->prim || !hits->t)
        return sg::set_error(SG_ERR_INVALID_ARGUMENT, "NULL material or output array");
    if (n > int64_t(0x7fffffff) * 128) return sg::set_error(SG_ERR_LIMIT, "batch too large");
    sg::TraceLaunch L;
    sg::DevTree tree;
    int device = 0;
    sg_status st = sg::scene_launch(scene, false, &L, &tree, &device);
    if (st != SG_OK) return st;
    int prev = -1;
    cudaGetDevice(&prev);
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) {
        const sg::DevRays r{rays->ox, rays->oy, rays->oz, rays->dx, rays->dy, rays->dz, rays->tmin, rays->tmax};
        cudaStream_t s = (cudaStream_t)stream;
        if (L.width == 8)
            e = L.q8 ? sg::launch_w<8, true>(L, tree, r, n, prim_material, ray_material, *hits, s)
                     : sg::launch_w<8, false>(L, tree, r, n, prim_material, ray_material, *hits, s);
        else
            e = L.q8 ? sg::launch_w<4, true>(L, tree, r, n, prim_material, ray_material, *hits, s)
                     : sg::launch_w<4, false>(L, tree, r, n, prim_material, ray_material, *hits, s);
    }
    if (prev >= 0) cudaSetDevice(prev);
    if (e != cudaSuccess) return sg::set_error(SG_ERR_CUDA, (std::string("multi-hit launch: ") + cudaGetErrorString(e)).c_str());
    return SG_OK;
}
