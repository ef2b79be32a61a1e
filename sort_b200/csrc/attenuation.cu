// sg_trace_attenuation: SORT's transparent-shadow query, batched.
//
// Restates Scene::GetAttenuation (core/scene.cpp:192-208), which loops
// Accelerator::GetAttenuation (accel/accelerator.cpp:26-69), whose query is
// Fbvh::GetIntersect with query_shadow set (accel/fast_bvh.hpp:345-370, SIMD
// branch). Per ray:
//   * the closest-hit traversal (same near-first order and t cull), except that
//     after each SIMD pack of W leaf slots (SORT's Triangle4/8, leaf order)
//     whose nearest hit became the current hit, the query ends as "blocked"
//     when that primitive's material has no transparency (only that hit is
//     checked, not the pack's other hits, as in SORT);
//   * blocked: the attenuation is 0; no hit: the loop ends;
//   * a transparent hit: att = the material's transparency; a black att is the
//     result; else the attenuation is multiplied by it and the ray restarts at
//     ray(t) = o + t * d with tmin 0.001 and tmax - t;
//   * the loop runs while the attenuation is not black.
// A ray stops after kMaxLayers transparent hits (status bit 2; SORT has no
// bound); a material id outside the table counts as opaque (status bit 4).
#include <cuda_runtime.h>

#include <cfloat>
#include <string>

#include "scene_access.h"
#include "sortgpu.h"
#include "trace_kernels.h"
#include "traversal.cuh"

namespace sg {
namespace {

constexpr int kMaxLayers = 4096;

template <int W, int STACK, bool Q8>
__global__ void __launch_bounds__(128)
    k_trace_attenuation(DevTree tr, DevRays rays, int64_t n, const int32_t* __restrict__ prim_mat,
                        const sg_transparency* __restrict__ mats, int32_t nmat, float* __restrict__ out,
                        int* __restrict__ err) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Traversal<W, false, STACK, false, Q8> tv;
    uint2 stk_mem[STACK];
    tv.stk = stk_mem;
    float o[3] = {rays.ox[i], rays.oy[i], rays.oz[i]};
    const float d[3] = {rays.dx[i], rays.dy[i], rays.dz[i]};
    float tmin = rays.tmin[i], tmax = rays.tmax[i];
    float att[3] = {1.0f, 1.0f, 1.0f};
    for (int layer = 0; !(att[0] == 0.0f && att[1] == 0.0f && att[2] == 0.0f); ++layer) {
        if (layer == kMaxLayers) {
            atomicOr(err, 2);
            break;
        }
        for (int a = 0; a < 3; ++a) {
            tv.r.o[a] = o[a];
            tv.r.d[a] = d[a];
        }
        tv.r.tmin = tmin;
        tv.r.tmax = tmax;
        bool blocked = false;
        if (tv.begin(tr)) {  // begin() clears the hit: best_prim = -1
            for (;;) {
                bool descend = false;
                if (!(tv.best_t < tv.cur_d)) {
                    if (tv.cur < 0) {
                        int64_t s = (int64_t)((uint32_t)tv.cur & 0x7fffffffu);
                        bool last = false;
                        while (!last && !blocked) {  // one SIMD pack of W leaf slots per pass
                            bool nearer = false;
                            for (int lane = 0; lane < W && !last; ++lane, ++s) {
                                const float4* q = tr.tris + 3 * s;
                                const float4 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2);
                                last = __float_as_int(b.w) != 0;
                                float t, u, v;
                                if (tri_test(tv.r, a, b, c, t, u, v) && t < tv.best_t) {
                                    tv.best_t = t;
                                    tv.best_u = u;
                                    tv.best_v = v;
                                    tv.best_prim = __float_as_int(a.w);
                                    nearer = true;
                                }
                            }
                            if (nearer) {
                                const int32_t m = __ldg(prim_mat + tv.best_prim);
                                if (m < 0 || m >= nmat) {
                                    atomicOr(err, 4);
                                    blocked = true;
                                } else {
                                    blocked = __ldg(&mats[m].transparent) == 0;
                                }
                            }
                        }
                        if (blocked) break;
                    } else if (tv.si + W > STACK) {  // cannot happen when STACK >= depth*(W-1)+1
                        atomicOr(err, 1);
                        blocked = true;
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
        if (blocked) {
            att[0] = att[1] = att[2] = 0.0f;
            break;
        }
        if (tv.best_prim < 0) break;  // GetIntersect found nothing
        // Every hit that became current was checked: this one is transparent.
        const sg_transparency* mt = mats + __ldg(prim_mat + tv.best_prim);
        const float a3[3] = {__ldg(&mt->rgb[0]), __ldg(&mt->rgb[1]), __ldg(&mt->rgb[2])};
        if (a3[0] == 0.0f && a3[1] == 0.0f && a3[2] == 0.0f) {  // if( att.IsBlack() ) return att;
            att[0] = a3[0];
            att[1] = a3[1];
            att[2] = a3[2];
            break;
        }
        for (int a = 0; a < 3; ++a) att[a] = __fmul_rn(att[a], a3[a]);
        const float t = tv.best_t;
        for (int a = 0; a < 3; ++a) o[a] = __fadd_rn(o[a], __fmul_rn(t, d[a]));  // Ray::operator()(t)
        tmin = 0.001f;
        tmax = __fsub_rn(tmax, t);
    }
    out[i] = att[0];
    out[n + i] = att[1];
    out[2 * n + i] = att[2];
}

template <int W, bool Q8>
cudaError_t launch_w(const TraceLaunch& L, const DevTree& tr, const DevRays& r, int64_t n, const int32_t* pm,
                     const sg_transparency* mats, int32_t nmat, float* out, cudaStream_t s) {
    const int64_t blocks = (n + 127) / 128;
#define SG_ATT_LAUNCH(ST) \
    k_trace_attenuation<W, ST, Q8><<<(unsigned)blocks, 128, 0, s>>>(tr, r, n, pm, mats, nmat, out, L.err)
    if (L.stack_need <= 64)
        SG_ATT_LAUNCH(64);
    else if (L.stack_need <= 128)
        SG_ATT_LAUNCH(128);
    else if (L.stack_need <= 256)
        SG_ATT_LAUNCH(256);
    else
        return cudaErrorInvalidValue;
#undef SG_ATT_LAUNCH
    return cudaGetLastError();
}

}  // namespace
}  // namespace sg

extern "C" sg_status sg_trace_attenuation(const sg_scene* scene, const sg_rays* rays, int64_t n,
                                          const sg_transparency* materials, int32_t nmat, float* attenuation,
                                          void* stream) {
    if (!scene || !rays || !attenuation) return sg::set_error(SG_ERR_INVALID_ARGUMENT, "NULL argument");
    if (n < 0 || nmat < 0) return sg::set_error(SG_ERR_INVALID_ARGUMENT, "negative count");
    if (n == 0) return SG_OK;
    if (!rays->ox || !rays->oy || !rays->oz || !rays->dx || !rays->dy || !rays->dz || !rays->tmin || !rays->tmax)
        return sg::set_error(SG_ERR_INVALID_ARGUMENT, "NULL ray array");
    if (nmat > 0 && !materials) return sg::set_error(SG_ERR_INVALID_ARGUMENT, "NULL material table");
    if (n > int64_t(0x7fffffff) * 128) return sg::set_error(SG_ERR_LIMIT, "batch too large");
    const int32_t* prim_material = sg::scene_materials(scene);
    if (!prim_material) return sg::set_error(SG_ERR_INVALID_ARGUMENT, "no primitive materials (sg_scene_set_materials)");
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
            e = L.q8 ? sg::launch_w<8, true>(L, tree, r, n, prim_material, materials, nmat, attenuation, s)
                     : sg::launch_w<8, false>(L, tree, r, n, prim_material, materials, nmat, attenuation, s);
        else
            e = L.q8 ? sg::launch_w<4, true>(L, tree, r, n, prim_material, materials, nmat, attenuation, s)
                     : sg::launch_w<4, false>(L, tree, r, n, prim_material, materials, nmat, attenuation, s);
    }
    if (prev >= 0) cudaSetDevice(prev);
    if (e != cudaSuccess)
        return sg::set_error(SG_ERR_CUDA, (std::string("attenuation launch: ") + cudaGetErrorString(e)).c_str());
    return SG_OK;
}
