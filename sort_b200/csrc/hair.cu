// Closest-hit and any-hit traversal for scenes with hair lines and area-light
// shapes.
//
// The tree and the box tests are the triangle path's (traversal.cuh); the leaf
// loop also runs SORT's ray-line test. SORT's leaf tests all its triangle
// packs, then all its line packs (accel/fast_bvh.hpp:346-390, with the packs
// made in accel/fast_bvh.hpp:221-252); the slots of a leaf hold its triangles
// first and its lines after them, each in SORT's leaf order, so testing the
// slots in order with a strictly-nearer rule picks the hit SORT's packs pick.
//
// Ray-line test: intersectLine_Inner and intersectLine_SIMD
// (simd/simd_line.h:232-330) per lane, in SORT's operation order, each
// multiply and add rounded on its own (SORT's simd_mad_ps is a multiply then
// an add): the ray in line space, the quadratic of the cone, the nearer root
// whose line-space y lies strictly inside (0, length), else the farther one;
// tmin < t < tmax; u = 1, v = lerp(v0, v1, y / length).
//
// Area shapes sit after a leaf's lines, as SORT's other_list follows its line
// packs (accel/fast_bvh.hpp:390-406), and are tested with Quad::GetIntersect
// (shape/quad.cpp:67-93) or Disk::GetIntersect (shape/disk.cpp): the ray taken
// to the shape's frame by Matrix::TransformPoint / TransformVector
// (math/matrix.cpp:70-92), t = -o.y / d.y with d.y != 0, kept when
// tmin < t <= tmax and t <= the nearest t so far, then p = o + t d inside the
// rectangle |x| <= sizeX/2, |z| <= sizeY/2, or the disk x^2 + z^2 <= r^2. A
// shape hit leaves u, v as they were, as SORT's shape test does.
#include <cuda_runtime.h>

#include <cfloat>

#include "hair.h"
#include "trace_kernels.h"
#include "traversal.cuh"

namespace sg {
namespace {

__device__ __forceinline__ float f_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float f_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float f_sub(float a, float b) { return __fsub_rn(a, b); }

// Returns true with t, v when the line is hit in (tmin, tmax).
__device__ __forceinline__ bool line_test(const RayState& r, const float4* __restrict__ rec, float& t_out,
                                          float& v_out) {
    const float4 m0 = __ldg(rec), m1 = __ldg(rec + 1), m2 = __ldg(rec + 2), g = __ldg(rec + 3), vv = __ldg(rec + 4);
    const float ox = f_add(f_add(f_add(f_mul(m0.x, r.o[0]), f_mul(m0.y, r.o[1])), f_mul(m0.z, r.o[2])), m0.w);
    const float oy = f_add(f_add(f_add(f_mul(m1.x, r.o[0]), f_mul(m1.y, r.o[1])), f_mul(m1.z, r.o[2])), m1.w);
    const float oz = f_add(f_add(f_add(f_mul(m2.x, r.o[0]), f_mul(m2.y, r.o[1])), f_mul(m2.z, r.o[2])), m2.w);
    const float dx = f_add(f_add(f_mul(m0.x, r.d[0]), f_mul(m0.y, r.d[1])), f_mul(m0.z, r.d[2]));
    const float dy = f_add(f_add(f_mul(m1.x, r.d[0]), f_mul(m1.y, r.d[1])), f_mul(m1.z, r.d[2]));
    const float dz = f_add(f_add(f_mul(m2.x, r.d[0]), f_mul(m2.y, r.d[1])), f_mul(m2.z, r.d[2]));
    const float w0 = g.x, length = g.z, slope = g.w;
    const float tmp0 = f_add(f_mul(oy, slope), w0);
    const float tmp1 = f_mul(dy, slope);
    const float a = f_sub(f_add(f_mul(dx, dx), f_mul(dz, dz)), f_mul(tmp1, tmp1));
    const float b = f_sub(f_add(f_mul(dx, ox), f_mul(dz, oz)), f_mul(tmp0, tmp1));
    const float c = f_sub(f_add(f_mul(ox, ox), f_mul(oz, oz)), f_mul(tmp0, tmp0));
    const float disc = f_sub(f_mul(b, b), f_mul(a, c));
    if (!(disc > 0.0f)) return false;
    const float s = __fsqrt_rn(disc);
    const float t0 = __fdiv_rn(f_sub(f_sub(0.0f, b), s), a);
    const float y0 = f_add(f_mul(dy, t0), oy);
    const bool near_in = y0 < length && y0 > 0.0f;
    const float t1 = __fdiv_rn(f_sub(s, b), a);
    const float y1 = f_add(f_mul(dy, t1), oy);
    const float y = near_in ? y0 : y1;
    if (!(y < length && y > 0.0f)) return false;
    const float t = near_in ? t0 : t1;
    if (!(t > r.tmin && t < r.tmax)) return false;
    const float q = __fdiv_rn(y, length);
    v_out = f_add(f_mul(vv.x, f_sub(1.0f, q)), f_mul(vv.y, q));  // slerp (math/utils.h:81)
    t_out = t;
    return true;
}

// Returns true with t when the area shape is hit (t <= limit, the nearest t so far).
__device__ __forceinline__ bool shape_test(const RayState& r, const float4* __restrict__ rec, float limit,
                                           float& t_out) {
    const float4 m0 = __ldg(rec), m1 = __ldg(rec + 1), m2 = __ldg(rec + 2), m3 = __ldg(rec + 3), g = __ldg(rec + 4);
    float ox = f_add(f_add(f_add(f_mul(r.o[0], m0.x), f_mul(r.o[1], m0.y)), f_mul(r.o[2], m0.z)), m0.w);
    float oy = f_add(f_add(f_add(f_mul(r.o[0], m1.x), f_mul(r.o[1], m1.y)), f_mul(r.o[2], m1.z)), m1.w);
    float oz = f_add(f_add(f_add(f_mul(r.o[0], m2.x), f_mul(r.o[1], m2.y)), f_mul(r.o[2], m2.z)), m2.w);
    const float ow = f_add(f_add(f_add(f_mul(r.o[0], m3.x), f_mul(r.o[1], m3.y)), f_mul(r.o[2], m3.z)), m3.w);
    if (ow != 1.0f) {  // Point / w multiplies by the reciprocal (math/point.h:126-129)
        const float inv = __fdiv_rn(1.0f, ow);
        ox = f_mul(ox, inv);
        oy = f_mul(oy, inv);
        oz = f_mul(oz, inv);
    }
    const float dx = f_add(f_add(f_mul(r.d[0], m0.x), f_mul(r.d[1], m0.y)), f_mul(r.d[2], m0.z));
    const float dy = f_add(f_add(f_mul(r.d[0], m1.x), f_mul(r.d[1], m1.y)), f_mul(r.d[2], m1.z));
    const float dz = f_add(f_add(f_mul(r.d[0], m2.x), f_mul(r.d[1], m2.y)), f_mul(r.d[2], m2.z));
    if (dy == 0.0f) return false;
    const float t = __fdiv_rn(-oy, dy);
    if (t > limit || t <= r.tmin || t > r.tmax) return false;
    const float px = f_add(ox, f_mul(t, dx)), pz = f_add(oz, f_mul(t, dz));
    if (__float_as_int(g.z) == SG_SHAPE_DISK) {
        if (f_add(f_mul(px, px), f_mul(pz, pz)) > g.y) return false;
    } else {
        if (px > g.x || px < -g.x) return false;
        if (pz > g.y || pz < -g.y) return false;
    }
    t_out = t;
    return true;
}

template <int W, bool ANY, int STACK, bool Q8>
__global__ void __launch_bounds__(128)
    k_trace_hair(DevTree tr, const float4* __restrict__ lines, DevRays rays, int64_t n, int32_t* __restrict__ prim_out,
                 float* __restrict__ t_out, float* __restrict__ u_out, float* __restrict__ v_out,
                 uint8_t* __restrict__ occ_out, int* __restrict__ err) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Traversal<W, false, STACK, false, Q8> tv;
    uint2 stk_mem[STACK];
    tv.stk = stk_mem;
    bool hit_any = false;
    if (tv.start(tr, rays, i)) {
        for (;;) {
            bool descend = false;
            if (!(tv.best_t < tv.cur_d)) {
                if (tv.cur < 0) {
                    int64_t s = (int64_t)((uint32_t)tv.cur & 0x7fffffffu);
                    for (;; ++s) {
                        const float4* q = tr.tris + 3 * s;
                        const float4 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2);
                        float t, u = tv.best_u, v = tv.best_v;
                        bool hit;
                        if (__float_as_int(c.w) == kShapeSlot) {
                            hit = shape_test(tv.r, lines + int64_t(__float_as_int(c.x)) * kLineF4, tv.best_t, t);
                        } else if (__float_as_int(c.w) == kLineSlot) {
                            u = 1.0f;
                            hit = line_test(tv.r, lines + int64_t(__float_as_int(c.x)) * kLineF4, t, v) &&
                                  t < tv.best_t;
                        } else {
                            hit = tri_test(tv.r, a, b, c, t, u, v) && t < tv.best_t;
                        }
                        if (hit) {
                            tv.best_t = t;
                            tv.best_u = u;
                            tv.best_v = v;
                            tv.best_prim = __float_as_int(a.w);
                            if (ANY) {
                                hit_any = true;
                                break;
                            }
                        }
                        if (__float_as_int(b.w)) break;
                    }
                    if (ANY && hit_any) break;
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
    if (ANY) {
        occ_out[i] = tv.best_prim >= 0 ? 1 : 0;
    } else {
        const bool h = tv.best_prim >= 0;
        prim_out[i] = tv.best_prim;
        t_out[i] = h ? tv.best_t : FLT_MAX;
        if (u_out) u_out[i] = h ? tv.best_u : 0.0f;
        if (v_out) v_out[i] = h ? tv.best_v : 0.0f;
    }
}

template <int W, bool ANY, bool Q8>
cudaError_t launch_wa(const TraceLaunch& L, const DevTree& tr, const float4* lines, const DevRays& r, int64_t n,
                      cudaStream_t s) {
    const unsigned blocks = (unsigned)((n + 127) / 128);
#define SG_HAIR_LAUNCH(ST)                                                                                       \
    k_trace_hair<W, ANY, ST, Q8><<<blocks, 128, 0, s>>>(tr, lines, r, n, L.prim, L.t, L.u, L.v, L.occ, L.err)
    if (L.stack_need <= 64)
        SG_HAIR_LAUNCH(64);
    else if (L.stack_need <= 128)
        SG_HAIR_LAUNCH(128);
    else if (L.stack_need <= 256)
        SG_HAIR_LAUNCH(256);
    else
        return cudaErrorInvalidValue;
#undef SG_HAIR_LAUNCH
    return cudaGetLastError();
}

template <int W, bool Q8>
cudaError_t launch_w(const TraceLaunch& L, const DevTree& tr, const float4* lines, const DevRays& r, int64_t n,
                     cudaStream_t s) {
    return L.any ? launch_wa<W, true, Q8>(L, tr, lines, r, n, s) : launch_wa<W, false, Q8>(L, tr, lines, r, n, s);
}

}  // namespace

cudaError_t launch_trace_hair(const TraceLaunch& L, const DevTree& tr, const float4* lines, const DevRays& rays,
                              int64_t n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    if (L.width == 8)
        return L.q8 ? launch_w<8, true>(L, tr, lines, rays, n, s) : launch_w<8, false>(L, tr, lines, rays, n, s);
    return L.q8 ? launch_w<4, true>(L, tr, lines, rays, n, s) : launch_w<4, false>(L, tr, lines, rays, n, s);
}

}  // namespace sg
