// Device-side ray setup, slab tests and the watertight triangle test.
//
// Every floating-point step that decides a hit is written with explicit
// round-to-nearest intrinsics (__fadd_rn, __fmul_rn, ...), which the compiler
// never fuses into FMA. Each step therefore rounds exactly like SORT's SSE/AVX
// code, where simd_mad_ps is a separate multiply and add
// (simd/simd_intel.h:128-130) and simd_rcp_ps is a true divide (125-127).
#pragma once

#include <cfloat>
#include <cstdint>

#include "layout.h"

namespace sg {

struct RayState {
    float o[3], d[3];
    float tmin, tmax;
    float rcp[3], od[3];  // resolveRayData: 1/d and -o/d with |d| clamped to >= 1e-5
    int nhi[3];           // 1 where rcp < 0: the ray enters a box through its upper bound
    int ly;               // Ray::Prepare major axis; x = (ly + 2) % 3, z = (ly + 1) % 3
    float ox, oy, oz;     // origin in the permuted (local x, y, z) frame
    float sx, sy, sz;     // shear constants
};

__device__ __forceinline__ float sse_min(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float sse_max(float a, float b) { return a > b ? a : b; }
// libstdc++ std::min / std::max
__device__ __forceinline__ float std_min(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float std_max(float a, float b) { return (a < b) ? b : a; }

__device__ __forceinline__ float pick3(int k, float a, float b, float c) { return k == 0 ? a : (k == 1 ? b : c); }

// resolveRayData (simd/simd_ray_utils.h:60-83) + Ray::Prepare (math/ray.h:60-69).
__device__ __forceinline__ void ray_setup(RayState& r) {
    const float delta = 0.00001f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float dk = fabsf(r.d[k]) < delta ? (r.d[k] < 0.0f ? -delta : delta) : r.d[k];
        r.rcp[k] = __frcp_rn(dk);
        r.od[k] = __fdiv_rn(-r.o[k], dk);
        r.nhi[k] = r.rcp[k] < 0.0f ? 1 : 0;
    }
    const float ax = fabsf(r.d[0]), ay = fabsf(r.d[1]), az = fabsf(r.d[2]);
    int y;
    if (ax > ay && ax > az)
        y = 0;
    else
        y = ay > az ? 1 : 2;
    const int z = (y + 1) % 3, x = (z + 1) % 3;
    r.ly = y;
    const float dxl = pick3(x, r.d[0], r.d[1], r.d[2]);
    const float dyl = pick3(y, r.d[0], r.d[1], r.d[2]);
    const float dzl = pick3(z, r.d[0], r.d[1], r.d[2]);
    r.sx = __fdiv_rn(-dxl, dyl);
    r.sz = __fdiv_rn(-dzl, dyl);
    r.sy = __frcp_rn(dyl);
    r.ox = pick3(x, r.o[0], r.o[1], r.o[2]);
    r.oy = pick3(y, r.o[0], r.o[1], r.o[2]);
    r.oz = pick3(z, r.o[0], r.o[1], r.o[2]);
}

// Scalar Intersect(ray, bbox) (math/bbox.h:124-155) for the root box.
__device__ __forceinline__ float root_intersect(const RayState& r, const float* lo, const float* hi) {
    float tmax = r.tmax, tmin = r.tmin;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (r.d[a] < 0.00001f && r.d[a] > -0.00001f) {
            if (r.o[a] > hi[a] || r.o[a] < lo[a]) return -1.0f;
        } else {
            const float ood = __frcp_rn(r.d[a]);
            float t1 = __fmul_rn(__fsub_rn(hi[a], r.o[a]), ood);
            float t2 = __fmul_rn(__fsub_rn(lo[a], r.o[a]), ood);
            if (t1 > t2) {
                const float tt = t1;
                t1 = t2;
                t2 = tt;
            }
            tmin = std_max(t1, tmin);
            tmax = std_min(t2, tmax);
            if (tmin > tmax) return -1.0f;
        }
    }
    return tmin;
}

// One lane of IntersectBBox_SIMD (simd/simd_bbox.h:62-85). Returns whether the
// slab interval is non-empty; d gets fmin on a hit and -1 on a miss, as SORT's
// simd_pick_ps leaves it (validity of the slot is checked by the caller).
//
// SORT's lanes use _mm_min_ps / _mm_max_ps (a < b ? a : b); here fminf / fmaxf,
// one instruction each. The two agree in value whenever neither input is NaN,
// and no input is: 1/d and -o/d are finite after the |d| >= 1e-5 clamp, box
// bounds are finite or +-FLT_MAX, so every t is finite or +-inf (rays must be
// finite, as SORT assumes). Where they may differ — which of +0 and -0 an equal
// pair returns — nothing downstream looks: entry distances are only compared.
__device__ __forceinline__ bool slab(const RayState& r, float lx, float hx, float ly, float hy, float lz, float hz,
                                     float& d) {
    float f_min = r.tmin, f_max = r.tmax;
    {
        const float t1 = __fadd_rn(r.od[0], __fmul_rn(r.rcp[0], hx));
        const float t2 = __fadd_rn(r.od[0], __fmul_rn(r.rcp[0], lx));
        f_min = fmaxf(f_min, fminf(t1, t2));
        f_max = fminf(f_max, fmaxf(t1, t2));
    }
    {
        const float t1 = __fadd_rn(r.od[1], __fmul_rn(r.rcp[1], hy));
        const float t2 = __fadd_rn(r.od[1], __fmul_rn(r.rcp[1], ly));
        f_min = fmaxf(f_min, fminf(t1, t2));
        f_max = fminf(f_max, fmaxf(t1, t2));
    }
    {
        const float t1 = __fadd_rn(r.od[2], __fmul_rn(r.rcp[2], hz));
        const float t2 = __fadd_rn(r.od[2], __fmul_rn(r.rcp[2], lz));
        f_min = fmaxf(f_min, fminf(t1, t2));
        f_max = fminf(f_max, fmaxf(t1, t2));
    }
    const bool hit = f_min <= f_max;
    d = hit ? f_min : -1.0f;
    return hit;
}

// slab() from each axis's entry plane n and exit plane f (n = lo, f = hi where
// 1/d > 0, swapped where 1/d < 0). With 1/d finite and non-zero and lo <= hi,
// t(b) = fl(-o/d + fl(b * 1/d)) is monotonic in b, so t(n) = min(t(lo), t(hi))
// and t(f) = max(...) exactly, and the interval's bounds are the same maxima and
// minima in another order: the result equals slab()'s for every box with
// lo <= hi. Only empty slots (lo = +FLT_MAX > hi = -FLT_MAX) differ, and the
// caller discards those by their -1 reference. Two flops and two comparisons
// fewer per axis.
__device__ __forceinline__ bool slab_near_far(const RayState& r, float nx, float fx, float ny, float fy, float nz,
                                              float fz, float& d) {
    const float tnx = __fadd_rn(r.od[0], __fmul_rn(r.rcp[0], nx));
    const float tfx = __fadd_rn(r.od[0], __fmul_rn(r.rcp[0], fx));
    const float tny = __fadd_rn(r.od[1], __fmul_rn(r.rcp[1], ny));
    const float tfy = __fadd_rn(r.od[1], __fmul_rn(r.rcp[1], fy));
    const float tnz = __fadd_rn(r.od[2], __fmul_rn(r.rcp[2], nz));
    const float tfz = __fadd_rn(r.od[2], __fmul_rn(r.rcp[2], fz));
    const float f_min = fmaxf(fmaxf(tnx, tny), fmaxf(tnz, r.tmin));
    const float f_max = fminf(fminf(tfx, tfy), fminf(tfz, r.tmax));
    const bool hit = f_min <= f_max;
    d = hit ? f_min : -1.0f;
    return hit;
}

// One lane of intersectTriangleInner_SIMD (simd/simd_triangle.h:212-300):
// translate, permute to the ray's major axis, shear, edge functions, det,
// t = (e0*p0y + e1*p1y + e2*p2y) / det with tmin < t <= tmax.
__device__ __forceinline__ bool tri_test(const RayState& r, const float4& a, const float4& b, const float4& c,
                                         float& t_out, float& u_out, float& v_out) {
    const int y = r.ly, z = (y + 1) % 3, x = (z + 1) % 3;
    const float p0x0 = __fsub_rn(pick3(x, a.x, a.y, a.z), r.ox);
    const float p0y0 = __fsub_rn(pick3(y, a.x, a.y, a.z), r.oy);
    const float p0z0 = __fsub_rn(pick3(z, a.x, a.y, a.z), r.oz);
    const float p1x0 = __fsub_rn(pick3(x, b.x, b.y, b.z), r.ox);
    const float p1y0 = __fsub_rn(pick3(y, b.x, b.y, b.z), r.oy);
    const float p1z0 = __fsub_rn(pick3(z, b.x, b.y, b.z), r.oz);
    const float p2x0 = __fsub_rn(pick3(x, c.x, c.y, c.z), r.ox);
    const float p2y0 = __fsub_rn(pick3(y, c.x, c.y, c.z), r.oy);
    const float p2z0 = __fsub_rn(pick3(z, c.x, c.y, c.z), r.oz);
    const float p0x = __fadd_rn(__fmul_rn(p0y0, r.sx), p0x0);
    const float p0z = __fadd_rn(__fmul_rn(p0y0, r.sz), p0z0);
    const float p1x = __fadd_rn(__fmul_rn(p1y0, r.sx), p1x0);
    const float p1z = __fadd_rn(__fmul_rn(p1y0, r.sz), p1z0);
    const float p2x = __fadd_rn(__fmul_rn(p2y0, r.sx), p2x0);
    const float p2z = __fadd_rn(__fmul_rn(p2y0, r.sz), p2z0);
    const float e0 = __fsub_rn(__fmul_rn(p1x, p2z), __fmul_rn(p1z, p2x));
    const float e1 = __fsub_rn(__fmul_rn(p2x, p0z), __fmul_rn(p2z, p0x));
    const float e2 = __fsub_rn(__fmul_rn(p0x, p1z), __fmul_rn(p0z, p1x));
    const bool c0 = (e0 >= 0.0f) && (e1 >= 0.0f) && (e2 >= 0.0f);
    const bool c1 = (e0 <= 0.0f) && (e1 <= 0.0f) && (e2 <= 0.0f);
    if (!(c0 || c1)) return false;
    const float det = __fadd_rn(e0, __fadd_rn(e1, e2));
    if (!(det != 0.0f)) return false;
    const float rcp_det = __frcp_rn(det);
    const float p0y = __fmul_rn(p0y0, r.sy);
    const float p1y = __fmul_rn(p1y0, r.sy);
    const float p2y = __fmul_rn(p2y0, r.sy);
    float t = __fmul_rn(e0, p0y);
    t = __fadd_rn(__fmul_rn(e1, p1y), t);
    t = __fadd_rn(__fmul_rn(e2, p2y), t);
    t = __fmul_rn(t, rcp_det);
    if (!(t > r.tmin && t <= r.tmax)) return false;
    t_out = t;
    u_out = __fmul_rn(e1, rcp_det);
    v_out = __fmul_rn(e2, rcp_det);
    return true;
}

}  // namespace sg
