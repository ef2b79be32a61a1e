// Device-side pieces of the wavefront path tracer shared by the single-render
// path (pt.cu) and the request server (serve.cu): SORT's constants, materials,
// area light, Philox random numbers, shading frame, BxDFs, queue appends, and
// the shading of one path vertex.
#pragma once

#include <cuda_runtime.h>

#include <cfloat>
#include <cstdint>

#include "pt_types.h"

namespace sg {

// SORT's constants (math/utils.h:28-32).
constexpr float kPi = 3.1415926f;
constexpr float kTwoPi = 6.2831852f;
constexpr float kInvPi = 0.3183099f;

struct Queue {
    float* ray;     // 8 * cap floats, SoA
    int* slot;      // path (pixel) per entry
    float* contrib; // shadow queue only: 3 * cap
};

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC'11): ten rounds of the round function below with the
// published multipliers and Weyl key increments.
__device__ __forceinline__ uint4 philox(uint4 c, uint2 k) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += 0x9E3779B9u;
        k.y += 0xBB67AE85u;
    }
    return c;
}
// 24 random bits in [0, 1), as SORT's sort_rand<float> (core/rand.cpp:104-107).
__device__ __forceinline__ float u01(uint32_t x) { return (float)(x >> 8) * (1.0f / 16777216.0f); }

__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator*(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float3 operator*(float3 a, float3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ float3 operator-(float3 a) { return f3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
    return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float3 normalize3(float3 v) { return v * (1.0f / sqrtf(dot3(v, v))); }
__device__ __forceinline__ bool black(float3 s) { return s.x == 0.0f && s.y == 0.0f && s.z == 0.0f; }
__device__ __forceinline__ float intensity(float3 s) { return 0.212671f * s.x + 0.715160f * s.y + 0.072169f * s.z; }
__device__ __forceinline__ float max_comp(float3 s) { return fmaxf(s.x, fmaxf(s.y, s.z)); }
__device__ __forceinline__ float mis(float f, float g) { return (f * f) / (f * f + g * g); }  // MisFactor

// Shading frame of ScatteringEvent (scatteringevent.cpp:42-59): y = normal.
struct Frame {
    float3 t, n, bt;
    __device__ float3 local(float3 v) const { return f3(dot3(v, t), dot3(v, n), dot3(v, bt)); }
    __device__ float3 world(float3 v) const { return t * v.x + n * v.y + bt * v.z; }
};
__device__ __forceinline__ Frame make_frame(float3 n) {
    const float3 a = fabsf(n.x) > 0.9f ? f3(0.0f, 1.0f, 0.0f) : f3(1.0f, 0.0f, 0.0f);
    const float3 tangent = normalize3(cross3(a, n));
    Frame fr;
    fr.n = normalize3(n);
    fr.bt = normalize3(cross3(fr.n, tangent));
    fr.t = normalize3(cross3(fr.bt, fr.n));
    return fr;
}

// UniformSampleDisk / CosSampleHemisphere (core/samplemethod.h: Shirley's mapping).
__device__ inline float3 cos_sample_hemisphere(float u, float v) {
    float r, theta, x, z;
    const float su = 2.0f * u - 1.0f, sv = 2.0f * v - 1.0f;
    const float asu = fabsf(su), asv = fabsf(sv);
    if (asu < asv) {
        r = asv;
        const float factor = sv > 0.0f ? -1.0f : 1.0f;
        theta = factor * su / r + 4.0f + 2.0f * factor;
    } else if (asv < asu) {
        r = asu;
        const float factor = su > 0.0f ? 1.0f : -1.0f;
        theta = factor * sv / r - 2.0f * factor + 2.0f;
        if (theta < 0.0f) theta += 8.0f;
    } else {
        return f3(0.0f, 1.0f, 0.0f);
    }
    theta *= kPi / 4.0f;
    x = cosf(theta) * r;
    z = sinf(theta) * r;
    return f3(x, sqrtf(fmaxf(0.0f, 1.0f - x * x - z * z)), z);
}

// ---- GGX (microfacet.cpp:229-299), isotropic ------------------------------
struct Ggx {
    float au, av, au2, av2, auv;
    __device__ explicit Ggx(float rough) {
        const float r = fmaxf(rough, 1e-3f);
        au = av = r * r;
        au2 = au * au;
        av2 = av * av;
        auv = au * av;
    }
    __device__ float D(float3 h) const {
        const float c2 = h.y * h.y;
        if (c2 <= 0.0f) return 0.0f;
        const float beta = c2 + (h.x * h.x / au2 + h.z * h.z / av2);
        return 1.0f / (kPi * auv * beta * beta);
    }
    __device__ float G1(float3 v) const {
        const float c2 = v.y * v.y;
        const float tan2 = 1.0f / c2 - 1.0f;
        if (isinf(tan2)) return 0.0f;
        const float sin_t = sqrtf(fmaxf(0.0f, 1.0f - c2));
        const float cphi = sin_t == 0.0f ? 1.0f : fminf(fmaxf(v.x / sin_t, -1.0f), 1.0f);
        const float cphi2 = cphi * cphi;
        const float a2 = cphi2 * au2 + (1.0f - cphi2) * av2;
        return 2.0f / (1.0f + sqrtf(1.0f + a2 * tan2));
    }
    __device__ float3 sample(float u, float v) const {
        const float theta = atanf(au * sqrtf(v / (1.0f - v)));
        const float phi = kTwoPi * u;
        const float st = sinf(theta);
        return f3(st * cosf(phi), cosf(theta), st * sinf(phi));
    }
};

__device__ inline float3 conductor_fresnel(float cosI, const float* eta, const float* k) {
    const float sq = cosI * cosI;
    float out[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float t = 2.0f * eta[c] * cosI;
        const float tmp_f = eta[c] * eta[c] + k[c] * k[c];
        const float tmp = tmp_f * sq;
        const float par = (tmp - t + 1.0f) / (tmp + t + 1.0f);
        const float perp = (tmp_f - t + sq) / (tmp_f + t + sq);
        out[c] = (par + perp) * 0.5f;
    }
    return f3(out[0], out[1], out[2]);
}

// BxDF value (includes |cos wi|, as SORT's f does) and pdf in the local frame.
// Both BxDFs are one-sided (doubleSided = false): zero unless wo and wi are
// above the surface (Bxdf::PointingUp, SameHemiSphere).
__device__ inline float3 bsdf_f(const PtMaterial& m, float3 wo, float3 wi) {
    if (!(wo.y > 0.0f) || !(wi.y > 0.0f)) return f3(0.0f, 0.0f, 0.0f);
    if (m.type != 1) {
        const float3 R = m.type == 2 ? f3(1.0f, 1.0f, 1.0f) : f3(m.a[0], m.a[1], m.a[2]);
        return R * (kInvPi * fabsf(wi.y));
    }
    const float nov = fabsf(wo.y);
    if (nov == 0.0f) return f3(0.0f, 0.0f, 0.0f);
    const Ggx g(m.rough);
    const float3 wh = normalize3(wi + wo);
    const float3 F = conductor_fresnel(dot3(wo, wh), m.a, m.k);
    return F * (g.D(wh) * g.G1(wo) * g.G1(wi) / (4.0f * nov));
}

__device__ inline float bsdf_pdf(const PtMaterial& m, float3 wo, float3 wi) {
    if (!(wo.y > 0.0f) || !(wi.y > 0.0f)) return 0.0f;
    if (m.type != 1) return fabsf(wi.y) * kInvPi;
    const Ggx g(m.rough);
    const float3 h = normalize3(wo + wi);
    const float eoh = fabsf(dot3(wo, h));
    return g.D(h) * fabsf(h.y) / (4.0f * eoh);
}

__device__ inline float3 bsdf_sample(const PtMaterial& m, float3 wo, float u, float v, float3& wi, float& pdf) {
    if (m.type != 1) {
        wi = cos_sample_hemisphere(u, v);
    } else {
        const Ggx g(m.rough);
        const float3 wh = g.sample(u, v);
        wi = wh * (2.0f * dot3(wo, wh)) - wo;  // reflect(wo, wh)
    }
    pdf = bsdf_pdf(m, wo, wi);
    return bsdf_f(m, wo, wi);
}

// ---- Area light over a quad facing -y (light/area.cpp, shape/quad.cpp) -----
__device__ __forceinline__ float3 light_normal() { return f3(0.0f, -1.0f, 0.0f); }

// Quad::Pdf via Shape::Pdf (shape/shape.h:90-100); also reports the hit distance.
__device__ inline float light_pdf_dir(const PtLight& L, float3 p, float3 wi, float& t_hit) {
    const float oy = -(p.y - L.c[1]), dy = -wi.y;  // the quad's local frame flips y and z
    if (dy == 0.0f) return 0.0f;
    const float t = -oy / dy;
    if (!(t > 0.0f)) return 0.0f;
    const float lx = (p.x - L.c[0]) + t * wi.x;
    const float lz = -(p.z - L.c[2]) + t * (-wi.z);
    if (lx > L.hx || lx < -L.hx || lz > L.hz || lz < -L.hz) return 0.0f;
    const float3 hit = p + wi * t;
    const float3 delta = p - hit;
    const float d = fmaxf(dot3(normalize3(delta), light_normal()), 0.0f);
    if (d <= 0.0f) return 0.0f;
    t_hit = t;
    return dot3(delta, delta) / (L.area * d);
}

__device__ __forceinline__ int warp_append(int* counter, bool want) {
    const unsigned m = __ballot_sync(__activemask(), want);
    if (!want) return -1;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(m) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(counter, __popc(m));
    base = __shfl_sync(m, base, leader);
    return base + __popc(m & ((1u << lane) - 1u));
}

__device__ __forceinline__ void put_ray(float* q, int cap, int i, float3 o, float3 d, float tmin, float tmax) {
    q[i] = o.x;
    q[cap + i] = o.y;
    q[2 * cap + i] = o.z;
    q[3 * cap + i] = d.x;
    q[4 * cap + i] = d.y;
    q[5 * cap + i] = d.z;
    q[6 * cap + i] = tmin;
    q[7 * cap + i] = tmax;
}

// Pinhole camera ray through pixel p (jittered by the sample's random numbers),
// as the reference harness's PerspectiveCamera builds it.
__device__ __forceinline__ float3 camera_dir(const Cam& cam, int width, int height, int p, uint2 key,
                                             uint32_t sample) {
    const int px = p % width, py = p / width;
    const uint4 r = philox(make_uint4((uint32_t)p, sample, 0xffffffffu, 0u), key);
    const float sx = (((float)px + u01(r.x)) / (float)width * 2.0f - 1.0f) * cam.half_w;
    const float sy = (1.0f - ((float)py + u01(r.y)) / (float)height * 2.0f) * cam.half_h;
    return normalize3(cam.fwd + cam.right * sx + cam.up * sy);
}

// What one path vertex produces (PathTracing::li, integrator/pathtracing.cpp:60-254).
struct Vertex {
    bool emit = false;   // add Le to the path's radiance (camera ray on the light, bounce 0)
    bool new_T = false;  // the path's throughput changed to T
    bool cont = false;   // the path continues along wi_next
    bool s1 = false;     // light-sample shadow ray (X, wi1, length len1) carrying c1
    bool s2 = false;     // BSDF-sample shadow ray (X, wi2, up to t2) carrying c2
    float3 Le = {0, 0, 0}, T = {0, 0, 0}, X = {0, 0, 0}, wi_next = {0, 0, 0}, wi1 = {0, 0, 0}, wi2 = {0, 0, 0},
           c1 = {0, 0, 0}, c2 = {0, 0, 0};
    float len1 = 0.0f, t2 = 0.0f;
};

// Shades the hit of ray (o, d) on primitive prim at distance t_hit, for the
// path of pixel p, sample `sample`, at `bounce`, with throughput T: emission
// at the first vertex, both samples of EvaluateDirect
// (integrator/integratormethod.cpp:100-192), the BSDF-sampled continuation and
// Russian roulette, in PathTracing::li's order. Random numbers: Philox keyed
// by the render, counter (p, sample, bounce, stream 0..2).
__device__ __forceinline__ Vertex shade_vertex(const PtDev& sc, uint2 key, uint32_t p, uint32_t sample, int bounce,
                                               int max_depth, float3 o, float3 d, int prim, float t_hit, float3 T) {
    Vertex v;
    v.X = o + d * t_hit;
    const float3 X = v.X;
    const float4 info = __ldg(sc.prim + prim);
    const int mid = __float_as_int(info.w);
    const PtMaterial m = mid < 0 ? PtMaterial{2, {1, 1, 1}, {0, 0, 0}, 0.0f} : sc.mats[mid];
    const PtLight& L = sc.light;
    const float3 Li = f3(L.I[0], L.I[1], L.I[2]);
    const float3 wo_w = -d;
    // Emission only where the camera ray lands (pathtracing.cpp:114-115).
    if (bounce == 0 && mid < 0 && dot3(wo_w, light_normal()) > 0.0f) {
        v.emit = true;
        v.Le = Li;
    }
    const Frame fr = make_frame(f3(info.x, info.y, info.z));
    const float3 wo = fr.local(wo_w);
    const uint4 r0 = philox(make_uint4(p, sample, (uint32_t)bounce, 0u), key);
    const uint4 r1 = philox(make_uint4(p, sample, (uint32_t)bounce, 1u), key);
    const uint4 r2 = philox(make_uint4(p, sample, (uint32_t)bounce, 2u), key);
    // EvaluateDirect, light sample (LightSample: t, u, v).
    {
        const float lu = 2.0f * u01(r0.y) - 1.0f, lv = 2.0f * u01(r0.z) - 1.0f;
        const float3 lp = f3(L.c[0] + L.hx * lu, L.c[1], L.c[2] - L.hz * lv);
        const float3 delta = lp - X;
        const float3 wi = normalize3(delta);
        const float dl = dot3(-wi, light_normal());
        const float lpdf = dl <= 0.0f ? 0.0f : dot3(delta, delta) / (L.area * dl);
        if (lpdf > 0.0f && !black(Li)) {
            const float3 wil = fr.local(wi);
            const float3 f = bsdf_f(m, wo, wil);
            if (!black(f)) {
                const float bpdf = bsdf_pdf(m, wo, wil);
                const float w = mis(lpdf, bpdf);
                v.c1 = T * Li * f * (w / lpdf);
                v.wi1 = wi;
                v.len1 = sqrtf(dot3(delta, delta));
                v.s1 = !black(v.c1);
            }
        }
    }
    // EvaluateDirect, BSDF sample toward the light.
    {
        float3 wil;
        float bpdf;
        const float3 f = bsdf_sample(m, wo, u01(r1.x), u01(r1.y), wil, bpdf);
        if (!black(f) && bpdf != 0.0f) {
            const float3 wi = fr.world(wil);
            float th = 0.0f;
            const float lpdf = light_pdf_dir(L, X, wi, th);
            if (lpdf > 0.0f && !black(Li)) {
                const float w = mis(bpdf, lpdf);
                v.c2 = T * Li * f * (w / bpdf);
                v.wi2 = wi;
                v.t2 = th;
                v.s2 = !black(v.c2);
            }
        }
    }
    // Continuation (pathtracing.cpp:180-254).
    {
        float3 wil;
        float pdf;
        const float3 f = bsdf_sample(m, wo, u01(r1.w), u01(r2.x), wil, pdf);
        if (!black(f) && pdf != 0.0f) {
            T = T * f * (1.0f / pdf);
            if (intensity(T) != 0.0f) {
                v.cont = true;
                if (bounce > 3 && max_comp(T) < 0.1f) {
                    const float cp = fmaxf(0.05f, 1.0f - max_comp(T));
                    if (u01(r2.y) < cp)
                        v.cont = false;
                    else
                        T = T * (1.0f / (1.0f - cp));
                }
                if (bounce + 1 >= max_depth) v.cont = false;
                v.wi_next = fr.world(wil);
                v.T = T;
                v.new_T = true;
            }
        }
    }
    return v;
}

}  // namespace sg
