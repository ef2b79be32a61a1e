// Wavefront path tracer with SORT's PathTracing estimator (integrator/pathtracing.cpp:44-258).
//
// One wave traces one sample for every pixel. Per bounce:
//   extend   closest-hit traversal of the compacted ray queue (trace.cu);
//   shade    for each hit: emission at the first vertex, next-event estimation
//            with both of EvaluateDirect's samples (integratormethod.cpp:100-192:
//            a light sample weighted by MIS against the BSDF, a BSDF sample that
//            hits the light weighted against the light), BSDF sampling of the
//            continuation, Russian roulette, all as PathTracing::li orders them;
//            shadow rays and the next rays are appended to compacted queues with
//            one atomic per warp;
//   shadow   any-hit traversal of the shadow queue;
//   resolve  unoccluded shadow contributions go to their path's two slots, and
//            are added to the path's radiance in a fixed order; at the end of
//            the wave each path's radiance is added to its pixel. Every sum has
//            one writer in a fixed order, so an image is bit-reproducible.
// Shading follows SORT's ScatteringEvent frame (scatteringevent.cpp:42-59) and
// BxDFs: Lambert (lambert.cpp:34-38), MicroFacetReflection with GGX and
// conductor Fresnel (microfacet.cpp:229-356, fresnel.h:119-130); the area light
// is SORT's AreaLight over a Quad (light/area.cpp, shape/quad.cpp), one-sided.
// Random numbers come from Philox4x32-10 (Salmon et al., SC'11), counter-based,
// keyed per render and indexed by (pixel, sample, bounce), so any schedule gives
// the same image. SORT draws from a Mersenne Twister seeded with the wall clock
// (core/rand.cpp:41-55), so images agree in distribution, not sample by sample.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "pt_common.cuh"
#include "pt_wave.h"
#include "scene_access.h"
#include "trace_kernels.h"

namespace sg {
namespace {

// Path p renders frame pixel p0 + p (a band of whole rows starts at p0).
__global__ void k_generate(Cam cam, int width, int height, int p0, int n, uint2 key, uint32_t sample, Queue q,
                           int cap, float* __restrict__ thr, int* __restrict__ count) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    put_ray(q.ray, cap, p, cam.eye, camera_dir(cam, width, height, p0 + p, key, sample), 0.0f, FLT_MAX);
    q.slot[p] = p;
    thr[p] = thr[cap + p] = thr[2 * cap + p] = 1.0f;          // throughput
    thr[3 * cap + p] = thr[4 * cap + p] = thr[5 * cap + p] = 0.0f;  // radiance of this sample
    if (p == 0) *count = n;
}

__global__ void k_shade(PtDev sc, uint2 key, int p0, uint32_t sample, int bounce, int max_depth, Queue in, int cap,
                        const int* __restrict__ in_count, const int32_t* __restrict__ hit_prim,
                        const float* __restrict__ hit_t, Queue next, int* __restrict__ next_count, Queue shadow,
                        int shadow_cap, int* __restrict__ shadow_count, float* __restrict__ thr,
                        float* __restrict__ vis) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= *in_count) return;
    const int p = in.slot[q];
    const int prim = hit_prim[q];
#pragma unroll
    for (int k = 0; k < 6; ++k) vis[k * cap + p] = 0.0f;  // this bounce's two shadow results
    Vertex v;
    if (prim >= 0) {
        const float3 o = f3(in.ray[q], in.ray[cap + q], in.ray[2 * cap + q]);
        const float3 d = f3(in.ray[3 * cap + q], in.ray[4 * cap + q], in.ray[5 * cap + q]);
        v = shade_vertex(sc, key, (uint32_t)(p0 + p), sample, bounce, max_depth, o, d, prim, hit_t[q],
                         f3(thr[p], thr[cap + p], thr[2 * cap + p]));
        if (v.emit) {
            thr[3 * cap + p] += v.Le.x;
            thr[4 * cap + p] += v.Le.y;
            thr[5 * cap + p] += v.Le.z;
        }
        if (v.new_T) {
            thr[p] = v.T.x;
            thr[cap + p] = v.T.y;
            thr[2 * cap + p] = v.T.z;
        }
    }
    const bool s1 = v.s1, s2 = v.s2, cont = v.cont;
    const float3 X = v.X, wi1 = v.wi1, wi2 = v.wi2, c1 = v.c1, c2 = v.c2, wi_next = v.wi_next;
    const float len1 = v.len1, t2 = v.t2;
    const int i1 = warp_append(shadow_count, s1);
    if (i1 >= 0) {
        put_ray(shadow.ray, shadow_cap, i1, X, wi1, 0.01f, len1 - 0.01f);
        shadow.slot[i1] = 2 * p;  // light-sample result
        shadow.contrib[i1] = c1.x;
        shadow.contrib[shadow_cap + i1] = c1.y;
        shadow.contrib[2 * shadow_cap + i1] = c1.z;
    }
    const int i2 = warp_append(shadow_count, s2);
    if (i2 >= 0) {
        put_ray(shadow.ray, shadow_cap, i2, X, wi2, 0.001f, t2 - 0.001f);
        shadow.slot[i2] = 2 * p + 1;  // BSDF-sample result
        shadow.contrib[i2] = c2.x;
        shadow.contrib[shadow_cap + i2] = c2.y;
        shadow.contrib[2 * shadow_cap + i2] = c2.z;
    }
    const int in_next = warp_append(next_count, cont);
    if (in_next >= 0) {
        put_ray(next.ray, cap, in_next, X, wi_next, 0.0001f, FLT_MAX);
        next.slot[in_next] = p;
    }
}

// Unoccluded shadow rays leave their contribution in their path's slot (one
// writer per slot, so the sums below do not depend on scheduling).
__global__ void k_resolve(Queue shadow, int shadow_cap, const int* __restrict__ count, const uint8_t* __restrict__ occ,
                          float* __restrict__ vis, int cap) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= *count || occ[i]) return;
    const int code = shadow.slot[i];
    const int p = code >> 1, which = code & 1;
    vis[(3 * which + 0) * cap + p] = shadow.contrib[i];
    vis[(3 * which + 1) * cap + p] = shadow.contrib[shadow_cap + i];
    vis[(3 * which + 2) * cap + p] = shadow.contrib[2 * shadow_cap + i];
}

// EvaluateDirect's two terms are added to the path's radiance in SORT's order
// (light sample, then BSDF sample), for every path shaded this bounce.
__global__ void k_accumulate(Queue in, const int* __restrict__ in_count, const float* __restrict__ vis,
                             float* __restrict__ thr, int cap) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= *in_count) return;
    const int p = in.slot[q];
#pragma unroll
    for (int c = 0; c < 3; ++c) thr[(3 + c) * cap + p] += vis[c * cap + p] + vis[(3 + c) * cap + p];
}

// End of a wave: each pixel's sample radiance goes into the image (one writer).
__global__ void k_flush(const float* __restrict__ thr, int cap, int n, float* __restrict__ image) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
#pragma unroll
    for (int c = 0; c < 3; ++c) image[3 * p + c] += thr[(3 + c) * cap + p];
}

__global__ void k_scale(float* __restrict__ image, int n, float s) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) image[i] *= s;
}

__global__ void k_zero(float* __restrict__ image, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) image[i] = 0.0f;
}

// Adds this bounce's queue lengths (extension rays, shadow rays) to the totals.
__global__ void k_count_rays(const int* __restrict__ extension, const int* __restrict__ shadow,
                             unsigned long long* __restrict__ totals) {
    if (threadIdx.x == 0) {  // waves of two samples may count at once
        atomicAdd(&totals[0], (unsigned long long)*extension);
        atomicAdd(&totals[1], (unsigned long long)*shadow);
    }
}

}  // namespace
}  // namespace sg

struct sg_pt_scene {
    const sg_scene* scene = nullptr;
    int device = 0;
    float4* d_prim = nullptr;
    sg::PtMaterial* d_mats = nullptr;
    sg::PtLight light{};
    // Per-render buffers, grown on demand.
    int cap = 0;
    void* d_buf = nullptr;
    size_t buf_bytes = 0;
    unsigned long long* d_totals = nullptr;  // rays traced by the last render: extension, shadow
    // kInFlight samples are in flight at once, each with its own buffers:
    // sample k runs on the caller's stream (k % kInFlight == 0) or on
    // extra[k % kInFlight], its shadow rays on side[k % kInFlight]
    // (pt_wave.h); the events order the hand-offs and the image additions.
    // Made by the first render.
    cudaStream_t extra[sg::kInFlight] = {};  // [0] unused: the caller's stream
    cudaStream_t side[sg::kInFlight] = {};
    cudaEvent_t shaded[sg::kInFlight] = {}, shadowed[sg::kInFlight] = {}, flushed[sg::kInFlight] = {};
    cudaEvent_t begun = nullptr;
};

extern "C" sg_status sg_pt_ray_counts(const sg_pt_scene* ps, int64_t* extension, int64_t* shadow, void* stream) {
    if (!ps || !extension || !shadow) return sg::set_error(SG_ERR_INVALID_ARGUMENT, "NULL argument");
    *extension = *shadow = 0;
    if (!ps->d_totals) return SG_OK;
    unsigned long long h[2] = {0, 0};
    cudaError_t e = cudaMemcpyAsync(h, ps->d_totals, sizeof(h), cudaMemcpyDeviceToHost, (cudaStream_t)stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e != cudaSuccess) return sg::set_error(SG_ERR_CUDA, cudaGetErrorString(e));
    *extension = (int64_t)h[0];
    *shadow = (int64_t)h[1];
    return SG_OK;
}

namespace {

sg_status pt_fail(cudaError_t e) { return sg::set_error(SG_ERR_CUDA, cudaGetErrorString(e)); }

}  // namespace

namespace sg {

// Perspective pinhole, as the oracle harness builds SORT's PerspectiveCamera.
Cam make_camera(const float* camera, int width, int height) {
    Cam cam;
    const float3 eye = make_float3(camera[0], camera[1], camera[2]);
    float3 fwd = make_float3(camera[3] - eye.x, camera[4] - eye.y, camera[5] - eye.z);
    const float fl = std::sqrt(fwd.x * fwd.x + fwd.y * fwd.y + fwd.z * fwd.z);
    fwd = make_float3(fwd.x / fl, fwd.y / fl, fwd.z / fl);
    const float3 up = make_float3(camera[6], camera[7], camera[8]);
    float3 right = make_float3(fwd.y * up.z - fwd.z * up.y, fwd.z * up.x - fwd.x * up.z, fwd.x * up.y - fwd.y * up.x);
    const float rl = std::sqrt(right.x * right.x + right.y * right.y + right.z * right.z);
    right = make_float3(right.x / rl, right.y / rl, right.z / rl);
    const float3 upv = make_float3(right.y * fwd.z - right.z * fwd.y, right.z * fwd.x - right.x * fwd.z,
                                   right.x * fwd.y - right.y * fwd.x);
    cam.eye = eye;
    cam.fwd = fwd;
    cam.right = right;
    cam.up = upv;
    cam.half_h = std::tan(camera[9] * 3.14159265358979f / 180.0f * 0.5f);
    cam.half_w = cam.half_h * (float)width / (float)height;
    return cam;
}

sg_status pt_scene_parts(const sg_pt_scene* ps, PtDev* dev, const sg_scene** scene) {
    if (!ps || !dev || !scene) return set_error(SG_ERR_INVALID_ARGUMENT, "NULL path-tracing scene");
    *dev = PtDev{ps->d_prim, ps->d_mats, ps->light};
    *scene = ps->scene;
    return SG_OK;
}

}  // namespace sg

extern "C" sg_status sg_pt_create(const sg_scene* scene, const float* triangles, int64_t ntri, const int32_t* mat_of_tri,
                                  const float* materials, int32_t nmat, const float* light, sg_pt_scene** out) {
    if (!scene || !out || !light || (ntri > 0 && (!triangles || !mat_of_tri)) || nmat < 0 || (nmat > 0 && !materials))
        return sg::set_error(SG_ERR_INVALID_ARGUMENT, "bad path-tracing scene description");
    *out = nullptr;
    sg::TraceLaunch L;
    sg::DevTree tree;
    int device = 0;
    sg_status st = sg::scene_launch(scene, false, &L, &tree, &device);
    if (st != SG_OK) return st;
    std::vector<float4> prim((size_t)std::max<int64_t>(ntri, 1));
    for (int64_t i = 0; i < ntri; ++i) {
        const float* v = triangles + i * 9;
        // SORT's geometric normal, cross(v2 - v0, v1 - v0) normalised (simd_triangle.h:331)
        const float ax = v[6] - v[0], ay = v[7] - v[1], az = v[8] - v[2];
        const float bx = v[3] - v[0], by = v[4] - v[1], bz = v[5] - v[2];
        float nx = ay * bz - az * by, ny = az * bx - ax * bz, nz = ax * by - ay * bx;
        const float len = std::sqrt(nx * nx + ny * ny + nz * nz);
        if (len > 0.0f) {
            nx /= len;
            ny /= len;
            nz /= len;
        } else {
            nx = 0.0f;
            ny = 1.0f;
            nz = 0.0f;
        }
        const int32_t mid = mat_of_tri[i];
        if (mid >= nmat) return sg::set_error(SG_ERR_INVALID_ARGUMENT, "material index out of range");
        float w;
        std::memcpy(&w, &mid, 4);
        prim[(size_t)i] = make_float4(nx, ny, nz, w);
    }
    std::vector<sg::PtMaterial> mats((size_t)std::max(nmat, 1));
    for (int m = 0; m < nmat; ++m) {
        const float* q = materials + (size_t)m * 10;
        sg::PtMaterial pm{};
        pm.type = (int)q[0];
        if (pm.type != 0 && pm.type != 1) return sg::set_error(SG_ERR_INVALID_ARGUMENT, "unknown material type");
        for (int c = 0; c < 3; ++c) {
            pm.a[c] = q[1 + c];
            pm.k[c] = q[4 + c];
        }
        pm.rough = q[7];
        mats[(size_t)m] = pm;
    }
    auto* ps = new sg_pt_scene();
    ps->scene = scene;
    ps->device = device;
    for (int c = 0; c < 3; ++c) {
        ps->light.c[c] = light[c];
        ps->light.I[c] = light[5 + c];
    }
    ps->light.hx = light[3] * 0.5f;
    ps->light.hz = light[4] * 0.5f;
    ps->light.area = light[3] * light[4];
    int prev = -1;
    cudaGetDevice(&prev);
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaMalloc(&ps->d_prim, prim.size() * sizeof(float4));
    if (e == cudaSuccess) e = cudaMalloc(&ps->d_mats, mats.size() * sizeof(sg::PtMaterial));
    if (e == cudaSuccess) e = cudaMemcpy(ps->d_prim, prim.data(), prim.size() * sizeof(float4), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(ps->d_mats, mats.data(), mats.size() * sizeof(sg::PtMaterial), cudaMemcpyHostToDevice);
    if (prev >= 0) cudaSetDevice(prev);
    if (e != cudaSuccess) {
        sg_pt_destroy(ps);
        return pt_fail(e);
    }
    *out = ps;
    return SG_OK;
}

extern "C" sg_status sg_pt_destroy(sg_pt_scene* ps) {
    if (!ps) return SG_OK;
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(ps->device);
    if (ps->d_prim) cudaFree(ps->d_prim);
    if (ps->d_mats) cudaFree(ps->d_mats);
    if (ps->d_buf) cudaFree(ps->d_buf);
    for (int k = 0; k < sg::kInFlight; ++k) {
        for (cudaStream_t t : {ps->extra[k], ps->side[k]})
            if (t) {
                cudaStreamSynchronize(t);
                cudaStreamDestroy(t);
            }
        for (cudaEvent_t ev : {ps->shaded[k], ps->shadowed[k], ps->flushed[k]})
            if (ev) cudaEventDestroy(ev);
    }
    if (ps->begun) cudaEventDestroy(ps->begun);
    if (prev >= 0) cudaSetDevice(prev);
    delete ps;
    return SG_OK;
}

namespace sg {

cudaError_t pt_scale(float* image, int64_t n, float s, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    if (n > int64_t(1) << 30) return cudaErrorInvalidValue;
    k_scale<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(image, (int)n, s);
    return cudaGetLastError();
}

cudaError_t pt_wave(const PtDev& dev, const TraceLaunch& base_in, const DevTree& tree, const Cam& cam, int width,
                    int height, int p0, int n, uint2 key, int sample, int max_depth, const PtWave& w, float* image,
                    cudaStream_t s) {
    const int cap = w.cap, scap = 2 * w.cap;
    if (n <= 0 || n > cap) return cudaErrorInvalidValue;
    TraceLaunch base = base_in;
    base.tuning.schedule = kScheduleThreadPerRay;  // queue lengths live on the device
    Queue qa{w.qa_ray, w.qa_slot, nullptr}, qb{w.qb_ray, w.qb_slot, nullptr};
    const Queue sq{w.sq_ray, w.sq_slot, w.sq_contrib};
    int* counters = w.counters;
    const int threads = 256;
    const int blocks = (n + threads - 1) / threads;
    cudaError_t e = cudaSuccess;
    Queue* cur = &qa;
    Queue* nxt = &qb;
    auto closest = [&](const Queue* q) {
        DevRays r{q->ray,           q->ray + cap,     q->ray + 2 * cap, q->ray + 3 * cap,
                  q->ray + 4 * cap, q->ray + 5 * cap, q->ray + 6 * cap, q->ray + 7 * cap};
        TraceLaunch Lc = base;
        Lc.any = false;
        Lc.prim = w.hit_prim;
        Lc.t = w.hit_t;
        Lc.n_dev = &counters[0];
        return launch_trace_fp32(Lc, tree, r, (int64_t)cap, s);
    };
    // Shadow rays, their results and the path radiance of bounce `cur` on
    // stream t; `shaded` is the length of the bounce's extension queue.
    auto shadows = [&](const Queue* q, const int* shaded, cudaStream_t t) {
        DevRays sr{sq.ray,            sq.ray + scap,     sq.ray + 2 * scap, sq.ray + 3 * scap,
                   sq.ray + 4 * scap, sq.ray + 5 * scap, sq.ray + 6 * scap, sq.ray + 7 * scap};
        TraceLaunch La = base;
        La.any = true;
        La.occ = w.occ;
        La.n_dev = &counters[2];
        cudaError_t r = launch_trace_fp32(La, tree, sr, (int64_t)scap, t);
        if (r != cudaSuccess) return r;
        k_resolve<<<(scap + threads - 1) / threads, threads, 0, t>>>(sq, scap, &counters[2], w.occ, w.vis, cap);
        k_accumulate<<<blocks, threads, 0, t>>>(*q, shaded, w.vis, w.thr, cap);
        k_count_rays<<<1, 32, 0, t>>>(shaded, &counters[2], w.totals);
        return cudaGetLastError();
    };
    k_generate<<<blocks, threads, 0, s>>>(cam, width, height, p0, n, key, (uint32_t)sample, *cur, cap, w.thr,
                                          &counters[0]);
    if ((e = closest(cur)) != cudaSuccess) return e;
    for (int bounce = 0; bounce < max_depth; ++bounce) {
        if ((e = cudaMemsetAsync(&counters[1], 0, 2 * sizeof(int), s)) != cudaSuccess) return e;
        k_shade<<<blocks, threads, 0, s>>>(dev, key, p0, (uint32_t)sample, bounce, max_depth, *cur, cap,
                                           &counters[0], w.hit_prim, w.hit_t, *nxt, &counters[1], sq, scap,
                                           &counters[2], w.thr, w.vis);
        const bool more = bounce + 1 < max_depth;
        if (!w.side) {
            if ((e = shadows(cur, &counters[0], s)) != cudaSuccess) return e;
        } else {
            // The shadow rays of this bounce go to the side stream and run
            // beside the next bounce's extension rays; the next shading (which
            // reuses the shadow queue, the path state and the counters) waits
            // for them.
            if ((e = cudaMemcpyAsync(&counters[3], &counters[0], sizeof(int), cudaMemcpyDeviceToDevice, s)) !=
                    cudaSuccess ||
                (e = cudaEventRecord(w.shaded, s)) != cudaSuccess ||
                (e = cudaStreamWaitEvent(w.side, w.shaded, 0)) != cudaSuccess ||
                (e = shadows(cur, &counters[3], w.side)) != cudaSuccess ||
                (e = cudaEventRecord(w.shadowed, w.side)) != cudaSuccess)
                return e;
        }
        // the next queue becomes the current one
        if ((e = cudaMemcpyAsync(&counters[0], &counters[1], sizeof(int), cudaMemcpyDeviceToDevice, s)) !=
            cudaSuccess)
            return e;
        Queue* t = cur;
        cur = nxt;
        nxt = t;
        if (more && (e = closest(cur)) != cudaSuccess) return e;
        if (w.side && (e = cudaStreamWaitEvent(s, w.shadowed, 0)) != cudaSuccess) return e;
    }
    if (w.flush_after && (e = cudaStreamWaitEvent(s, w.flush_after, 0)) != cudaSuccess) return e;
    k_flush<<<blocks, threads, 0, s>>>(w.thr, cap, n, image);
    if (w.flush_done && (e = cudaEventRecord(w.flush_done, s)) != cudaSuccess) return e;
    return cudaGetLastError();
}

}  // namespace sg

extern "C" sg_status sg_pt_render(sg_pt_scene* ps, const float* camera, int32_t width, int32_t height, int32_t spp,
                                  int32_t max_depth, uint64_t seed, float* image, void* stream) {
    return sg_pt_render_rows(ps, camera, width, height, 0, height, spp, max_depth, seed, image, stream);
}

extern "C" sg_status sg_pt_render_rows(sg_pt_scene* ps, const float* camera, int32_t width, int32_t height,
                                       int32_t row_begin, int32_t row_end, int32_t spp, int32_t max_depth,
                                       uint64_t seed, float* image, void* stream) {
    if (!ps || !camera || !image || width <= 0 || height <= 0 || spp <= 0 || max_depth <= 0)
        return sg::set_error(SG_ERR_INVALID_ARGUMENT, "bad render arguments");
    if ((int64_t)width * height > (int64_t)1 << 28) return sg::set_error(SG_ERR_LIMIT, "image too large");
    if (row_begin < 0 || row_end > height || row_begin >= row_end)
        return sg::set_error(SG_ERR_INVALID_ARGUMENT, "bad row range");
    const int P = width * (row_end - row_begin);  // pixels of the band
    const int p0 = width * row_begin;
    sg::TraceLaunch base;
    sg::DevTree tree;
    int device = 0;
    sg_status st = sg::scene_launch(ps->scene, false, &base, &tree, &device);
    if (st != SG_OK) return st;
    base.tuning.schedule = sg::kScheduleThreadPerRay;  // queue lengths live on the device
    int prev = -1;
    cudaGetDevice(&prev);
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return pt_fail(e);
    struct Restore {
        int dev;
        ~Restore() {
            if (dev >= 0) cudaSetDevice(dev);
        }
    } restore{prev};
    cudaStream_t s = (cudaStream_t)stream;

    // Buffers, kInFlight times (samples in flight): two extension queues (rays +
    // slots), hits, one shadow queue of 2 entries per path (rays + slots +
    // contributions), occlusion flags, throughput, shadow results, 4
    // counters; then the shared ray totals.
    const size_t cap = (size_t)P, scap = 2 * (size_t)P;
    auto align = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t qbytes = align(cap * 8 * 4) + align(cap * 4);
    const size_t set = 2 * qbytes + align(cap * 4) * 2 + align(scap * 8 * 4) + align(scap * 4) +
                       align(scap * 3 * 4) + align(scap) + align(cap * 6 * 4) + align(cap * 6 * 4) + align(16);
    const size_t need = sg::kInFlight * set + align(16);
    if (ps->buf_bytes < need) {
        if (ps->d_buf) cudaFree(ps->d_buf);
        ps->d_buf = nullptr;
        ps->buf_bytes = 0;
        if ((e = cudaMalloc(&ps->d_buf, need)) != cudaSuccess) return pt_fail(e);
        ps->buf_bytes = need;
    }
    char* b = (char*)ps->d_buf;
    auto take = [&](size_t bytes) {
        char* r = b;
        b += align(bytes);
        return r;
    };
    bool made = true;
    for (int k = 0; k < sg::kInFlight; ++k) {
        for (cudaStream_t* t : {&ps->extra[k], &ps->side[k]})
            if (t != &ps->extra[0])
                made = made && (*t || cudaStreamCreateWithFlags(t, cudaStreamNonBlocking) == cudaSuccess);
        for (cudaEvent_t* ev : {&ps->shaded[k], &ps->shadowed[k], &ps->flushed[k]})
            made = made && (*ev || cudaEventCreateWithFlags(ev, cudaEventDisableTiming) == cudaSuccess);
    }
    made = made && (ps->begun || cudaEventCreateWithFlags(&ps->begun, cudaEventDisableTiming) == cudaSuccess);
    if (!made) return sg::set_error(SG_ERR_CUDA, "render streams and events");
    sg::PtWave w[sg::kInFlight] = {};
    for (int k = 0; k < sg::kInFlight; ++k) {
        w[k].qa_ray = (float*)take(cap * 32);
        w[k].qa_slot = (int*)take(cap * 4);
        w[k].qb_ray = (float*)take(cap * 32);
        w[k].qb_slot = (int*)take(cap * 4);
        w[k].hit_prim = (int32_t*)take(cap * 4);
        w[k].hit_t = (float*)take(cap * 4);
        w[k].sq_ray = (float*)take(scap * 32);
        w[k].sq_slot = (int*)take(scap * 4);
        w[k].sq_contrib = (float*)take(scap * 12);
        w[k].occ = (uint8_t*)take(scap);
        w[k].thr = (float*)take(cap * 24);  // throughput and radiance per path
        w[k].vis = (float*)take(cap * 24);  // two shadow results per path
        w[k].counters = (int*)take(16);     // current, next, shadow queue; the shaded queue's length
        w[k].cap = (int)cap;
        w[k].side = ps->side[k];
        w[k].shaded = ps->shaded[k];
        w[k].shadowed = ps->shadowed[k];
        w[k].flush_done = ps->flushed[k];
    }
    unsigned long long* totals = (unsigned long long*)take(16);  // rays traced: extension, shadow
    if ((size_t)(b - (char*)ps->d_buf) > need) return sg::set_error(SG_ERR_INTERNAL, "render buffer layout overflow");
    for (sg::PtWave& x : w) x.totals = totals;
    ps->d_totals = totals;
    if ((e = cudaMemsetAsync(totals, 0, 16, s)) != cudaSuccess) return pt_fail(e);

    const sg::Cam cam = sg::make_camera(camera, width, height);
    const uint2 key = make_uint2((uint32_t)seed, (uint32_t)(seed >> 32));
    sg::PtDev dev{ps->d_prim, ps->d_mats, ps->light};
    const int threads = 256;
    const int img_n = 3 * P;
    sg::k_zero<<<(img_n + threads - 1) / threads, threads, 0, s>>>(image, img_n);
    // The other streams start after everything the caller put on `stream`.
    if ((e = cudaEventRecord(ps->begun, s)) != cudaSuccess) return pt_fail(e);
    for (int k = 1; k < sg::kInFlight; ++k)
        if ((e = cudaStreamWaitEvent(ps->extra[k], ps->begun, 0)) != cudaSuccess) return pt_fail(e);
    for (int sample = 0; sample < spp; ++sample) {
        const int set = sample % sg::kInFlight;
        sg::PtWave& ws = w[set];
        ws.flush_after = sample > 0 ? ps->flushed[(sample - 1) % sg::kInFlight] : nullptr;  // image sums in order
        const cudaStream_t on = set ? ps->extra[set] : s;
        if ((e = sg::pt_wave(dev, base, tree, cam, width, height, p0, P, key, sample, max_depth, ws, image, on)) !=
            cudaSuccess)
            return pt_fail(e);
    }
    // Every stream's work is done before the scale: the last addition closes
    // the chain, and every other stream's last sample precedes it.
    if ((e = cudaStreamWaitEvent(s, ps->flushed[(spp - 1) % sg::kInFlight], 0)) != cudaSuccess) return pt_fail(e);
    sg::k_scale<<<(img_n + threads - 1) / threads, threads, 0, s>>>(image, img_n, 1.0f / (float)spp);
    if ((e = cudaGetLastError()) != cudaSuccess) return pt_fail(e);
    return SG_OK;
}
