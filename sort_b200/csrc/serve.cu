// Bounce steps of the render server: a path pool shared by every admitted
// request, refilled from the ring of pixel samples, traced through
// multi-scene extension and shadow queues and shaded with the single-render
// vertex code (pt_common.cuh), so each path's radiance is bit-identical to
// sg_pt_render's for the same request, pixel and sample.
//
// One step:
//   regen       slots holding a pixel start its next sample; idle slots
//               claim ring entries (one atomic per warp); each starts the
//               camera path of that pixel sample;
//   settle      the claim counter is pulled back to the ring's end if warps
//               over-claimed;
//   extend      closest-hit traversal of the extension queue, each ray in its
//               own scene's tree (after a replay's first step only the camera
//               rays: the continuations were traced on the side stream during
//               the previous step's shadow rays);
//   shade       shade_vertex per hit; shadow rays and continuations appended
//               with their scene;
//   shadow      any-hit traversal of the shadow queue;
//   resolve     unoccluded shadow results to their slot;
//   accumulate  both results added to the path's radiance (sg_pt_render's
//               order); an ended path adds its radiance to its pixel; the slot
//               keeps the pixel for its next sample, or at the end of a claim
//               appends that sample to the ring, or after the last sample
//               scales the pixel by 1/spp and counts it finished;
//   advance     the next extension queue becomes the current one.
// Every kernel's grid covers the pool (or the shadow queue) and reads its
// length on the device, so a step is a fixed sequence of launches that a
// CUDA graph can replay.
#include <cuda_runtime.h>

#include "pt_common.cuh"
#include "serve_kernels.h"
#include "traversal.cuh"

namespace sg {
namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ unsigned long long warp_append64(unsigned long long* counter, bool want) {
    const unsigned m = __ballot_sync(__activemask(), want);
    if (!want) return ~0ull;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(m) - 1;
    unsigned long long base = 0;
    if (lane == leader) base = atomicAdd(counter, (unsigned long long)__popc(m));
    base = __shfl_sync(m, base, leader);
    return base + __popc(m & ((1u << lane) - 1u));
}

__device__ __forceinline__ void pixel_finished(const SrvBuffers& b, int r) {
    if (atomicSub(&b.units_left[r], 1u) == 1u) b.done[r] = 1;
}

// This replay's admissions: the first sample to render of every pixel, appended after the ring's end.
__global__ void k_srv_admit(SrvBuffers b) {
    const SrvControl* c = b.control;
    const int64_t total = c->admit_total;
    const unsigned long long tail = b.counters->tail;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        int lo = 0, hi = c->nadmit - 1;  // last admission whose first pixel is <= i
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (c->admit[mid].first <= i)
                lo = mid;
            else
                hi = mid - 1;
        }
        const SrvAdmit ad = c->admit[lo];
        b.ring[(tail + (unsigned long long)i) % (unsigned long long)b.ring_cap] =
            srv_unit(ad.request, ad.sample0, (int)(i - ad.first));
    }
}

__global__ void k_srv_admit_commit(SrvBuffers b) {
    if (threadIdx.x == 0 && blockIdx.x == 0) b.counters->tail += (unsigned long long)b.control->admit_total;
}

__global__ void k_srv_regen(SrvBuffers b, float* __restrict__ qray, int* __restrict__ qslot,
                            int* __restrict__ qscene) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = s < b.slots;
    const unsigned long long tail = b.counters->tail;
    const int state = in ? b.st_state[s] : kSlotActive;
    const bool want = state == kSlotIdle;
    const unsigned long long idx = warp_append64(&b.counters->head, want);
    int r, sample, pix;
    if (state == kSlotNext) {  // the next sample of the pixel this slot holds
        r = b.st_req[s];
        pix = b.st_pix[s];
        sample = b.st_sample[s];
    } else if (want && idx < tail) {
        const unsigned long long u = b.ring[idx % (unsigned long long)b.ring_cap];
        r = (int)(u >> 48);
        sample = (int)((u >> 32) & 0xffffu);
        pix = (int)(u & 0xffffffffu);
    } else {
        return;
    }
    const SrvRequest& q = b.requests[r];
    if (q.cancelled) {
        pixel_finished(b, r);
        b.st_state[s] = kSlotIdle;
        return;
    }
    const int C = (int)b.slots;
    const float3 d = camera_dir(q.cam, q.width, q.height, pix, q.key, (uint32_t)sample);
    const int i = warp_append(&b.counters->queue[0], true);
    put_ray(qray, C, i, q.cam.eye, d, 0.0f, FLT_MAX);
    qslot[i] = (int)s;
    qscene[i] = q.scene;
    b.st_req[s] = r;
    b.st_pix[s] = pix;
    b.st_sample[s] = sample;
    b.st_bounce[s] = 0;
    b.st_state[s] = kSlotActive;
    b.thr[s] = b.thr[C + s] = b.thr[2 * C + s] = 1.0f;
    b.thr[3 * C + s] = b.thr[4 * C + s] = b.thr[5 * C + s] = 0.0f;
}

__global__ void k_srv_settle(SrvBuffers b) {
    if (threadIdx.x == 0 && blockIdx.x == 0 && b.counters->head > b.counters->tail)
        b.counters->head = b.counters->tail;
}

// One ray per thread over a queue of rays from many scenes. Held to 9 blocks
// of 128 per SM (56 registers; 12 bytes spilled for width-8 FP32 trees):
// serve_27m's closed loop runs 3.6% faster than at the compiler's 60-80
// registers.
// Rays begin (null: 0) .. count - 1 of the queue.
template <int W, bool ANY, int STACK, bool Q8>
__global__ void __launch_bounds__(128, 9) k_srv_trace(const SrvScene* __restrict__ scenes, const float* __restrict__ ray,
                                                   const int* __restrict__ scene_of, int cap,
                                                   const int* __restrict__ begin, const int* __restrict__ count,
                                                   int32_t* __restrict__ prim, float* __restrict__ t,
                                                   uint8_t* __restrict__ occ, int* __restrict__ err) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= *count || (begin && i < *begin)) return;
    const DevTree tr = scenes[scene_of[i]].tree;
    const DevRays rays{ray, ray + cap, ray + 2 * cap, ray + 3 * cap, ray + 4 * cap, ray + 5 * cap, ray + 6 * cap,
                       ray + 7 * cap};
    RayWalk<W, ANY, STACK, Q8> tv;
    uint2 stk[STACK];
    if (tv.start(tr, rays, i))
        while (!tv.step(tr, stk, err)) {
        }
    tv.finish(tr, i, prim, t, nullptr, nullptr, occ);
}

__global__ void k_srv_shade(SrvBuffers b, const float* __restrict__ qray, const int* __restrict__ qslot,
                            const int* __restrict__ qscene, float* __restrict__ nray, int* __restrict__ nslot,
                            int* __restrict__ nscene) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= b.counters->queue[0]) return;
    const int C = (int)b.slots, SC = 2 * C;
    const int s = qslot[q];
    const int sc = qscene[q];
    const int prim = b.hit_prim[q];
    float* thr = b.thr;
#pragma unroll
    for (int k = 0; k < 6; ++k) b.vis[k * C + s] = 0.0f;
    Vertex v;
    if (prim >= 0) {
        const SrvRequest& rq = b.requests[b.st_req[s]];
        const float3 o = f3(qray[q], qray[C + q], qray[2 * C + q]);
        const float3 d = f3(qray[3 * C + q], qray[4 * C + q], qray[5 * C + q]);
        v = shade_vertex(b.scenes[sc].pt, rq.key, (uint32_t)b.st_pix[s], (uint32_t)b.st_sample[s], b.st_bounce[s],
                         rq.max_depth, o, d, prim, b.hit_t[q], f3(thr[s], thr[C + s], thr[2 * C + s]));
        if (v.emit) {
            thr[3 * C + s] += v.Le.x;
            thr[4 * C + s] += v.Le.y;
            thr[5 * C + s] += v.Le.z;
        }
        if (v.new_T) {
            thr[s] = v.T.x;
            thr[C + s] = v.T.y;
            thr[2 * C + s] = v.T.z;
        }
    }
    const int i1 = warp_append(&b.counters->queue[2], v.s1);
    if (i1 >= 0) {
        put_ray(b.sq_ray, SC, i1, v.X, v.wi1, 0.01f, v.len1 - 0.01f);
        b.sq_slot[i1] = 2 * s;
        b.sq_scene[i1] = sc;
        b.sq_contrib[i1] = v.c1.x;
        b.sq_contrib[SC + i1] = v.c1.y;
        b.sq_contrib[2 * SC + i1] = v.c1.z;
    }
    const int i2 = warp_append(&b.counters->queue[2], v.s2);
    if (i2 >= 0) {
        put_ray(b.sq_ray, SC, i2, v.X, v.wi2, 0.001f, v.t2 - 0.001f);
        b.sq_slot[i2] = 2 * s + 1;
        b.sq_scene[i2] = sc;
        b.sq_contrib[i2] = v.c2.x;
        b.sq_contrib[SC + i2] = v.c2.y;
        b.sq_contrib[2 * SC + i2] = v.c2.z;
    }
    const int in = warp_append(&b.counters->queue[1], v.cont);
    if (in >= 0) {
        put_ray(nray, C, in, v.X, v.wi_next, 0.0001f, FLT_MAX);
        nslot[in] = s;
        nscene[in] = sc;
        b.st_bounce[s] += 1;
    } else {
        b.st_state[s] = kSlotFinished;
    }
}

__global__ void k_srv_resolve(SrvBuffers b) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= b.counters->queue[2] || b.occ[i]) return;
    const int C = (int)b.slots, SC = 2 * C;
    const int code = b.sq_slot[i];
    const int s = code >> 1, which = code & 1;
    b.vis[(3 * which + 0) * C + s] = b.sq_contrib[i];
    b.vis[(3 * which + 1) * C + s] = b.sq_contrib[SC + i];
    b.vis[(3 * which + 2) * C + s] = b.sq_contrib[2 * SC + i];
}

__global__ void k_srv_accumulate(SrvBuffers b, const int* __restrict__ qslot) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= b.counters->queue[0]) return;
    const int C = (int)b.slots;
    const int s = qslot[q];
    float* thr = b.thr;
#pragma unroll
    for (int c = 0; c < 3; ++c) thr[(3 + c) * C + s] += b.vis[c * C + s] + b.vis[(3 + c) * C + s];
    const bool ended = b.st_state[s] == kSlotFinished;
    bool requeue = false, pixel_done = false;
    int r = 0, pix = 0, sample = 0;
    if (ended) {
        r = b.st_req[s];
        pix = b.st_pix[s];
        sample = b.st_sample[s];
        const SrvRequest& rq = b.requests[r];
        bool more = false;
        if (!rq.cancelled) {
            float* px = rq.image + 3 * (int64_t)pix;
#pragma unroll
            for (int c = 0; c < 3; ++c) px[c] += thr[(3 + c) * C + s];
            more = sample + 1 < rq.spp;
            if (!more) {
#pragma unroll
                for (int c = 0; c < 3; ++c) px[c] *= rq.inv_spp;
            }
        }
        if (more && (sample + 1) % b.samples_per_claim != 0) {  // keep the pixel
            b.st_sample[s] = sample + 1;
            b.st_state[s] = kSlotNext;
        } else {
            requeue = more;
            pixel_done = !more;
            b.st_state[s] = kSlotIdle;
        }
    }
    const unsigned long long at = warp_append64(&b.counters->tail, requeue);
    if (requeue) b.ring[at % (unsigned long long)b.ring_cap] = srv_unit(r, sample + 1, pix);
    // Finished pixels, one atomic per warp and request (a request's pixels
    // finish together, so one counter per request would otherwise serialise).
    const unsigned fm = __ballot_sync(__activemask(), pixel_done);
    if (pixel_done) {
        const unsigned peers = __match_any_sync(fm, r);
        if ((int)(threadIdx.x & 31) == __ffs(peers) - 1) {
            const unsigned c = (unsigned)__popc(peers);
            if (atomicSub(&b.units_left[r], c) == c) b.done[r] = 1;
        }
    }
}

__global__ void k_srv_advance(SrvBuffers b) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    SrvCounters* c = b.counters;
    c->ext_rays += (unsigned long long)c->queue[0];
    c->shadow_rays += (unsigned long long)c->queue[2];
    c->queue[0] = c->queue[1];
    c->queue[1] = 0;
    c->queue[2] = 0;
}

template <int W, bool Q8, int STACK>
cudaError_t enqueue_stack(const SrvBuffers& b, int iterations, const SrvStreams& st) {
    const cudaStream_t s = st.main;
    const int C = (int)b.slots;
    const int pool_blocks = (C + kThreads - 1) / kThreads;
    const int trace_blocks = (C + 127) / 128;
    const int shadow_blocks = (2 * C + 127) / 128;
    cudaError_t e = cudaSuccess;
    for (int it = 0; it < iterations; ++it) {
        const bool a_cur = (it % 2) == 0;  // even steps read queue A and write queue B
        float* cray = a_cur ? b.qa_ray : b.qb_ray;
        int* cslot = a_cur ? b.qa_slot : b.qb_slot;
        int* cscene = a_cur ? b.qa_scene : b.qb_scene;
        float* nray = a_cur ? b.qb_ray : b.qa_ray;
        int* nslot = a_cur ? b.qb_slot : b.qa_slot;
        int* nscene = a_cur ? b.qb_scene : b.qa_scene;
        // Continuations of this queue traced by the previous step on the side stream.
        const bool traced = st.side && it > 0;
        if (it == 0) {
            k_srv_admit<<<1184, kThreads, 0, s>>>(b);
            k_srv_admit_commit<<<1, 32, 0, s>>>(b);
        }
        k_srv_regen<<<pool_blocks, kThreads, 0, s>>>(b, cray, cslot, cscene);
        k_srv_settle<<<1, 32, 0, s>>>(b);
        k_srv_trace<W, false, STACK, Q8><<<trace_blocks, 128, 0, s>>>(
            b.scenes, cray, cscene, C, traced ? &b.counters->queue[3] : nullptr, &b.counters->queue[0], b.hit_prim,
            b.hit_t, nullptr, b.err);
        if (traced && (e = cudaStreamWaitEvent(s, st.joined, 0)) != cudaSuccess) return e;
        k_srv_shade<<<pool_blocks, kThreads, 0, s>>>(b, cray, cslot, cscene, nray, nslot, nscene);
        if (st.side && it + 1 < iterations) {
            // The next queue's continuation rays are complete: trace them on the
            // side stream (their count fixed in queue[3]; advance resets queue[1]).
            if ((e = cudaMemcpyAsync(&b.counters->queue[3], &b.counters->queue[1], sizeof(int),
                                     cudaMemcpyDeviceToDevice, s)) != cudaSuccess ||
                (e = cudaEventRecord(st.forked, s)) != cudaSuccess ||
                (e = cudaStreamWaitEvent(st.side, st.forked, 0)) != cudaSuccess)
                return e;
            k_srv_trace<W, false, STACK, Q8><<<trace_blocks, 128, 0, st.side>>>(
                b.scenes, nray, nscene, C, nullptr, &b.counters->queue[3], b.hit_prim, b.hit_t, nullptr, b.err);
            if ((e = cudaEventRecord(st.joined, st.side)) != cudaSuccess) return e;
        }
        k_srv_trace<W, true, STACK, Q8><<<shadow_blocks, 128, 0, s>>>(
            b.scenes, b.sq_ray, b.sq_scene, 2 * C, nullptr, &b.counters->queue[2], nullptr, nullptr, b.occ, b.err);
        k_srv_resolve<<<(2 * C + kThreads - 1) / kThreads, kThreads, 0, s>>>(b);
        k_srv_accumulate<<<pool_blocks, kThreads, 0, s>>>(b, cslot);
        k_srv_advance<<<1, 32, 0, s>>>(b);
    }
    return cudaGetLastError();
}

template <int W, bool Q8>
cudaError_t enqueue_w(const SrvBuffers& b, int iterations, int stack, const SrvStreams& st) {
    if (stack <= 64) return enqueue_stack<W, Q8, 64>(b, iterations, st);
    if (stack <= 128) return enqueue_stack<W, Q8, 128>(b, iterations, st);
    if (stack <= 256) return enqueue_stack<W, Q8, 256>(b, iterations, st);
    return cudaErrorInvalidValue;
}

}  // namespace

cudaError_t srv_enqueue_steps(const SrvBuffers& b, int iterations, int width, int stack, bool q8,
                              const SrvStreams& st) {
    if (iterations < 2 || iterations % 2 != 0) return cudaErrorInvalidValue;
    if (width == 8)
        return q8 ? enqueue_w<8, true>(b, iterations, stack, st) : enqueue_w<8, false>(b, iterations, stack, st);
    if (width == 4)
        return q8 ? enqueue_w<4, true>(b, iterations, stack, st) : enqueue_w<4, false>(b, iterations, stack, st);
    return cudaErrorInvalidValue;
}

}  // namespace sg
