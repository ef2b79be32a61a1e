// One wave of the wavefront path tracer (pt.cu): one sample for every pixel
// of a band, on caller-provided buffers. sg_pt_render_rows runs one wave per
// sample on the render's own buffers; the render server (server.cpp) runs
// waves on its idle path pool for a request that has the GPU to itself.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "pt_types.h"
#include "trace_kernels.h"

namespace sg {

// Samples sg_pt_render keeps in flight, each on its own buffers and streams.
constexpr int kInFlight = 2;

// Device buffers of a wave, with the layouts the server's pool uses: two
// extension queues (8 floats per ray with stride cap, a path index per
// entry), the hits (cap each), the shadow queue (stride 2 * cap, three
// contribution planes) and its occlusion flags, per-path throughput and
// radiance (6 * cap floats) and shadow results (6 * cap), four queue
// counters (current, next, shadow, and the shaded queue's length for the side
// stream) and two ray totals (extension, shadow).
struct PtWave {
    float* qa_ray;
    int* qa_slot;
    float* qb_ray;
    int* qb_slot;
    float* sq_ray;
    int* sq_slot;
    float* sq_contrib;
    int32_t* hit_prim;
    float* hit_t;
    uint8_t* occ;
    float* thr;
    float* vis;
    int* counters;  // 4: current, next and shadow queue lengths, the shaded queue's length
    unsigned long long* totals;
    int cap;
    // Optional: a second stream on which each bounce's shadow rays run beside
    // the next bounce's extension rays, with two events for the hand-offs.
    cudaStream_t side;
    cudaEvent_t shaded, shadowed;
    // Optional: the radiance is added to the image only after `flush_after`
    // (the previous sample's addition, when samples run on several streams),
    // and `flush_done` is recorded after it.
    cudaEvent_t flush_after, flush_done;
};

// Sample `sample` of pixels p0 .. p0 + n - 1 (n <= w.cap) of a width x height
// frame: each pixel's radiance is added to image[3 * (p - p0) + c]; nothing is
// zeroed or scaled. Every pixel draws the random numbers of its place in the
// frame, so waves over bands and over whole frames give the same sums.
// `base` is the scene's launch (scene_launch), `tree` its tree.
// image[i] *= s for i < n (the 1/spp of a finished render), on stream st.
cudaError_t pt_scale(float* image, int64_t n, float s, cudaStream_t st);

cudaError_t pt_wave(const PtDev& dev, const TraceLaunch& base, const DevTree& tree, const Cam& cam, int width,
                    int height, int p0, int n, uint2 key, int sample, int max_depth, const PtWave& w, float* image,
                    cudaStream_t s);

}  // namespace sg
