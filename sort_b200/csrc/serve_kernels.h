// Device tables of the render server (server.cpp) and the launcher of its
// bounce steps (serve.cu).
//
// Work is a ring of pixel samples: entry = (request, pixel, sample). Admission
// appends the admission's first sample to render of every pixel of a request; free path slots claim entries
// from the ring's head. A path that ends adds its radiance to its pixel; its
// slot then renders the pixel's next sample itself, up to samples_per_claim
// samples per claim, and after that appends the pixel's next sample at the
// ring's end. So a pixel has at most one sample in flight (its samples
// accumulate in order), requests take turns chunk by chunk, and slots keep
// runs of neighbouring pixels (coherent camera and bounce rays).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "layout.h"
#include "pt_types.h"

namespace sg {

struct SrvRequest {
    Cam cam;
    uint2 key;
    float* image;  // width * height * 3 floats (device)
    int32_t scene;
    int32_t width;
    int32_t height;
    int32_t spp;
    int32_t max_depth;
    float inv_spp;  // 1 / spp, rounded once on the host like sg_pt_render's scale
    int32_t cancelled;
    int32_t pad;
};

struct SrvScene {
    DevTree tree;
    PtDev pt;
};

constexpr int kSrvMaxAdmit = 256;  // admissions per graph replay

struct SrvAdmit {
    int32_t request;  // request-table index
    int32_t pixels;
    int64_t first;    // offset among this replay's admitted pixels
    int32_t sample0;  // first sample to render (earlier ones are in the image already; 0 today)
    int32_t pad;
};

// Staged by the host before each replay.
struct SrvControl {
    int32_t nadmit;
    int32_t pad;
    int64_t admit_total;
    SrvAdmit admit[kSrvMaxAdmit];
};

struct SrvCounters {
    int queue[4];               // [0] current extension queue, [1] next, [2] shadow queue,
                                // [3] continuation rays of the current queue already traced
    unsigned long long head;    // ring entries claimed
    unsigned long long tail;    // ring entries appended
    unsigned long long ext_rays, shadow_rays;
};

// Ring entry: request (16 bits) | sample (16 bits) | pixel (32 bits).
__host__ __device__ inline unsigned long long srv_unit(int request, int sample, int pixel) {
    return ((unsigned long long)(unsigned)request << 48) | ((unsigned long long)(unsigned)sample << 32) |
           (unsigned long long)(unsigned)pixel;
}

constexpr int kSlotIdle = 0;      // claims a ring entry at the next regen
constexpr int kSlotActive = 1;    // a path is in flight
constexpr int kSlotFinished = 2;  // its path ended this step (accumulate settles it)
constexpr int kSlotNext = 3;      // starts its pixel's next sample at the next regen

struct SrvBuffers {
    const SrvRequest* requests;
    const SrvScene* scenes;
    const SrvControl* control;
    SrvCounters* counters;
    unsigned int* units_left;  // per request: pixels not yet finished
    int* done;                 // per request: 1 once every pixel is finished
    unsigned long long* ring;
    int64_t ring_cap;
    int64_t slots;          // path pool size C
    int samples_per_claim;  // samples a slot renders of its pixel before returning it to the ring
    int* st_req;
    int* st_pix;
    int* st_sample;
    int* st_bounce;
    int* st_state;
    float* thr;  // 6 * C: throughput, radiance of the current sample
    float* vis;  // 6 * C: this bounce's two shadow-ray results
    float* qa_ray;
    int* qa_slot;
    int* qa_scene;
    float* qb_ray;
    int* qb_slot;
    int* qb_scene;
    int32_t* hit_prim;
    float* hit_t;
    float* sq_ray;  // shadow queue, 2 * C entries
    int* sq_slot;
    int* sq_scene;
    float* sq_contrib;
    uint8_t* occ;
    int* err;
};

// Bytes of path state per pool slot (the buffers above, per slot).
constexpr int64_t kSrvBytesPerSlot = 5 * 4 + 6 * 4 * 2 + 2 * (8 * 4 + 4 + 4) + 4 + 4 + 2 * (8 * 4 + 4 + 4 + 3 * 4 + 1);

// Stream pair of the bounce steps: with a side stream, a step's continuation
// rays are traced on it beside the step's shadow rays (the next step then
// traces only the camera rays its regeneration adds); `forked` and `joined`
// are the hand-off events.
struct SrvStreams {
    cudaStream_t main;
    cudaStream_t side;  // may be null: everything on `main`
    cudaEvent_t forked, joined;
};

// Enqueues `iterations` bounce steps; the first takes this replay's
// admissions. Tree width / stack / node format are those of every scene.
cudaError_t srv_enqueue_steps(const SrvBuffers& b, int iterations, int width, int stack, bool q8,
                              const SrvStreams& st);

}  // namespace sg
