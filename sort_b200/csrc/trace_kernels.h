// Host-side launch wrappers of the traversal kernels (implemented in trace.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "layout.h"

namespace sg {

constexpr int kScheduleThreadPerRay = 0;  // one ray per thread for the whole launch
constexpr int kSchedulePersistent = 1;    // persistent warps refilling idle lanes
constexpr int kScheduleWhileWhile = 2;    // warp alternates interior and leaf phases
constexpr int kScheduleSpeculative = 3;   // while-while, lanes keep descending past their first leaf
constexpr int kScheduleSorted = 4;        // one ray per thread, rays taken in the order of a coherence key
constexpr int kScheduleAuto = 5;          // sorted for large closest-hit batches, else thread per ray

struct TraceTuning {
    int schedule = kScheduleAuto;
    int refill_threshold = 8;  // idle lanes of a warp that trigger a refill (1..32)
};

struct TraceLaunch {
    int width = 8;
    bool any = false;
    int stack_need = 1;  // depth * (width - 1) + 1, the deepest the stack can grow
    TraceTuning tuning;
    int32_t* prim = nullptr;
    float* t = nullptr;
    float* u = nullptr;
    float* v = nullptr;
    uint8_t* occ = nullptr;
    int* err = nullptr;
    unsigned long long* stats = nullptr;  // non-null: also accumulate SORT's traversal counters
    unsigned long long* counter = nullptr;  // persistent schedule: ray counter, zeroed on the stream first
    const int* n_dev = nullptr;  // if set, the batch is min(n, *n_dev) (one-ray-per-thread kernel)
    bool q8 = false;             // interior nodes in the 8-bit format
};

cudaError_t launch_trace_fp32(const TraceLaunch& L, const DevTree& tr, const DevRays& rays, int64_t n,
                              cudaStream_t s);
}  // namespace sg
