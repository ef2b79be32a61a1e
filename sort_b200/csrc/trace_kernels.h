// Host-side launch wrappers of the traversal kernels (implemented in trace.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "layout.h"

namespace sg {

// stack_need = depth * (width - 1) + 1, the deepest the traversal stack can grow.
cudaError_t launch_trace_fp32(int width, bool any, const DevTree& tr, const DevRays& rays, int64_t n, int stack_need,
                              int32_t* prim, float* t, float* u, float* v, uint8_t* occ, int* err, cudaStream_t s);
// Same traversal, also accumulating SORT's counters into stats[0] (interior
// nodes tested) and stats[1] (primitives tested).
cudaError_t launch_trace_fp32_stats(int width, bool any, const DevTree& tr, const DevRays& rays, int64_t n,
                                    int stack_need, int32_t* prim, float* t, float* u, float* v, uint8_t* occ,
                                    int* err, unsigned long long* stats, cudaStream_t s);

}  // namespace sg
