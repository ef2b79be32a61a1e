// Device tables and launchers of the multi-scene batch traversal (batch.cu),
// shared with the host side of sg_batcher (batch.cpp).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "layout.h"

namespace sg {

// At most this many kernel groups (width x node format x query) in one run.
constexpr int kMaxBatchGroups = 8;

// Status bits of a run.
constexpr int kBatchStackOverflow = 1;  // a traversal stack bound was exceeded (never, by construction)
constexpr int kBatchBudgetCut = 2;      // the time budget stopped the run before every ray was claimed

// One batch of a run, in the run's table order (grouped, then in caller order).
struct BatchDesc {
    const float* rays;  // plane k of ray i at rays[k * stride + i]
    int64_t stride;
    int64_t start;  // first ray of this batch in its group's ray sequence
    int64_t n;
    int32_t* prim;
    float* t;
    float* u;
    float* v;
    uint8_t* occ;
    int32_t tree;  // index into the run's tree table
    int32_t pad;
};

struct GroupDesc {
    int32_t first;  // first batch of the group in the table
    int32_t count;
    int64_t total;  // rays in the group
};

// Written by the host before every run (copied inside the stream order).
struct RunHeader {
    int32_t nbatches;
    int32_t refill;     // idle lanes at which a warp claims new rays (1..32)
    int64_t budget_ns;  // 0 = none
    GroupDesc groups[kMaxBatchGroups];
};

// Written by the device during a run.
struct RunState {
    unsigned long long counter[kMaxBatchGroups];
    unsigned long long start_ns;
    int status;
    int pad;
};

struct BatchArgs {
    const RunHeader* header;
    const BatchDesc* batches;
    const DevTree* trees;
    RunState* state;
    unsigned long long* remaining;  // rays of each batch not yet finished
    long long* done_ns;             // per batch: ns from the run's start to its last ray, -1 until then
    int group;
};

// One compiled configuration of the group kernel.
struct BatchKernel {
    // Enqueues the kernel with `grid` blocks on s.
    cudaError_t (*launch)(const BatchArgs& a, int grid, cudaStream_t s);
    // Resident blocks per SM (occupancy calculator).
    int (*blocks_per_sm)();
};

// Returns the kernel for width 4/8, any-hit, stack 64/128/256, block threads
// 64/128/256 and 8-bit nodes; launch == nullptr for an unsupported combination.
BatchKernel batch_kernel(int width, bool any, int stack, int block, bool q8);

// Initialises the run state and the per-batch counters (one kernel).
cudaError_t launch_batch_begin(const RunHeader* header, const BatchDesc* batches, RunState* state,
                               unsigned long long* remaining, long long* done_ns, int max_batches, cudaStream_t s);

}  // namespace sg
