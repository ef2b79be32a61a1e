// Multi-scene batch traversal: one persistent kernel per group of batches that
// share a tree width, node format and query (closest / any hit) drains every
// batch of the group, whatever scene each one traces.
//
// The group's batches form one ray sequence (batch after batch, in table
// order). A warp claims as many consecutive rays of it as it has idle lanes,
// each lane finds its ray's batch by its position in that sequence, loads the
// ray from the batch's planes and traverses its batch's tree with the same
// per-ray traversal as the single-batch kernels (traversal.cuh), so every hit
// is the one sg_trace_closest / sg_trace_any returns for that batch alone.
// Like the persistent single-batch schedule, a warp refills once `refill`
// lanes are idle (ray compaction between traversal steps).
//
// Each finished ray is counted against its batch (one atomic per batch per
// warp step); the warp that finishes a batch's last ray stamps the batch's
// completion time. A run may carry a time budget: once it has passed, warps
// stop claiming rays, finish the ones they hold and the run reports the cut.
#include <cuda_runtime.h>

#include "batch_kernels.h"
#include "traversal.cuh"

namespace sg {

namespace {

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Largest k with batches[k].start <= idx (idx < the group's total, so that
// batch holds idx: empty batches share their start with the next one).
__device__ __forceinline__ int find_batch(const BatchDesc* __restrict__ bt, int count, int64_t idx, int hint) {
    const int64_t hs = __ldg(&bt[hint].start);
    if (idx >= hs && idx < hs + __ldg(&bt[hint].n)) return hint;
    int lo = 0, hi = count - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&bt[mid].start) <= idx)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// Counts the lanes that finished a ray this step against their batches.
__device__ __forceinline__ void count_finished(bool fin, int b, const BatchArgs& a, int first, unsigned lane) {
    const unsigned fm = __ballot_sync(0xffffffffu, fin);
    if (fm == 0) return;
    const int leader = __ffs(fm) - 1;
    const int b0 = __shfl_sync(0xffffffffu, b, leader);
    const unsigned same = __ballot_sync(0xffffffffu, fin && b == b0);
    unsigned peers;
    if (same == fm)
        peers = fm;  // the usual case: one batch
    else
        peers = __match_any_sync(0xffffffffu, fin ? b : -1);
    if (fin && (unsigned)(__ffs(peers) - 1) == lane) {
        const unsigned long long c = (unsigned long long)__popc(peers);
        const unsigned long long old = atomicAdd(&a.remaining[first + b], 0ull - c);
        if (old == c) a.done_ns[first + b] = (long long)(global_ns() - a.state->start_ns);
    }
}

// Held to 1,152 resident threads per SM (56 registers, nine blocks of 128):
// with the traversal in RayWalk, batched_31m runs at 1,903 Mrays/s there
// against 1,868 at 1,024 threads (64 registers) and 1,873 at 896 (72).
template <int W, bool ANY, int STACK, int BLOCK, bool Q8>
__global__ void __launch_bounds__(BLOCK, 1152 / BLOCK) k_trace_batches(BatchArgs a) {
    const unsigned lane = threadIdx.x & 31u;
    const unsigned lt_mask = (1u << lane) - 1u;
    const GroupDesc g = a.header->groups[a.group];
    const int refill = a.header->refill;
    const long long budget = a.header->budget_ns;
    const BatchDesc* __restrict__ bt = a.batches + g.first;
    RayWalk<W, ANY, STACK, Q8> tv;
    uint2 stk[STACK];
    DevTree tr;
    tr.nodes = nullptr;
    tr.tris = nullptr;
    int b = 0;       // this lane's batch within the group
    int64_t j = 0;   // its ray within that batch
    bool alive = false;
    bool drained = false;  // warp-uniform: nothing left to claim
    if (g.count <= 0) return;
    for (;;) {
        const unsigned idle = __ballot_sync(0xffffffffu, !alive);
        if (idle != 0 && !drained) {
            unsigned long long base = 0;
            if (lane == 0) {
                if (budget > 0 && (long long)(global_ns() - a.state->start_ns) > budget) {
                    atomicOr(&a.state->status, kBatchBudgetCut);
                    base = (unsigned long long)g.total;
                } else {
                    base = atomicAdd(&a.state->counter[a.group], (unsigned long long)__popc(idle));
                }
            }
            base = __shfl_sync(0xffffffffu, base, 0);
            if ((int64_t)base >= g.total) drained = true;
            bool fin = false;
            if (!alive) {
                const int64_t idx = (int64_t)base + __popc(idle & lt_mask);
                if (idx < g.total) {
                    b = find_batch(bt, g.count, idx, b);
                    const float* p = bt[b].rays;
                    const int64_t stride = __ldg(&bt[b].stride);
                    j = idx - __ldg(&bt[b].start);
                    p += j;
                    tv.r.o[0] = __ldg(p);
                    tv.r.o[1] = __ldg(p + stride);
                    tv.r.o[2] = __ldg(p + 2 * stride);
                    tv.r.d[0] = __ldg(p + 3 * stride);
                    tv.r.d[1] = __ldg(p + 4 * stride);
                    tv.r.d[2] = __ldg(p + 5 * stride);
                    tv.r.tmin = __ldg(p + 6 * stride);
                    tv.r.tmax = __ldg(p + 7 * stride);
                    tr = a.trees[__ldg(&bt[b].tree)];
                    alive = tv.begin(tr);
                    if (!alive) {
                        tv.finish(tr, j, bt[b].prim, bt[b].t, bt[b].u, bt[b].v, bt[b].occ);
                        fin = true;
                    }
                }
            }
            count_finished(fin, b, a, g.first, lane);
        }
        const unsigned busy0 = __ballot_sync(0xffffffffu, alive);
        if (busy0 == 0) {
            if (drained) break;
            continue;
        }
        // Traverse until enough lanes are idle to be worth refilling.
        for (;;) {
            bool fin = false;
            if (alive && tv.step(tr, stk, &a.state->status)) {
                tv.finish(tr, j, bt[b].prim, bt[b].t, bt[b].u, bt[b].v, bt[b].occ);
                alive = false;
                fin = true;
            }
            count_finished(fin, b, a, g.first, lane);
            const unsigned busy = __ballot_sync(0xffffffffu, alive);
            if (busy == 0) break;
            if (!drained && 32 - __popc(busy) >= refill) break;
        }
    }
}

__global__ void k_batch_begin(const RunHeader* __restrict__ h, const BatchDesc* __restrict__ batches,
                              RunState* __restrict__ st, unsigned long long* __restrict__ remaining,
                              long long* __restrict__ done_ns) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        for (int g = 0; g < kMaxBatchGroups; ++g) st->counter[g] = 0;
        st->status = 0;
        st->start_ns = global_ns();
    }
    if (i < h->nbatches) {
        const int64_t n = batches[i].n;
        remaining[i] = (unsigned long long)n;
        done_ns[i] = n == 0 ? 0 : -1;
    }
}

template <int W, bool ANY, int STACK, int BLOCK, bool Q8>
cudaError_t launch_group(const BatchArgs& a, int grid, cudaStream_t s) {
    k_trace_batches<W, ANY, STACK, BLOCK, Q8><<<grid, BLOCK, 0, s>>>(a);
    return cudaGetLastError();
}

template <int W, bool ANY, int STACK, int BLOCK, bool Q8>
int group_occupancy() {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_trace_batches<W, ANY, STACK, BLOCK, Q8>, BLOCK, 0) !=
        cudaSuccess)
        return 0;
    return n;
}

template <int W, bool ANY, int STACK, int BLOCK, bool Q8>
BatchKernel make_kernel() {
    return BatchKernel{&launch_group<W, ANY, STACK, BLOCK, Q8>, &group_occupancy<W, ANY, STACK, BLOCK, Q8>};
}

template <int W, bool ANY, int STACK, bool Q8>
BatchKernel pick_block(int block) {
    if (block == 64) return make_kernel<W, ANY, STACK, 64, Q8>();
    if (block == 128) return make_kernel<W, ANY, STACK, 128, Q8>();
    if (block == 256) return make_kernel<W, ANY, STACK, 256, Q8>();
    return BatchKernel{nullptr, nullptr};
}

template <int W, bool ANY, bool Q8>
BatchKernel pick_stack(int stack, int block) {
    if (stack == 64) return pick_block<W, ANY, 64, Q8>(block);
    if (stack == 128) return pick_block<W, ANY, 128, Q8>(block);
    if (stack == 256) return pick_block<W, ANY, 256, Q8>(block);
    return BatchKernel{nullptr, nullptr};
}

template <int W>
BatchKernel pick_query(bool any, int stack, int block, bool q8) {
    if (any) return q8 ? pick_stack<W, true, true>(stack, block) : pick_stack<W, true, false>(stack, block);
    return q8 ? pick_stack<W, false, true>(stack, block) : pick_stack<W, false, false>(stack, block);
}

}  // namespace

BatchKernel batch_kernel(int width, bool any, int stack, int block, bool q8) {
    if (width == 8) return pick_query<8>(any, stack, block, q8);
    if (width == 4) return pick_query<4>(any, stack, block, q8);
    return BatchKernel{nullptr, nullptr};
}

cudaError_t launch_batch_begin(const RunHeader* header, const BatchDesc* batches, RunState* state,
                               unsigned long long* remaining, long long* done_ns, int max_batches, cudaStream_t s) {
    const int threads = 256;
    const int blocks = (max_batches + threads - 1) / threads;
    k_batch_begin<<<blocks < 1 ? 1 : blocks, threads, 0, s>>>(header, batches, state, remaining, done_ns);
    return cudaGetLastError();
}

}  // namespace sg
