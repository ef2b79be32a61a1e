// Closest-hit and any-hit traversal of SORT-topology wide BVHs on sm_100a.
//
// The per-ray traversal restates Fbvh::GetIntersect
// (accel/fast_bvh.hpp:305-504, SIMD branch):
//   * root slab test against the enlarged scene box (scalar Intersect);
//   * a stack of (node, entry distance) pairs; a popped entry is skipped when
//     the current hit is nearer than its entry distance (strict <, line 343);
//   * a leaf tests its triangles in SIMD-lane packing order and keeps a hit only
//     when strictly nearer (simd/simd_triangle.h:359-369), so the first of equal
//     distances wins;
//   * an interior node's hit children are visited nearest first; equal distances
//     visit the higher child slot first (the 1-, 2- and >=3-hit cases of lines
//     416-455 all reduce to that order);
//   * any-hit returns at the first triangle hit (opaque early exit, 362-373).
// With FP32 child boxes and the same rounding, hits, distances and barycentrics
// are bit-identical to SORT's.
//
// GPU-side choices that leave that order intact:
//   * the entry SORT would pop right after pushing a node's children (the
//     nearest) stays in registers and is descended into directly;
//   * leaf triangles are fetched two at a time (the triangle array carries one
//     padding slot), so the second's loads overlap the first's test;
//   * two schedules: one ray per thread for the whole launch, or persistent
//     warps in which a lane whose ray finished takes the next ray of the batch,
//     so warps stay full instead of idling on their slowest ray.
#include <cuda_runtime.h>

#include "trace_common.cuh"
#include "trace_kernels.h"

namespace sg {

template <int W>
struct NodeData {
    float lo[3][W], hi[3][W];
    int32_t ch[W];
};

template <int W>
__device__ __forceinline__ void load_node(const float4* __restrict__ nodes, int32_t ref, NodeData<W>& nd) {
    const float4* p = nodes + (size_t)ref * NodeShape<W>::kF4;
    constexpr int Q = W / 4;  // float4 per plane
#pragma unroll
    for (int a = 0; a < 3; ++a) {
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const float4 l = __ldg(p + (2 * a) * Q + q);
            const float4 h = __ldg(p + (2 * a + 1) * Q + q);
            nd.lo[a][4 * q + 0] = l.x;
            nd.lo[a][4 * q + 1] = l.y;
            nd.lo[a][4 * q + 2] = l.z;
            nd.lo[a][4 * q + 3] = l.w;
            nd.hi[a][4 * q + 0] = h.x;
            nd.hi[a][4 * q + 1] = h.y;
            nd.hi[a][4 * q + 2] = h.z;
            nd.hi[a][4 * q + 3] = h.w;
        }
    }
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int4 c = __ldg(reinterpret_cast<const int4*>(p + 6 * Q + q));
        nd.ch[4 * q + 0] = c.x;
        nd.ch[4 * q + 1] = c.y;
        nd.ch[4 * q + 2] = c.z;
        nd.ch[4 * q + 3] = c.w;
    }
}

// 8-bit node (layout.h, quantize.cpp): decode every child bound to
// fl(origin + q * 2^e) (one rounding: q * 2^e is exact), giving FP32 boxes that
// contain SORT's, which the unchanged slab test then uses.
__device__ __forceinline__ float q8_bound(uint32_t word, int byte, float s, float origin) {
    const float q = __uint_as_float(__byte_perm(word, 0x4B000000u, 0x7540u | (unsigned)byte)) - 8388608.0f;
    return fmaf(q, s, origin);
}

template <int W>
__device__ __forceinline__ void load_node_q8(const float4* __restrict__ nodes, int32_t ref, NodeData<W>& nd) {
    const float4* p = nodes + (size_t)ref * (W == 8 ? kQ8F4W8 : kQ8F4W4);
    const float4 h = __ldg(p);
    const uint32_t eb = __float_as_uint(h.w);
    const float org[3] = {h.x, h.y, h.z};
    float s[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) s[a] = __uint_as_float(((eb >> (8 * a)) & 0xffu) << 23);
    if (W == 8) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const uint4 q = __ldg(reinterpret_cast<const uint4*>(p + 1 + a));
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                nd.lo[a][j] = q8_bound(q.x, j, s[a], org[a]);
                nd.lo[a][4 + j] = q8_bound(q.y, j, s[a], org[a]);
                nd.hi[a][j] = q8_bound(q.z, j, s[a], org[a]);
                nd.hi[a][4 + j] = q8_bound(q.w, j, s[a], org[a]);
            }
        }
        const int4 c0 = __ldg(reinterpret_cast<const int4*>(p + 4));
        const int4 c1 = __ldg(reinterpret_cast<const int4*>(p + 5));
        nd.ch[0] = c0.x;
        nd.ch[1] = c0.y;
        nd.ch[2] = c0.z;
        nd.ch[3] = c0.w;
        nd.ch[4 % W] = c1.x;
        nd.ch[5 % W] = c1.y;
        nd.ch[6 % W] = c1.z;
        nd.ch[7 % W] = c1.w;
    } else {
        const uint4 q01 = __ldg(reinterpret_cast<const uint4*>(p + 1));
        const uint4 q2 = __ldg(reinterpret_cast<const uint4*>(p + 2));
        const int4 c = __ldg(reinterpret_cast<const int4*>(p + 3));
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            nd.lo[0][j] = q8_bound(q01.x, j, s[0], org[0]);
            nd.hi[0][j] = q8_bound(q01.y, j, s[0], org[0]);
            nd.lo[1][j] = q8_bound(q01.z, j, s[1], org[1]);
            nd.hi[1][j] = q8_bound(q01.w, j, s[1], org[1]);
            nd.lo[2][j] = q8_bound(q2.x, j, s[2], org[2]);
            nd.hi[2][j] = q8_bound(q2.y, j, s[2], org[2]);
        }
        nd.ch[0] = c.x;
        nd.ch[1 % W] = c.y;
        nd.ch[2 % W] = c.z;
        nd.ch[3 % W] = c.w;
    }
}

// One ray's traversal state. STATS adds SORT's traversal counters
// (accel/fast_bvh.hpp:50-96): interior nodes box-tested, and primitives tested
// counted per leaf entered (sIntersectionTest += pri_cnt).
template <int W, bool ANY, int STACK, bool STATS, bool Q8 = false>
struct Traversal {
    RayState r;
    float best_t, best_u, best_v;
    int32_t best_prim;
    int32_t cur;
    float cur_d;
    int si;
    unsigned node_tests, prim_tests;
    uint2 stk[STACK];

    // Loads ray i and runs the root test; returns false when the ray is already
    // finished (root miss or empty tree).
    __device__ __forceinline__ bool start(const DevTree& tr, const DevRays& rays, int64_t i) {
        r.o[0] = rays.ox[i];
        r.o[1] = rays.oy[i];
        r.o[2] = rays.oz[i];
        r.d[0] = rays.dx[i];
        r.d[1] = rays.dy[i];
        r.d[2] = rays.dz[i];
        r.tmin = rays.tmin[i];
        r.tmax = rays.tmax[i];
        ray_setup(r);
        best_t = FLT_MAX;
        best_u = best_v = 0.0f;
        best_prim = -1;
        node_tests = prim_tests = 0;
        si = 0;
        const float f0 = root_intersect(r, tr.box_lo, tr.box_hi);
        cur = tr.root;
        cur_d = f0;
        return f0 >= 0.0f && tr.root != kEmpty;
    }

    __device__ __forceinline__ void finish(int64_t i, int32_t* __restrict__ prim_out, float* __restrict__ t_out,
                                           float* __restrict__ u_out, float* __restrict__ v_out,
                                           uint8_t* __restrict__ occ_out, unsigned long long* __restrict__ stats) {
        if (STATS) {
            atomicAdd(stats, (unsigned long long)node_tests);
            atomicAdd(stats + 1, (unsigned long long)prim_tests);
        }
        if (ANY) {
            occ_out[i] = best_prim >= 0 ? 1 : 0;
        } else {
            prim_out[i] = best_prim;
            t_out[i] = best_prim >= 0 ? best_t : FLT_MAX;
            if (u_out) u_out[i] = best_prim >= 0 ? best_u : 0.0f;
            if (v_out) v_out[i] = best_prim >= 0 ? best_v : 0.0f;
        }
    }

    // Processes the entry `cur` (a leaf, an interior node, or a culled entry).
    // Returns true when the ray is finished.
    __device__ __forceinline__ bool step(const DevTree& tr, int* __restrict__ err) {
        bool descend = false;
        if (!(best_t < cur_d)) {  // fast_bvh.hpp:343: skip when the hit is nearer than the entry
            if (cur < 0) {
                if (leaf(tr, cur)) return true;
            } else {
                if (si + W > STACK) {  // cannot happen when STACK >= depth*(W-1)+1; reported, never overrun
                    atomicOr(err, 1);
                    return true;
                }
                descend = interior(tr);
            }
        }
        if (!descend) {
            if (si == 0) return true;
            const uint2 e = stk[--si];
            cur = (int32_t)e.x;
            cur_d = __uint_as_float(e.y);
        }
        return false;
    }

    // Leaf: triangles in leaf order; returns true on an any-hit early exit.
    __device__ __forceinline__ bool leaf(const DevTree& tr, int32_t ref) {
        int64_t s = (int64_t)((uint32_t)ref & 0x7fffffffu);
        unsigned tested = 0;
        bool found = false;
        for (;;) {
            const float4* q = tr.tris + 3 * s;
            const float4 a0 = __ldg(q), b0 = __ldg(q + 1), c0 = __ldg(q + 2);
            const float4 a1 = __ldg(q + 3), b1 = __ldg(q + 4), c1 = __ldg(q + 5);
            float t, u, v;
            ++tested;
            if (tri_test(r, a0, b0, c0, t, u, v) && t < best_t) {
                best_t = t;
                best_u = u;
                best_v = v;
                best_prim = __float_as_int(a0.w);
                if (ANY) {
                    found = true;
                    break;
                }
            }
            if (__float_as_int(b0.w)) break;
            ++tested;
            if (tri_test(r, a1, b1, c1, t, u, v) && t < best_t) {
                best_t = t;
                best_u = u;
                best_v = v;
                best_prim = __float_as_int(a1.w);
                if (ANY) {
                    ++s;
                    found = true;
                    break;
                }
            }
            if (__float_as_int(b1.w)) break;
            s += 2;
        }
        if (STATS) {
            if (ANY && found)  // whole leaf, as SORT counts it
                for (int64_t q = s; !__float_as_int(__ldg(tr.tris + 3 * q + 1).w); ++q) ++tested;
            prim_tests += tested;
        }
        return ANY && found;
    }

    // Interior node: box-test the children, push all hits but the nearest and
    // descend into that one. Returns false when no child is hit.
    __device__ __forceinline__ bool interior(const DevTree& tr) {
        NodeData<W> nd;
        if (Q8)
            load_node_q8<W>(tr.nodes, cur, nd);
        else
            load_node<W>(tr.nodes, cur, nd);
        if (STATS) ++node_tests;
        float d[W];
        unsigned mask = 0;
#pragma unroll
        for (int j = 0; j < W; ++j) {
            const bool hit = slab(r, nd.lo[0][j], nd.hi[0][j], nd.lo[1][j], nd.hi[1][j], nd.lo[2][j], nd.hi[2][j], d[j]);
            if (hit && nd.ch[j] != kEmpty) mask |= 1u << j;
        }
        const int cnt = __popc(mask);
        if (cnt == 0) return false;
        if (cnt == 1) {
#pragma unroll
            for (int j = 0; j < W; ++j)
                if (mask & (1u << j)) {
                    cur = nd.ch[j];
                    cur_d = d[j];
                }
            return true;
        }
        if (cnt == 2) {
            // SORT pushes the far one first when t0 < t1, else the second slot
            // last; the one it would pop next is descended into.
            int32_t c0 = 0, c1 = 0;
            float t0 = 0.0f, t1 = 0.0f;
            bool first = true;
#pragma unroll
            for (int j = 0; j < W; ++j) {
                if (mask & (1u << j)) {
                    if (first) {
                        c0 = nd.ch[j];
                        t0 = d[j];
                        first = false;
                    } else {
                        c1 = nd.ch[j];
                        t1 = d[j];
                    }
                }
            }
            if (t0 < t1) {
                stk[si++] = make_uint2((uint32_t)c1, __float_as_uint(t1));
                cur = c0;
                cur_d = t0;
            } else {
                stk[si++] = make_uint2((uint32_t)c0, __float_as_uint(t0));
                cur = c1;
                cur_d = t1;
            }
            return true;
        }
        // >= 3 hits: SORT's selection loop (fast_bvh.hpp:438-453) pushes by
        // decreasing distance, ties lowest slot first, only distances > -1; the
        // last one it pushes is descended into instead.
        unsigned left = 0;
#pragma unroll
        for (int j = 0; j < W; ++j) left |= (((mask >> j) & 1u) && d[j] > -1.0f) ? (1u << j) : 0u;
        if (left == 0) return false;
        for (;;) {
            float best = -1.0f;
            int32_t ref = 0;
            unsigned pick = 0;
#pragma unroll
            for (int j = 0; j < W; ++j) {
                if ((left & (1u << j)) && d[j] > best) {
                    best = d[j];
                    ref = nd.ch[j];
                    pick = 1u << j;
                }
            }
            left &= ~pick;
            if (left == 0) {
                cur = ref;
                cur_d = best;
                return true;
            }
            stk[si++] = make_uint2((uint32_t)ref, __float_as_uint(best));
        }
    }
};

// While-while traversal, one ray per thread: the warp alternates an interior
// phase and a leaf phase, so lanes walking interior nodes and lanes testing
// triangles do not split every iteration.
//
// Interior phase: a lane pops / descends until its entry is an un-culled leaf,
// which it parks as its pending leaf. With SPEC, a lane that already holds a
// pending leaf keeps descending (speculatively) while other lanes still lack
// one, and stops at its next leaf. Leaf phase: every lane with a pending leaf
// re-checks the cull against its current hit and tests the leaf.
//
// Leaves are tested in SORT's order and each is culled with the hit found so
// far, so results are SORT's: a speculative visit only sees interior nodes
// that SORT visits too, or that SORT culls — and then every leaf below is culled
// here as well, because a child's entry distance is never below its parent's
// (each slab bound of a child lies inside the parent's, and the rounded
// t = -o/d + b/d is monotonic in b).
template <int W, bool ANY, int STACK, bool SPEC>
__global__ void __launch_bounds__(128) k_trace_fp32_ww(DevTree tr, DevRays rays, int64_t n,
                                                       int32_t* __restrict__ prim_out, float* __restrict__ t_out,
                                                       float* __restrict__ u_out, float* __restrict__ v_out,
                                                       uint8_t* __restrict__ occ_out, int* __restrict__ err) {
    const int64_t i0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i0 < n;
    const int64_t i = valid ? i0 : n - 1;  // lanes past the batch end idle through the loop
    Traversal<W, ANY, STACK, false> tv;
    const bool started = tv.start(tr, rays, i);
    bool have = valid && started;  // `cur` holds an entry still to process
    bool pend = false;             // a parked leaf is waiting for the leaf phase
    int32_t lf = 0;
    float lf_d = 0.0f;
    while (__any_sync(0xffffffffu, have || pend)) {
        // Interior phase (warp-uniform loop; each lane does at most one unit per pass).
        for (;;) {
            const bool needs = have && !pend;
            const bool spec = SPEC && have && pend;
            if (!__any_sync(0xffffffffu, needs)) break;
            if (needs || spec) {
                bool descend = false;
                bool blocked = false;
                if (!(tv.best_t < tv.cur_d)) {
                    if (tv.cur < 0) {
                        if (!pend) {
                            lf = tv.cur;
                            lf_d = tv.cur_d;
                            pend = true;
                        } else {
                            blocked = true;  // second leaf: wait for the leaf phase
                        }
                    } else if (tv.si + W > STACK) {  // cannot happen when STACK >= depth*(W-1)+1
                        atomicOr(err, 1);
                        have = false;
                        blocked = true;
                    } else {
                        descend = tv.interior(tr);
                    }
                }
                if (!descend && !blocked) {
                    if (tv.si == 0) {
                        have = false;
                    } else {
                        const uint2 e = tv.stk[--tv.si];
                        tv.cur = (int32_t)e.x;
                        tv.cur_d = __uint_as_float(e.y);
                    }
                }
            }
        }
        // Leaf phase.
        if (pend) {
            pend = false;
            if (!(tv.best_t < lf_d) && tv.leaf(tr, lf)) have = false;  // any-hit: done
        }
    }
    if (valid) tv.finish(i, prim_out, t_out, u_out, v_out, occ_out, nullptr);
}

// One ray per thread for the whole launch. With n_dev set, the batch size is
// min(n, *n_dev), read on the device (queues whose length only the GPU knows).
// Q8 reads 8-bit nodes.
template <int W, bool ANY, int STACK, bool STATS, bool Q8 = false>
__global__ void __launch_bounds__(128) k_trace_fp32(DevTree tr, DevRays rays, int64_t n, int32_t* __restrict__ prim_out,
                                                    float* __restrict__ t_out, float* __restrict__ u_out,
                                                    float* __restrict__ v_out, uint8_t* __restrict__ occ_out,
                                                    int* __restrict__ err, unsigned long long* __restrict__ stats,
                                                    const int* __restrict__ n_dev) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n_dev && i >= (int64_t)*n_dev) return;
    if (i >= n) return;
    Traversal<W, ANY, STACK, STATS, Q8> tv;
    if (tv.start(tr, rays, i))
        while (!tv.step(tr, err)) {
        }
    tv.finish(i, prim_out, t_out, u_out, v_out, occ_out, stats);
}

// Persistent warps: a lane whose ray finished takes the next ray in batch order
// once at least `refill` lanes of its warp are idle; the warp's leader claims
// those rays from a launch-wide counter, so the whole GPU still advances
// through the batch in order (neighbouring rays share tree nodes in L1/L2).
template <int W, bool ANY, int STACK, bool STATS>
__global__ void __launch_bounds__(128) k_trace_fp32_persistent(DevTree tr, DevRays rays, int64_t n,
                                                               unsigned long long* __restrict__ counter, int refill,
                                                               int32_t* __restrict__ prim_out, float* __restrict__ t_out,
                                                               float* __restrict__ u_out, float* __restrict__ v_out,
                                                               uint8_t* __restrict__ occ_out, int* __restrict__ err,
                                                               unsigned long long* __restrict__ stats) {
    const unsigned lane = threadIdx.x & 31u;
    const unsigned lt_mask = (1u << lane) - 1u;
    Traversal<W, ANY, STACK, STATS> tv;
    bool alive = false;
    bool drained = false;  // warp-uniform: the counter has passed n
    int64_t ray = -1;
    for (;;) {
        const unsigned idle = __ballot_sync(0xffffffffu, !alive);
        if (idle != 0 && !drained) {
            unsigned long long base = 0;
            if (lane == 0) base = atomicAdd(counter, (unsigned long long)__popc(idle));
            base = __shfl_sync(0xffffffffu, base, 0);
            if ((int64_t)base >= n) drained = true;
            if (!alive) {
                const int64_t idx = (int64_t)base + __popc(idle & lt_mask);
                if (idx < n) {
                    ray = idx;
                    alive = tv.start(tr, rays, idx);
                    if (!alive) tv.finish(idx, prim_out, t_out, u_out, v_out, occ_out, stats);
                }
            }
        }
        const unsigned busy0 = __ballot_sync(0xffffffffu, alive);
        if (busy0 == 0) {
            if (drained) break;
            continue;
        }
        // Traverse until enough lanes are idle to be worth refilling.
        for (;;) {
            if (alive && tv.step(tr, err)) {
                tv.finish(ray, prim_out, t_out, u_out, v_out, occ_out, stats);
                alive = false;
            }
            const unsigned busy = __ballot_sync(0xffffffffu, alive);
            if (busy == 0) break;
            if (!drained && 32 - __popc(busy) >= refill) break;
        }
    }
}

template <int W, bool ANY, int STACK, bool STATS>
static cudaError_t launch_stack(const TraceLaunch& L, const DevTree& tr, const DevRays& rays, int64_t n,
                                cudaStream_t s) {
    const int threads = 128;
    // Counting launches keep the one-entry-per-step loop, whose interior-node
    // visits are exactly SORT's (speculation visits extra ones).
    // 8-bit nodes are read by the one-ray-per-thread kernel.
    if (L.q8) {
        const int64_t blocks = (n + threads - 1) / threads;
        k_trace_fp32<W, ANY, STACK, STATS, true><<<(unsigned)blocks, threads, 0, s>>>(
            tr, rays, n, L.prim, L.t, L.u, L.v, L.occ, L.err, L.stats, L.n_dev);
        return cudaGetLastError();
    }
    // A device-side batch size is only read by the one-ray-per-thread kernel.
    if (!STATS && !L.n_dev &&
        (L.tuning.schedule == kScheduleWhileWhile || L.tuning.schedule == kScheduleSpeculative)) {
        const int64_t blocks = (n + threads - 1) / threads;
        if (L.tuning.schedule == kScheduleSpeculative)
            k_trace_fp32_ww<W, ANY, STACK, true><<<(unsigned)blocks, threads, 0, s>>>(tr, rays, n, L.prim, L.t, L.u,
                                                                                      L.v, L.occ, L.err);
        else
            k_trace_fp32_ww<W, ANY, STACK, false><<<(unsigned)blocks, threads, 0, s>>>(tr, rays, n, L.prim, L.t, L.u,
                                                                                       L.v, L.occ, L.err);
        return cudaGetLastError();
    }
    if (L.tuning.schedule == kSchedulePersistent && !L.n_dev) {
        int dev = 0, sms = 0, blocks_per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, k_trace_fp32_persistent<W, ANY, STACK, STATS>,
                                                      threads, 0);
        if (blocks_per_sm < 1) blocks_per_sm = 1;
        if (sms < 1) sms = 1;
        int64_t blocks = (int64_t)sms * blocks_per_sm;
        const int64_t needed = (n + threads - 1) / threads;
        if (blocks > needed) blocks = needed;
        const int refill = L.tuning.refill_threshold < 1 ? 1 : (L.tuning.refill_threshold > 32 ? 32 : L.tuning.refill_threshold);
        cudaError_t e = cudaMemsetAsync(L.counter, 0, sizeof(unsigned long long), s);
        if (e != cudaSuccess) return e;
        k_trace_fp32_persistent<W, ANY, STACK, STATS><<<(unsigned)blocks, threads, 0, s>>>(
            tr, rays, n, L.counter, refill, L.prim, L.t, L.u, L.v, L.occ, L.err, L.stats);
    } else {
        const int64_t blocks = (n + threads - 1) / threads;
        k_trace_fp32<W, ANY, STACK, STATS><<<(unsigned)blocks, threads, 0, s>>>(tr, rays, n, L.prim, L.t, L.u, L.v,
                                                                                L.occ, L.err, L.stats, L.n_dev);
    }
    return cudaGetLastError();
}

template <int W, bool ANY, bool STATS>
static cudaError_t launch_w(const TraceLaunch& L, const DevTree& tr, const DevRays& rays, int64_t n, cudaStream_t s) {
    if (L.stack_need <= 64) return launch_stack<W, ANY, 64, STATS>(L, tr, rays, n, s);
    if (L.stack_need <= 128) return launch_stack<W, ANY, 128, STATS>(L, tr, rays, n, s);
    if (L.stack_need <= 256) return launch_stack<W, ANY, 256, STATS>(L, tr, rays, n, s);
    return cudaErrorInvalidValue;
}

template <bool STATS>
static cudaError_t launch_any_width(const TraceLaunch& L, const DevTree& tr, const DevRays& rays, int64_t n,
                                    cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    if (L.width == 8)
        return L.any ? launch_w<8, true, STATS>(L, tr, rays, n, s) : launch_w<8, false, STATS>(L, tr, rays, n, s);
    return L.any ? launch_w<4, true, STATS>(L, tr, rays, n, s) : launch_w<4, false, STATS>(L, tr, rays, n, s);
}

cudaError_t launch_trace_fp32(const TraceLaunch& L, const DevTree& tr, const DevRays& rays, int64_t n,
                              cudaStream_t s) {
    return L.stats ? launch_any_width<true>(L, tr, rays, n, s) : launch_any_width<false>(L, tr, rays, n, s);
}

}  // namespace sg
