// Per-ray wide-BVH traversal shared by the traversal kernels (trace.cu, batch.cu).
//
// Restates Fbvh::GetIntersect (accel/fast_bvh.hpp:305-504, SIMD branch); the
// ordering rules are listed at the top of trace.cu.
#pragma once

#include <cuda_runtime.h>

#include "trace_common.cuh"

namespace sg {

// A node's child boxes as each ray sees them: per axis the plane it enters
// through (nr, the lower bound when the direction is positive) and the plane
// it leaves through (fr); see slab_near_far.
template <int W>
struct NodeData {
    float nr[3][W], fr[3][W];
    int32_t ch[W];
};

template <int W>
__device__ __forceinline__ void load_node(const float4* __restrict__ nodes, int32_t ref, const RayState& r,
                                          NodeData<W>& nd) {
    const float4* p = nodes + (size_t)ref * NodeShape<W>::kF4;
    constexpr int Q = W / 4;  // float4 per plane
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float4* pn = p + (2 * a + r.nhi[a]) * Q;      // lo plane, or hi for a negative direction
        const float4* pf = p + (2 * a + 1 - r.nhi[a]) * Q;  // the other one
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const float4 l = __ldg(pn + q);
            const float4 h = __ldg(pf + q);
            nd.nr[a][4 * q + 0] = l.x;
            nd.nr[a][4 * q + 1] = l.y;
            nd.nr[a][4 * q + 2] = l.z;
            nd.nr[a][4 * q + 3] = l.w;
            nd.fr[a][4 * q + 0] = h.x;
            nd.fr[a][4 * q + 1] = h.y;
            nd.fr[a][4 * q + 2] = h.z;
            nd.fr[a][4 * q + 3] = h.w;
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
__device__ __forceinline__ void load_node_q8(const float4* __restrict__ nodes, int32_t ref, const RayState& r,
                                             NodeData<W>& nd) {
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
            const bool flip = r.nhi[a] != 0;
            const uint32_t n0 = flip ? q.z : q.x, n1 = flip ? q.w : q.y;
            const uint32_t f0 = flip ? q.x : q.z, f1 = flip ? q.y : q.w;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                nd.nr[a][j] = q8_bound(n0, j, s[a], org[a]);
                nd.nr[a][4 + j] = q8_bound(n1, j, s[a], org[a]);
                nd.fr[a][j] = q8_bound(f0, j, s[a], org[a]);
                nd.fr[a][4 + j] = q8_bound(f1, j, s[a], org[a]);
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
        const uint32_t lo[3] = {q01.x, q01.z, q2.x}, hi[3] = {q01.y, q01.w, q2.y};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const uint32_t n = r.nhi[a] ? hi[a] : lo[a], f = r.nhi[a] ? lo[a] : hi[a];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                nd.nr[a][j] = q8_bound(n, j, s[a], org[a]);
                nd.fr[a][j] = q8_bound(f, j, s[a], org[a]);
            }
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
//
// STEP_SKIPS_EMPTY: the caller drives the traversal through step(), which
// passes over empty child entries itself, so interior() need not test each
// hit child against kEmpty. An empty FP32 slot holds the empty box
// (+FLT_MAX .. -FLT_MAX), which a ray with finite origin and direction never
// hits (per axis the entry distance is >= +FLT_MAX/|d| - |o/d| > 0 and the exit
// distance the negative of that), so only a ray with a NaN or infinite
// component can reach one. An empty 8-bit slot decodes to an inverted box
// (lower bound 255 steps above the upper one), which such a ray misses too.
// Dropping the per-child test saves two instructions per child and six
// registers in the closest-hit kernel; skipping in step() keeps any empty
// entry that is reached harmless.
template <int W, bool ANY, int STACK, bool STATS, bool Q8 = false, bool STEP_SKIPS_EMPTY = false>
struct Traversal {
    static constexpr bool kTestEmpty = !STEP_SKIPS_EMPTY;
    RayState r;
    float best_t, best_u, best_v;
    int32_t best_prim;
    int32_t cur;
    float cur_d;
    int si;
    unsigned node_tests, prim_tests;
    uint2* stk;  // STACK entries owned by the kernel (see RayWalk: a stack array
                 // inside this object would put every field in local memory)

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
        return begin(tr);
    }

    // Same as start, for a ray already stored in r.o, r.d, r.tmin, r.tmax.
    __device__ __forceinline__ bool begin(const DevTree& tr) {
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
                if (cur != kEmpty && leaf(tr, cur)) return true;
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
            load_node_q8<W>(tr.nodes, cur, r, nd);
        else
            load_node<W>(tr.nodes, cur, r, nd);
        if (STATS) ++node_tests;
        float d[W];
        unsigned mask = 0;
#pragma unroll
        for (int j = 0; j < W; ++j) {
            const bool hit =
                slab_near_far(r, nd.nr[0][j], nd.fr[0][j], nd.nr[1][j], nd.fr[1][j], nd.nr[2][j], nd.fr[2][j], d[j]);
            if (hit && (!kTestEmpty || nd.ch[j] != kEmpty)) mask |= 1u << j;
        }
        const int cnt = __popc(mask);
        if (cnt == 0) return false;
        if (ANY && !STATS) {
            // Any hit: before the first hit nothing is culled (the current hit
            // distance stays FLT_MAX), so the answer is whether any triangle of
            // the nodes the slab tests reach is hit, whatever the visit order.
            // Descend into the lowest hit slot, push the others; SORT's
            // near-first order is kept only where its counts are wanted.
            const unsigned first = mask & (0u - mask);  // lowest set bit
            int32_t fc = 0;
#pragma unroll
            for (int j = 0; j < W; ++j) {
                if (!(mask & (1u << j))) continue;
                if ((1u << j) == first)
                    fc = nd.ch[j];
                else
                    stk[si++] = make_uint2((uint32_t)nd.ch[j], 0u);  // entry distance 0: never culled
            }
            cur = fc;
            cur_d = 0.0f;
            return true;
        }
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

// ---------------------------------------------------------------------------
// RayWalk: the closest-hit / any-hit traversal of the hot kernels. Same visit
// order, culling, leaf order and per-operation rounding as Traversal, so the
// same hits, distances and barycentrics; arranged so that a ray's state stays
// in registers:
//  * The stack is not part of the walker: the kernel owns it (a per-thread
//    local array) and passes it in. An object holding a dynamically indexed
//    array is placed in local memory as a whole, so a stack inside the walker
//    put every ray field in local memory too (Traversal: a 1,160-byte frame of
//    which 136 bytes are ray fields; RayWalk: 1,024 bytes, the stack alone).
//  * The best hit is (t, leaf slot). u, v and the primitive id are recomputed
//    from that slot once, when the ray finishes: the test is deterministic, so
//    they are the values the hit had when it was found.
//  * An interior node is box-tested in groups of four children, and its child
//    references are read after the box test, only when a child is hit.
// Measured on 4,194,304 incoherent rays (21M triangles, OBVH): 1,031 Mrays/s
// sorted closest-hit against Traversal's 950, any-hit 1,174 against 1,066. A
// shared-memory short stack (the first 8 or 16 entries per thread in shared
// memory, the rest local) was slower (1,004 / 977): the local stack's top
// entries stay in L1, and shared memory takes L1 capacity the nodes need.
// Packed FP32 pairs (add.rn.f32x2 / mul.rn.f32x2) in the slab test changed 2
// of 524,288 hits against SORT (a packed multiply-add evidently does not keep
// the product's rounding), so the slab test stays scalar.
template <int W, bool ANY, int STACK, bool Q8 = false>
struct RayWalk {
    RayState r;
    float best_t;
    int32_t best_slot;  // leaf slot of the nearest hit so far, -1 none
    int32_t cur;
    float cur_d;
    int si;

    __device__ __forceinline__ bool start(const DevTree& tr, const DevRays& rays, int64_t i) {
        r.o[0] = rays.ox[i];
        r.o[1] = rays.oy[i];
        r.o[2] = rays.oz[i];
        r.d[0] = rays.dx[i];
        r.d[1] = rays.dy[i];
        r.d[2] = rays.dz[i];
        r.tmin = rays.tmin[i];
        r.tmax = rays.tmax[i];
        return begin(tr);
    }

    // Same as start, for a ray already stored in r.o, r.d, r.tmin, r.tmax.
    __device__ __forceinline__ bool begin(const DevTree& tr) {
        ray_setup(r);
        best_t = FLT_MAX;
        best_slot = -1;
        si = 0;
        const float f0 = root_intersect(r, tr.box_lo, tr.box_hi);
        cur = tr.root;
        cur_d = f0;
        return f0 >= 0.0f && tr.root != kEmpty;
    }

    // The nearest hit's primitive, t, u, v (closest-hit), re-testing its slot.
    __device__ __forceinline__ int32_t result(const DevTree& tr, float& t, float& u, float& v) const {
        t = FLT_MAX;
        u = v = 0.0f;
        if (best_slot < 0) return -1;
        const float4* q = tr.tris + 3 * (int64_t)best_slot;
        const float4 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2);
        tri_test(r, a, b, c, t, u, v);  // hits again: same inputs, same rounding
        return __float_as_int(a.w);
    }

    // Writes the ray's answer.
    __device__ __forceinline__ void finish(const DevTree& tr, int64_t i, int32_t* __restrict__ prim_out,
                                           float* __restrict__ t_out, float* __restrict__ u_out,
                                           float* __restrict__ v_out, uint8_t* __restrict__ occ_out) const {
        if (ANY) {
            occ_out[i] = best_slot >= 0 ? 1 : 0;
            return;
        }
        float t, u, v;
        prim_out[i] = result(tr, t, u, v);
        t_out[i] = t;
        if (u_out) u_out[i] = u;
        if (v_out) v_out[i] = v;
    }

    // Processes the entry `cur` (a leaf, an interior node, an empty slot or a
    // culled entry). Returns true when the ray is finished.
    __device__ __forceinline__ bool step(const DevTree& tr, uint2* stk, int* __restrict__ err) {
        bool descend = false;
        if (!(best_t < cur_d)) {  // fast_bvh.hpp:343
            if (cur < 0) {
                if (cur != kEmpty && leaf(tr, cur)) return true;
            } else {
                if (si + W > STACK) {  // cannot happen when STACK >= depth*(W-1)+1; reported, never overrun
                    atomicOr(err, 1);
                    return true;
                }
                descend = interior(tr, stk);
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

    // Leaf: triangles in leaf order, two fetched at a time; true on an any-hit.
    __device__ __forceinline__ bool leaf(const DevTree& tr, int32_t ref) {
        int32_t s = ref & 0x7fffffff;
        for (;;) {
            const float4* q = tr.tris + 3 * (int64_t)s;
            const float4 a0 = __ldg(q), b0 = __ldg(q + 1), c0 = __ldg(q + 2);
            const float4 a1 = __ldg(q + 3), b1 = __ldg(q + 4), c1 = __ldg(q + 5);
            float t, u, v;
            if (tri_test(r, a0, b0, c0, t, u, v) && t < best_t) {
                best_t = t;
                best_slot = s;
                if (ANY) return true;
            }
            if (__float_as_int(b0.w)) break;
            if (tri_test(r, a1, b1, c1, t, u, v) && t < best_t) {
                best_t = t;
                best_slot = s + 1;
                if (ANY) return true;
            }
            if (__float_as_int(b1.w)) break;
            s += 2;
        }
        return false;
    }

    // Slab test of four children from their near planes n[axis][c] and far
    // planes f[axis][c] (slab_near_far per child).
    __device__ __forceinline__ void test4(const float (&n)[3][4], const float (&f)[3][4], float* d, unsigned& mask,
                                          int g) const {
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const bool hit = slab_near_far(r, n[0][c], f[0][c], n[1][c], f[1][c], n[2][c], f[2][c], d[c]);
            mask |= hit ? (1u << (4 * g + c)) : 0u;
        }
    }

    // Children 4g .. 4g+3 of the node at p.
    __device__ __forceinline__ void test_group(const float4* __restrict__ p, int g, float* d, unsigned& mask) const {
        float n[3][4], f[3][4];
        if (Q8) {
            // 8-bit node (layout.h, quantize.cpp): each bound decodes to
            // fl(origin + q * 2^e), a box containing SORT's.
            const float4 h = __ldg(p);
            const uint32_t eb = __float_as_uint(h.w);
            const float org[3] = {h.x, h.y, h.z};
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const float sc = __uint_as_float(((eb >> (8 * a)) & 0xffu) << 23);
                uint32_t lo, hi;
                if (W == 8) {
                    const uint4 qv = __ldg(reinterpret_cast<const uint4*>(p + 1 + a));
                    lo = g == 0 ? qv.x : qv.y;
                    hi = g == 0 ? qv.z : qv.w;
                } else {
                    const uint4 q01 = __ldg(reinterpret_cast<const uint4*>(p + 1));
                    const uint4 q2 = __ldg(reinterpret_cast<const uint4*>(p + 2));
                    lo = a == 0 ? q01.x : (a == 1 ? q01.z : q2.x);
                    hi = a == 0 ? q01.y : (a == 1 ? q01.w : q2.y);
                }
                const uint32_t nw = r.nhi[a] ? hi : lo, fw = r.nhi[a] ? lo : hi;
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    n[a][c] = q8_bound(nw, c, sc, org[a]);
                    f[a][c] = q8_bound(fw, c, sc, org[a]);
                }
            }
        } else {
            constexpr int Q = W / 4;  // float4 per plane
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const float4 l = __ldg(p + (2 * a + r.nhi[a]) * Q + g);
                const float4 h = __ldg(p + (2 * a + 1 - r.nhi[a]) * Q + g);
                n[a][0] = l.x;
                n[a][1] = l.y;
                n[a][2] = l.z;
                n[a][3] = l.w;
                f[a][0] = h.x;
                f[a][1] = h.y;
                f[a][2] = h.z;
                f[a][3] = h.w;
            }
        }
        test4(n, f, d, mask, g);
    }

    __device__ __forceinline__ void push(uint2* stk, int32_t ref, float dist) {
        stk[si++] = make_uint2((uint32_t)ref, __float_as_uint(dist));
    }

    // Interior node: box-test the children, push all hits but the nearest and
    // descend into that one (SORT's order, as Traversal::interior). Returns
    // false when no child is hit.
    __device__ __forceinline__ bool interior(const DevTree& tr, uint2* stk) {
        constexpr int kF4 = Q8 ? (W == 8 ? kQ8F4W8 : kQ8F4W4) : NodeShape<W>::kF4;
        constexpr int kChild = Q8 ? (W == 8 ? 4 : 3) : 6 * (W / 4);  // float4 index of child[0:4]
        const float4* p = tr.nodes + (size_t)cur * kF4;
        float d[W];
        unsigned mask = 0;
#pragma unroll
        for (int g = 0; g < W / 4; ++g) test_group(p, g, d + 4 * g, mask);
        if (mask == 0) return false;
        int32_t ch[W];
#pragma unroll
        for (int q = 0; q < W / 4; ++q) {
            const int4 c = __ldg(reinterpret_cast<const int4*>(p + kChild + q));
            ch[4 * q + 0] = c.x;
            ch[4 * q + 1] = c.y;
            ch[4 * q + 2] = c.z;
            ch[4 * q + 3] = c.w;
        }
        if (ANY) {
            // Before the first hit nothing is culled, so any order finds the
            // same answer: descend into the lowest hit slot, push the others.
            const unsigned first = mask & (0u - mask);
            int32_t fc = 0;
#pragma unroll
            for (int j = 0; j < W; ++j) {
                if (!(mask & (1u << j))) continue;
                if ((1u << j) == first)
                    fc = ch[j];
                else
                    push(stk, ch[j], 0.0f);
            }
            cur = fc;
            cur_d = 0.0f;
            return true;
        }
        const int cnt = __popc(mask);
        if (cnt == 1) {
#pragma unroll
            for (int j = 0; j < W; ++j)
                if (mask & (1u << j)) {
                    cur = ch[j];
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
                        c0 = ch[j];
                        t0 = d[j];
                        first = false;
                    } else {
                        c1 = ch[j];
                        t1 = d[j];
                    }
                }
            }
            if (t0 < t1) {
                push(stk, c1, t1);
                cur = c0;
                cur_d = t0;
            } else {
                push(stk, c0, t0);
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
                    ref = ch[j];
                    pick = 1u << j;
                }
            }
            left &= ~pick;
            if (left == 0) {
                cur = ref;
                cur_d = best;
                return true;
            }
            push(stk, ref, best);
        }
    }
};

}  // namespace sg
