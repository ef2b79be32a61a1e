// Device tree layout shared by the host upload code and the kernels.
#pragma once

#include <vector_types.h>

#include <cstdint>

namespace sg {

// Interior node, FP32 child boxes, child-major: child j of node k occupies
// float4 [k*kF4 + 2j] = {lo_x, lo_y, lo_z, child reference bits} and
// float4 [k*kF4 + 2j + 1] = {hi_x, hi_y, hi_z, 0}. A node is 2*W float4:
// 256 B for W = 8, 128 B for W = 4. One lane can fetch one child with two
// 128-bit loads; W lanes fetch a whole node in one coalesced sweep.
//
// Child reference: >= 0 interior node index; bit 31 set: leaf whose first
// triangle slot is the low 31 bits; -1: empty slot (SORT's unused SIMD lane,
// with the empty box +FLT_MAX..-FLT_MAX).
//
// Triangles: 3 float4 per leaf slot, slots in leaf order:
//   {v0.xyz, primitive index bits}, {v1.xyz, last-in-leaf flag bits}, {v2.xyz, 0}.
// kPadSlots zero slots follow the last one so a kernel may fetch up to 8 slots
// past any leaf start without leaving the allocation.
template <int W>
struct NodeShape {
    static constexpr int kF4 = 2 * W;
};

constexpr int32_t kEmpty = -1;
constexpr int kPadSlots = 8;

struct DevTree {
    const float4* nodes;
    const float4* tris;
    int32_t root;
    float box_lo[3];
    float box_hi[3];
};

struct DevRays {
    const float* ox;
    const float* oy;
    const float* oz;
    const float* dx;
    const float* dy;
    const float* dz;
    const float* tmin;
    const float* tmax;
};

}  // namespace sg
