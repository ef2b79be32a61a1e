// Device tree layout shared by the host upload code and the kernels.
#pragma once

#include <vector_types.h>

#include <cstdint>

namespace sg {

// Device tree layout.
//   W = 8: 14 float4 per interior node: lo_x[0:4], lo_x[4:8], hi_x[0:4],
//          hi_x[4:8], lo_y.., hi_y.., lo_z.., hi_z.., child[0:4], child[4:8].
//   W = 4:  8 float4 per interior node: lo_x, hi_x, lo_y, hi_y, lo_z, hi_z,
//          child[0:4], (padding to 128 bytes).
//   Triangles: 3 float4 per leaf slot: {v0, prim id}, {v1, last-in-leaf flag},
//          {v2, 0}, slots in leaf order.
//   Child reference: >= 0 interior node index; bit 31 set: leaf whose first
//   slot is the low 31 bits; -1: empty slot.
template <int W>
struct NodeShape;
template <>
struct NodeShape<8> {
    static constexpr int kF4 = 14;
};
template <>
struct NodeShape<4> {
    static constexpr int kF4 = 8;
};

constexpr int32_t kEmpty = -1;

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
