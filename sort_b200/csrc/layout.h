// Device tree layout shared by the host upload code and the kernels.
#pragma once

#include <vector_types.h>

#include <cstdint>

namespace sg {

// Interior node, FP32 child boxes, plane-major (structure of arrays):
//   W = 8: 14 float4 = 224 B: lo_x[0:4], lo_x[4:8], hi_x[0:4], hi_x[4:8],
//          lo_y.., hi_y.., lo_z.., hi_z.., child[0:4], child[4:8];
//   W = 4:  8 float4 = 128 B: lo_x, hi_x, lo_y, hi_y, lo_z, hi_z, child[0:4],
//          and 16 B of padding.
// A thread reads a node with 14 (7) 128-bit loads covering 7 (4) sectors.
//
// Child reference: >= 0 interior node index; bit 31 set: leaf whose first
// triangle slot is the low 31 bits; -1: empty slot (SORT's unused SIMD lane,
// with the empty box +FLT_MAX..-FLT_MAX).
//
// Triangles: 3 float4 per leaf slot, slots in leaf order:
//   {v0.xyz, primitive index bits}, {v1.xyz, last-in-leaf flag bits}, {v2.xyz, 0}.
// kPadSlots zero slots follow the last one so a kernel may fetch slots past a
// leaf's last one without leaving the allocation.
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
constexpr int kPadSlots = 8;

// Interior node, 8-bit child boxes (SG_NODES_QUANT8; see quantize.cpp):
//   float4 0: origin x, y, z; w = the three scale exponents e + 127, one byte
//             per axis (x in the low byte), scale = 2^e;
//   W = 8: float4 1..3: per axis 8 lower-bound bytes then 8 upper-bound bytes;
//          float4 4..5: child[0:8].  96 B.
//   W = 4: float4 1: lo_x[4] hi_x[4] lo_y[4] hi_y[4]; float4 2: lo_z[4] hi_z[4]
//          and 8 B of padding; float4 3: child[0:4].  64 B.
// A bound decodes to fl(origin + q * scale). An empty slot has lower bytes 255
// and upper bytes 0: an inverted box.
constexpr int kQ8F4W8 = 6;
constexpr int kQ8F4W4 = 4;

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
