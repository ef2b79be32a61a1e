// Primitives other than triangles (hair line segments, area-light shapes):
// the records the traversal reads and their set-up.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "layout.h"
#include "sortgpu.h"

namespace sg {

// A line's record, 5 float4 per line in primitive order:
//   [m00 m01 m02 m03] [m10 m11 m12 m13] [m20 m21 m22 m23]  world-to-line matrix rows
//   [w0 w1 length (w1-w0)/length] [v0 v1 0 0]
// A leaf slot that holds a line is {0, 0, 0, primitive index},
// {0, 0, 0, last-in-leaf flag}, {line index, 0, 0, kLineSlot} (int bits).
constexpr int kLineF4 = 5;
constexpr int32_t kLineSlot = 1;

// An area shape's record (SORT's Quad / Disk), 5 float4 like a line's, after
// the lines in the same buffer:
//   [inv m00 .. m03] [inv m10 .. m13] [inv m20 .. m23] [inv m30 .. m33]
//   [a b kind 0]  quad: a, b = sizeX / 2, sizeY / 2; disk: a = radius, b = radius^2
// A leaf slot that holds one is {0, 0, 0, primitive index},
// {0, 0, 0, last-in-leaf flag}, {record index, 0, 0, kShapeSlot}.
constexpr int32_t kShapeSlot = 2;

// The record (20 floats) and box (min xyz, max xyz) of an area shape.
void shape_setup(const sg_area_shape& shape, float* record20, float* box6);

// One segment, 10 floats (p0 xyz, p1 xyz, v0, v1, w0, w1 half widths), in
// the space `transform` (SORT's row-major 4x4 Matrix; NULL = the identity)
// maps to world space: its record (20 floats) and its box (min xyz, max xyz).
void line_setup(const float* segment10, float* record20, float* box6, const float* transform16 = nullptr);

// Matrix::TransformPoint (math/matrix.cpp:70-82) of a row-major 4x4.
void transform_point16(const float* m16, const float* p, float* out);

struct TraceLaunch;
// Closest-hit or any-hit (L.any) over a tree whose leaves hold triangles,
// lines and area shapes (hair.cu); `extra` holds the line records, then the
// shape records.
cudaError_t launch_trace_hair(const TraceLaunch& L, const DevTree& tr, const float4* extra, const DevRays& rays,
                              int64_t n, cudaStream_t s);

}  // namespace sg
