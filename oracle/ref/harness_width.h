// Per-width entry points of the oracle harness (test infrastructure only).
// QBVH and OBVH are compiled from the same SORT header under different SIMD
// macros (accel/qbvh.cpp:20-31, accel/obvh.cpp:20-31), so each lives in its own
// translation unit: harness_qbvh.cpp and harness_obvh.cpp.
#pragma once
#include <cstdint>
#include <unordered_map>
#include <vector>

class Accelerator;
class Primitive;

using HarnessIndexMap = std::unordered_map<const Primitive*, int32_t>;

// The accelerator harness scenes are built with: SORT's Qbvh (width 4) or
// Obvh (width 8), unless g_harness_accel_factory is set (harness_gbvh.cpp sets
// it to the Gbvh adapter in the library that links the GPU engine).
using HarnessAccelFactory = Accelerator* (*)(int width, unsigned max_depth, unsigned max_leaf);
extern HarnessAccelFactory g_harness_accel_factory;
Accelerator* harness_make_accel(int width, unsigned max_depth, unsigned max_leaf);

Accelerator* harness_make_qbvh(unsigned max_depth, unsigned max_leaf);
Accelerator* harness_make_obvh(unsigned max_depth, unsigned max_leaf);
unsigned harness_qbvh_depth(const Accelerator* a);
unsigned harness_obvh_depth(const Accelerator* a);
// Pre-order topology stream:
//   interior node: [child_cnt, child0 ..., child_{n-1} ...]
//   leaf:          [0, pri_cnt, primitive indices in SIMD-lane packing order]
void harness_qbvh_topology(const Accelerator* a, const HarnessIndexMap& idx, std::vector<int32_t>& out);
void harness_obvh_topology(const Accelerator* a, const HarnessIndexMap& idx, std::vector<int32_t>& out);
