// Oracle harness, obvh half (test infrastructure only): creates SORT's
// Obvh and walks the tree it built (Fbvh::m_root is private, so it is opened
// up in this translation unit only). The SIMD helper that simd/simd_ray_utils.h
// defines out of line is renamed here so it does not clash with SORT's own copy
// in accel/obvh.cpp.
#include <cstdint>
#include <memory>
#include <queue>
#include <unordered_map>
#include <vector>
#define resolveRayData harness_unused_resolveRayData_obvh
#define private public
#define protected public
#include "accel/obvh.h"
#undef private
#undef protected
#include "harness_width.h"

namespace {
using Node = Obvh_Node;
using Accel = Obvh;

void export_node(const HarnessIndexMap& idx, const Node* node, std::vector<int32_t>& out) {
    out.push_back((int32_t)node->child_cnt);
    if (node->child_cnt == 0) {
        const size_t cnt_pos = out.size();
        out.push_back(0);
        int32_t n = 0;
        for (unsigned i = 0; i < node->tri_cnt; ++i)
            for (int l = 0; l < SIMD_CHANNEL; ++l) {
                const Primitive* p = node->tri_list[i].m_ori_pri[l];
                if (!p) continue;
                out.push_back(idx.at(p));
                ++n;
            }
        for (unsigned i = 0; i < node->line_cnt; ++i)  // then the line packs, as the leaf tests them
            for (int l = 0; l < SIMD_CHANNEL; ++l) {
                const Primitive* p = node->line_list[i].m_ori_pri[l];
                if (!p) continue;
                out.push_back(idx.at(p));
                ++n;
            }
        for (const Primitive* p : node->other_list) {
            out.push_back(idx.at(p));
            ++n;
        }
        out[cnt_pos] = n;
        return;
    }
    for (unsigned j = 0; j < node->child_cnt; ++j) export_node(idx, node->children[j].get(), out);
}
}  // namespace

Accelerator* harness_make_obvh(unsigned max_depth, unsigned max_leaf) {
    auto* a = new Accel();
    a->m_maxNodeDepth = max_depth;
    a->m_maxPriInLeaf = max_leaf;
    return a;
}

unsigned harness_obvh_depth(const Accelerator* a) { return ((const Accel*)a)->m_depth; }

void harness_obvh_topology(const Accelerator* a, const HarnessIndexMap& idx, std::vector<int32_t>& out) {
    const Accel* acc = (const Accel*)a;
    if (acc->m_root) export_node(idx, acc->m_root.get(), out);
}
