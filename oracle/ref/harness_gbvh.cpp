// The Gbvh adapter (sort_b200/integration/gbvh.h) inside SORT's own code
// (TEST INFRASTRUCTURE ONLY). Compiled with SORT's unmodified sources and the
// rest of the harness into oracle/_ref/libsortref_gbvh.so, which also links
// the GPU engine (libsortgpu.so). sortref_use_gbvh(1) makes every harness
// scene built afterwards (sortref_scene_create*, sortref_scene_from_stream,
// sortref_pt_scene_create) use Gbvh instead of SORT's Qbvh / Obvh, so SORT's
// Scene::GetIntersect / GetAttenuation and its PathTracing integrator run on
// the GPU through the adapter, one ray per call, exactly as SORT would call
// an accelerator it loaded from a scene stream.
//
// gbvh.h reads shape members SORT keeps protected or private (sizes,
// transforms, line end points); a SORT build grants that with friend
// declarations, this harness by opening the headers, as harness.cpp does.
#define private public
#define protected public
#include "core/scene.h"
#include "entity/visual.h"
#include "shape/disk.h"
#include "shape/line.h"
#include "shape/quad.h"
#include "shape/triangle.h"
#undef private
#undef protected

#include "gbvh.h"
#include "harness_width.h"

namespace {
Accelerator* make_gbvh(int width, unsigned max_depth, unsigned max_leaf) {
    return new Gbvh(width, max_depth, max_leaf);
}
}  // namespace

extern "C" void sortref_use_gbvh(int on) { g_harness_accel_factory = on ? make_gbvh : nullptr; }
