// Internal (not exported) access to a scene's launch parameters, for entry
// points implemented outside api.cpp.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "sortgpu.h"
#include "trace_kernels.h"

namespace sg {

// Primitives of a scene: triangles (9 floats), hair segments (10 floats; with
// transforms set, segment k is in the object space that the row-major 4x4
// transforms[16 * line_transform[k]] maps to world space, else in world
// space), area shapes, and optionally the order SORT's builder sees them in
// (sg_shapes).
struct MixedInput {
    const float* triangles = nullptr;
    int64_t ntri = 0;
    const float* lines = nullptr;
    int64_t nlines = 0;
    const float* transforms = nullptr;
    const int32_t* line_transform = nullptr;
    const sg_area_shape* shapes = nullptr;
    int64_t nshapes = 0;
    const int32_t* order = nullptr;
};

struct BuiltTree;
struct BuildParams;
// SORT's tree over every primitive of `in` and the non-triangle primitives'
// records (20 floats each, lines then shapes). Throws as build_tree does.
BuiltTree build_mixed(const MixedInput& in, BuildParams bp, int builder, int device, std::vector<float>& recs);

sg_status scene_create_mixed(const MixedInput& in, const sg_build_opts* opts, sg_scene** out);

// Records msg for sg_last_error() and returns s.
sg_status set_error(sg_status s, const char* msg);

// Fills the launch description (width, stack bound, tuning, status word,
// persistent-schedule counter slot) and the device tree of scene s.
sg_status scene_launch(const sg_scene* s, bool any, TraceLaunch* L, DevTree* tree, int* device);

// The per-primitive material ids of scene s on its device (sg_scene_set_materials), or NULL.
const int32_t* scene_materials(const sg_scene* s);

// Synchronises st and reports the traversal status word of scene s.
sg_status scene_status(const sg_scene* s, cudaStream_t st);

struct PtDev;
// The shading tables of a path-tracing scene and the traversal scene it uses.
sg_status pt_scene_parts(const sg_pt_scene* ps, PtDev* dev, const sg_scene** scene);

}  // namespace sg
