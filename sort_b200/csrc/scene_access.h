// Internal (not exported) access to a scene's launch parameters, for entry
// points implemented outside api.cpp.
#pragma once

#include <cuda_runtime.h>

#include "sortgpu.h"
#include "trace_kernels.h"

namespace sg {

// Scene creation with hair segments in object space: segment k is mapped to
// world space by the row-major 4x4 transforms[16 * line_transform[k]] (both
// NULL: the segments are in world space).
sg_status scene_create_mixed(const float* triangles, int64_t ntri, const float* lines, int64_t nlines,
                             const float* transforms, const int32_t* line_transform, const sg_build_opts* opts,
                             sg_scene** out);

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
