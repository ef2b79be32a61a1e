// Plain data of the path tracer shared by host and device code: materials, the
// area light, a scene's shading tables and the pinhole camera.
#pragma once

#include <vector_types.h>

namespace sg {

struct PtMaterial {
    int type;  // 0 Lambert, 1 GGX conductor reflection, 2 the light's own surface (white Lambert)
    float a[3];
    float k[3];
    float rough;
};

struct PtLight {
    float c[3];
    float hx, hz;
    float I[3];
    float area;
};

struct PtDev {
    const float4* prim;  // per primitive: geometric normal, material id (bits of w)
    const PtMaterial* mats;
    PtLight light;
};

struct Cam {
    float3 eye, fwd, right, up;
    float half_w, half_h;
};

// Camera from eye xyz, target xyz, up xyz, vertical fov in degrees, for an
// image of width x height (implemented in pt.cu).
Cam make_camera(const float* camera, int width, int height);

}  // namespace sg
