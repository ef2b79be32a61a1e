// Hair line and area-shape set-up on the host. Lines: what SORT computes once per Line before any
// ray is traced (shape/line.cpp:117-135 Line::SetTransform, 98-106
// Line::GetBBox), in SORT's operation order (this file is compiled without
// floating-point contraction, as SORT is), so the per-line constants and boxes
// are bit-identical to SORT's.
//
// SORT's HairVisual builds its lines in object space and applies the entity's
// transform (entity/visual.cpp:41-102); lines given in world space take the
// identity, which SORT would still apply through Matrix::TransformPoint (a -0
// coordinate becomes +0), and lines read from a scene stream take their
// entity's transform.
#include "hair.h"

#include <cmath>
#include <cstring>

namespace sg {
namespace {

struct V3 {
    float x, y, z;
};

V3 transform_point(const float* m, const V3& p) {
    const float in[3] = {p.x, p.y, p.z};
    float out[3];
    transform_point16(m, in, out);
    return V3{out[0], out[1], out[2]};
}

// normalize (math/vector3.h:163-168).
V3 normalize(const V3& v) {
    const float len = std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z);
    if (len == 0.0f) return v;
    return V3{v.x / len, v.y / len, v.z / len};
}

}  // namespace

void transform_point16(const float* m, const float* p, float* out) {
    const float x = p[0] * m[0] + p[1] * m[1] + p[2] * m[2] + m[3];
    const float y = p[0] * m[4] + p[1] * m[5] + p[2] * m[6] + m[7];
    const float z = p[0] * m[8] + p[1] * m[9] + p[2] * m[10] + m[11];
    const float w = p[0] * m[12] + p[1] * m[13] + p[2] * m[14] + m[15];
    if (w == 1.0f) {
        out[0] = x;
        out[1] = y;
        out[2] = z;
    } else {  // Point / w multiplies by the reciprocal (math/point.h:126-129)
        const float t = 1.0f / w;
        out[0] = x * t;
        out[1] = y * t;
        out[2] = z * t;
    }
}

void line_setup(const float* in, float* rec, float* box, const float* transform16) {
    const V3 p0{in[0], in[1], in[2]}, p1{in[3], in[4], in[5]};
    const float v0 = in[6], v1 = in[7], w0 = in[8], w1 = in[9];
    static const float identity[16] = {1.0f, 0.0f, 0.0f, 0.0f, 0.0f, 1.0f, 0.0f, 0.0f,
                                       0.0f, 0.0f, 1.0f, 0.0f, 0.0f, 0.0f, 0.0f, 1.0f};
    const float* t16 = transform16 ? transform16 : identity;
    const V3 gp0 = transform_point(t16, p0), gp1 = transform_point(t16, p1);
    const V3 y = normalize(V3{gp1.x - gp0.x, gp1.y - gp0.y, gp1.z - gp0.z});
    // coordinateSystem (math/vector3.h:171-180)
    V3 x;
    if (std::fabs(y.x) > std::fabs(y.y)) {
        const float inv = 1.0f / sqrtf(y.x * y.x + y.z * y.z);
        x = V3{-y.z * inv, 0.0f, y.x * inv};
    } else {
        const float inv = 1.0f / sqrtf(y.y * y.y + y.z * y.z);
        x = V3{0.0f, y.z * inv, -y.y * inv};
    }
    const V3 z{y.y * x.z - y.z * x.y, y.z * x.x - y.x * x.z, y.x * x.y - y.y * x.x};  // cross(y, x)
    const float m[16] = {x.x, x.y, x.z, -(x.x * gp0.x + x.y * gp0.y + x.z * gp0.z),
                         y.x, y.y, y.z, -(y.x * gp0.x + y.y * gp0.y + y.z * gp0.z),
                         z.x, z.y, z.z, -(z.x * gp0.x + z.y * gp0.y + z.z * gp0.z),
                         0.0f, 0.0f, 0.0f, 1.0f};
    const V3 lp0 = transform_point(m, gp0), lp1 = transform_point(m, gp1);
    const float length = lp1.y - lp0.y;
    for (int k = 0; k < 12; ++k) rec[k] = m[k];
    rec[12] = w0;
    rec[13] = w1;
    rec[14] = length;
    rec[15] = (w1 - w0) / length;  // formed per test by intersectLine_Inner (simd/simd_line.h:239)
    rec[16] = v0;
    rec[17] = v1;
    rec[18] = 0.0f;
    rec[19] = 0.0f;
    // Line::GetBBox: BBox() then Union(gp0), Union(gp1) (math/bbox.cpp:106-113), Expend(max(w0, w1)).
    float mn[3] = {3.402823466e+38f, 3.402823466e+38f, 3.402823466e+38f};
    float mx[3] = {-3.402823466e+38f, -3.402823466e+38f, -3.402823466e+38f};
    for (const V3& p : {gp0, gp1}) {
        const float c[3] = {p.x, p.y, p.z};
        for (int a = 0; a < 3; ++a) {
            if (c[a] < mn[a]) mn[a] = c[a];
            if (c[a] > mx[a]) mx[a] = c[a];
        }
    }
    const float grow = w0 < w1 ? w1 : w0;  // std::max(w0, w1)
    for (int a = 0; a < 3; ++a) {
        box[a] = mn[a] - grow;
        box[3 + a] = mx[a] + grow;
    }
}

void shape_setup(const sg_area_shape& shape, float* rec, float* box) {
    const bool disk = shape.kind == SG_SHAPE_DISK;
    // Quad: halfx = sizeX * 0.5f, halfy = sizeY * 0.5f (shape/quad.cpp:71-80, 86-89);
    // Disk: the radius and its square as Disk::GetIntersect forms it.
    const float a = disk ? shape.size[0] : shape.size[0] * 0.5f;
    const float b = disk ? shape.size[0] * shape.size[0] : shape.size[1] * 0.5f;
    for (int k = 0; k < 16; ++k) rec[k] = shape.inverse[k];
    rec[16] = a;
    rec[17] = b;
    const int32_t kind = shape.kind;
    std::memcpy(&rec[18], &kind, 4);
    rec[19] = 0.0f;
    // Quad::GetBBox / Disk::GetBBox: BBox() then Union of four corners of the
    // shape in its plane through m_transform.TransformPoint.
    const float ex = a, ez = disk ? a : b;
    const float corners[4][3] = {{ex, 0.0f, ez}, {ex, 0.0f, -ez}, {-ex, 0.0f, ez}, {-ex, 0.0f, -ez}};
    float mn[3] = {3.402823466e+38f, 3.402823466e+38f, 3.402823466e+38f};
    float mx[3] = {-3.402823466e+38f, -3.402823466e+38f, -3.402823466e+38f};
    for (const auto& c : corners) {
        float w[3];
        transform_point16(shape.matrix, c, w);
        for (int k = 0; k < 3; ++k) {
            if (w[k] < mn[k]) mn[k] = w[k];
            if (w[k] > mx[k]) mx[k] = w[k];
        }
    }
    for (int k = 0; k < 3; ++k) {
        box[k] = mn[k];
        box[3 + k] = mx[k];
    }
}

}  // namespace sg
