// sg_stream_*: reading SORT's binary scene stream (the file the Blender
// exporter writes and SORT loads), for the GPU path.
//
// The stream is read in SORT's order (work/image_evaluation/image_evaluation.cpp:
// 62-108): the global configuration (loadConfig, 354-377, with the integrator's
// Serialize), the material section (MatManager::ParseMatFile,
// material/matmanager.cpp:50-270, and Material::Serialize,
// material/material.cpp:153-225), the entities (Scene::LoadScene,
// core/scene.cpp:112-180), then the accelerator's class and parameters.
// Scalars are 4 bytes (float, int, unsigned), bool 1 byte, strings end with a
// NUL byte, a StringID is the 32-bit CRC SORT hashes class names with
// (core/strid.h:40-65), a Transform is its 16-float matrix.
//
// What the GPU path uses is kept: triangles in world space (MeshVisual::
// Serialize and Mesh::ApplyTransform, entity/visual.cpp:25-39,
// core/mesh.cpp:26-38, 111-178) with their material indices, hair segments as
// HairVisual makes them (entity/visual.cpp:41-97) with their entity's
// transform, the camera, area lights, the integrator's parameters, material
// names and flags, and the accelerator. Materials' TSL shader graphs, resource
// files, volume data and the other light types are read past (their counts and
// types are reported). Each area light's shape (a Quad for SQUARE and
// RECTANGLE, a Disk for DISK) is a primitive of the scene, with the transform
// AreaLightEntity::Serialize leaves it (entity/light_entity.cpp:97-154: the
// streamed matrix, its inverse by Matrix::Inverse, the scale taken out of
// both). The order of the primitives as SORT's ScenePrimitiveIterator visits
// them (entity by entity) is recorded; the scene is built in that order.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "hair.h"
#include "scene_access.h"
#include "sortgpu.h"

struct sg_stream {
    sg_stream_info info{};
    std::vector<float> triangles;  // 9 per triangle, world space
    std::vector<int32_t> tri_material;
    std::vector<float> lines;         // 10 per segment, object space of their entity
    std::vector<int32_t> line_material;
    std::vector<int32_t> line_transform;  // index into transforms
    std::vector<float> transforms;        // 16 per hair entity
    sg_stream_camera camera{};
    std::vector<sg_stream_area_light> area_lights;
    std::vector<sg_area_shape> shapes;  // one per area light, as the scene holds it
    std::vector<std::pair<int, int64_t>> runs;  // (kind 0 triangle / 1 line / 2 shape, count) in entity order
    std::vector<std::string> material_names;
    std::vector<int32_t> material_flags;  // bit 0 transparency node, bit 1 SSS node
};

namespace {

constexpr uint32_t sid(const char* s) {
    // crc32_bitwise of core/strid.h:40-57: reflected polynomial, zero start, inverted end.
    uint32_t crc = 0;
    for (; *s; ++s) {
        crc ^= uint32_t(uint8_t(*s));
        for (int k = 0; k < 8; ++k) crc = (crc >> 1) ^ ((0u - (crc & 1u)) & 0xEDB88320u);
    }
    return ~crc;
}

// Matrix::Inverse (math/matrix.cpp:115-143, Cramer's rule, with the
// determinant of 104-112), each entry in SORT's expression order so the
// inverse is bit-identical; false (out untouched) when |det| < 1e-8.
bool inverse16(const float* m, float* out) {
    float d = (m[0] * m[5] - m[1] * m[4]) * (m[10] * m[15] - m[11] * m[14]) -
              (m[0] * m[6] - m[2] * m[4]) * (m[9] * m[15] - m[11] * m[13]) +
              (m[0] * m[7] - m[3] * m[4]) * (m[9] * m[14] - m[10] * m[13]) +
              (m[1] * m[6] - m[2] * m[5]) * (m[8] * m[15] - m[11] * m[12]) -
              (m[1] * m[7] - m[3] * m[5]) * (m[8] * m[14] - m[10] * m[12]) +
              (m[2] * m[7] - m[3] * m[6]) * (m[8] * m[13] - m[9] * m[12]);
    if (std::fabs(d) < 0.00000001f) return false;
    d = 1.0f / d;
    // Entry (r, c) is a cofactor written as a sum of three products; the table
    // gives, per entry, the three (m[a], m[b] * m[c] - m[e] * m[f]) terms.
    static const int8_t T[16][15] = {
        {5, 10, 15, 11, 14, 6, 11, 13, 9, 15, 7, 9, 14, 10, 13},
        {9, 2, 15, 3, 14, 10, 3, 13, 1, 15, 11, 1, 14, 2, 13},
        {13, 2, 7, 3, 6, 14, 3, 5, 1, 7, 15, 1, 6, 2, 5},
        {1, 7, 10, 6, 11, 2, 5, 11, 7, 9, 3, 6, 9, 5, 10},
        {6, 8, 15, 11, 12, 7, 10, 12, 8, 14, 4, 11, 14, 10, 15},
        {10, 0, 15, 3, 12, 11, 2, 12, 0, 14, 8, 3, 14, 2, 15},
        {14, 0, 7, 3, 4, 15, 2, 4, 0, 6, 12, 3, 6, 2, 7},
        {2, 7, 8, 4, 11, 3, 4, 10, 6, 8, 0, 6, 11, 7, 10},
        {7, 8, 13, 9, 12, 4, 9, 15, 11, 13, 5, 11, 12, 8, 15},
        {11, 0, 13, 1, 12, 8, 1, 15, 3, 13, 9, 3, 12, 0, 15},
        {15, 0, 5, 1, 4, 12, 1, 7, 3, 5, 13, 3, 4, 0, 7},
        {3, 5, 8, 4, 9, 0, 7, 9, 5, 11, 1, 4, 11, 7, 8},
        {4, 10, 13, 9, 14, 5, 8, 14, 10, 12, 6, 9, 12, 8, 13},
        {8, 2, 13, 1, 14, 9, 0, 14, 2, 12, 10, 1, 12, 0, 13},
        {12, 2, 5, 1, 6, 13, 0, 6, 2, 4, 14, 1, 4, 0, 5},
        {0, 5, 10, 6, 9, 1, 6, 8, 4, 10, 2, 4, 9, 5, 8}};
    for (int k = 0; k < 16; ++k) {
        const int8_t* t = T[k];
        const float a = m[t[0]] * (m[t[1]] * m[t[2]] - m[t[3]] * m[t[4]]);
        const float b = m[t[5]] * (m[t[6]] * m[t[7]] - m[t[8]] * m[t[9]]);
        const float c = m[t[10]] * (m[t[11]] * m[t[12]] - m[t[13]] * m[t[14]]);
        out[k] = d * (a + b + c);
    }
    return true;
}

// Matrix::operator* (math/matrix.cpp:51-67): each entry summed from 0 over k.
void multiply16(const float* a, const float* b, float* out) {
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            float v = 0.0f;
            for (int k = 0; k < 4; ++k) v += a[i * 4 + k] * b[k * 4 + j];
            out[i * 4 + j] = v;
        }
}

// The shape of an area light as AreaLightEntity::Serialize leaves it
// (entity/light_entity.cpp:97-150): the transform without its scale, a Quad
// of size (SetSizeX / SetSizeY clamp to 0.0001) or a Disk of radius.
sg_area_shape light_shape(const sg_stream_area_light& a) {
    const float* m = a.light2world;
    float inv[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};  // Matrix() when not invertible
    inverse16(m, inv);
    auto length = [](float x, float y, float z) { return std::sqrt(x * x + y * y + z * z); };
    const float sx = length(m[0], m[4], m[8]), sy = length(m[1], m[5], m[9]), sz = length(m[2], m[6], m[10]);
    const float unscale[16] = {1 / sx, 0, 0, 0, 0, 1 / sy, 0, 0, 0, 0, 1 / sz, 0, 0, 0, 0, 1};
    const float scale[16] = {sx, 0, 0, 0, 0, sy, 0, 0, 0, 0, sz, 0, 0, 0, 0, 1};
    sg_area_shape out{};
    multiply16(m, unscale, out.matrix);
    multiply16(scale, inv, out.inverse);
    if (a.shape == sid("DISK")) {
        out.kind = SG_SHAPE_DISK;
        out.size[0] = a.size_x;
    } else {
        out.kind = SG_SHAPE_QUAD;
        const float y = a.shape == sid("SQUARE") ? a.size_x : a.size_y;
        out.size[0] = std::max(0.0001f, a.size_x);
        out.size[1] = std::max(0.0001f, y);
    }
    return out;
}

void add_run(sg_stream& s, int kind, int64_t count) {
    if (count <= 0) return;
    if (!s.runs.empty() && s.runs.back().first == kind)
        s.runs.back().second += count;
    else
        s.runs.emplace_back(kind, count);
}

class Reader {
public:
    explicit Reader(const char* path) : f_(std::fopen(path, "rb")) {
        if (!f_) throw std::invalid_argument(std::string("cannot open ") + path);
    }
    ~Reader() {
        if (f_) std::fclose(f_);
    }
    void bytes(void* dst, size_t n, const char* what) {
        if (n && std::fread(dst, 1, n, f_) != n) throw std::runtime_error(std::string("stream ends inside ") + what);
    }
    void skip(uint64_t n, const char* what) {
        char buf[4096];
        while (n) {
            const size_t k = n < sizeof(buf) ? size_t(n) : sizeof(buf);
            bytes(buf, k, what);
            n -= k;
        }
    }
    uint32_t u32(const char* what) {
        uint32_t v;
        bytes(&v, 4, what);
        return v;
    }
    int32_t i32(const char* what) { return int32_t(u32(what)); }
    float f32(const char* what) {
        float v;
        bytes(&v, 4, what);
        return v;
    }
    bool boolean(const char* what) {
        uint8_t v;
        bytes(&v, 1, what);
        return v != 0;
    }
    std::string str(const char* what) {
        std::string s;
        for (;;) {
            char c;
            bytes(&c, 1, what);
            if (c == 0) return s;
            s.push_back(c);
        }
    }
    int64_t offset() const { return int64_t(std::ftell(f_)); }

private:
    FILE* f_;
};

// Shader units with their parameter defaults, then connections (the list both
// ShaderGroupTemplate and a material's shaders use).
void skip_shader_graph(Reader& r) {
    const uint32_t units = r.u32("shader units");
    for (uint32_t i = 0; i < units; ++i) {
        r.str("shader unit name");
        r.str("shader unit type");
        const uint32_t params = r.u32("shader parameters");
        for (uint32_t j = 0; j < params; ++j) {
            r.str("parameter name");
            const int32_t channels = r.i32("parameter channels");
            if (channels == 1)
                r.f32("parameter value");
            else if (channels == 3)
                r.skip(12, "parameter value");
            else if (channels == 4)
                r.str("parameter reference");
        }
    }
    const uint32_t connections = r.u32("shader connections");
    for (uint32_t i = 0; i < connections; ++i)
        for (int k = 0; k < 4; ++k) r.str("shader connection");
}

void read_config(Reader& r, sg_stream_info& in) {
    in.version = r.i32("version");
    if (in.version != 0) throw std::runtime_error("unknown scene stream version");
    r.str("resource path");
    in.threads = r.i32("thread count");
    in.spp = r.i32("samples per pixel");
    in.image_width = r.i32("image width");
    in.image_height = r.i32("image height");
    in.clamp = r.f32("clamp");
    in.integrator = r.u32("integrator");
    in.max_depth = r.i32("max recursive depth");  // Integrator::Serialize
    if (in.integrator == sid("PathTracing")) {
        in.bssrdf_bounces = r.i32("BSSRDF bounces");
    } else if (in.integrator == sid("AmbientOcclusion")) {
        in.ao_max_distance = r.f32("AO distance");
    } else if (in.integrator == sid("BidirPathTracing") || in.integrator == sid("LightTracing")) {
        in.mis = r.boolean("MIS") ? 1 : 0;
    } else if (in.integrator == sid("InstantRadiosity")) {
        in.ir_path_sets = r.i32("light path sets");
        in.ir_paths = r.i32("light paths");
        in.ir_min_distance = r.f32("minimum distance");
    } else if (in.integrator != sid("DirectLight") && in.integrator != sid("WhittedRT")) {
        throw std::runtime_error("unknown integrator in the scene stream");
    }
}

void read_materials(Reader& r, sg_stream& s) {
    const uint32_t resources = r.u32("resource count");
    for (uint32_t i = 0; i < resources; ++i) {
        r.str("resource file");
        r.u32("resource type");
    }
    for (;;) {
        const uint32_t kind = r.u32("material section");
        if (kind == sid("End of Material")) return;
        if (kind == sid("ShaderUnitTemplate")) {
            r.str("shader unit type");
            r.str("shader source");
            const uint32_t bindings = r.u32("resource bindings");
            for (uint32_t i = 0; i < bindings; ++i) {
                r.str("resource handle");
                r.str("resource name");
            }
        } else if (kind == sid("ShaderGroupTemplate")) {
            r.str("shader group type");
            skip_shader_graph(r);
            r.str("root shader");
            const uint32_t out_args = r.u32("exposed outputs");
            for (uint32_t i = 0; i < out_args; ++i) r.str("exposed output");
            const std::string input = r.str("group input");
            if (!input.empty()) {
                const uint32_t in_args = r.u32("exposed inputs");
                for (uint32_t i = 0; i < in_args; ++i) r.str("exposed input");
            }
        } else if (kind == sid("Material")) {
            s.material_names.push_back(r.str("material name"));
            if (r.u32("surface shader tag") == sid("Surface Shader")) skip_shader_graph(r);
            if (r.u32("volume shader tag") == sid("Volume Shader")) skip_shader_graph(r);
            int32_t flags = r.boolean("transparency flag") ? 1 : 0;
            flags |= r.boolean("SSS flag") ? 2 : 0;
            r.f32("volume step");
            r.u32("volume step count");
            s.material_flags.push_back(flags);
        } else {
            throw std::runtime_error("unknown entry in the material section");
        }
    }
}

void read_matrix(Reader& r, float* m) {
    for (int k = 0; k < 16; ++k) m[k] = r.f32("transform");
}

// MeshVisual::Serialize then ApplyTransform: world-space triangles.
void read_mesh(Reader& r, const float* xf, sg_stream& s) {
    r.boolean("has uv");
    const uint32_t nv = r.u32("vertex count");
    std::vector<float> pos(size_t(nv) * 3);
    for (uint32_t i = 0; i < nv; ++i) {
        float v[8];  // position, normal, texture coordinate
        r.bytes(v, sizeof(v), "vertices");
        sg::transform_point16(xf, v, &pos[size_t(i) * 3]);
    }
    const uint32_t nt = r.u32("triangle count");
    for (uint32_t i = 0; i < nt; ++i) {
        int32_t id[4];  // three vertex indices, material index
        r.bytes(id, sizeof(id), "triangles");
        for (int k = 0; k < 3; ++k) {
            if (id[k] < 0 || uint32_t(id[k]) >= nv) throw std::runtime_error("triangle index out of range");
            for (int a = 0; a < 3; ++a) s.triangles.push_back(pos[size_t(id[k]) * 3 + a]);
        }
        s.tri_material.push_back(id[3]);
    }
    const uint32_t volume = r.u32("volume tag");
    if (volume == sid("has_volume")) {  // MediumDensity::Serialize (medium/mediumdata.cpp:26-38)
        const uint32_t w = r.u32("volume width"), h = r.u32("volume height"), d = r.u32("volume depth");
        if (w && h && d) r.skip(uint64_t(w) * h * d * 4, "volume density");
        s.info.volumes++;
    } else if (volume != sid("no_volume")) {
        throw std::runtime_error("bad volume tag in a mesh");
    }
    if (r.u32("end of mesh") != sid("end of mesh")) throw std::runtime_error("mesh does not end where expected");
}

// HairVisual::Serialize: one segment per step, width and v by length fraction.
void read_hair(Reader& r, int32_t xf_index, sg_stream& s) {
    const uint32_t count = r.u32("hair count");
    const float width_tip = r.f32("tip width"), width_bottom = r.f32("bottom width");
    const int32_t mat = r.i32("hair material");
    for (uint32_t i = 0; i < count; ++i) {
        const uint32_t steps = r.u32("hair steps");
        if (steps == 0) continue;  // SORT reads no point for such a strand
        std::vector<float> p(size_t(steps + 1) * 3);
        r.bytes(p.data(), p.size() * sizeof(float), "hair points");
        std::vector<float> len(steps, 0.0f);
        for (uint32_t j = 0; j < steps; ++j) {
            const float dx = p[3 * j] - p[3 * (j + 1)], dy = p[3 * j + 1] - p[3 * (j + 1) + 1],
                        dz = p[3 * j + 2] - p[3 * (j + 1) + 2];
            len[j] += std::sqrt(dx * dx + dy * dy + dz * dz);  // distance (math/point.h)
        }
        float total = 0.0f;
        for (float l : len) total += l;  // std::accumulate
        if (total <= 0.0f) continue;
        float prev_v = 0.0f, prev_w = width_bottom, cur_len = 0.0f;
        for (uint32_t j = 1; j <= steps; ++j) {
            cur_len += len[j - 1];
            const float t = cur_len / total;
            const float cur_w = width_bottom * (1.0f - t) + width_tip * t;  // slerp (math/utils.h:81)
            const float cur_v = 0.0f * (1.0f - t) + 1.0f * t;
            const float seg[10] = {p[3 * (j - 1)], p[3 * (j - 1) + 1], p[3 * (j - 1) + 2], p[3 * j], p[3 * j + 1],
                                   p[3 * j + 2], prev_v, cur_v, prev_w, cur_w};
            s.lines.insert(s.lines.end(), seg, seg + 10);
            s.line_material.push_back(mat);
            s.line_transform.push_back(xf_index);
            prev_w = cur_w;
            prev_v = cur_v;
        }
    }
}

void read_entities(Reader& r, sg_stream& s) {
    if (r.u32("verification bits") != sid("verification bits")) throw std::runtime_error("not a SORT scene stream");
    s.info.entity_offset = r.offset() - 4;
    for (;;) {
        const uint32_t kind = r.u32("entity class");
        if (kind == sid("End of Entities")) return;
        if (kind == sid("VisualEntity")) {
            float xf[16];
            read_matrix(r, xf);
            const uint32_t visuals = r.u32("visual count");
            for (uint32_t v = 0; v < visuals; ++v) {
                const uint32_t vk = r.u32("visual class");
                if (vk == sid("MeshVisual")) {
                    const size_t before = s.tri_material.size();
                    read_mesh(r, xf, s);
                    add_run(s, 0, int64_t(s.tri_material.size() - before));
                } else if (vk == sid("HairVisual")) {
                    s.transforms.insert(s.transforms.end(), xf, xf + 16);
                    const size_t before = s.line_material.size();
                    read_hair(r, int32_t(s.transforms.size() / 16 - 1), s);
                    add_run(s, 1, int64_t(s.line_material.size() - before));
                } else {
                    throw std::runtime_error("unknown visual class in the scene stream");
                }
            }
        } else if (kind == sid("PerspectiveCameraEntity")) {
            sg_stream_camera& c = s.camera;
            for (float* v : {c.eye, c.up, c.target})
                for (int a = 0; a < 3; ++a) v[a] = r.f32("camera");
            c.image_width = r.i32("camera width");
            c.image_height = r.i32("camera height");
            c.lens_radius = r.f32("lens radius");
            c.sensor_w = r.f32("sensor width");
            c.sensor_h = r.f32("sensor height");
            c.aspect_fit = r.i32("sensor fit");
            c.aspect_ratio_w = r.f32("aspect ratio");
            c.aspect_ratio_h = r.f32("aspect ratio");
            c.fov = r.f32("field of view");
            s.info.has_camera = 1;
        } else if (kind == sid("AreaLightEntity")) {
            sg_stream_area_light a{};
            read_matrix(r, a.light2world);
            a.energy = r.f32("light energy");
            for (int k = 0; k < 3; ++k) a.intensity[k] = r.f32("light intensity");
            a.shape = r.u32("area light shape");
            if (a.shape == sid("SQUARE") || a.shape == sid("DISK")) {
                a.size_x = r.f32("area light size");
            } else if (a.shape == sid("RECTANGLE")) {
                a.size_x = r.f32("area light size");
                a.size_y = r.f32("area light size");
            } else {
                throw std::runtime_error("unknown area light shape");
            }
            s.area_lights.push_back(a);
            s.shapes.push_back(light_shape(a));  // the light's Primitive (entity/light_entity.cpp:153-154)
            add_run(s, 2, 1);
        } else if (kind == sid("PointLightEntity") || kind == sid("DirLightEntity") ||
                   kind == sid("SpotLightEntity")) {
            float m[16];
            read_matrix(r, m);
            r.f32("light energy");
            r.skip(12, "light intensity");
            if (kind == sid("SpotLightEntity")) r.skip(8, "spot light falloff");
            s.info.other_lights++;
        } else if (kind == sid("SkyLightEntity")) {
            float m[16];
            read_matrix(r, m);
            r.f32("sky intensity");
            r.skip(12, "sky colour");
            r.str("sky image");
            s.info.other_lights++;
        } else {
            throw std::runtime_error("unknown entity class in the scene stream");
        }
    }
}

void read_accelerator(Reader& r, sg_stream_info& in) {
    in.accelerator = r.u32("accelerator");
    if (in.accelerator == sid("Qbvh") || in.accelerator == sid("Obvh") || in.accelerator == sid("Bvh") ||
        in.accelerator == sid("KDTree") || in.accelerator == sid("OcTree")) {
        in.accel_max_depth = r.i32("accelerator depth");
        in.accel_max_leaf = r.i32("accelerator leaf size");
    }
}

}  // namespace

extern "C" {

sg_status sg_stream_open(const char* path, sg_stream** out) {
    if (!path || !out) return sg::set_error(SG_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = nullptr;
    std::unique_ptr<sg_stream> s(new (std::nothrow) sg_stream());
    if (!s) return sg::set_error(SG_ERR_OUT_OF_MEMORY, "host allocation failed");
    try {
        Reader r(path);
        read_config(r, s->info);
        read_materials(r, *s);
        read_entities(r, *s);
        read_accelerator(r, s->info);
    } catch (const std::invalid_argument& e) {
        return sg::set_error(SG_ERR_INVALID_ARGUMENT, e.what());
    } catch (const std::bad_alloc&) {
        return sg::set_error(SG_ERR_OUT_OF_MEMORY, "host memory exhausted reading the stream");
    } catch (const std::exception& e) {
        return sg::set_error(SG_ERR_UNSUPPORTED, e.what());
    }
    sg_stream_info& in = s->info;
    in.triangles = int64_t(s->tri_material.size());
    in.lines = int64_t(s->line_material.size());
    in.materials = int32_t(s->material_names.size());
    in.area_lights = int32_t(s->area_lights.size());
    *out = s.release();
    return SG_OK;
}

sg_status sg_stream_info_get(const sg_stream* s, sg_stream_info* info) {
    if (!s || !info) return sg::set_error(SG_ERR_INVALID_ARGUMENT, "NULL argument");
    *info = s->info;
    return SG_OK;
}

sg_status sg_stream_triangles(const sg_stream* s, float* tri9, int32_t* material) {
    if (!s) return sg::set_error(SG_ERR_INVALID_ARGUMENT, "NULL stream");
    if (tri9 && !s->triangles.empty()) std::memcpy(tri9, s->triangles.data(), s->triangles.size() * sizeof(float));
    if (material && !s->tri_material.empty())
        std::memcpy(material, s->tri_material.data(), s->tri_material.size() * sizeof(int32_t));
    return SG_OK;
}

sg_status sg_stream_lines(const sg_stream* s, float* seg10_world, int32_t* material) {
    if (!s) return sg::set_error(SG_ERR_INVALID_ARGUMENT, "NULL stream");
    for (size_t k = 0; seg10_world && k < s->line_material.size(); ++k) {
        const float* xf = &s->transforms[size_t(s->line_transform[k]) * 16];
        const float* in = &s->lines[k * 10];
        float* o = seg10_world + k * 10;
        sg::transform_point16(xf, in, o);
        sg::transform_point16(xf, in + 3, o + 3);
        for (int j = 6; j < 10; ++j) o[j] = in[j];
    }
    if (material && !s->line_material.empty())
        std::memcpy(material, s->line_material.data(), s->line_material.size() * sizeof(int32_t));
    return SG_OK;
}

sg_status sg_stream_camera_get(const sg_stream* s, sg_stream_camera* camera) {
    if (!s || !camera) return sg::set_error(SG_ERR_INVALID_ARGUMENT, "NULL argument");
    if (!s->info.has_camera) return sg::set_error(SG_ERR_INVALID_ARGUMENT, "the stream has no camera");
    *camera = s->camera;
    return SG_OK;
}

sg_status sg_stream_area_light_get(const sg_stream* s, int32_t k, sg_stream_area_light* light) {
    if (!s || !light) return sg::set_error(SG_ERR_INVALID_ARGUMENT, "NULL argument");
    if (k < 0 || size_t(k) >= s->area_lights.size()) return sg::set_error(SG_ERR_INVALID_ARGUMENT, "no such light");
    *light = s->area_lights[size_t(k)];
    return SG_OK;
}

sg_status sg_stream_material(const sg_stream* s, int32_t k, char* name, int64_t cap, int32_t* flags) {
    if (!s) return sg::set_error(SG_ERR_INVALID_ARGUMENT, "NULL stream");
    if (k < 0 || size_t(k) >= s->material_names.size()) return sg::set_error(SG_ERR_INVALID_ARGUMENT, "no such material");
    const std::string& n = s->material_names[size_t(k)];
    if (name) {
        if (cap < int64_t(n.size()) + 1) return sg::set_error(SG_ERR_LIMIT, "name buffer too small");
        std::memcpy(name, n.c_str(), n.size() + 1);
    }
    if (flags) *flags = s->material_flags[size_t(k)];
    return SG_OK;
}

sg_status sg_stream_close(sg_stream* s) {
    delete s;
    return SG_OK;
}

sg_status sg_stream_scene_create(const sg_stream* s, const sg_build_opts* opts, sg_scene** out) {
    if (!s || !out) return sg::set_error(SG_ERR_INVALID_ARGUMENT, "NULL argument");
    sg_build_opts o;
    if (opts) {
        o = *opts;
    } else {
        // The stream's accelerator: Obvh and Qbvh keep their width and
        // parameters; anything else takes SORT's fallback, a QBVH
        // (core/scene.cpp:169-177), with Fbvh's default parameters.
        sg_default_build_opts(&o);
        const sg_stream_info& in = s->info;
        o.width = in.accelerator == sid("Obvh") ? 8 : 4;
        if (in.accelerator == sid("Obvh") || in.accelerator == sid("Qbvh")) {
            o.max_depth = in.accel_max_depth;
            o.max_leaf = in.accel_max_leaf;
        }
    }
    sg::MixedInput in;
    in.triangles = s->triangles.data();
    in.ntri = int64_t(s->tri_material.size());
    in.lines = s->lines.data();
    in.nlines = int64_t(s->line_material.size());
    in.transforms = s->transforms.data();
    in.line_transform = s->line_transform.data();
    in.shapes = s->shapes.data();
    in.nshapes = int64_t(s->shapes.size());
    // SORT's primitive order: the runs of each kind in entity order. Left out
    // (NULL) when it is triangles, then lines, then shapes anyway.
    std::vector<int32_t> order;
    bool natural = true;
    int last = 0;
    for (const auto& run : s->runs) {
        if (run.first < last) natural = false;
        last = run.first;
    }
    if (!natural) {
        int64_t next[3] = {0, in.ntri, in.ntri + in.nlines};
        try {
            order.reserve(size_t(in.ntri + in.nlines + in.nshapes));
            for (const auto& run : s->runs)
                for (int64_t k = 0; k < run.second; ++k) order.push_back(int32_t(next[run.first]++));
        } catch (const std::bad_alloc&) {
            return sg::set_error(SG_ERR_OUT_OF_MEMORY, "host allocation failed");
        }
        in.order = order.data();
    }
    return sg::scene_create_mixed(in, &o, out);
}

sg_status sg_stream_primitive_order(const sg_stream* s, int32_t* order) {
    if (!s || !order) return sg::set_error(SG_ERR_INVALID_ARGUMENT, "NULL argument");
    const int64_t ntri = int64_t(s->tri_material.size()), nlines = int64_t(s->line_material.size());
    int64_t next[3] = {0, ntri, ntri + nlines}, k = 0;
    for (const auto& run : s->runs)
        for (int64_t j = 0; j < run.second; ++j) order[k++] = int32_t(next[run.first]++);
    return SG_OK;
}

sg_status sg_stream_area_shapes(const sg_stream* s, sg_area_shape* shapes) {
    if (!s || (!shapes && !s->shapes.empty())) return sg::set_error(SG_ERR_INVALID_ARGUMENT, "NULL argument");
    if (!s->shapes.empty()) std::memcpy(shapes, s->shapes.data(), s->shapes.size() * sizeof(sg_area_shape));
    return SG_OK;
}

}  // extern "C"
