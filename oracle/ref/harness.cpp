// Oracle harness around SORT's own accelerator code.
//
// TEST INFRASTRUCTURE ONLY. This file is compiled together with SORT's
// unmodified sources (accel/qbvh.cpp, accel/obvh.cpp, shape/triangle.cpp, ...)
// by oracle/Makefile into oracle/_ref/libsortref.so. Only the test suite, the
// smoke check and bench.py's CPU-baseline leg load that library; the product
// (sort_b200) never links or calls it.
//
// What the harness supplies, because SORT's scene loader needs the absent TSL
// library and a .sort stream:
//   * the Scene / ScenePrimitiveIterator members the accelerator calls
//     (core/scene.cpp:43-80, 112-185 restated over a harness-owned triangle list,
//     including the 0.1% scene-box enlargement of core/scene.cpp:150-154);
//   * an opaque MaterialBase (HasTransparency() == false) so any-hit queries take
//     SORT's opaque early exit (accel/fast_bvh.hpp:362-373);
//   * a thread pool that calls Accelerator::GetIntersect / GetAttenuation per ray,
//     one RenderContext per worker, as SORT's tile workers do
//     (work/image_evaluation/image_evaluation.cpp:184-264).
//
// Hit identity: SORT returns a const Primitive*; the harness maps it to the
// primitive's index in ScenePrimitiveIterator order (= input triangle order).
// Each triangle gets its own three vertices with texture coordinates
// (0,0), (1,0), (0,1), so SORT's interpolated SurfaceInteraction::u/v
// (simd/simd_triangle.h:327-337) equal the barycentric coordinates exactly.

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <queue>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

// Scene's members are private and only core/scene.cpp (not linked) touches them;
// the harness stands in for that file, so it opens them up here.
#define private public
#define protected public
#include "core/scene.h"
#include "entity/visual.h"
#include "material/material.h"
#include "core/render_context.h"
#include "math/interaction.h"
#include "scatteringevent/bssrdf/bssrdf.h"
#include "shape/disk.h"
#include "shape/line.h"
#include "shape/quad.h"
#include "stream/fstream.h"
#undef private
#undef protected

#include "harness_width.h"

// ---------------------------------------------------------------------------------
// Harness-side entity / visual / material.

namespace {

class OpaqueMaterial : public MaterialBase {
public:
    void UpdateScatteringEvent(ScatteringEvent&, RenderContext&) const override {}
    void UpdateMediumStack(const MediumInteraction&, const SE_Interaction, MediumStack&, RenderContext&) const override {}
    void EvaluateMediumSample(const MediumInteraction&, MediumSample&) const override {}
    Spectrum EvaluateTransparency(const SurfaceInteraction&) const override { return 0.0f; }
    void BuildMaterial(Tsl_Namespace::ShadingContext*) override {}
    StringID GetUniqueID() const override { return StringID(1u); }
    bool HasTransparency() const override { return false; }
    bool HasSSS() const override { return false; }
    bool HasVolumeAttached() const override { return false; }
    float GetVolumeStep() const override { return 0.0f; }
    unsigned int GetVolumeStepCnt() const override { return 0; }
    void Serialize(IStreamBase&) override {}
};

OpaqueMaterial g_opaque;

// Material with its own unique id, for the BSSRDF multi-hit query, which keeps
// only hits on primitives of one material (by GetUniqueID), and for the
// transparent-shadow query: a transparent material answers HasTransparency and
// EvaluateTransparency with a constant, in place of the TSL shader's value
// (material/material.h:159-165, 189-191).
class TaggedMaterial : public OpaqueMaterial {
public:
    explicit TaggedMaterial(sid_t id, bool transparent = false, Spectrum transparency = Spectrum(0.0f))
        : m_id(id), m_transparent(transparent), m_transparency(transparency) {}
    StringID GetUniqueID() const override { return StringID(m_id); }
    bool HasTransparency() const override { return m_transparent; }
    Spectrum EvaluateTransparency(const SurfaceInteraction&) const override {
        return m_transparent ? m_transparency : Spectrum(0.0f);
    }

private:
    sid_t m_id;
    bool m_transparent;
    Spectrum m_transparency;
};

// Material index k of a harness scene maps to unique id kMaterialIdBase + k.
constexpr sid_t kMaterialIdBase = 1000;

// A MeshVisual filled directly from a flat triangle list (one triangle per three
// vertices), mirroring what MeshVisual::Serialize does (entity/visual.cpp:26-33).
class HarnessVisual : public MeshVisual {
public:
    void Fill(const float* tri, int ntri, MaterialBase* const* mats = nullptr) {
        m_memory = std::make_unique<Mesh>();
        m_memory->m_vertices.resize((size_t)ntri * 3);
        m_memory->m_indices.resize((size_t)ntri);
        for (int i = 0; i < ntri; ++i) {
            const float* p = tri + (size_t)i * 9;
            Point a(p[0], p[1], p[2]), b(p[3], p[4], p[5]), c(p[6], p[7], p[8]);
            Vector n = cross(c - a, b - a);
            const float len = n.Length();
            n = len > 0.0f ? n / len : Vector(0.0f, 1.0f, 0.0f);
            const Point pts[3] = {a, b, c};
            const float uv[3][2] = {{0.0f, 0.0f}, {1.0f, 0.0f}, {0.0f, 1.0f}};
            for (int k = 0; k < 3; ++k) {
                MeshVertex& mv = m_memory->m_vertices[(size_t)i * 3 + k];
                mv.m_position = pts[k];
                mv.m_normal = n;
                mv.m_tangent = Vector(1.0f, 0.0f, 0.0f);
                mv.m_texCoord = Vector2f(uv[k][0], uv[k][1]);
            }
            MeshFaceIndex& fi = m_memory->m_indices[(size_t)i];
            fi.m_id[0] = i * 3;
            fi.m_id[1] = i * 3 + 1;
            fi.m_id[2] = i * 3 + 2;
            fi.m_mat = mats ? mats[i] : &g_opaque;
        }
        m_memory->m_hasUV = true;
        for (const auto& mi : m_memory->m_indices) {
            m_triangles.push_back(std::make_unique<Triangle>(this, mi));
            m_primitives.push_back(std::make_unique<Primitive>(m_memory.get(), mi.m_mat, m_triangles.back().get()));
        }
    }
};

// Hair line segments as SORT's HairVisual makes them (entity/visual.cpp:41-102):
// one Line per segment, its transform applied (the identity here: the segments
// are given in world space), one Primitive per Line.
class HarnessHair : public Visual {
public:
    void Fill(const float* seg, int n) {
        for (int i = 0; i < n; ++i) {
            const float* s = seg + (size_t)i * 10;
            m_lines.push_back(std::make_unique<Line>(Point(s[0], s[1], s[2]), Point(s[3], s[4], s[5]), s[6], s[7],
                                                     s[8], s[9], -1));
            m_lines.back()->SetTransform(Transform());
            m_primitives.push_back(std::make_unique<Primitive>(nullptr, &g_opaque, m_lines.back().get()));
        }
    }
    void Serialize(IStreamBase&) override {}
    void ApplyTransform(const Transform&) override {}

private:
    std::vector<std::unique_ptr<Line>> m_lines;
};

// Area-light shapes as the accelerator sees them: one Quad or Disk with its
// Transform per primitive (entity/light_entity.cpp:112-154 makes one per
// light; the light itself plays no part in intersection).
// Record per shape, 35 floats: kind (int bits; 0 quad, 1 disk), size x, size y
// (a disk's radius in size x), matrix[16], inverse[16] (row-major).
class HarnessShapes : public Visual {
public:
    void Fill(const float* rec, int n) {
        for (int i = 0; i < n; ++i) {
            const float* r = rec + (size_t)i * 35;
            int32_t kind;
            std::memcpy(&kind, r, 4);
            const Transform xf(Matrix(r + 3), Matrix(r + 19));
            std::unique_ptr<Shape> shape;
            if (kind == 1) {
                auto d = std::make_unique<Disk>();
                d->SetRadius(r[1]);
                shape = std::move(d);
            } else {
                auto q = std::make_unique<Quad>();
                q->SetSizeX(r[1]);
                q->SetSizeY(r[2]);
                shape = std::move(q);
            }
            shape->SetTransform(xf);
            m_primitives.push_back(std::make_unique<Primitive>(nullptr, &g_opaque, shape.get()));
            m_shapes.push_back(std::move(shape));
        }
    }
    void Add(std::unique_ptr<Shape> shape) {
        m_primitives.push_back(std::make_unique<Primitive>(nullptr, &g_opaque, shape.get()));
        m_shapes.push_back(std::move(shape));
    }
    void Serialize(IStreamBase&) override {}
    void ApplyTransform(const Transform&) override {}

private:
    std::vector<std::unique_ptr<Shape>> m_shapes;
};

class HarnessEntity : public Entity {
public:
    void Serialize(IStreamBase&) override {}
    HarnessVisual* AddVisual() {
        auto v = std::make_unique<HarnessVisual>();
        HarnessVisual* raw = v.get();
        m_visuals.push_back(std::move(v));
        return raw;
    }
    void Push(std::unique_ptr<Visual> v) { m_visuals.push_back(std::move(v)); }
    HarnessHair* AddHair() {
        auto v = std::make_unique<HarnessHair>();
        HarnessHair* raw = v.get();
        m_visuals.push_back(std::move(v));
        return raw;
    }
    HarnessShapes* AddShapes() {
        auto v = std::make_unique<HarnessShapes>();
        HarnessShapes* raw = v.get();
        m_visuals.push_back(std::move(v));
        return raw;
    }
};

struct RefScene {
    Scene scene;
    int width = 4;
    std::unordered_map<const Primitive*, int32_t> index_of;
    std::vector<const Primitive*> prims;
    std::vector<std::unique_ptr<TaggedMaterial>> materials;
    double build_seconds = 0.0;  // Accelerator::Build alone
};

}  // namespace

// ---------------------------------------------------------------------------------
// Scene members SORT's accelerator calls (restated from core/scene.cpp:43-80).

ScenePrimitiveIterator::ScenePrimitiveIterator(const Scene& scene) : m_scene(scene) { Reset(); }

void ScenePrimitiveIterator::Reset() {
    m_indices[0] = 0;
    m_indices[1] = 0;
    m_indices[2] = -1;
}

const Primitive* ScenePrimitiveIterator::Next() {
    int eid = m_indices[0], vid = m_indices[1], pid = m_indices[2] + 1;
    while (eid < (int)m_scene.m_entities.size()) {
        m_indices[0] = eid;
        const auto entity = m_scene.m_entities[eid].get();
        while (vid < (int)entity->m_visuals.size()) {
            m_indices[1] = vid;
            const auto visual = entity->m_visuals[vid].get();
            if (pid < (int)visual->m_primitives.size()) {
                m_indices[2] = pid;
                return visual->m_primitives[pid].get();
            }
            pid = 0;
            ++vid;
        }
        vid = 0;
        ++eid;
    }
    m_indices[0] = eid;
    return nullptr;
}

unsigned Scene::GetPrimitiveCount() const {
    unsigned cnt = 0;
    for (const auto& e : m_entities) cnt += e->GetPrimitiveCount();
    return cnt;
}

HarnessAccelFactory g_harness_accel_factory = nullptr;

Accelerator* harness_make_accel(int width, unsigned max_depth, unsigned max_leaf) {
    if (g_harness_accel_factory) return g_harness_accel_factory(width, max_depth, max_leaf);
    return width == 4 ? harness_make_qbvh(max_depth, max_leaf) : harness_make_obvh(max_depth, max_leaf);
}

// Symbols referenced from linked SORT objects on paths the harness never reaches.
Spectrum EvaluateTransparency(Tsl_Namespace::ShaderInstance*, const SurfaceInteraction&) { return 0.0f; }

// ---------------------------------------------------------------------------------
// Topology export: pre-order walk of SORT's tree.
//   interior node: [child_cnt, child0 ..., child_{n-1} ...]
//   leaf:          [0, pri_cnt, prim indices in SIMD-lane packing order]

namespace {

template <class Fn>
void parallel_chunks(int64_t n, int nthreads, Fn&& fn) {
    if (nthreads <= 0) nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
    std::atomic<int64_t> next{0};
    const int64_t chunk = 4096;
    auto worker = [&]() {
        RenderContext rc;
        rc.Init();
        for (;;) {
            const int64_t s = next.fetch_add(chunk);
            if (s >= n) break;
            const int64_t e = std::min(n, s + chunk);
            for (int64_t i = s; i < e; ++i) fn(rc, i);
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nthreads; ++t) pool.emplace_back(worker);
    worker();
    for (auto& th : pool) th.join();
}

}  // namespace

extern "C" {

// Build SORT's QBVH (width 4) or OBVH (width 8) over ntri triangles given as
// 9 floats each (v0, v1, v2). max_depth / max_leaf are Fbvh's m_maxNodeDepth /
// m_maxPriInLeaf (accel/fast_bvh.h:176-181, read from the scene stream in SORT).
static void* make_ref_scene(int width, const float* tri, int ntri, const float* lines, int nlines,
                            const int32_t* mat_of_tri, int nmat, const int32_t* transparent, const float* rgb,
                            int max_depth, int max_leaf) {
    if ((width != 4 && width != 8) || ntri < 0 || nmat < 0 || nlines < 0) return nullptr;
    auto* rs = new RefScene();
    rs->width = width;
    std::vector<MaterialBase*> mats;
    if (mat_of_tri) {
        for (int k = 0; k < nmat; ++k) {
            const bool tr = transparent && transparent[k];
            const Spectrum c = rgb ? Spectrum(rgb[3 * k], rgb[3 * k + 1], rgb[3 * k + 2]) : Spectrum(0.0f);
            rs->materials.push_back(std::make_unique<TaggedMaterial>(kMaterialIdBase + k, tr, c));
        }
        mats.resize((size_t)ntri);
        for (int i = 0; i < ntri; ++i) {
            if (mat_of_tri[i] < 0 || mat_of_tri[i] >= nmat) {
                delete rs;
                return nullptr;
            }
            mats[(size_t)i] = rs->materials[(size_t)mat_of_tri[i]].get();
        }
    }
    auto entity = std::make_unique<HarnessEntity>();
    HarnessVisual* visual = entity->AddVisual();
    visual->Fill(tri, ntri, mat_of_tri ? mats.data() : nullptr);
    if (nlines > 0) entity->AddHair()->Fill(lines, nlines);
    rs->scene.m_entities.push_back(std::move(entity));

    ScenePrimitiveIterator iter(rs->scene);
    int32_t idx = 0;
    while (auto p = iter.Next()) {
        rs->index_of[p] = idx++;
        rs->prims.push_back(p);
        rs->scene.m_bbox.Union(p->GetBBox());
    }
    // core/scene.cpp:150-154
    static const auto threshold = 0.001f;
    auto delta = (rs->scene.m_bbox.m_Max - rs->scene.m_bbox.m_Min) * threshold;
    rs->scene.m_bbox.m_Min -= delta;
    rs->scene.m_bbox.m_Max += delta;

    rs->scene.m_accelerator.reset(harness_make_accel(width, (unsigned)max_depth, (unsigned)max_leaf));
    const auto t0 = std::chrono::steady_clock::now();
    rs->scene.m_accelerator->Build(rs->scene);
    rs->build_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return rs;
}

// Triangles (9 floats each), hair segments (10 floats: p0, p1, v0, v1, w0, w1)
// and area shapes (35-float records, see HarnessShapes): primitive ids in that
// order. `order` (or NULL: increasing ids) lists the ids in the order the
// scene presents them: each run of one kind is one entity, so SORT's
// ScenePrimitiveIterator (core/scene.cpp:43-80) visits the primitives in that
// order and Accelerator::Build sees them so. NULL on a bad argument.
void* sortref_scene_create_shapes(int width, const float* tri, int ntri, const float* lines, int nlines,
                                  const float* shapes, int nshapes, const int32_t* order, int max_depth,
                                  int max_leaf) {
    if ((width != 4 && width != 8) || ntri < 0 || nlines < 0 || nshapes < 0) return nullptr;
    const int nall = ntri + nlines + nshapes;
    std::vector<int32_t> ord((size_t)nall);
    std::vector<uint8_t> seen((size_t)nall, 0);
    for (int k = 0; k < nall; ++k) {
        const int32_t id = order ? order[k] : k;
        if (id < 0 || id >= nall || seen[(size_t)id]) return nullptr;
        seen[(size_t)id] = 1;
        ord[(size_t)k] = id;
    }
    auto kind_of = [&](int32_t id) { return id < ntri ? 0 : (id < ntri + nlines ? 1 : 2); };
    auto* rs = new RefScene();
    rs->width = width;
    for (int k = 0; k < nall;) {
        const int kind = kind_of(ord[(size_t)k]);
        int e = k;
        while (e < nall && kind_of(ord[(size_t)e]) == kind) ++e;
        std::vector<float> buf;
        const int per = kind == 0 ? 9 : (kind == 1 ? 10 : 35);
        const float* src = kind == 0 ? tri : (kind == 1 ? lines : shapes);
        const int first = kind == 0 ? 0 : (kind == 1 ? ntri : ntri + nlines);
        for (int i = k; i < e; ++i) {
            const float* x = src + (size_t)(ord[(size_t)i] - first) * per;
            buf.insert(buf.end(), x, x + per);
        }
        auto entity = std::make_unique<HarnessEntity>();
        if (kind == 0)
            entity->AddVisual()->Fill(buf.data(), e - k);
        else if (kind == 1)
            entity->AddHair()->Fill(buf.data(), e - k);
        else
            entity->AddShapes()->Fill(buf.data(), e - k);
        rs->scene.m_entities.push_back(std::move(entity));
        k = e;
    }
    ScenePrimitiveIterator iter(rs->scene);
    rs->prims.assign((size_t)nall, nullptr);
    int32_t pos = 0;
    while (auto p = iter.Next()) {
        const int32_t id = ord[(size_t)pos++];
        rs->index_of[p] = id;
        rs->prims[(size_t)id] = p;
        rs->scene.m_bbox.Union(p->GetBBox());
    }
    // core/scene.cpp:150-154
    static const auto threshold = 0.001f;
    auto delta = (rs->scene.m_bbox.m_Max - rs->scene.m_bbox.m_Min) * threshold;
    rs->scene.m_bbox.m_Min -= delta;
    rs->scene.m_bbox.m_Max += delta;
    rs->scene.m_accelerator.reset(harness_make_accel(width, (unsigned)max_depth, (unsigned)max_leaf));
    const auto t0 = std::chrono::steady_clock::now();
    rs->scene.m_accelerator->Build(rs->scene);
    rs->build_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return rs;
}

// An area light's shape as AreaLightEntity::Serialize makes it
// (entity/light_entity.cpp:97-150), with SORT's own arithmetic: the inverse
// by Matrix::Inverse (what reading a Transform does), the scale taken out by
// Matrix::operator* with Scale(). shape: 0 SQUARE (a), 1 RECTANGLE (a, b),
// 2 DISK (radius a). out: the 35-word record of HarnessShapes (kind, sizes
// as the shape holds them after SetSizeX / SetSizeY / SetRadius, matrix,
// inverse).
void sortref_light_shape(const float* m16, int shape, float a, float b, float* out) {
    Transform xf;
    xf.matrix = Matrix(m16);
    xf.matrix.Inverse(xf.invMatrix);
    const auto sx = Vector(xf.matrix.m[0], xf.matrix.m[4], xf.matrix.m[8]).Length();
    const auto sy = Vector(xf.matrix.m[1], xf.matrix.m[5], xf.matrix.m[9]).Length();
    const auto sz = Vector(xf.matrix.m[2], xf.matrix.m[6], xf.matrix.m[10]).Length();
    const auto mat = xf.matrix * Scale(1 / sx, 1 / sy, 1 / sz).matrix;
    const auto inv_mat = Scale(sx, sy, sz).matrix * xf.invMatrix;
    int32_t kind = shape == 2 ? 1 : 0;
    std::memcpy(out, &kind, 4);
    if (shape == 2) {
        Disk d;
        d.SetRadius(a);
        out[1] = a;
        out[2] = 0.0f;
    } else {
        Quad q;
        q.SetSizeX(a);
        q.SetSizeY(shape == 0 ? a : b);
        out[1] = q.sizeX;
        out[2] = q.sizeY;
    }
    for (int k = 0; k < 16; ++k) {
        out[3 + k] = mat.m[k];
        out[19 + k] = inv_mat.m[k];
    }
}

double sortref_build_seconds(void* h) { return ((RefScene*)h)->build_seconds; }

void* sortref_scene_create_transparent(int width, const float* tri, int ntri, const int32_t* mat_of_tri, int nmat,
                                       const int32_t* transparent, const float* rgb, int max_depth, int max_leaf) {
    return make_ref_scene(width, tri, ntri, nullptr, 0, mat_of_tri, nmat, transparent, rgb, max_depth, max_leaf);
}

// The entity section of a SORT scene stream, from byte `offset` (its
// "verification bits"), read with SORT's own IFileStream and visuals: each
// VisualEntity's transform (VisualEntity::Serialize, entity/visual_entity.h:
// 31-43) with its MeshVisual / HairVisual Serialize and ApplyTransform
// (entity/visual.cpp). Cameras and lights are read past with their fields
// (entity/camera_entity.cpp:21-33, entity/light_entity.cpp:25-150). Then the
// accelerator of the given width over the primitives in SORT's order.
void* sortref_scene_from_stream(const char* path, int64_t offset, int width, int max_depth, int max_leaf) {
    if (width != 4 && width != 8) return nullptr;
    IFileStream file(path);
    IStreamBase& stream = file;  // the composite readers (StringID, Point, Transform) live on the base
    std::vector<char> skip((size_t)offset);
    if (offset > 0) stream.Load(skip.data(), (int)offset);
    StringID check;
    stream >> check;
    if (!(check == StringID("verification bits"))) return nullptr;
    auto* rs = new RefScene();
    rs->width = width;
    auto entity = std::make_unique<HarnessEntity>();
    for (;;) {
        StringID cls;
        stream >> cls;
        if (cls == StringID("End of Entities")) break;
        if (cls == StringID("VisualEntity")) {
            Transform xf;
            stream >> xf;
            unsigned cnt = 0;
            stream >> cnt;
            while (cnt-- > 0) {
                StringID vc;
                stream >> vc;
                std::unique_ptr<Visual> v;
                if (vc == StringID("MeshVisual"))
                    v = std::make_unique<MeshVisual>();
                else if (vc == StringID("HairVisual"))
                    v = std::make_unique<HairVisual>();
                else {
                    delete rs;
                    return nullptr;
                }
                v->Serialize(stream);
                v->ApplyTransform(xf);
                entity->Push(std::move(v));
            }
        } else if (cls == StringID("PerspectiveCameraEntity")) {
            Point eye, target;
            Vector up;
            unsigned w, h;
            float lens, sw, sh, arw, arh, fov;
            int fit;
            stream >> eye >> up >> target >> w >> h >> lens >> sw >> sh >> fit >> arw >> arh >> fov;
        } else if (cls == StringID("AreaLightEntity")) {
            // AreaLightEntity::Serialize's steps (entity/light_entity.cpp:97-154)
            // with SORT's own arithmetic: the Transform read (its inverse by
            // Matrix::Inverse), the scale taken out by Matrix::operator* with
            // Scale(), and the shape SORT makes, as one primitive.
            Transform xf;
            float energy;
            Spectrum in;
            StringID shape;
            stream >> xf >> energy >> in >> shape;
            const auto sx = Vector(xf.matrix.m[0], xf.matrix.m[4], xf.matrix.m[8]).Length();
            const auto sy = Vector(xf.matrix.m[1], xf.matrix.m[5], xf.matrix.m[9]).Length();
            const auto sz = Vector(xf.matrix.m[2], xf.matrix.m[6], xf.matrix.m[10]).Length();
            const auto mat = xf.matrix * Scale(1 / sx, 1 / sy, 1 / sz).matrix;
            const auto inv_mat = Scale(sx, sy, sz).matrix * xf.invMatrix;
            const Transform l2w(mat, inv_mat);
            std::unique_ptr<Shape> sh;
            float a = 0.0f, b = 0.0f;
            if (shape == StringID("RECTANGLE")) {
                stream >> a >> b;
                auto q = std::make_unique<Quad>();
                q->SetSizeX(a);
                q->SetSizeY(b);
                sh = std::move(q);
            } else if (shape == StringID("SQUARE")) {
                stream >> a;
                auto q = std::make_unique<Quad>();
                q->SetSizeX(a);
                q->SetSizeY(a);
                sh = std::move(q);
            } else {
                stream >> a;
                auto d = std::make_unique<Disk>();
                d->SetRadius(a);
                sh = std::move(d);
            }
            sh->SetTransform(l2w);
            auto v = std::make_unique<HarnessShapes>();
            v->Add(std::move(sh));
            entity->Push(std::move(v));
        } else if (cls == StringID("PointLightEntity") || cls == StringID("DirLightEntity") ||
                   cls == StringID("SpotLightEntity")) {
            Transform xf;
            float energy;
            Spectrum in;
            stream >> xf >> energy >> in;
            if (cls == StringID("SpotLightEntity")) {
                float a, b;
                stream >> a >> b;
            }
        } else if (cls == StringID("SkyLightEntity")) {
            Transform xf;
            float intensity;
            Spectrum color;
            std::string file;
            stream >> xf >> intensity >> color >> file;
        } else {
            delete rs;
            return nullptr;
        }
    }
    rs->scene.m_entities.push_back(std::move(entity));
    ScenePrimitiveIterator iter(rs->scene);
    int32_t idx = 0;
    while (auto p = iter.Next()) {
        rs->index_of[p] = idx++;
        rs->prims.push_back(p);
        rs->scene.m_bbox.Union(p->GetBBox());
    }
    static const auto threshold = 0.001f;  // core/scene.cpp:150-154
    auto delta = (rs->scene.m_bbox.m_Max - rs->scene.m_bbox.m_Min) * threshold;
    rs->scene.m_bbox.m_Min -= delta;
    rs->scene.m_bbox.m_Max += delta;
    rs->scene.m_accelerator.reset(harness_make_accel(width, (unsigned)max_depth, (unsigned)max_leaf));
    rs->scene.m_accelerator->Build(rs->scene);
    return rs;
}

// Triangles followed by hair segments (10 floats each: p0, p1, v0, v1, w0, w1),
// all opaque; primitive order: the triangles, then the lines.
void* sortref_scene_create_hair(int width, const float* tri, int ntri, const float* lines, int nlines, int max_depth,
                                int max_leaf) {
    return make_ref_scene(width, tri, ntri, lines, nlines, nullptr, 0, nullptr, nullptr, max_depth, max_leaf);
}

void* sortref_scene_create_mat(int width, const float* tri, int ntri, const int32_t* mat_of_tri, int nmat,
                               int max_depth, int max_leaf) {
    return sortref_scene_create_transparent(width, tri, ntri, mat_of_tri, nmat, nullptr, nullptr, max_depth,
                                            max_leaf);
}

void* sortref_scene_create(int width, const float* tri, int ntri, int max_depth, int max_leaf) {
    return sortref_scene_create_mat(width, tri, ntri, nullptr, 0, max_depth, max_leaf);
}

// BSSRDF probe query through Scene::GetIntersect(const Ray&, BSSRDFIntersections&,
// RenderContext&, StringID) (core/scene.cpp:221-225): up to
// TOTAL_SSS_INTERSECTION_CNT (4) hits on primitives of material ray_mat[i], in
// the slots SORT leaves them in. count[i] = hits kept; per ray 4 entries of
// prim / t / u / v at [4 * i + k], entries past count are prim -1, t FLT_MAX.
void sortref_trace_multi(void* h, const float* rays, int64_t n, const int32_t* ray_mat, int32_t* count,
                         int32_t* prim, float* t, float* u, float* v, int nthreads) {
    RefScene* rs = (RefScene*)h;
    const bool valid = rs->scene.m_accelerator->GetIsValid();
    parallel_chunks(n, nthreads, [&](RenderContext& rc, int64_t i) {
        Ray r(Point(rays[i], rays[n + i], rays[2 * n + i]), Vector(rays[3 * n + i], rays[4 * n + i], rays[5 * n + i]), 0,
              rays[6 * n + i], rays[7 * n + i]);
        BSSRDFIntersections inter;  // what Scene::GetIntersect forwards to the accelerator
        if (valid)
            rs->scene.m_accelerator->GetIntersect(r, inter, rc, StringID(kMaterialIdBase + (sid_t)ray_mat[i]));
        count[i] = (int32_t)inter.cnt;
        for (unsigned k = 0; k < TOTAL_SSS_INTERSECTION_CNT; ++k) {
            const int64_t o = 4 * i + k;
            if (k < inter.cnt) {
                const SurfaceInteraction& s = inter.intersections[k]->intersection;
                prim[o] = rs->index_of.at(s.primitive);
                t[o] = s.t;
                u[o] = s.u;
                v[o] = s.v;
            } else {
                prim[o] = -1;
                t[o] = FLT_MAX;
                u[o] = v[o] = 0.0f;
            }
        }
        rc.m_memory_arena->Reset();
    });
}

void sortref_scene_destroy(void* h) { delete (RefScene*)h; }

int sortref_is_valid(void* h) { return ((RefScene*)h)->scene.m_accelerator->GetIsValid() ? 1 : 0; }

// Scene box after the 0.1% enlargement: min xyz, max xyz.
void sortref_scene_bbox(void* h, float* out6) {
    const BBox& b = ((RefScene*)h)->scene.m_bbox;
    for (int k = 0; k < 3; ++k) {
        out6[k] = b.m_Min[k];
        out6[3 + k] = b.m_Max[k];
    }
}

// Tree depth SORT recorded (Fbvh::m_depth).
int sortref_depth(void* h) {
    RefScene* rs = (RefScene*)h;
    if (g_harness_accel_factory) return -1;  // not SORT's Fbvh: no tree to walk
    if (rs->width == 4) return (int)harness_qbvh_depth(rs->scene.m_accelerator.get());
    return (int)harness_obvh_depth(rs->scene.m_accelerator.get());
}

// Pre-order topology stream (format above). Returns the number of int32 written,
// or the required size (negated) if cap is too small.
int64_t sortref_topology(void* h, int32_t* out, int64_t cap) {
    RefScene* rs = (RefScene*)h;
    std::vector<int32_t> v;
    if (g_harness_accel_factory || !rs->scene.m_accelerator->GetIsValid()) return 0;
    if (rs->width == 4)
        harness_qbvh_topology(rs->scene.m_accelerator.get(), rs->index_of, v);
    else
        harness_obvh_topology(rs->scene.m_accelerator.get(), rs->index_of, v);
    if ((int64_t)v.size() > cap) return -(int64_t)v.size();
    std::memcpy(out, v.data(), v.size() * sizeof(int32_t));
    return (int64_t)v.size();
}

// Closest hit for n rays given SoA (ox, oy, oz, dx, dy, dz, tmin, tmax; each n
// floats, packed one after the other). Follows Scene::GetIntersect
// (core/scene.cpp:182-185): t is reset to FLT_MAX, then the accelerator runs.
// Miss: prim = -1, t = FLT_MAX, u = v = 0.
void sortref_trace_closest(void* h, const float* rays, int64_t n, int32_t* prim, float* t, float* u, float* v,
                           int nthreads) {
    RefScene* rs = (RefScene*)h;
    const Accelerator* acc = rs->scene.m_accelerator.get();
    const bool valid = acc->GetIsValid();
    parallel_chunks(n, nthreads, [&](RenderContext& rc, int64_t i) {
        Ray r(Point(rays[i], rays[n + i], rays[2 * n + i]), Vector(rays[3 * n + i], rays[4 * n + i], rays[5 * n + i]), 0,
              rays[6 * n + i], rays[7 * n + i]);
        SurfaceInteraction inter;
        inter.t = FLT_MAX;
        const bool hit = valid && acc->GetIntersect(rc, r, inter);
        if (hit && inter.primitive) {
            prim[i] = rs->index_of.at(inter.primitive);
            t[i] = inter.t;
            u[i] = inter.u;
            v[i] = inter.v;
        } else {
            prim[i] = -1;
            t[i] = FLT_MAX;
            u[i] = 0.0f;
            v[i] = 0.0f;
        }
    });
}

// Any-hit (shadow) query through Accelerator::GetAttenuation
// (accel/accelerator.cpp:26-69), as Scene::GetAttenuation calls it: occluded = 1 when
// an opaque primitive lies in (tmin, tmax].
void sortref_trace_any(void* h, const float* rays, int64_t n, uint8_t* occluded, int nthreads) {
    RefScene* rs = (RefScene*)h;
    const Accelerator* acc = rs->scene.m_accelerator.get();
    const bool valid = acc->GetIsValid();
    parallel_chunks(n, nthreads, [&](RenderContext& rc, int64_t i) {
        Ray r(Point(rays[i], rays[n + i], rays[2 * n + i]), Vector(rays[3 * n + i], rays[4 * n + i], rays[5 * n + i]), 0,
              rays[6 * n + i], rays[7 * n + i]);
        Spectrum att(1.0f);
        bool blocked = false;
        if (valid) blocked = acc->GetAttenuation(r, att, rc, nullptr) && att.IsBlack();
        occluded[i] = blocked ? 1 : 0;
    });
}

// Scene::GetAttenuation (core/scene.cpp:192-208), restated over SORT's own
// Accelerator::GetAttenuation (accel/accelerator.cpp:26-69, no medium): rgb
// planes [0,n), [n,2n), [2n,3n).
void sortref_trace_attenuation(void* h, const float* rays, int64_t n, float* out, int nthreads) {
    RefScene* rs = (RefScene*)h;
    const Accelerator* acc = rs->scene.m_accelerator.get();
    const bool valid = acc->GetIsValid();
    parallel_chunks(n, nthreads, [&](RenderContext& rc, int64_t i) {
        Ray ray(Point(rays[i], rays[n + i], rays[2 * n + i]), Vector(rays[3 * n + i], rays[4 * n + i], rays[5 * n + i]),
                0, rays[6 * n + i], rays[7 * n + i]);
        Spectrum attenuation(1.0f);
        while (valid && !attenuation.IsBlack()) {
            Spectrum att;
            if (!acc->GetAttenuation(ray, att, rc, nullptr)) break;
            if (att.IsBlack()) {
                attenuation = att;
                break;
            }
            attenuation *= att;
        }
        out[i] = attenuation.r;
        out[n + i] = attenuation.g;
        out[2 * n + i] = attenuation.b;
    });
}

// Ray::Prepare (math/ray.h:60-69) for one direction: the major axis it picks and
// the shear constants. Exposed so the restated oracle can be pinned on it.
void sortref_ray_prepare(const float* d, int* local_xyz, float* scale_xyz) {
    Ray r(Point(0.0f), Vector(d[0], d[1], d[2]));
    r.Prepare();
    local_xyz[0] = r.m_local_x;
    local_xyz[1] = r.m_local_y;
    local_xyz[2] = r.m_local_z;
    scale_xyz[0] = r.m_scale_x;
    scale_xyz[1] = r.m_scale_y;
    scale_xyz[2] = r.m_scale_z;
}

int sortref_hardware_threads(void) { return (int)std::max(1u, std::thread::hardware_concurrency()); }

}  // extern "C"
