// Gbvh: SORT's Accelerator interface (accel/accelerator.h:55-156) answered by
// libsortgpu (include/sortgpu.h). A header a SORT build compiles in beside
// accel/qbvh.cpp and accel/obvh.cpp; it registers itself as "Gbvh", so a
// scene stream that names that accelerator class gets it
// (core/scene.cpp:163-177).
//
// What SORT needs to change to build it: Quad::sizeX/sizeY, Disk::radius,
// Shape::m_transform and Line's end points, widths and v (all protected or
// private in shape/*.h) must be readable here, for instance with
// `friend class Gbvh;` in Shape and Line.
//
// The tree is SORT's: the primitives are handed over in ScenePrimitiveIterator
// order (with sg_shapes.order), so the GPU builds the tree Fbvh::Build builds,
// and every query returns the primitive SORT's Obvh / Qbvh returns. The
// per-ray interface (GetIntersect) makes one library call per ray: it works,
// and it is how SORT's own integrators drive it, but one ray per call cannot
// keep a GPU busy; the batch calls at the end are the throughput path.
#pragma once

#include <cfloat>
#include <memory>
#include <unordered_map>
#include <vector>

#include "accel/accelerator.h"
#include "core/primitive.h"
#include "core/scene.h"
#include "entity/visual.h"
#include "material/material.h"
#include "math/interaction.h"
#include "scatteringevent/bssrdf/bssrdf.h"
#include "shape/disk.h"
#include "shape/line.h"
#include "shape/quad.h"
#include "shape/triangle.h"
#include "sortgpu.h"

class Gbvh : public Accelerator {
public:
    DEFINE_RTTI(Gbvh, Accelerator);

    Gbvh() = default;
    explicit Gbvh(int width, unsigned max_depth = 16, unsigned max_leaf = 8)
        : m_width(width == 4 ? 4 : 8), m_maxNodeDepth(max_depth), m_maxPriInLeaf(max_leaf) {}

    ~Gbvh() override {
        if (m_gpu) sg_scene_destroy(m_gpu);
    }

    // Fbvh::Serialize reads the same two parameters (accel/fast_bvh.h:159-162).
    void Serialize(IStreamBase& stream) override {
        stream >> m_maxNodeDepth;
        stream >> m_maxPriInLeaf;
    }

    // Every primitive of the scene, by kind, in the order SORT's iterator
    // gives them: triangles (world-space vertices of their mesh), hair lines
    // (their world-space end points, v and widths), area-light Quads and Disks
    // (size and Transform). Hit indices map back through m_prims.
    void Build(const Scene& scene) override {
        m_bbox = scene.GetBBox();
        std::vector<float> tri, lines;
        std::vector<sg_area_shape> shapes;
        std::vector<const Primitive*> by_kind[3];
        std::vector<std::pair<int, int32_t>> seq;  // (kind, index within kind) in iterator order
        ScenePrimitiveIterator iter(scene);
        while (const Primitive* p = iter.Next()) {
            const Shape* shape = p->GetShape();
            if (const auto* t = dynamic_cast<const Triangle*>(shape)) {
                const auto& mem = t->m_meshVisual->m_memory;
                for (int k = 0; k < 3; ++k) {
                    const Point& v = mem->m_vertices[t->m_index.m_id[k]].m_position;
                    tri.insert(tri.end(), {v.x, v.y, v.z});
                }
                seq.emplace_back(0, int32_t(by_kind[0].size()));
                by_kind[0].push_back(p);
            } else if (const auto* l = dynamic_cast<const Line*>(shape)) {
                // World-space segment as Line::SetTransform left it; the library
                // derives Line's per-segment constants from it as SORT does.
                lines.insert(lines.end(), {l->m_gp0.x, l->m_gp0.y, l->m_gp0.z, l->m_gp1.x, l->m_gp1.y, l->m_gp1.z,
                                           l->m_v0, l->m_v1, l->m_w0, l->m_w1});
                seq.emplace_back(1, int32_t(by_kind[1].size()));
                by_kind[1].push_back(p);
            } else if (dynamic_cast<const Quad*>(shape) || dynamic_cast<const Disk*>(shape)) {
                sg_area_shape a{};
                if (const auto* q = dynamic_cast<const Quad*>(shape)) {
                    a.kind = SG_SHAPE_QUAD;
                    a.size[0] = q->sizeX;
                    a.size[1] = q->sizeY;
                } else {
                    a.kind = SG_SHAPE_DISK;
                    a.size[0] = static_cast<const Disk*>(shape)->radius;
                }
                for (int k = 0; k < 16; ++k) {
                    a.matrix[k] = shape->m_transform.matrix.m[k];
                    a.inverse[k] = shape->m_transform.invMatrix.m[k];
                }
                shapes.push_back(a);
                seq.emplace_back(2, int32_t(by_kind[2].size()));
                by_kind[2].push_back(p);
            } else {
                m_unsupported = true;  // another shape kind: this accelerator does not take the scene
            }
        }
        // Library indices: triangles, then lines, then shapes.
        const int32_t base[3] = {0, int32_t(by_kind[0].size()), int32_t(by_kind[0].size() + by_kind[1].size())};
        m_prims.clear();
        for (const auto& v : by_kind) m_prims.insert(m_prims.end(), v.begin(), v.end());
        std::vector<int32_t> order;
        for (const auto& e : seq) order.push_back(base[e.first] + e.second);
        m_first_line = base[1];
        m_first_shape = base[2];

        sg_build_opts opts;
        sg_default_build_opts(&opts);
        opts.width = m_width;
        opts.max_depth = (int32_t)m_maxNodeDepth;
        opts.max_leaf = (int32_t)m_maxPriInLeaf;
        const sg_shapes in{tri.data(), (int64_t)by_kind[0].size(), lines.data(), (int64_t)by_kind[1].size(),
                           shapes.data(), (int64_t)shapes.size(), order.data()};
        m_isValid = !m_unsupported && !m_prims.empty() && sg_scene_create_shapes(&in, &opts, &m_gpu) == SG_OK;
        if (!m_isValid || !by_kind[1].empty() || !by_kind[2].empty()) return;
        // Material of every triangle, as a small index, for the BSSRDF query
        // and the transparent-shadow batch (triangle scenes only).
        std::vector<int32_t> mats;
        for (const Primitive* p : m_prims) {
            const sid_t sid = p->GetMaterial()->GetUniqueID().m_sid;
            mats.push_back(m_matIndex.emplace(sid, (int32_t)m_matIndex.size()).first->second);
        }
        m_isValid = sg_scene_set_materials(m_gpu, mats.data(), (int64_t)mats.size()) == SG_OK;
        // The transparency of each material, taken as a constant per material.
        m_transparency.assign(m_matIndex.size(), sg_transparency{0, {0.0f, 0.0f, 0.0f}});
        for (const Primitive* p : m_prims) {
            const MaterialBase* m = p->GetMaterial();
            sg_transparency& tr = m_transparency[(size_t)m_matIndex.at(m->GetUniqueID().m_sid)];
            tr.transparent = m->HasTransparency() ? 1 : 0;
            if (tr.transparent) {
                const Spectrum c = m->EvaluateTransparency(SurfaceInteraction());
                tr.rgb[0] = c.r;
                tr.rgb[1] = c.g;
                tr.rgb[2] = c.b;
            }
        }
    }

    // Accelerator::GetIntersect (accel/accelerator.h:74), one ray per call.
    // query_shadow: the any-hit query, answered as SORT's opaque early exit
    // answers it (primitive = nullptr and true when blocked,
    // accel/fast_bvh.hpp:362-373): correct for opaque scenes; scenes with
    // transparent materials take GetAttenuationBatch instead of SORT's loop.
    // Closest hit: a triangle's interaction is filled from the GPU's t, u, v
    // as SORT's SIMD path fills it (setupIntersection, simd/simd_triangle.h:
    // 311-341), so it is SORT's bit for bit. A line or an area shape fills it
    // with SORT's own shape test at the GPU's distance (what Fbvh runs for an
    // other_list primitive); a shape hit then keeps u, v as the caller's
    // interaction had them, where SORT keeps those of the hit it replaced.
    bool GetIntersect(RenderContext& rc, const Ray& r, SurfaceInteraction& intersect) const override {
        (void)rc;
        if (!m_isValid) return false;
        const float rays8[8] = {r.m_Ori.x, r.m_Ori.y, r.m_Ori.z, r.m_Dir.x, r.m_Dir.y, r.m_Dir.z, r.m_fMin, r.m_fMax};
        if (intersect.query_shadow) {
            uint8_t occluded = 0;
            if (sg_trace_any_host(m_gpu, rays8, 1, &occluded) != SG_OK || !occluded) return false;
            intersect.primitive = nullptr;
            return true;
        }
        int32_t prim = -1;
        float t = FLT_MAX, u = 0.0f, v = 0.0f;
        if (sg_trace_closest_host(m_gpu, rays8, 1, &prim, &t, &u, &v) != SG_OK || prim < 0) return false;
        return fill(prim, r, t, u, v, &intersect);
    }

    // BSSRDF probe query (accel/accelerator.h:122): up to 4 hits on primitives
    // of material matID, the same hits in the same slots as Fbvh keeps them
    // (triangle scenes).
    void GetIntersect(const Ray& r, BSSRDFIntersections& intersect, RenderContext& rc,
                      const StringID matID) const override {
        intersect.cnt = 0;
        intersect.maxt = FLT_MAX;
        const auto it = m_matIndex.find(matID.m_sid);
        if (!m_isValid || it == m_matIndex.end()) return;
        const float rays8[8] = {r.m_Ori.x, r.m_Ori.y, r.m_Ori.z, r.m_Dir.x, r.m_Dir.y, r.m_Dir.z, r.m_fMin, r.m_fMax};
        int32_t count = 0, prim[4];
        float t[4], u[4], v[4];
        if (sg_trace_multi_host(m_gpu, rays8, 1, &it->second, &count, prim, t, u, v) != SG_OK) return;
        for (int32_t k = 0; k < count; ++k) {
            auto* hit = SORT_MALLOC(rc.m_memory_arena, BSSRDFIntersection)();
            fill(prim[k], r, t[k], u[k], v[k], &hit->intersection);
            intersect.intersections[intersect.cnt++] = hit;
        }
    }

    // Batch extension the wavefront integrator calls: rays8 = ox[n] oy[n] oz[n]
    // dx[n] dy[n] dz[n] tmin[n] tmax[n]; prim[i] indexes PrimitiveAt (or -1).
    sg_status GetIntersectBatch(const float* rays8, int64_t n, int32_t* prim, float* t, float* u, float* v) const {
        return sg_trace_closest_host(m_gpu, rays8, n, prim, t, u, v);
    }
    sg_status GetOcclusionBatch(const float* rays8, int64_t n, uint8_t* occluded) const {
        return sg_trace_any_host(m_gpu, rays8, n, occluded);
    }
    // Scene::GetAttenuation's whole loop for a batch (core/scene.cpp:192-208):
    // rgb = r[n] g[n] b[n] (triangle scenes).
    sg_status GetAttenuationBatch(const float* rays8, int64_t n, float* rgb) const {
        return sg_trace_attenuation_host(m_gpu, rays8, n, m_transparency.data(), (int32_t)m_transparency.size(), rgb);
    }
    const Primitive* PrimitiveAt(int32_t i) const { return m_prims[(size_t)i]; }

    std::unique_ptr<Accelerator> Clone() const override {
        return std::make_unique<Gbvh>(m_width, m_maxNodeDepth, m_maxPriInLeaf);
    }

private:
    // The interaction of primitive `prim` hit at t (u, v: barycentric weights
    // of vertices 1 and 2 for a triangle).
    bool fill(int32_t prim, const Ray& r, float t, float u, float v, SurfaceInteraction* out) const {
        const Primitive* p = m_prims[(size_t)prim];
        if (prim < m_first_line) {
            // setupIntersection (simd/simd_triangle.h:311-341), term for term.
            const auto* tri = static_cast<const Triangle*>(p->GetShape());
            const auto w = 1 - u - v;
            const auto& mem = tri->m_meshVisual->m_memory;
            const auto& mv0 = mem->m_vertices[tri->m_index.m_id[0]];
            const auto& mv1 = mem->m_vertices[tri->m_index.m_id[1]];
            const auto& mv2 = mem->m_vertices[tri->m_index.m_id[2]];
            out->intersect = r(t);
            out->t = t;
            out->gnormal = normalize(cross((mv2.m_position - mv0.m_position), (mv1.m_position - mv0.m_position)));
            out->normal = (w * mv0.m_normal + u * mv1.m_normal + v * mv2.m_normal).Normalize();
            out->tangent = (w * mv0.m_tangent + u * mv1.m_tangent + v * mv2.m_tangent).Normalize();
            out->view = -r.m_Dir;
            const auto uv = w * mv0.m_texCoord + u * mv1.m_texCoord + v * mv2.m_texCoord;
            out->u = uv.x;
            out->v = uv.y;
            out->primitive = p;
            return true;
        }
        // A shape's own test at the GPU's distance: an area shape accepts
        // t <= the interaction's t, so it finds the same hit and fills the rest.
        out->t = prim < m_first_shape ? FLT_MAX : t;
        if (p->GetIntersect(r, out)) return true;
        // The scalar line test can round differently from the SIMD one the
        // GPU follows; keep the GPU's hit with what it determines.
        out->t = t;
        out->intersect = r(t);
        out->view = -r.m_Dir;
        out->u = u;
        out->v = v;
        out->primitive = p;
        return true;
    }

    sg_scene* m_gpu = nullptr;
    int m_width = 8;
    unsigned m_maxNodeDepth = 16;
    unsigned m_maxPriInLeaf = 8;
    bool m_unsupported = false;
    int32_t m_first_line = 0, m_first_shape = 0;  // library indices where lines / area shapes start
    std::vector<const Primitive*> m_prims;        // by library index
    std::unordered_map<sid_t, int32_t> m_matIndex;
    std::vector<sg_transparency> m_transparency;  // by material index
};
