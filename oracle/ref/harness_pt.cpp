// Oracle harness, path-tracing half (TEST INFRASTRUCTURE ONLY).
//
// Runs SORT's own PathTracing::Li (integrator/pathtracing.cpp:37-258) with its
// EvaluateDirect (integrator/integratormethod.cpp:100-192), ScatteringEvent,
// Lambert, MicroFacetReflection + GGX + FresnelConductor, AreaLight and Quad —
// all compiled unmodified from SORT's sources by oracle/Makefile — over a
// harness-built scene:
//   * triangles with one material each: Lambert(albedo) or GGX conductor
//     (eta, k, roughness), added to the ScatteringEvent exactly as SORT's closures
//     do (material/closures.cpp:165-170, 252-258);
//   * one rectangular AreaLight whose Quad is also a primitive of the tree, as
//     AreaLightEntity sets it up (entity/light_entity.cpp:99-158); the quad's
//     primitive has no material, and SORT's default material makes it a white
//     Lambert surface (material/material.cpp:230-235) — given explicitly here;
//   * the Scene members the integrator calls, restated from core/scene.cpp
//     (GetIntersect, GetAttenuation, SampleLight, Le, light distribution);
//   * a pinhole camera with one uniformly jittered ray per sample.
// Every pixel re-seeds its RenderContext's Mersenne Twister from (seed, pixel)
// with the generator's standard initialisation, so a render does not depend on
// how pixels are spread over threads.
#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <queue>
#include <thread>
#include <vector>

#define private public
#define protected public
#include "core/rand.h"
#include "core/render_context.h"
#include "core/samplemethod.h"
#include "core/scene.h"
#include "entity/visual.h"
#include "integrator/pathtracing.h"
#include "light/area.h"
#include "material/material.h"
#include "math/interaction.h"
#include "sampler/sample.h"
#include "scatteringevent/bsdf/lambert.h"
#include "scatteringevent/bsdf/microfacet.h"
#include "scatteringevent/scatteringevent.h"
#include "shape/quad.h"
#undef private
#undef protected

#include "harness_width.h"

namespace {

struct MatDesc {
    int type = 0;            // 0 Lambert, 1 GGX conductor reflection
    Spectrum albedo;         // Lambert base colour
    Spectrum eta, k;         // conductor Fresnel
    float roughness = 0.5f;  // GGX, isotropic
};

class HarnessMaterial : public MaterialBase {
public:
    explicit HarnessMaterial(const MatDesc& d) : m(d) {}
    void UpdateScatteringEvent(ScatteringEvent& se, RenderContext& rc) const override {
        const Tsl_Namespace::float3 up{0.0f, 1.0f, 0.0f};
        if (m.type == 0) {
            const ClosureTypeLambert p{{m.albedo.r, m.albedo.g, m.albedo.b}, up};
            se.AddBxdf(SORT_MALLOC(rc.m_memory_arena, Lambert)(rc, p, FULL_WEIGHT));
        } else {
            const ClosureTypeMicrofacetReflectionGGX p{{m.eta.r, m.eta.g, m.eta.b},
                                                        {m.k.r, m.k.g, m.k.b},
                                                        m.roughness,
                                                        m.roughness,
                                                        {1.0f, 1.0f, 1.0f},
                                                        up};
            se.AddBxdf(SORT_MALLOC(rc.m_memory_arena, MicroFacetReflection)(rc, p, FULL_WEIGHT));
        }
    }
    void UpdateMediumStack(const MediumInteraction&, const SE_Interaction, MediumStack&, RenderContext&) const override {}
    void EvaluateMediumSample(const MediumInteraction&, MediumSample&) const override {}
    Spectrum EvaluateTransparency(const SurfaceInteraction&) const override { return 0.0f; }
    void BuildMaterial(Tsl_Namespace::ShadingContext*) override {}
    StringID GetUniqueID() const override { return StringID(2u); }
    bool HasTransparency() const override { return false; }
    bool HasSSS() const override { return false; }
    bool HasVolumeAttached() const override { return false; }
    float GetVolumeStep() const override { return 0.0f; }
    unsigned int GetVolumeStepCnt() const override { return 0; }
    void Serialize(IStreamBase&) override {}

private:
    MatDesc m;
};

Vector any_perpendicular(const Vector& n) {
    const Vector a = std::fabs(n.x) > 0.9f ? Vector(0.0f, 1.0f, 0.0f) : Vector(1.0f, 0.0f, 0.0f);
    return normalize(cross(a, n));
}

class PtVisual : public MeshVisual {
public:
    void Fill(const float* tri, int ntri, const int32_t* mat_of_tri, const std::vector<std::unique_ptr<HarnessMaterial>>& mats) {
        m_memory = std::make_unique<Mesh>();
        m_memory->m_vertices.resize((size_t)ntri * 3);
        m_memory->m_indices.resize((size_t)ntri);
        for (int i = 0; i < ntri; ++i) {
            const float* p = tri + (size_t)i * 9;
            Point a(p[0], p[1], p[2]), b(p[3], p[4], p[5]), c(p[6], p[7], p[8]);
            Vector n = cross(c - a, b - a);  // SORT's geometric normal (simd_triangle.h:331)
            const float len = n.Length();
            n = len > 0.0f ? n / len : Vector(0.0f, 1.0f, 0.0f);
            const Vector tg = any_perpendicular(n);
            const Point pts[3] = {a, b, c};
            for (int k = 0; k < 3; ++k) {
                MeshVertex& mv = m_memory->m_vertices[(size_t)i * 3 + k];
                mv.m_position = pts[k];
                mv.m_normal = n;  // flat shading: shading normal = geometric normal
                mv.m_tangent = tg;
                mv.m_texCoord = Vector2f(0.0f, 0.0f);
            }
            MeshFaceIndex& fi = m_memory->m_indices[(size_t)i];
            fi.m_id[0] = i * 3;
            fi.m_id[1] = i * 3 + 1;
            fi.m_id[2] = i * 3 + 2;
            fi.m_mat = mats[(size_t)mat_of_tri[i]].get();
        }
        m_memory->m_hasUV = true;
        for (const auto& mi : m_memory->m_indices) {
            m_triangles.push_back(std::make_unique<Triangle>(this, mi));
            m_primitives.push_back(std::make_unique<Primitive>(m_memory.get(), mi.m_mat, m_triangles.back().get()));
        }
    }
};

class PtEntity : public Entity {
public:
    void Serialize(IStreamBase&) override {}
    void Add(std::unique_ptr<Visual> v) { m_visuals.push_back(std::move(v)); }
};

struct PtScene {
    Scene scene;
    std::vector<std::unique_ptr<HarnessMaterial>> mats;
    std::unique_ptr<HarnessMaterial> light_surface;  // white Lambert
    std::unique_ptr<AreaLight> light;
    std::unique_ptr<float[]> light_power;
};

// MT19937 init_genrand (Matsumoto & Nishimura), the initialisation SORT's
// RandomNumberGenerator::init runs with its time(0) seed (core/rand.cpp:41-55).
void reseed(RenderContext& rc, uint32_t seed) {
    auto& g = *rc.m_random_num_generator;
    g.mt[0] = seed & 0xffffffffUL;
    for (g.mti = 1; g.mti < MT_CNT; g.mti++)
        g.mt[g.mti] = (1812433253UL * (g.mt[g.mti - 1] ^ (g.mt[g.mti - 1] >> 30)) + (unsigned long)g.mti) & 0xffffffffUL;
}

uint32_t mix32(uint32_t x) {  // integer hash (finaliser of MurmurHash3) to spread per-pixel seeds
    x ^= x >> 16;
    x *= 0x85ebca6bu;
    x ^= x >> 13;
    x *= 0xc2b2ae35u;
    x ^= x >> 16;
    return x;
}

}  // namespace

// ---------------------------------------------------------------------------------
// Scene members PathTracing / EvaluateDirect call (restated from core/scene.cpp).

bool Scene::GetIntersect(RenderContext& rc, const Ray& r, SurfaceInteraction& intersect) const {
    intersect.t = FLT_MAX;
    return m_accelerator->GetIntersect(rc, r, intersect);
}

Spectrum Scene::GetAttenuation(const Ray& const_ray, RenderContext& rc, MediumStack* ms) const {
    auto ray = const_ray;
    Spectrum attenuation(1.0f);
    while (!attenuation.IsBlack()) {
        Spectrum att;
        if (!m_accelerator->GetAttenuation(ray, att, rc, ms)) break;
        if (att.IsBlack()) return att;
        attenuation *= att;
    }
    return attenuation;
}

// No participating media in these scenes: the stack stays empty.
void Scene::RestoreMediumStack(const Point&, RenderContext&, MediumStack&) const {}

const Light* Scene::SampleLight(float u, float* pdf) const {
    float _pdf;
    const int id = m_lightsDis->SampleDiscrete(u, &_pdf);
    if (id >= 0 && id < (int)m_lights.size() && _pdf != 0.0f) {
        if (pdf) *pdf = _pdf;
        return m_lights[id];
    }
    return nullptr;
}

Spectrum Scene::Le(const Ray& ray) const {
    if (m_skyLight) {
        Spectrum r;
        m_skyLight->Le(ray, 0, r);
        return r;
    }
    return 0.0f;
}

extern "C" {

// mat_params: 10 floats per material: type (0 Lambert, 1 GGX conductor),
//   Lambert: albedo r g b;  GGX: eta r g b, k r g b, roughness.
// light: centre x y z, size x, size z, intensity r g b (a rectangle facing -y).
void* sortref_pt_scene_create(int width, const float* tri, int ntri, const int32_t* mat_of_tri, int nmat,
                              const float* mat_params, const float* light, int max_depth, int max_leaf) {
    if ((width != 4 && width != 8) || ntri < 0 || nmat < 1) return nullptr;
    auto* ps = new PtScene();
    for (int m = 0; m < nmat; ++m) {
        const float* q = mat_params + (size_t)m * 10;
        MatDesc d;
        d.type = (int)q[0];
        if (d.type == 0) {
            d.albedo = Spectrum(q[1], q[2], q[3]);
        } else {
            d.eta = Spectrum(q[1], q[2], q[3]);
            d.k = Spectrum(q[4], q[5], q[6]);
            d.roughness = q[7];
        }
        ps->mats.push_back(std::make_unique<HarnessMaterial>(d));
    }
    MatDesc white;
    white.type = 0;
    white.albedo = Spectrum(1.0f);
    ps->light_surface = std::make_unique<HarnessMaterial>(white);

    auto mesh_entity = std::make_unique<PtEntity>();
    auto visual = std::make_unique<PtVisual>();
    visual->Fill(tri, ntri, mat_of_tri, ps->mats);
    mesh_entity->Add(std::move(visual));
    ps->scene.m_entities.push_back(std::move(mesh_entity));

    // The area light: a Quad in the x-z plane of its local frame (normal +y),
    // placed at the centre and turned to face -y.
    ps->light = std::make_unique<AreaLight>();
    auto quad = std::make_unique<Quad>();
    quad->SetSizeX(light[3]);
    quad->SetSizeY(light[4]);
    const Matrix m(1.0f, 0.0f, 0.0f, light[0], 0.0f, -1.0f, 0.0f, light[1], 0.0f, 0.0f, -1.0f, light[2], 0.0f, 0.0f,
                   0.0f, 1.0f);
    const Matrix inv(1.0f, 0.0f, 0.0f, -light[0], 0.0f, -1.0f, 0.0f, light[1], 0.0f, 0.0f, -1.0f, light[2], 0.0f,
                     0.0f, 0.0f, 1.0f);
    const Transform xf(m, inv);
    quad->SetTransform(xf);
    ps->light->m_light2world = xf;
    ps->light->intensity = Spectrum(light[5], light[6], light[7]);
    ps->light->m_shape = std::move(quad);
    auto light_prim = std::make_unique<Primitive>(nullptr, ps->light_surface.get(), ps->light->m_shape.get(),
                                                  ps->light.get());
    auto light_entity = std::make_unique<PtEntity>();
    light_entity->Add(std::make_unique<SinglePrimitiveVisual>(std::move(light_prim)));
    ps->scene.m_entities.push_back(std::move(light_entity));
    ps->scene.m_lights.push_back(ps->light.get());
    ps->light->SetupScene(&ps->scene);
    // Scene::genLightDistribution (core/scene.cpp:227-244) for one light.
    ps->light_power = std::make_unique<float[]>(1);
    ps->light_power[0] = ps->light->Power().GetIntensity();
    ps->light->SetPickPDF(1.0f);
    ps->scene.m_lightsDis = std::make_unique<Distribution1D>(ps->light_power.get(), 1u);

    ScenePrimitiveIterator iter(ps->scene);
    while (auto p = iter.Next()) ps->scene.m_bbox.Union(p->GetBBox());
    static const auto threshold = 0.001f;
    auto delta = (ps->scene.m_bbox.m_Max - ps->scene.m_bbox.m_Min) * threshold;
    ps->scene.m_bbox.m_Min -= delta;
    ps->scene.m_bbox.m_Max += delta;
    ps->scene.m_accelerator.reset(harness_make_accel(width, (unsigned)max_depth, (unsigned)max_leaf));
    ps->scene.m_accelerator->Build(ps->scene);
    return ps;
}

void sortref_pt_scene_destroy(void* h) { delete (PtScene*)h; }

// cam: eye xyz, target xyz, up xyz, vertical field of view in degrees.
// Writes the mean radiance of spp samples per pixel, RGB, row-major from the top.
void sortref_pt_render(void* h, int max_recursive_depth, const float* cam, int width, int height, int spp,
                       uint32_t seed, float* out_rgb, int nthreads) {
    PtScene* ps = (PtScene*)h;
    PathTracing integrator;
    integrator.max_recursive_depth = max_recursive_depth;
    const Vector eye(cam[0], cam[1], cam[2]);
    Vector fwd = Vector(cam[3], cam[4], cam[5]) - eye;
    fwd = normalize(fwd);
    Vector right = normalize(cross(fwd, Vector(cam[6], cam[7], cam[8])));
    const Vector upv = cross(right, fwd);
    const float half_h = std::tan(cam[9] * 3.14159265358979f / 180.0f * 0.5f);
    const float half_w = half_h * (float)width / (float)height;
    if (nthreads <= 0) nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
    std::atomic<int> next{0};
    const int npix = width * height;
    auto worker = [&]() {
        RenderContext rc;
        rc.Init();
        PixelSample pxs;
        for (;;) {
            const int pix = next.fetch_add(1);
            if (pix >= npix) break;
            reseed(rc, mix32(seed ^ mix32((uint32_t)pix * 2654435761u)));
            const int px = pix % width, py = pix / width;
            Spectrum sum;
            for (int s = 0; s < spp; ++s) {
                const float jx = sort_rand<float>(rc), jy = sort_rand<float>(rc);
                const float sx = (((float)px + jx) / (float)width * 2.0f - 1.0f) * half_w;
                const float sy = (1.0f - ((float)py + jy) / (float)height * 2.0f) * half_h;
                const Vector d = normalize(fwd + right * sx + upv * sy);
                const Ray ray(Point(eye.x, eye.y, eye.z), d, 0, 0.0f, FLT_MAX);
                sum += integrator.Li(ray, pxs, ps->scene, rc);
                rc.m_memory_arena->Reset();
            }
            sum /= (float)spp;
            out_rgb[(size_t)pix * 3 + 0] = sum.r;
            out_rgb[(size_t)pix * 3 + 1] = sum.g;
            out_rgb[(size_t)pix * 3 + 2] = sum.b;
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nthreads; ++t) pool.emplace_back(worker);
    worker();
    for (auto& th : pool) th.join();
}

}  // extern "C"
