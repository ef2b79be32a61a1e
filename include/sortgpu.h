/* sortgpu: B200-native ray-query engine behind SORT's Accelerator API.
 *
 * C ABI of libsortgpu.so. Plain pointers and sizes only; every entry point
 * returns an sg_status (SG_OK == 0) and records a message for sg_last_error().
 *
 * What each entry point replaces in SORT (paths relative to SORT's src/):
 *
 *   sg_scene_create   Accelerator::Build (accel/accelerator.h:128) as
 *                     Fbvh::Build (accel/fast_bvh.hpp:109-136), together with the
 *                     scene box Scene::LoadScene computes first
 *                     (core/scene.cpp:146-154) and Fbvh::Serialize's two
 *                     parameters (accel/fast_bvh.h:159-162).
 *   sg_trace_closest  Accelerator::GetIntersect(RenderContext&, const Ray&,
 *                     SurfaceInteraction&) (accel/accelerator.h:74), as called by
 *                     Scene::GetIntersect (core/scene.cpp:182-185), for a batch.
 *   sg_trace_any      Accelerator::GetAttenuation (accel/accelerator.h:96,
 *                     accel/accelerator.cpp:26-69) for opaque scenes, i.e. the
 *                     any-hit query SORT builds from GetIntersect with
 *                     query_shadow set (accel/fast_bvh.hpp:362-373); also stands in
 *                     for IsOccluded (accel/accelerator.h:76-86), which SORT
 *                     compiles out under ENABLE_TRANSPARENT_SHADOW.
 *   sg_scene_destroy  the Accelerator's destructor (Scene owns it, core/scene.h).
 *   sg_scene_info     Fbvh's build statistics (accel/fast_bvh.hpp:50-96 counters)
 *                     and Accelerator::GetBBox / GetIsValid (accelerator.h:133-142).
 *   sg_scene_topology no SORT counterpart as an API; exports the tree in the
 *                     pre-order form the tests compare against SORT's own tree.
 *   sg_build_topology_host
 *                     Fbvh::Build alone, on the host, without a GPU: builds the
 *                     tree and returns the same pre-order topology stream.
 *   sg_trace_stats    SORT's traversal statistics for a batch (accel/fast_bvh.hpp:50-96
 *                     and accel/accelerator.cpp:21-23: sRayCount, sIntersectionTest)
 *                     plus the interior-node box tests; runs the same traversal.
 *   sg_scene_set_tuning / sg_scene_get_tuning
 *                     no SORT counterpart: launch schedule of the traversal
 *                     kernels (SORT's scheduling knob is its thread count,
 *                     work/image_evaluation/image_evaluation.cpp:70-75).
 *   sg_trace_closest_host / sg_trace_any_host
 *                     the same queries on host buffers, with the host<->device
 *                     copies done inside the call (what a caller that holds rays in
 *                     host memory, like SORT's integrators, binds).
 *   sg_trace_multi / sg_trace_multi_host
 *                     Accelerator::GetIntersect(const Ray&, BSSRDFIntersections&,
 *                     RenderContext&, StringID) (accel/accelerator.h:122), the
 *                     BSSRDF probe query, for a batch.
 *   sg_trace_attenuation / sg_trace_attenuation_host
 *                     Scene::GetAttenuation (core/scene.cpp:192-208) with
 *                     Accelerator::GetAttenuation (accel/accelerator.cpp:26-69) on
 *                     scenes with transparent materials (ENABLE_TRANSPARENT_SHADOW).
 *   sg_scene_create_hair / sg_scene_create_shapes
 *                     Fbvh::Build over scenes whose primitives include hair
 *                     Lines (Line4/8 packs) and area-light Quads and Disks (a
 *                     leaf's other_list, accel/fast_bvh.hpp:221-264, 375-406).
 *
 * Semantics carried over from SORT:
 *   - hit identity is the primitive's index in input order (SORT returns a
 *     Primitive*, whose index in ScenePrimitiveIterator order this is);
 *   - a triangle hit needs tmin < t <= tmax and is taken only if strictly
 *     nearer than the current one (a line hit: tmin < t < tmax, strictly
 *     nearer; an area-shape hit: tmin < t <= tmax and t <= the current t, as
 *     each SORT shape tests); a miss returns prim = -1 and t = FLT_MAX;
 *   - u, v are the barycentric weights of vertex 1 and vertex 2.
 *
 * Rays and hits are device pointers unless the function name ends in _host.
 * Calls are ordered on the given CUDA stream (NULL = legacy default stream) and
 * do not synchronise it; sg_*_host calls synchronise before returning.
 */
#ifndef SORTGPU_H
#define SORTGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    SG_OK = 0,
    SG_ERR_INVALID_ARGUMENT = 1,
    SG_ERR_CUDA = 2,
    SG_ERR_OUT_OF_MEMORY = 3,
    SG_ERR_UNSUPPORTED = 4,
    SG_ERR_LIMIT = 5,
    SG_ERR_INTERNAL = 6,
    SG_ERR_CANCELLED = 7
} sg_status;

/* Child-box storage of the device tree. */
typedef enum {
    SG_NODES_FP32 = 0,   /* FP32 child boxes: hits and visit order bit-identical to SORT */
    SG_NODES_QUANT8 = 1  /* 8-bit child boxes relative to the parent, rounded outward */
} sg_node_format;

typedef struct {
    int32_t width;          /* 4 = SORT's Qbvh, 8 = SORT's Obvh */
    int32_t max_depth;      /* Fbvh::m_maxNodeDepth (SORT default 16) */
    int32_t max_leaf;       /* Fbvh::m_maxPriInLeaf (SORT default 8) */
    int32_t node_format;    /* sg_node_format */
    int32_t device;         /* CUDA device ordinal the tree lives on */
    int32_t build_threads;  /* host threads for the build, 0 = all */
    int32_t builder;        /* sg_builder: which builder makes the tree */
} sg_build_opts;

/* SG_BUILDER_HOST and SG_BUILDER_GPU produce SORT's Fbvh tree (same
 * topology, leaf order, boxes). SG_BUILDER_LBVH builds a wide BVH in Morton
 * order entirely on the device, for fast scene admission: not SORT's tree (the
 * same hits and distances except near-ties, where two triangles are hit within
 * rounding of each other (1e-6 of the distance, more when the ray starts close
 * to large triangles) and a rounded box entry distance decides which one is
 * kept, and rays whose slab test misses the hit triangle's own box by
 * rounding, so that finding it depends on the leaf boxes), FP32 nodes only,
 * max_depth ignored. SG_BUILDER_PLOC builds a wide BVH
 * by parallel locally-ordered clustering over the Morton order (Meister and
 * Bittner 2018) on the device: tighter boxes than the LBVH, a few more passes,
 * the same promises and limits. */
typedef enum {
    SG_BUILDER_HOST = 0, /* host threads, one subtree per thread below the top */
    SG_BUILDER_GPU = 1,  /* data-parallel passes on the scene's device */
    SG_BUILDER_LBVH = 2, /* Morton-order wide BVH on the scene's device */
    SG_BUILDER_PLOC = 3  /* clustered (PLOC) wide BVH on the scene's device */
} sg_builder;

/* Structure-of-arrays ray batch: n entries in each array. */
typedef struct {
    const float* ox;
    const float* oy;
    const float* oz;
    const float* dx;
    const float* dy;
    const float* dz;
    const float* tmin;
    const float* tmax;
} sg_rays;

typedef struct {
    int32_t* prim;  /* primitive index, -1 on a miss */
    float* t;       /* FLT_MAX on a miss */
    float* u;       /* may be NULL */
    float* v;       /* may be NULL */
} sg_hits;

typedef struct {
    int64_t triangles;
    int64_t interior_nodes;
    int64_t leaves;
    int32_t depth;           /* Fbvh::m_depth */
    int32_t width;
    int32_t node_format;
    int32_t valid;           /* Accelerator::GetIsValid */
    float bbox[6];           /* enlarged scene box: min xyz, max xyz */
    int64_t device_bytes;    /* HBM held by the tree (nodes + triangles) */
    double build_seconds;    /* build time (host clock, whole build) */
    int32_t build_rounds;    /* GPU builders: split rounds (SG_BUILDER_GPU) or wide-tree levels (LBVH); 0 on the host */
    int32_t build_launches;  /* GPU builders: their split / collapse kernels launched (prefix sums and sorts not counted) */
} sg_scene_info;

/* Traversal launch schedule (results never depend on it). */
typedef enum {
    SG_SCHEDULE_THREAD_PER_RAY = 0, /* one ray per thread for the whole launch */
    SG_SCHEDULE_PERSISTENT = 1,     /* persistent warps; a finished lane takes the batch's next ray */
    SG_SCHEDULE_WHILE_WHILE = 2,    /* each warp alternates an interior phase and a leaf phase */
    SG_SCHEDULE_SPECULATIVE = 3,    /* while-while; lanes keep descending past their first leaf */
    SG_SCHEDULE_SORTED = 4,         /* one ray per thread, threads given rays in the order of a 30-bit key
                                       (direction octant, origin cell, coarse direction) so that a warp's
                                       rays take similar paths; batches of 65,536 rays or more; scratch
                                       (16 B per ray) from a stream-ordered pool */
    SG_SCHEDULE_AUTO = 5            /* a new scene's default: SORTED for closest-hit batches of 2M rays or
                                       more (measured faster on 4M incoherent rays, slower on 1M coherent
                                       primary rays), THREAD_PER_RAY otherwise */
} sg_schedule;

typedef struct {
    int32_t schedule;          /* sg_schedule */
    int32_t refill_threshold;  /* idle lanes (1..32) that make a persistent warp fetch new rays */
} sg_trace_tuning;

typedef struct sg_scene sg_scene;

void sg_default_build_opts(sg_build_opts* opts);

sg_status sg_scene_create(const float* triangles, int64_t ntri, const sg_build_opts* opts, sg_scene** out);

/* A scene of triangles and hair line segments: SORT's Line shapes as a
 * HairVisual makes them (entity/visual.cpp:41-97, shape/line.cpp), tested with
 * Line4/8's ray-line test (simd/simd_line.h:232-330). lines: 10 floats per
 * segment in world space: p0 xyz, p1 xyz, v0, v1 (texture v at the two ends),
 * w0, w1 (half widths at the two ends). Primitive indices: the triangles
 * 0 .. ntri-1, then the lines ntri .. ntri+nlines-1 (a mesh visual followed by
 * a hair visual in SORT's primitive order). A line hit reports u = 1 and SORT's
 * v. Such a scene answers sg_trace_closest / sg_trace_any and their _host
 * forms; the other queries return SG_ERR_UNSUPPORTED, and so does
 * SG_BUILDER_LBVH. sg_scene_info's triangle count is the primitive count. */
sg_status sg_scene_create_hair(const float* triangles, int64_t ntri, const float* lines, int64_t nlines,
                               const sg_build_opts* opts, sg_scene** out);

/* ---- Area-light shapes in the accelerator --------------------------------
 * SORT puts each area light's shape into the accelerator as a primitive
 * (entity/light_entity.cpp:153-154); Fbvh keeps such primitives in a leaf's
 * other_list and tests them after the leaf's triangle and line packs
 * (accel/fast_bvh.hpp:244-247, 390-406) with the shape's own scalar test:
 * Quad::GetIntersect (shape/quad.cpp:67-93) for SQUARE and RECTANGLE lights,
 * Disk::GetIntersect (shape/disk.cpp) for DISK lights. That test takes a hit
 * when t <= the current nearest t (not only when nearer), and a shape hit
 * leaves u and v at the values of the hit it replaced (0 when none).
 * sg_area_shape: the shape in its local frame (a sizeX x sizeY rectangle, or a
 * disk of the given radius, in the x-z plane around the origin, normal +y)
 * and Shape::m_transform (math/transform.h) as SORT holds it. */
typedef enum { SG_SHAPE_QUAD = 0, SG_SHAPE_DISK = 1 } sg_shape_kind;
typedef struct {
    int32_t kind;       /* sg_shape_kind */
    float size[2];      /* quad: sizeX, sizeY (shape/quad.h:107-108); disk: radius, unused */
    float matrix[16];   /* local to world, row-major (Transform::matrix) */
    float inverse[16];  /* world to local (Transform::invMatrix) */
} sg_area_shape;

/* Primitives of every kind, and the order SORT's builder sees them in.
 * Primitive indices: triangles 0 .. ntri-1, then the hair segments (10 floats
 * each, as sg_scene_create_hair takes them), then the area shapes. order:
 * NULL (that order) or the ntri + nlines + nshapes indices in the order
 * SORT's ScenePrimitiveIterator visits the primitives (entity by entity,
 * core/scene.cpp:43-80), which decides the tree SORT builds. Hits report the
 * indices above. Such a scene answers sg_trace_closest / sg_trace_any and
 * their _host forms (the others: SG_ERR_UNSUPPORTED, as for hair), and is
 * built by SG_BUILDER_HOST or SG_BUILDER_GPU. */
typedef struct {
    const float* triangles;
    int64_t ntri;
    const float* lines;
    int64_t nlines;
    const sg_area_shape* shapes;
    int64_t nshapes;
    const int32_t* order;
} sg_shapes;
sg_status sg_scene_create_shapes(const sg_shapes* shapes, const sg_build_opts* opts, sg_scene** out);

/* SORT's binary scene stream (what the Blender exporter writes and
 * ImageEvaluation loads, work/image_evaluation/image_evaluation.cpp:62-108),
 * read for the GPU path: the configuration with the integrator's parameters
 * (loadConfig, 354-377), the material section (MatManager::ParseMatFile,
 * material/matmanager.cpp:50-270: names and flags are kept, TSL shader graphs
 * and resources are read past), the entities (Scene::LoadScene,
 * core/scene.cpp:112-180: meshes and hair with their transforms, the camera,
 * area lights; other lights are counted) and the accelerator. Triangles are in
 * world space (Mesh::ApplyTransform); hair segments as HairVisual makes them
 * (entity/visual.cpp:41-97). StringIDs are SORT's 32-bit hashes of the class
 * names. Unknown classes or a broken stream: SG_ERR_UNSUPPORTED. */
typedef struct sg_stream sg_stream;
typedef struct {
    int32_t version, threads, spp, image_width, image_height;
    float clamp;
    uint32_t integrator;     /* StringID of the integrator class (PathTracing, ...) */
    int32_t max_depth;       /* Integrator::max_recursive_depth */
    int32_t bssrdf_bounces;  /* PathTracing */
    float ao_max_distance;   /* AmbientOcclusion */
    int32_t mis;             /* BidirPathTracing, LightTracing */
    int32_t ir_path_sets, ir_paths;
    float ir_min_distance;   /* InstantRadiosity */
    int64_t triangles, lines;
    int32_t materials, area_lights, other_lights, has_camera, volumes;
    uint32_t accelerator;    /* StringID of the accelerator class (Qbvh, Obvh, ...) */
    int32_t accel_max_depth, accel_max_leaf;
    int64_t entity_offset;   /* byte offset of the entity section ("verification bits") */
} sg_stream_info;
typedef struct {
    float eye[3], up[3], target[3];
    int32_t image_width, image_height;
    float lens_radius, sensor_w, sensor_h;
    int32_t aspect_fit;
    float aspect_ratio_w, aspect_ratio_h, fov;
} sg_stream_camera; /* PerspectiveCameraEntity::Serialize (entity/camera_entity.cpp:21-33) */
typedef struct {
    float light2world[16]; /* as streamed (SORT removes the scale afterwards, entity/light_entity.cpp:99-106) */
    float energy;
    float intensity[3];
    uint32_t shape;        /* StringID: SQUARE, RECTANGLE or DISK */
    float size_x, size_y;  /* SQUARE: size_x; RECTANGLE: both; DISK: size_x is the radius */
} sg_stream_area_light;
sg_status sg_stream_open(const char* path, sg_stream** out);
sg_status sg_stream_info_get(const sg_stream* stream, sg_stream_info* info);
/* 9 floats per triangle (world space) and its material index (-1: none). */
sg_status sg_stream_triangles(const sg_stream* stream, float* triangles, int32_t* material);
/* 10 floats per hair segment in world space (as sg_scene_create_hair takes
 * them) and its material index. */
sg_status sg_stream_lines(const sg_stream* stream, float* lines, int32_t* material);
sg_status sg_stream_camera_get(const sg_stream* stream, sg_stream_camera* camera);
sg_status sg_stream_area_light_get(const sg_stream* stream, int32_t index, sg_stream_area_light* light);
/* Name (NUL-terminated, cap bytes available) and flags (bit 0: a transparency
 * node, bit 1: an SSS node) of material `index` in the stream's order. */
sg_status sg_stream_material(const sg_stream* stream, int32_t index, char* name, int64_t cap, int32_t* flags);
/* The area lights' shapes (sg_stream_info.area_lights of them, in stream
 * order) as SORT's scene holds them: a Quad for SQUARE / RECTANGLE lights, a
 * Disk for DISK, with the transform AreaLightEntity::Serialize leaves the
 * shape (entity/light_entity.cpp:97-150: the streamed matrix and its inverse
 * by Matrix::Inverse, the scale taken out of both). */
sg_status sg_stream_area_shapes(const sg_stream* stream, sg_area_shape* shapes);
/* The scene's primitive indices (triangles, segments, shapes) in the order
 * SORT's ScenePrimitiveIterator visits them (entity by entity): triangles +
 * lines + area lights entries, the order sg_stream_scene_create builds in. */
sg_status sg_stream_primitive_order(const sg_stream* stream, int32_t* order);
/* The stream's scene as an sg_scene: its triangles, its hair segments (their
 * entity's transform applied as SORT's Line::SetTransform applies it) and its
 * area lights' shapes, built in the order SORT's scene presents them (entity
 * by entity). Primitive indices: triangles, then segments, then shapes.
 * opts NULL: the stream's accelerator (Obvh: width 8, Qbvh: width 4, with
 * their depth and leaf size; any other class: SORT's fallback, a QBVH with
 * default parameters). */
sg_status sg_stream_scene_create(const sg_stream* stream, const sg_build_opts* opts, sg_scene** out);
sg_status sg_stream_close(sg_stream* stream);
sg_status sg_scene_destroy(sg_scene* scene);
sg_status sg_scene_info_get(const sg_scene* scene, sg_scene_info* info);
sg_status sg_scene_topology(const sg_scene* scene, int32_t* out, int64_t cap, int64_t* written);
/* Topology stream: interior node [child_cnt, children...], leaf [0, count,
 * primitive indices in leaf order]; pre-order from the root. Call with
 * out = NULL / cap = 0 to learn the size (returns SG_ERR_LIMIT and sets written). */
sg_status sg_build_topology_host(const float* triangles, int64_t ntri, const sg_build_opts* opts, int32_t* out,
                                 int64_t cap, int64_t* written, int32_t* depth);
/* The same for a scene with hair segments (as sg_scene_create_hair takes
 * them): SORT's tree over the triangles and the lines' boxes. */
sg_status sg_build_topology_host_hair(const float* triangles, int64_t ntri, const float* lines, int64_t nlines,
                                      const sg_build_opts* opts, int32_t* out, int64_t cap, int64_t* written,
                                      int32_t* depth);
/* The same for primitives of every kind (as sg_scene_create_shapes takes
 * them); a leaf lists its triangles, then its lines, then its area shapes. */
sg_status sg_build_topology_host_shapes(const sg_shapes* shapes, const sg_build_opts* opts, int32_t* out,
                                        int64_t cap, int64_t* written, int32_t* depth);

sg_status sg_scene_set_tuning(sg_scene* scene, const sg_trace_tuning* tuning);
sg_status sg_scene_get_tuning(const sg_scene* scene, sg_trace_tuning* tuning);

sg_status sg_trace_closest(const sg_scene* scene, const sg_rays* rays, int64_t n, const sg_hits* hits, void* stream);
sg_status sg_trace_any(const sg_scene* scene, const sg_rays* rays, int64_t n, uint8_t* occluded, void* stream);

/* BSSRDF probe query: Accelerator::GetIntersect(const Ray&, BSSRDFIntersections&,
 * RenderContext&, StringID) (accel/accelerator.h:122, accel/fast_bvh.hpp:656-819)
 * for a batch. Per ray up to 4 (TOTAL_SSS_INTERSECTION_CNT) hits on primitives
 * whose material equals ray_material[i], gathered and replaced exactly as SORT
 * does (intersectTriangleMulti_SIMD, simd/simd_triangle.h:412-455), so the kept
 * set and the slot of each hit are SORT's. prim_material: one material id per
 * primitive (input order), device; ray_material: one per ray, device.
 * hits: count[i] = hits kept; prim / t / u / v hold 4 entries per ray at
 * [4*i + k] (prim -1, t FLT_MAX past count); u, v may be NULL. */
typedef struct {
    int32_t* count;
    int32_t* prim;
    float* t;
    float* u;
    float* v;
} sg_multi_hits;
sg_status sg_trace_multi(const sg_scene* scene, const sg_rays* rays, int64_t n, const int32_t* prim_material,
                         const int32_t* ray_material, const sg_multi_hits* hits, void* stream);
/* Host-buffer form for callers like SORT's per-ray integrators: the scene keeps
 * one material id per primitive (sg_scene_set_materials, host array of the
 * scene's triangle count, copied to the device); rays8 as sg_trace_closest_host;
 * ray_material one per ray; outputs 1 (count) or 4 (prim, t, u, v) per ray.
 * Synchronous. */
sg_status sg_scene_set_materials(sg_scene* scene, const int32_t* material, int64_t n);
sg_status sg_trace_multi_host(const sg_scene* scene, const float* rays8, int64_t n, const int32_t* ray_material,
                              int32_t* count, int32_t* prim, float* t, float* u, float* v);

/* Transparent-shadow query: Scene::GetAttenuation (core/scene.cpp:192-208)
 * over Accelerator::GetAttenuation (accel/accelerator.cpp:26-69) and Fbvh's
 * query_shadow traversal (accel/fast_bvh.hpp:345-370). Per ray, from its
 * [tmin, tmax] segment: find the nearest hit, leaving early when a SIMD pack's
 * nearest hit is on an opaque material (then the attenuation is 0); on a
 * transparent hit multiply by the material's transparency (a black one is
 * returned as it is) and restart at the hit point with tmin 0.001 and
 * tmax - t; no hit ends the loop. attenuation[0..n), [n..2n), [2n..3n): r, g, b.
 * Primitive materials come from sg_scene_set_materials; materials[nmat] is a
 * device array for sg_trace_attenuation, a host array for the _host form. A
 * ray that crosses more than 4096 transparent surfaces stops there (reported
 * as SG_ERR_LIMIT); a primitive material id outside [0, nmat) counts as opaque
 * (reported as SG_ERR_INVALID_ARGUMENT). The _host form reports both; the
 * device form records them in the scene's status word, which the next
 * host-buffer call on that scene reports. */
typedef struct {
    int32_t transparent; /* MaterialBase::HasTransparency (material/material.h:100) */
    float rgb[3];        /* MaterialBase::EvaluateTransparency (material/material.h:85), constant per material */
} sg_transparency;
sg_status sg_trace_attenuation(const sg_scene* scene, const sg_rays* rays, int64_t n, const sg_transparency* materials,
                               int32_t nmat, float* attenuation, void* stream);
sg_status sg_trace_attenuation_host(const sg_scene* scene, const float* rays8, int64_t n,
                                    const sg_transparency* materials, int32_t nmat, float* attenuation);

/* Counts over one batch (synchronises the stream): interior nodes box-tested and
 * primitives tested, the latter counted per leaf entered as SORT's
 * sIntersectionTest does. any = 0 closest-hit traversal, 1 any-hit traversal. */
sg_status sg_trace_stats(const sg_scene* scene, const sg_rays* rays, int64_t n, int32_t any, int64_t* node_tests,
                         int64_t* prim_tests, void* stream);

/* Host-buffer forms. rays8 is one block of 8*n floats: ox[n], oy[n], oz[n],
 * dx[n], dy[n], dz[n], tmin[n], tmax[n]. */
sg_status sg_trace_closest_host(const sg_scene* scene, const float* rays8, int64_t n, int32_t* prim, float* t,
                                float* u, float* v);
sg_status sg_trace_any_host(const sg_scene* scene, const float* rays8, int64_t n, uint8_t* occluded);

/* sg_trace_closest_host without any device allocation. No counterpart in SORT:
 * it exists for callers that must not call cudaMalloc while they query (a
 * host that owns the whole GPU memory budget, a real-time loop that must not
 * take the allocator's locks or wait on an implicit synchronisation). Rays and hits are staged in a 24 MiB array compiled into
 * the library, held on every GPU that loads it until exit; at most 524,288 rays
 * per call (SG_ERR_LIMIT beyond). All calls share that array, so calls whose
 * work overlaps on the GPU race. Every batch runs one ray per thread, whatever
 * schedule sg_scene_set_tuning chose (the sorted schedule would take scratch
 * from a pool); results are the same under every schedule. Scenes with hair
 * lines are rejected (SG_ERR_UNSUPPORTED). The first call on a device looks up
 * the array's address (cudaGetSymbolAddress); make that first call before any
 * stream capture begins on that device. Ordered on `stream` (NULL = legacy
 * default stream); the call ends by synchronising `stream` to read the
 * traversal status. */
sg_status sg_trace_closest_host_static(const sg_scene* scene, const float* rays8, int64_t n, int32_t* prim, float* t,
                                       float* u, float* v, void* stream);

/* ---- Batched multi-scene traversal --------------------------------------
 * A batcher traces many ray batches, over many resident scenes and of uneven
 * sizes, in one replay of a captured CUDA graph: per group of batches sharing
 * a tree width, node format and query, one persistent kernel drains all of
 * them as one ray sequence, instead of one launch per batch. No SORT
 * counterpart as an API: it stands in for SORT's render workers, which each
 * call Accelerator::GetIntersect / GetAttenuation for their own rays
 * (work/image_evaluation/image_evaluation.cpp:70-75, 153-279). A batch's
 * results are exactly those of sg_trace_closest / sg_trace_any on its scene
 * alone, whatever shares the run.
 *
 * sg_batch: rays are device SoA planes ox, oy, oz, dx, dy, dz, tmin, tmax;
 *   plane k of ray i is rays[k * stride + i] (stride 0 = n), so a batch may be
 *   a slice of a larger ray array. any = 0 writes hits, 1 writes occluded.
 * sg_batcher_run: enqueues the run on `stream` (no synchronisation). Runs of
 *   one batcher share its device tables: order them on one stream. budget_ns
 *   > 0 stops warps from claiming rays once that long has passed since the
 *   run's start; the rays they hold still finish. Up to max_batches batches.
 * sg_batcher_wait: synchronises `stream`; per batch of the LAST run (caller
 *   order) the ns from the run's start to the completion of its last ray, or
 *   -1 if the budget left it incomplete (then returns SG_ERR_LIMIT).
 * sg_batcher_autotune: picks, by timing runs of `batches` on `stream`, the
 *   tree width per scene (alternatives[i]: the same triangles built at the
 *   other width, or NULL; use_alternative[i] = 1 where that one is faster) and
 *   the kernel tuning (block threads, stack, refill threshold), which it
 *   installs in the batcher and returns in `best`. reps: timed runs per
 *   candidate (0 = 3). */
typedef struct {
    const sg_scene* scene;
    const float* rays;
    int64_t stride;
    int64_t n;
    int32_t any;
    int32_t reserved;
    sg_hits hits;
    uint8_t* occluded;
} sg_batch;

typedef struct {
    int32_t block_threads;    /* rays per block: 64, 128 or 256 */
    int32_t stack;            /* stack entries 64, 128 or 256; 0 or less than a tree needs = the least that fits */
    int32_t refill_threshold; /* idle lanes (1..32) at which a warp claims new rays */
    int32_t blocks_per_sm;    /* resident blocks per SM, 0 = as many as fit */
} sg_batch_tuning;

typedef struct sg_batcher sg_batcher;
sg_status sg_batcher_create(int32_t device, int32_t max_batches, sg_batcher** out);
sg_status sg_batcher_destroy(sg_batcher* batcher);
sg_status sg_batcher_set_tuning(sg_batcher* batcher, const sg_batch_tuning* tuning);
sg_status sg_batcher_get_tuning(const sg_batcher* batcher, sg_batch_tuning* tuning);
sg_status sg_batcher_run(sg_batcher* batcher, const sg_batch* batches, int32_t count, int64_t budget_ns, void* stream);
sg_status sg_batcher_wait(sg_batcher* batcher, int64_t* done_ns, int32_t count, void* stream);
sg_status sg_batcher_autotune(sg_batcher* batcher, const sg_batch* batches, const sg_scene* const* alternatives,
                              int32_t count, int32_t reps, int32_t* use_alternative, sg_batch_tuning* best,
                              void* stream);

/* ---- Path tracing -------------------------------------------------------
 * SORT's PathTracing integrator (integrator/pathtracing.cpp:37-258) with its
 * next-event estimation (integrator/integratormethod.cpp:100-192), Lambert and
 * GGX-conductor BxDFs and one rectangular AreaLight, run as a wavefront over a
 * scene built by sg_scene_create; replaces ImageEvaluation's per-pixel loop
 * (work/image_evaluation/image_evaluation.cpp:210-238) for those materials.
 *
 * sg_pt_create: triangles/ntri as given to sg_scene_create (same order);
 *   mat_of_tri[i] indexes materials (10 floats each: type 0 Lambert with albedo
 *   r g b; type 1 GGX conductor reflection with eta r g b, k r g b, roughness),
 *   or is -1 for the light's own surface (the light quad's two triangles, which
 *   must be in the scene as SORT puts the quad in its accelerator);
 *   light = centre x y z, size x, size z, intensity r g b of a rectangle facing -y.
 * sg_pt_render: camera = eye xyz, target xyz, up xyz, vertical fov (degrees);
 *   writes the mean radiance of spp samples per pixel to `image` (device,
 *   width*height*3 floats, row-major from the top); max_depth as SORT's
 *   max_recursive_depth; ordered on `stream`. */
typedef struct sg_pt_scene sg_pt_scene;
sg_status sg_pt_create(const sg_scene* scene, const float* triangles, int64_t ntri, const int32_t* mat_of_tri,
                       const float* materials, int32_t nmat, const float* light, sg_pt_scene** out);
sg_status sg_pt_render(sg_pt_scene* pt, const float* camera, int32_t width, int32_t height, int32_t spp,
                       int32_t max_depth, uint64_t seed, float* image, void* stream);
/* sg_pt_render_rows: rows [row_begin, row_end) of the same width x height
 * frame into `image` (width*(row_end-row_begin)*3 floats): every pixel gets
 * the random numbers of its place in the whole frame, so bands rendered
 * separately (on one GPU or on several) put together are bit-identical to
 * sg_pt_render of the frame. No SORT counterpart: SORT's render threads split
 * a frame into tiles (work/image_evaluation/image_evaluation.cpp:153-279). */
sg_status sg_pt_render_rows(sg_pt_scene* pt, const float* camera, int32_t width, int32_t height, int32_t row_begin,
                            int32_t row_end, int32_t spp, int32_t max_depth, uint64_t seed, float* image,
                            void* stream);
sg_status sg_pt_destroy(sg_pt_scene* pt);
/* Rays the last sg_pt_render traced: extension (closest-hit) and shadow
 * (any-hit) rays; synchronises `stream`. The counterpart of SORT's sRayCount /
 * sShadowRayCount (accel/accelerator.cpp:21-23). */
sg_status sg_pt_ray_counts(const sg_pt_scene* pt, int64_t* extension, int64_t* shadow, void* stream);

/* ---- Render server ------------------------------------------------------
 * A serving loop that keeps path-tracing scenes resident and renders requests
 * of uneven sizes concurrently: every admitted request's pixels share one pool
 * of in-flight paths and one set of wavefront queues (extension, shadow) over
 * all scenes; a pool slot whose path ends takes the next pixel sample of any
 * admitted request, and requests are admitted as soon as the pixel budget
 * frees up (continuous batching). The bounce steps run as replays of a
 * captured CUDA graph. Each pixel's samples are accumulated in sample order
 * with the arithmetic of sg_pt_render, so a request's image is bit-identical to
 * sg_pt_render of the same request, alone or in any mix.
 * No SORT counterpart as an API: SORT renders one image per process
 * (work/image_evaluation/image_evaluation.cpp:120-305).
 *
 * sg_server_opts: path_slots = paths in flight (each holds about 250 bytes of
 *   path state in HBM); pixel_budget = pixels of admitted, unfinished requests
 *   (20 bytes each: image + work queue entry); max_requests = requests admitted
 *   at once; steps_per_poll = bounce steps per graph replay (even, >= 2);
 *   samples_per_claim = samples a pool slot renders of one pixel before the
 *   pixel goes back to the shared work queue (1 = strict turn-taking between
 *   requests; larger keeps neighbouring pixels together in the queues);
 *   solo_pixels = requests of at least this many pixels and 2 or more
 *   samples take one of the server's solo lanes, in queue order: rendered as
 *   sg_pt_render renders, one wave per sample (two in flight) on the lane's
 *   own buffers, beside the pool, the oldest lane's waves at the highest
 *   stream priority; the lane scales and completes the request (the image
 *   is the same either way). The pool renders the other requests.
 *   0 = 1 (every multi-sample request), < 0 = never.
 * sg_server_add_scene: all scenes of a server share one tree width and node
 *   format (SG_ERR_UNSUPPORTED otherwise); the sg_pt_scene and its sg_scene
 *   must outlive the server.
 * sg_server_submit: queues a request; image is a host buffer of
 *   width*height*3 floats that holds the result when the request completes.
 *   A request larger than pixel_budget fails with SG_ERR_LIMIT.
 * sg_server_wait: blocks until the ticket completes or timeout_ns passes
 *   (SG_ERR_LIMIT, the request keeps running); timeout_ns < 0 waits forever.
 *   Each completed ticket can be waited for once.
 * sg_server_cancel: a queued request is dropped; an admitted one stops taking
 *   new pixel samples and completes once its paths in flight end; either way
 *   its result reports SG_ERR_CANCELLED and its image is not written. */
typedef struct {
    int32_t device;
    int32_t max_requests;
    int64_t path_slots;
    int64_t pixel_budget;
    int32_t steps_per_poll;
    int32_t samples_per_claim;
    int64_t solo_pixels;
} sg_server_opts;

typedef struct {
    int32_t scene;  /* from sg_server_add_scene */
    int32_t width;
    int32_t height;
    int32_t spp;
    int32_t max_depth;
    int32_t reserved;
    uint64_t seed;
    float camera[10]; /* as sg_pt_render */
    float* image;     /* host, width*height*3 floats */
} sg_request;

typedef struct {
    int64_t ticket;
    int32_t status;     /* SG_OK, SG_ERR_CANCELLED, or the error that ended it */
    int32_t reserved;
    int64_t submit_ns;  /* steady clock of the host */
    int64_t admit_ns;
    int64_t done_ns;    /* image in host memory */
} sg_request_result;

typedef struct {
    int64_t requests_done;
    int64_t samples_done;     /* pixel samples of the requests completed (not cancelled) */
    int64_t extension_rays;   /* closest-hit rays traced */
    int64_t shadow_rays;      /* any-hit rays traced */
    int64_t graph_replays;
    int64_t queued;           /* submitted, not admitted */
    int64_t admitted;         /* admitted, not complete */
    int64_t solo_waves;       /* samples rendered as whole-request waves (solo_pixels) */
} sg_server_stats;

typedef struct sg_server sg_server;
void sg_default_server_opts(sg_server_opts* opts);
sg_status sg_server_create(const sg_server_opts* opts, sg_server** out);
sg_status sg_server_add_scene(sg_server* server, const sg_pt_scene* pt, int32_t* scene_id);
sg_status sg_server_submit(sg_server* server, const sg_request* request, int64_t* ticket);
sg_status sg_server_wait(sg_server* server, int64_t ticket, int64_t timeout_ns, sg_request_result* result);
sg_status sg_server_cancel(sg_server* server, int64_t ticket);
sg_status sg_server_stats_get(sg_server* server, sg_server_stats* stats);
sg_status sg_server_destroy(sg_server* server);

/* Measurement aid, no SORT counterpart: the L2 read bandwidth (GB/s) a kernel
 * reaches on `device`, reading a buffer of `bytes` (1..96 MiB, resident in L2)
 * `reps` times with L1-bypassing 128-bit loads. The roofline of a workload
 * whose tree fits in L2 is this figure, not HBM's. */
sg_status sg_probe_l2_read_gbs(int32_t device, int64_t bytes, int32_t reps, double* gbs);

const char* sg_last_error(void);
const char* sg_version(void);

#ifdef __cplusplus
}
#endif

#endif /* SORTGPU_H */
