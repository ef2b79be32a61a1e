/* Restated CPU oracle for SORT's QBVH/OBVH ray-query path (TEST INFRASTRUCTURE).
 *
 * Plain C restatement of:
 *   accel/fast_bvh.hpp:109-270   Fbvh::Build / splitNode / makeLeaf
 *   accel/bvh_utils.h:27-118     Bvh_Primitive centroid, sah, pickBestSplit (16 bins)
 *   core/scene.cpp:146-154       scene box = union of primitive boxes, enlarged by 0.1%
 *   accel/fast_bvh.hpp:305-504   Fbvh::GetIntersect (SIMD branch): root slab test,
 *                                (node, tmin) stack, t-culling, near-first push order
 *   simd/simd_ray_utils.h:60-83  resolveRayData (|d| < 1e-5 clamp, 1/d, -o/d)
 *   simd/simd_bbox.h:62-85       IntersectBBox_SIMD
 *   simd/simd_triangle.h:212-383 intersectTriangleInner_SIMD / intersectTriangle_SIMD
 *   math/ray.h:26-69             majorAxis / Ray::Prepare
 *   math/bbox.h:124-155          scalar Intersect (root test)
 *   accel/accelerator.cpp:26-69  any-hit through GetAttenuation (opaque early exit)
 *
 * Parity is pinned against SORT's own code compiled from its sources
 * (oracle/_ref/libsortref.so, see oracle/Makefile): tests compare this port's
 * topology and hits with the reference library's, and commit golden vectors
 * produced by the reference under tests/golden/.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load
 * this library. The product (sort_b200) never calls it.
 */
#ifndef SORT_ORACLE_H
#define SORT_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_tree orc_tree;

/* Build the W-wide tree (W = 4: QBVH, 8: OBVH) over ntri triangles given as
 * 9 floats each. max_depth / max_leaf = Fbvh::m_maxNodeDepth / m_maxPriInLeaf. */
orc_tree* orc_build(int width, const float* tri, int64_t ntri, int max_depth, int max_leaf);
void orc_free(orc_tree* t);

/* Pre-order topology stream, same format as the reference harness:
 *   interior node: [child_cnt, child0 ..., child_{n-1} ...]
 *   leaf:          [0, pri_cnt, primitive indices in leaf order]
 * Returns the count written, or minus the required size if cap is too small. */
int64_t orc_topology(const orc_tree* t, int32_t* out, int64_t cap);
int orc_depth(const orc_tree* t);
void orc_scene_bbox(const orc_tree* t, float* out6);

/* Rays: SoA block of 8*n floats (ox, oy, oz, dx, dy, dz, tmin, tmax). */
void orc_trace_closest(const orc_tree* t, const float* rays, int64_t n, int32_t* prim, float* tt, float* u, float* v,
                       int nthreads);
void orc_trace_any(const orc_tree* t, const float* rays, int64_t n, uint8_t* occluded, int nthreads);

/* Per-ray work counters of the closest-hit (any = 0) or any-hit (any = 1)
 * traversal: interior-node box tests and primitives tested, SORT's
 * sIntersectionTest convention (whole leaf counted, accel/fast_bvh.hpp:409). */
void orc_count(const orc_tree* t, const float* rays, int64_t n, int any, int64_t* node_tests, int64_t* prim_tests,
               int nthreads);

/* Ray::Prepare for one direction (math/ray.h:60-69). */
void orc_ray_prepare(const float* d, int* local_xyz, float* scale_xyz);

/* SORT's FP32 watertight test of ray i against triangle prim alone
 * (tmin < t <= tmax); returns 1 and t on a hit. */
int orc_tri_test(const float* tri, int64_t prim, const float* rays, int64_t n, int64_t i, float* t_out);

/* FP64 re-intersection of ray i with triangle prim (same watertight
 * formulation in doubles); returns t, or -1 on a miss. */
double orc_fp64_intersect(const float* tri, int64_t prim, const float* rays, int64_t n, int64_t i);

/* orc_fp64_intersect of every ray i with triangle prim[i]; -1 where prim[i] < 0. */
void orc_fp64_t_batch(const float* tri, const int32_t* prim, const float* rays, int64_t n, double* t_out);

#ifdef __cplusplus
}
#endif
#endif
