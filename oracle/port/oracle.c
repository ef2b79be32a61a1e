/* Restated CPU oracle for SORT's QBVH/OBVH ray-query path (TEST INFRASTRUCTURE).
 * See oracle.h for the list of reference functions restated here and how the
 * restatement is pinned. Compiled with -ffp-contract=off: every a*b+c below is a
 * rounded multiply followed by a rounded add, as SORT's SSE/AVX simd_mad_ps is
 * (simd/simd_intel.h:128-130).
 *
 * The product never links this file.
 */
#include "oracle.h"

#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------- */
/* BBox helpers (math/bbox.cpp:22-125)                                        */

typedef struct {
    float mn[3], mx[3];
} obox;

static void box_empty(obox* b) {
    for (int k = 0; k < 3; ++k) {
        b->mn[k] = FLT_MAX;
        b->mx[k] = -FLT_MAX;
    }
}
/* std::min(a, b) and std::max(a, b) exactly as libstdc++ defines them. */
static float std_min(float a, float b) { return (b < a) ? b : a; }
static float std_max(float a, float b) { return (a < b) ? b : a; }
/* BBox::Union(const Point&) (math/bbox.cpp:106-113): strict compares. */
static void box_add_point(obox* b, const float* p) {
    for (int k = 0; k < 3; ++k) {
        if (p[k] < b->mn[k]) b->mn[k] = p[k];
        if (p[k] > b->mx[k]) b->mx[k] = p[k];
    }
}
/* BBox::Union(const BBox&) (math/bbox.cpp:115-120) and the free Union (bbox.h). */
static void box_add_box(obox* b, const obox* o) {
    for (int k = 0; k < 3; ++k) {
        b->mn[k] = std_min(b->mn[k], o->mn[k]);
        b->mx[k] = std_max(b->mx[k], o->mx[k]);
    }
}
static float box_half_area(const obox* b) {
    const float ox = b->mx[0] - b->mn[0], oy = b->mx[1] - b->mn[1], oz = b->mx[2] - b->mn[2];
    return ox * oy + oy * oz + oz * ox;
}
static int box_max_axis(const obox* b) {
    const float ox = b->mx[0] - b->mn[0], oy = b->mx[1] - b->mn[1], oz = b->mx[2] - b->mn[2];
    if (ox > oy && ox > oz) return 0;
    if (oy > ox && oy > oz) return 1;
    return 2;
}

/* ------------------------------------------------------------------------- */
/* Tree                                                                      */

typedef struct {
    int32_t child_cnt;
    int32_t child[8];
    int32_t pri_offset, pri_cnt;
    float lo[3][8], hi[3][8]; /* child boxes (calcBoundingBoxSIMD), axis-major */
} onode;

struct orc_tree {
    int width, max_depth, max_leaf, depth;
    int64_t ntri;
    const float* tri; /* caller's triangles (9 floats each); kept for FP64 re-checks */
    float* tri_copy;
    obox scene;       /* enlarged scene box (Fbvh::m_bbox) */
    obox* pbox;       /* per-primitive boxes (Triangle::GetBBox) */
    int32_t* order;   /* m_bvhpri order: primitive index per slot */
    float* cent;      /* centroid per slot (moves with order) */
    onode* nodes;
    int64_t nnodes, cap;
    int root;
};

typedef struct {
    int32_t idx;
    float c[3];
} bprim;

static int new_node(orc_tree* t) {
    if (t->nnodes == t->cap) {
        t->cap = t->cap ? t->cap * 2 : 1024;
        t->nodes = (onode*)realloc(t->nodes, (size_t)t->cap * sizeof(onode));
    }
    onode* n = &t->nodes[t->nnodes];
    memset(n, 0, sizeof(*n));
    return (int)t->nnodes++;
}

/* pickBestSplit (accel/bvh_utils.h:69-118). */
static float pick_best_split(int* axis_out, float* split_pos, const bprim* pr, const obox* pbox, const obox* node_box,
                             int64_t start, int64_t end) {
    enum { SPLITS = 16 };
    const float inv_split_count = 1.0f / (float)SPLITS;
    obox inner;
    box_empty(&inner);
    for (int64_t i = start; i < end; ++i) box_add_point(&inner, pr[i].c);
    const unsigned primitive_num = (unsigned)(end - start);
    const int axis = box_max_axis(&inner);
    *axis_out = axis;
    float min_sah = FLT_MAX;
    unsigned bin[SPLITS];
    obox bbox[SPLITS], rbox[SPLITS - 1];
    memset(bin, 0, sizeof(bin));
    for (int i = 0; i < SPLITS; ++i) box_empty(&bbox[i]);
    for (int i = 0; i < SPLITS - 1; ++i) box_empty(&rbox[i]);
    const float split_start = inner.mn[axis];
    const float split_delta = (inner.mx[axis] - inner.mn[axis]) * inv_split_count;
    if (split_delta == 0.0f) return FLT_MAX;
    const float inv_split_delta = 1.0f / split_delta;
    for (int64_t i = start; i < end; ++i) {
        int index = (int)((pr[i].c[axis] - split_start) * inv_split_delta);
        if (index > SPLITS - 1) index = SPLITS - 1;
        ++bin[index];
        box_add_box(&bbox[index], &pbox[pr[i].idx]);
    }
    box_add_box(&rbox[SPLITS - 2], &bbox[SPLITS - 1]);
    for (int i = SPLITS - 3; i >= 0; i--) {
        obox u = rbox[i + 1];
        box_add_box(&u, &bbox[i + 1]);
        rbox[i] = u;
    }
    unsigned left = bin[0];
    obox lbox = bbox[0];
    float pos = split_delta + split_start;
    const float node_area = box_half_area(node_box);
    for (int i = 0; i < SPLITS - 1; i++) {
        const unsigned right = primitive_num - left;
        const float sah_value =
            ((float)left * box_half_area(&lbox) + (float)right * box_half_area(&rbox[i])) / node_area;
        if (sah_value < min_sah) {
            min_sah = sah_value;
            *split_pos = pos;
        }
        left += bin[i + 1];
        box_add_box(&lbox, &bbox[i + 1]);
        pos += split_delta;
    }
    return min_sah;
}

/* std::partition over a bidirectional range, as libstdc++ implements it: scan
 * from the front for an element failing the predicate, from the back for one
 * passing it, swap, repeat. Returns the partition point. */
static int64_t partition_by(bprim* pr, int64_t first, int64_t last, int axis, float split_pos) {
    for (;;) {
        for (;;) {
            if (first == last) return first;
            if (pr[first].c[axis] < split_pos)
                ++first;
            else
                break;
        }
        --last;
        for (;;) {
            if (first == last) return first;
            if (!(pr[last].c[axis] < split_pos))
                --last;
            else
                break;
        }
        bprim tmp = pr[first];
        pr[first] = pr[last];
        pr[last] = tmp;
        ++first;
    }
}

static obox range_box(const bprim* pr, const obox* pbox, int64_t start, int64_t cnt) {
    obox b;
    box_empty(&b);
    for (int64_t i = start; i < start + cnt; ++i) box_add_box(&b, &pbox[pr[i].idx]);
    return b;
}

typedef struct {
    int64_t s[32], e[32];
    int head, tail;
} rqueue;
static void q_push(rqueue* q, int64_t s, int64_t e) {
    q->s[q->tail] = s;
    q->e[q->tail] = e;
    q->tail++;
}
static int q_size(const rqueue* q) { return q->tail - q->head; }

static void make_leaf(orc_tree* t, int node, int64_t start, int64_t end, int depth) {
    onode* n = &t->nodes[node];
    n->pri_cnt = (int32_t)(end - start);
    n->pri_offset = (int32_t)start;
    n->child_cnt = 0;
    if (depth > t->depth) t->depth = depth;
}

/* splitNode (accel/fast_bvh.hpp:138-211). */
static void split_node(orc_tree* t, bprim* pr, int node, const obox* node_box, int depth) {
    const int W = t->width;
    const int64_t start = t->nodes[node].pri_offset;
    const int64_t end = start + t->nodes[node].pri_cnt;
    if (t->nodes[node].pri_cnt <= t->max_leaf || depth == t->max_depth) {
        make_leaf(t, node, start, end, depth);
        return;
    }
    rqueue to_split = {{0}, {0}, 0, 0}, done = {{0}, {0}, 0, 0};
    q_push(&to_split, start, end);
    while (q_size(&to_split) > 0 && q_size(&to_split) + q_size(&done) < W) {
        const int64_t s = to_split.s[to_split.head], e = to_split.e[to_split.head];
        to_split.head++;
        const unsigned prim_cnt = (unsigned)(e - s);
        int axis = 0;
        float split_pos = 0.0f;
        const float sah = pick_best_split(&axis, &split_pos, pr, t->pbox, node_box, s, e);
        if (sah >= (float)prim_cnt || prim_cnt <= (unsigned)t->max_leaf) {
            q_push(&done, s, e);
        } else {
            const int64_t mid = partition_by(pr, s, e, axis, split_pos);
            if (mid == s || mid == e) {
                q_push(&done, s, e);
            } else {
                q_push(&to_split, s, mid);
                q_push(&to_split, mid, e);
            }
        }
    }
    if (q_size(&to_split) + q_size(&done) == 1) {
        make_leaf(t, node, start, end, depth);
        return;
    }
    int kids[8];
    int cnt = 0;
    for (int i = to_split.head; i < to_split.tail; ++i) {
        const int c = new_node(t);
        t->nodes[c].pri_offset = (int32_t)to_split.s[i];
        t->nodes[c].pri_cnt = (int32_t)(to_split.e[i] - to_split.s[i]);
        kids[cnt++] = c;
    }
    for (int i = done.head; i < done.tail; ++i) {
        const int c = new_node(t);
        t->nodes[c].pri_offset = (int32_t)done.s[i];
        t->nodes[c].pri_cnt = (int32_t)(done.e[i] - done.s[i]);
        kids[cnt++] = c;
    }
    t->nodes[node].child_cnt = cnt;
    for (int j = 0; j < cnt; ++j) t->nodes[node].child[j] = kids[j];
    for (int j = 0; j < cnt; ++j) {
        const obox cb = range_box(pr, t->pbox, t->nodes[kids[j]].pri_offset, t->nodes[kids[j]].pri_cnt);
        split_node(t, pr, kids[j], &cb, depth + 1);
    }
    /* calcBoundingBoxSIMD (fast_bvh.hpp:273-302): empty lanes keep the default box. */
    onode* n = &t->nodes[node];
    for (int j = 0; j < 8; ++j)
        for (int k = 0; k < 3; ++k) {
            n->lo[k][j] = FLT_MAX;
            n->hi[k][j] = -FLT_MAX;
        }
    for (int j = 0; j < cnt; ++j) {
        const obox cb = range_box(pr, t->pbox, t->nodes[n->child[j]].pri_offset, t->nodes[n->child[j]].pri_cnt);
        for (int k = 0; k < 3; ++k) {
            n->lo[k][j] = cb.mn[k];
            n->hi[k][j] = cb.mx[k];
        }
    }
}

orc_tree* orc_build(int width, const float* tri, int64_t ntri, int max_depth, int max_leaf) {
    if ((width != 4 && width != 8) || ntri < 0) return NULL;
    orc_tree* t = (orc_tree*)calloc(1, sizeof(orc_tree));
    t->width = width;
    t->max_depth = max_depth;
    t->max_leaf = max_leaf;
    t->ntri = ntri;
    t->tri_copy = (float*)malloc((size_t)(ntri > 0 ? ntri : 1) * 9 * sizeof(float));
    if (ntri > 0) memcpy(t->tri_copy, tri, (size_t)ntri * 9 * sizeof(float));
    t->tri = t->tri_copy;
    t->root = -1;
    t->pbox = (obox*)malloc((size_t)(ntri > 0 ? ntri : 1) * sizeof(obox));
    box_empty(&t->scene);
    for (int64_t i = 0; i < ntri; ++i) {
        box_empty(&t->pbox[i]);
        for (int k = 0; k < 3; ++k) box_add_point(&t->pbox[i], tri + i * 9 + 3 * k);
        box_add_box(&t->scene, &t->pbox[i]);
    }
    {   /* core/scene.cpp:150-154 */
        const float threshold = 0.001f;
        float delta[3];
        for (int k = 0; k < 3; ++k) delta[k] = (t->scene.mx[k] - t->scene.mn[k]) * threshold;
        for (int k = 0; k < 3; ++k) {
            t->scene.mn[k] -= delta[k];
            t->scene.mx[k] += delta[k];
        }
    }
    if (ntri == 0) return t;
    bprim* pr = (bprim*)malloc((size_t)ntri * sizeof(bprim));
    for (int64_t i = 0; i < ntri; ++i) {
        pr[i].idx = (int32_t)i;
        for (int k = 0; k < 3; ++k) pr[i].c[k] = (t->pbox[i].mx[k] + t->pbox[i].mn[k]) * 0.5f;
    }
    t->root = new_node(t);
    t->nodes[t->root].pri_offset = 0;
    t->nodes[t->root].pri_cnt = (int32_t)ntri;
    split_node(t, pr, t->root, &t->scene, 1);
    t->order = (int32_t*)malloc((size_t)ntri * sizeof(int32_t));
    for (int64_t i = 0; i < ntri; ++i) t->order[i] = pr[i].idx;
    free(pr);
    return t;
}

void orc_free(orc_tree* t) {
    if (!t) return;
    free(t->tri_copy);
    free(t->pbox);
    free(t->order);
    free(t->nodes);
    free(t);
}

static void topo_rec(const orc_tree* t, int node, int32_t* out, int64_t cap, int64_t* k) {
    const onode* n = &t->nodes[node];
    if (*k < cap) out[*k] = n->child_cnt;
    (*k)++;
    if (n->child_cnt == 0) {
        if (*k < cap) out[*k] = n->pri_cnt;
        (*k)++;
        for (int32_t i = 0; i < n->pri_cnt; ++i) {
            if (*k < cap) out[*k] = t->order[n->pri_offset + i];
            (*k)++;
        }
        return;
    }
    for (int j = 0; j < n->child_cnt; ++j) topo_rec(t, n->child[j], out, cap, k);
}

int64_t orc_topology(const orc_tree* t, int32_t* out, int64_t cap) {
    if (t->root < 0) return 0;
    int64_t k = 0;
    topo_rec(t, t->root, out, cap, &k);
    return k <= cap ? k : -k;
}

int orc_depth(const orc_tree* t) { return t->depth; }

void orc_scene_bbox(const orc_tree* t, float* out6) {
    for (int k = 0; k < 3; ++k) {
        out6[k] = t->scene.mn[k];
        out6[3 + k] = t->scene.mx[k];
    }
}

/* ------------------------------------------------------------------------- */
/* Ray setup                                                                 */

typedef struct {
    float o[3], d[3], tmin, tmax;
    float rcp[3], ori_dir[3];          /* resolveRayData */
    int lx, ly, lz;                    /* Ray::Prepare */
    float sx, sy, sz;
} oray;

static float sgn(float x) { return x < 0.0f ? -1.0f : 1.0f; }

static void prepare_axes(const float* d, int* lx, int* ly, int* lz, float* sx, float* sy, float* sz) {
    int y;
    if (fabsf(d[0]) > fabsf(d[1]) && fabsf(d[0]) > fabsf(d[2]))
        y = 0;
    else
        y = fabsf(d[1]) > fabsf(d[2]) ? 1 : 2;
    const int z = (y + 1) % 3, x = (z + 1) % 3;
    *lx = x;
    *ly = y;
    *lz = z;
    *sx = -d[x] / d[y];
    *sz = -d[z] / d[y];
    *sy = 1.0f / d[y];
}

void orc_ray_prepare(const float* d, int* local_xyz, float* scale_xyz) {
    prepare_axes(d, &local_xyz[0], &local_xyz[1], &local_xyz[2], &scale_xyz[0], &scale_xyz[1], &scale_xyz[2]);
}

static void load_ray(oray* r, const float* rays, int64_t n, int64_t i) {
    for (int k = 0; k < 3; ++k) {
        r->o[k] = rays[k * n + i];
        r->d[k] = rays[(3 + k) * n + i];
    }
    r->tmin = rays[6 * n + i];
    r->tmax = rays[7 * n + i];
    const float delta = 0.00001f;
    for (int k = 0; k < 3; ++k) {
        const float dk = fabsf(r->d[k]) < delta ? sgn(r->d[k]) * delta : r->d[k];
        r->rcp[k] = 1.0f / dk;
        r->ori_dir[k] = -r->o[k] / dk;
    }
    prepare_axes(r->d, &r->lx, &r->ly, &r->lz, &r->sx, &r->sy, &r->sz);
}

/* Scalar Intersect(ray, bbox) (math/bbox.h:124-155). */
static float root_intersect(const oray* r, const obox* bb) {
    float tmax = r->tmax, tmin = r->tmin;
    for (int axis = 0; axis < 3; axis++) {
        if (r->d[axis] < 0.00001f && r->d[axis] > -0.00001f) {
            if (r->o[axis] > bb->mx[axis] || r->o[axis] < bb->mn[axis]) return -1.0f;
        } else {
            const float ood = 1.0f / r->d[axis];
            float t1 = (bb->mx[axis] - r->o[axis]) * ood;
            float t2 = (bb->mn[axis] - r->o[axis]) * ood;
            if (t1 > t2) {
                const float tt = t1;
                t1 = t2;
                t2 = tt;
            }
            tmin = std_max(t1, tmin);
            tmax = std_min(t2, tmax);
            if (tmin > tmax) return -1.0f;
        }
    }
    return tmin;
}

/* SSE/AVX min/max lane semantics: min(a, b) = a < b ? a : b. */
static float sse_min(float a, float b) { return a < b ? a : b; }
static float sse_max(float a, float b) { return a > b ? a : b; }

/* IntersectBBox_SIMD (simd/simd_bbox.h:62-85): fmin per child, -1 on a miss.
 * Returns the hit mask. */
static int node_boxes(const oray* r, const onode* n, float* fmin_out) {
    int mask = 0;
    for (int j = 0; j < 8; ++j) {
        float f_min = r->tmin, f_max = r->tmax;
        for (int k = 0; k < 3; ++k) {
            const float t1 = r->ori_dir[k] + r->rcp[k] * n->hi[k][j];
            const float t2 = r->ori_dir[k] + r->rcp[k] * n->lo[k][j];
            f_min = sse_max(f_min, sse_min(t1, t2));
            f_max = sse_min(f_max, sse_max(t1, t2));
        }
        const int valid = j < n->child_cnt;
        if (valid && f_min <= f_max) {
            mask |= 1 << j;
            fmin_out[j] = f_min;
        } else {
            fmin_out[j] = -1.0f;
        }
    }
    return mask;
}

/* One lane of intersectTriangleInner_SIMD (simd/simd_triangle.h:212-300). */
static int tri_test(const oray* r, const float* v, float* t_out, float* u_out, float* v_out) {
    float p[3][3];
    for (int i = 0; i < 3; ++i)
        for (int k = 0; k < 3; ++k) p[i][k] = v[i * 3 + k] - r->o[k];
    float px[3], py[3], pz[3];
    for (int i = 0; i < 3; ++i) {
        px[i] = p[i][r->lx];
        py[i] = p[i][r->ly];
        pz[i] = p[i][r->lz];
    }
    for (int i = 0; i < 3; ++i) {
        px[i] = py[i] * r->sx + px[i];
        pz[i] = py[i] * r->sz + pz[i];
    }
    const float e0 = px[1] * pz[2] - pz[1] * px[2];
    const float e1 = px[2] * pz[0] - pz[2] * px[0];
    const float e2 = px[0] * pz[1] - pz[0] * px[1];
    const int c0 = (e0 >= 0.0f) && (e1 >= 0.0f) && (e2 >= 0.0f);
    const int c1 = (e0 <= 0.0f) && (e1 <= 0.0f) && (e2 <= 0.0f);
    if (!(c0 || c1)) return 0;
    const float det = e0 + (e1 + e2);
    if (!(det != 0.0f)) return 0;
    const float rcp_det = 1.0f / det;
    for (int i = 0; i < 3; ++i) py[i] = py[i] * r->sy;
    float t = e0 * py[0];
    t = e1 * py[1] + t;
    t = e2 * py[2] + t;
    t = t * rcp_det;
    if (!(t > r->tmin && t <= r->tmax)) return 0;
    *t_out = t;
    *u_out = e1 * rcp_det;
    *v_out = e2 * rcp_det;
    return 1;
}

typedef struct {
    int32_t prim;
    float t, u, v;
    int64_t node_tests, prim_tests;
} ohit;

/* Fbvh::GetIntersect, SIMD branch (accel/fast_bvh.hpp:305-455). any != 0 runs
 * the query_shadow variant (opaque early exit, 362-373). Returns 1 on a hit. */
static int traverse(const orc_tree* t, const oray* r, int any, ohit* h, int32_t* stack_node, float* stack_t) {
    h->prim = -1;
    h->t = FLT_MAX;
    h->u = h->v = 0.0f;
    h->node_tests = h->prim_tests = 0;
    if (t->root < 0) return 0;
    const float f0 = root_intersect(r, &t->scene);
    if (f0 < 0.0f) return 0;
    int si = 0;
    stack_node[si] = t->root;
    stack_t[si] = f0;
    si++;
    while (si > 0) {
        --si;
        const onode* n = &t->nodes[stack_node[si]];
        const float fmin = stack_t[si];
        if (h->t < fmin) continue;
        if (n->child_cnt == 0) {
            for (int32_t i = 0; i < n->pri_cnt; ++i) {
                const int32_t prim = t->order[n->pri_offset + i];
                float tt, uu, vv;
                if (tri_test(r, t->tri + (int64_t)prim * 9, &tt, &uu, &vv) && tt < h->t) {
                    h->t = tt;
                    h->u = uu;
                    h->v = vv;
                    h->prim = prim;
                    if (any) {
                        h->prim_tests += n->pri_cnt;
                        return 1;
                    }
                }
            }
            h->prim_tests += n->pri_cnt;
            continue;
        }
        h->node_tests++;
        float fm[8];
        int m = node_boxes(r, n, fm);
        if (m == 0) continue;
        int k0 = __builtin_ctz((unsigned)m);
        const float t0 = fm[k0];
        m &= m - 1;
        if (m == 0) {
            stack_node[si] = n->child[k0];
            stack_t[si] = t0;
            si++;
        } else {
            const int k1 = __builtin_ctz((unsigned)m);
            m &= m - 1;
            if (m == 0) {
                const float t1 = fm[k1];
                if (t0 < t1) {
                    stack_node[si] = n->child[k1]; stack_t[si] = t1; si++;
                    stack_node[si] = n->child[k0]; stack_t[si] = t0; si++;
                } else {
                    stack_node[si] = n->child[k0]; stack_t[si] = t0; si++;
                    stack_node[si] = n->child[k1]; stack_t[si] = t1; si++;
                }
            } else {
                for (int i = 0; i < n->child_cnt; ++i) {
                    int k = -1;
                    float max_dist = -1.0f;
                    for (int j = 0; j < n->child_cnt; ++j)
                        if (fm[j] > max_dist) {
                            max_dist = fm[j];
                            k = j;
                        }
                    if (k == -1) break;
                    fm[k] = -1.0f;
                    stack_node[si] = n->child[k];
                    stack_t[si] = max_dist;
                    si++;
                }
            }
        }
    }
    return h->prim >= 0;
}

/* ------------------------------------------------------------------------- */
/* Threaded drivers                                                          */

typedef struct {
    const orc_tree* t;
    const float* rays;
    int64_t n;
    int mode; /* 0 closest, 1 any, 2 count-closest, 3 count-any */
    int32_t* prim;
    float *tt, *u, *v;
    uint8_t* occ;
    int64_t node_tests, prim_tests;
    int64_t* next;
    pthread_mutex_t* lock;
} job;

static void* worker(void* arg) {
    job* j = (job*)arg;
    const int64_t chunk = 4096;
    const int ssize = j->t->depth * j->t->width + j->t->width + 8;
    int32_t* sn = (int32_t*)malloc((size_t)ssize * sizeof(int32_t));
    float* st = (float*)malloc((size_t)ssize * sizeof(float));
    for (;;) {
        pthread_mutex_lock(j->lock);
        const int64_t s = *j->next;
        *j->next += chunk;
        pthread_mutex_unlock(j->lock);
        if (s >= j->n) break;
        const int64_t e = s + chunk < j->n ? s + chunk : j->n;
        for (int64_t i = s; i < e; ++i) {
            oray r;
            ohit h;
            load_ray(&r, j->rays, j->n, i);
            const int any = (j->mode == 1 || j->mode == 3);
            const int hit = traverse(j->t, &r, any, &h, sn, st);
            if (j->mode == 0) {
                j->prim[i] = h.prim;
                j->tt[i] = h.prim >= 0 ? h.t : FLT_MAX;
                j->u[i] = h.prim >= 0 ? h.u : 0.0f;
                j->v[i] = h.prim >= 0 ? h.v : 0.0f;
            } else if (j->mode == 1) {
                j->occ[i] = (uint8_t)(hit ? 1 : 0);
            } else {
                j->node_tests += h.node_tests;
                j->prim_tests += h.prim_tests;
            }
        }
    }
    free(sn);
    free(st);
    return NULL;
}

static void run(job* proto, int nthreads) {
    if (nthreads <= 0) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    pthread_t th[256];
    job jobs[256];
    int64_t next = 0;
    pthread_mutex_t lock;
    pthread_mutex_init(&lock, NULL);
    for (int i = 0; i < nthreads; ++i) {
        jobs[i] = *proto;
        jobs[i].next = &next;
        jobs[i].lock = &lock;
        jobs[i].node_tests = jobs[i].prim_tests = 0;
        pthread_create(&th[i], NULL, worker, &jobs[i]);
    }
    proto->node_tests = proto->prim_tests = 0;
    for (int i = 0; i < nthreads; ++i) {
        pthread_join(th[i], NULL);
        proto->node_tests += jobs[i].node_tests;
        proto->prim_tests += jobs[i].prim_tests;
    }
    pthread_mutex_destroy(&lock);
}

void orc_trace_closest(const orc_tree* t, const float* rays, int64_t n, int32_t* prim, float* tt, float* u, float* v,
                       int nthreads) {
    job j;
    memset(&j, 0, sizeof(j));
    j.t = t; j.rays = rays; j.n = n; j.mode = 0; j.prim = prim; j.tt = tt; j.u = u; j.v = v;
    run(&j, nthreads);
}

void orc_trace_any(const orc_tree* t, const float* rays, int64_t n, uint8_t* occluded, int nthreads) {
    job j;
    memset(&j, 0, sizeof(j));
    j.t = t; j.rays = rays; j.n = n; j.mode = 1; j.occ = occluded;
    run(&j, nthreads);
}

void orc_count(const orc_tree* t, const float* rays, int64_t n, int any, int64_t* node_tests, int64_t* prim_tests,
               int nthreads) {
    job j;
    memset(&j, 0, sizeof(j));
    j.t = t; j.rays = rays; j.n = n; j.mode = any ? 3 : 2;
    run(&j, nthreads);
    *node_tests = j.node_tests;
    *prim_tests = j.prim_tests;
}

int orc_tri_test(const float* tri, int64_t prim, const float* rays, int64_t n, int64_t i, float* t_out) {
    oray r;
    float u, v;
    load_ray(&r, rays, n, i);
    return tri_test(&r, tri + prim * 9, t_out, &u, &v);
}

double orc_fp64_intersect(const float* tri, int64_t prim, const float* rays, int64_t n, int64_t i) {
    double o[3], d[3], p[3][3];
    for (int k = 0; k < 3; ++k) {
        o[k] = rays[k * n + i];
        d[k] = rays[(3 + k) * n + i];
    }
    int y;
    if (fabs(d[0]) > fabs(d[1]) && fabs(d[0]) > fabs(d[2]))
        y = 0;
    else
        y = fabs(d[1]) > fabs(d[2]) ? 1 : 2;
    const int z = (y + 1) % 3, x = (z + 1) % 3;
    const double sx = -d[x] / d[y], sz = -d[z] / d[y], sy = 1.0 / d[y];
    double px[3], py[3], pz[3];
    for (int a = 0; a < 3; ++a) {
        for (int k = 0; k < 3; ++k) p[a][k] = (double)tri[prim * 9 + a * 3 + k] - o[k];
        px[a] = p[a][x] + sx * p[a][y];
        pz[a] = p[a][z] + sz * p[a][y];
        py[a] = p[a][y] * sy;
    }
    const double e0 = px[1] * pz[2] - pz[1] * px[2];
    const double e1 = px[2] * pz[0] - pz[2] * px[0];
    const double e2 = px[0] * pz[1] - pz[0] * px[1];
    if ((e0 < 0 || e1 < 0 || e2 < 0) && (e0 > 0 || e1 > 0 || e2 > 0)) return -1.0;
    const double det = e0 + e1 + e2;
    if (det == 0.0) return -1.0;
    return (e0 * py[0] + e1 * py[1] + e2 * py[2]) / det;
}

void orc_fp64_t_batch(const float* tri, const int32_t* prim, const float* rays, int64_t n, double* t_out) {
    for (int64_t i = 0; i < n; ++i) t_out[i] = prim[i] >= 0 ? orc_fp64_intersect(tri, prim[i], rays, n, i) : -1.0;
}
