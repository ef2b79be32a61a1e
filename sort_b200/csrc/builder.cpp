// Wide-BVH builder with SORT's Fbvh::Build split rules (see builder.h).
#include "builder.h"

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cstring>
#include <future>
#include <memory>
#include <stdexcept>
#include <thread>

namespace sg {
namespace {

// libstdc++'s std::min / std::max argument order matters for signed zeros, so
// they are spelled out: min(a, b) = b < a ? b : a; max(a, b) = a < b ? b : a.
inline float smin(float a, float b) { return (b < a) ? b : a; }
inline float smax(float a, float b) { return (a < b) ? b : a; }

inline Box empty_box() {
    Box b;
    for (int k = 0; k < 3; ++k) {
        b.mn[k] = FLT_MAX;
        b.mx[k] = -FLT_MAX;
    }
    return b;
}
// BBox::Union(const Point&) (math/bbox.cpp:106-113).
inline void add_point(Box& b, const float* p) {
    for (int k = 0; k < 3; ++k) {
        if (p[k] < b.mn[k]) b.mn[k] = p[k];
        if (p[k] > b.mx[k]) b.mx[k] = p[k];
    }
}
// BBox::Union(const BBox&) (math/bbox.cpp:115-120).
inline void add_box(Box& b, const Box& o) {
    for (int k = 0; k < 3; ++k) {
        b.mn[k] = smin(b.mn[k], o.mn[k]);
        b.mx[k] = smax(b.mx[k], o.mx[k]);
    }
}
inline float half_area(const Box& b) {
    const float ox = b.mx[0] - b.mn[0], oy = b.mx[1] - b.mn[1], oz = b.mx[2] - b.mn[2];
    const float a = ox * oy;
    const float c = oy * oz;
    const float e = oz * ox;
    return (a + c) + e;
}
inline int max_axis(const Box& b) {
    const float ox = b.mx[0] - b.mn[0], oy = b.mx[1] - b.mn[1], oz = b.mx[2] - b.mn[2];
    if (ox > oy && ox > oz) return 0;
    if (oy > ox && oy > oz) return 1;
    return 2;
}

struct Prim {  // Bvh_Primitive (accel/bvh_utils.h:27-45): centroid + primitive
    float c[3];
    int32_t idx;
};

struct TNode {
    int64_t off = 0, cnt = 0;
    int nkids = 0;
    std::unique_ptr<TNode> kids[8];
    Box kid_box[8];
};

struct Ctx {
    BuildParams p;
    const Box* pbox = nullptr;
    Prim* prims = nullptr;
    std::atomic<int> depth{0};
    std::atomic<int> free_threads{0};
};

// 16-bin SAH split search (accel/bvh_utils.h:69-118).
float pick_best_split(int& axis, float& split_pos, const Ctx& c, const Box& node_box, int64_t start, int64_t end) {
    constexpr int kBins = 16;
    const float inv_bins = 1.0f / float(kBins);
    Box inner = empty_box();
    for (int64_t i = start; i < end; ++i) add_point(inner, c.prims[i].c);
    const unsigned n = unsigned(end - start);
    axis = max_axis(inner);
    float min_sah = FLT_MAX;
    unsigned bin[kBins];
    Box bbox[kBins], rbox[kBins - 1];
    std::memset(bin, 0, sizeof(bin));
    for (auto& b : bbox) b = empty_box();
    for (auto& b : rbox) b = empty_box();
    const float split_start = inner.mn[axis];
    const float split_delta = (inner.mx[axis] - inner.mn[axis]) * inv_bins;
    if (split_delta == 0.0f) return FLT_MAX;
    const float inv_split_delta = 1.0f / split_delta;
    for (int64_t i = start; i < end; ++i) {
        const float d = c.prims[i].c[axis] - split_start;
        int index = int(d * inv_split_delta);
        index = std::min(index, kBins - 1);
        ++bin[index];
        add_box(bbox[index], c.pbox[c.prims[i].idx]);
    }
    add_box(rbox[kBins - 2], bbox[kBins - 1]);
    for (int i = kBins - 3; i >= 0; i--) {
        Box u = rbox[i + 1];
        add_box(u, bbox[i + 1]);
        rbox[i] = u;
    }
    unsigned left = bin[0];
    Box lbox = bbox[0];
    float pos = split_delta + split_start;
    const float node_area = half_area(node_box);
    for (int i = 0; i < kBins - 1; i++) {
        const float l = float(left) * half_area(lbox);
        const float r = float(n - left) * half_area(rbox[i]);
        const float sah = (l + r) / node_area;
        if (sah < min_sah) {
            min_sah = sah;
            split_pos = pos;
        }
        left += bin[i + 1];
        add_box(lbox, bbox[i + 1]);
        pos += split_delta;
    }
    return min_sah;
}

Box range_box(const Ctx& c, int64_t off, int64_t cnt) {
    Box b = empty_box();
    for (int64_t i = off; i < off + cnt; ++i) add_box(b, c.pbox[c.prims[i].idx]);
    return b;
}

struct Range {
    int64_t s, e;
};

// splitNode (accel/fast_bvh.hpp:138-211).
void split_node(Ctx& c, TNode* node, const Box& node_box, int depth) {
    const int W = c.p.width;
    const int64_t start = node->off, end = node->off + node->cnt;
    if (node->cnt <= c.p.max_leaf || depth == c.p.max_depth) {
        int d = c.depth.load();
        while (depth > d && !c.depth.compare_exchange_weak(d, depth)) {
        }
        return;
    }
    Range to_split[32], done[32];
    int ts_head = 0, ts_tail = 0, dn_tail = 0;
    to_split[ts_tail++] = {start, end};
    while (ts_tail > ts_head && (ts_tail - ts_head) + dn_tail < W) {
        const Range cur = to_split[ts_head++];
        const unsigned prim_cnt = unsigned(cur.e - cur.s);
        int axis = 0;
        float split_pos = 0.0f;
        const float sah = pick_best_split(axis, split_pos, c, node_box, cur.s, cur.e);
        if (sah >= float(prim_cnt) || prim_cnt <= unsigned(c.p.max_leaf)) {
            done[dn_tail++] = cur;
        } else {
            Prim* mid_ptr = std::partition(c.prims + cur.s, c.prims + cur.e,
                                           [axis, split_pos](const Prim& p) { return p.c[axis] < split_pos; });
            const int64_t mid = mid_ptr - c.prims;
            if (mid == cur.s || mid == cur.e) {
                done[dn_tail++] = cur;
            } else {
                to_split[ts_tail++] = {cur.s, mid};
                to_split[ts_tail++] = {mid, cur.e};
            }
        }
    }
    if ((ts_tail - ts_head) + dn_tail == 1) {
        int d = c.depth.load();
        while (depth > d && !c.depth.compare_exchange_weak(d, depth)) {
        }
        return;
    }
    for (int i = ts_head; i < ts_tail; ++i) {
        auto k = std::make_unique<TNode>();
        k->off = to_split[i].s;
        k->cnt = to_split[i].e - to_split[i].s;
        node->kids[node->nkids++] = std::move(k);
    }
    for (int i = 0; i < dn_tail; ++i) {
        auto k = std::make_unique<TNode>();
        k->off = done[i].s;
        k->cnt = done[i].e - done[i].s;
        node->kids[node->nkids++] = std::move(k);
    }
    // Children only permute their own ranges, so they can be built concurrently.
    constexpr int64_t kGrain = 1 << 15;
    std::future<void> pending[8];
    for (int j = 0; j < node->nkids; ++j) {
        TNode* kid = node->kids[j].get();
        const Box kb = range_box(c, kid->off, kid->cnt);
        bool spawned = false;
        if (kid->cnt >= kGrain) {
            int f = c.free_threads.load();
            while (f > 0 && !c.free_threads.compare_exchange_weak(f, f - 1)) {
            }
            if (f > 0) {
                pending[j] = std::async(std::launch::async, [&c, kid, kb, depth]() {
                    split_node(c, kid, kb, depth + 1);
                    c.free_threads.fetch_add(1);
                });
                spawned = true;
            }
        }
        if (!spawned) split_node(c, kid, kb, depth + 1);
    }
    for (int j = 0; j < node->nkids; ++j)
        if (pending[j].valid()) pending[j].get();
    // calcBoundingBoxSIMD (fast_bvh.hpp:273-302), after the children settled.
    for (int j = 0; j < node->nkids; ++j) node->kid_box[j] = range_box(c, node->kids[j]->off, node->kids[j]->cnt);
}

struct Flattener {
    BuiltTree& t;
    const Ctx& c;
    int W;
    int32_t alloc(int n) {
        const int32_t base = int32_t(t.first_interior.size());
        t.first_interior.resize(t.first_interior.size() + n, -1);
        t.child.resize(t.child.size() + size_t(n) * W, kEmptyRef);
        t.lo.resize(t.lo.size() + size_t(n) * 3 * W, FLT_MAX);
        t.hi.resize(t.hi.size() + size_t(n) * 3 * W, -FLT_MAX);
        return base;
    }
    void leaf(const TNode* n) {
        t.leaves++;
        t.leaf_last[size_t(n->off + n->cnt - 1)] = 1;
    }
    void fill(const TNode* n, int32_t idx) {
        int interior = 0;
        for (int j = 0; j < n->nkids; ++j) interior += n->kids[j]->nkids > 0;
        const int32_t base = interior ? alloc(interior) : -1;
        t.first_interior[idx] = base;
        int k = 0;
        for (int j = 0; j < n->nkids; ++j) {
            const TNode* kid = n->kids[j].get();
            int32_t ref;
            if (kid->nkids == 0) {
                ref = leaf_ref(kid->off);
                leaf(kid);
            } else {
                ref = base + k++;
            }
            t.child[size_t(idx) * W + j] = ref;
            for (int a = 0; a < 3; ++a) {
                t.lo[(size_t(idx) * 3 + a) * W + j] = n->kid_box[j].mn[a];
                t.hi[(size_t(idx) * 3 + a) * W + j] = n->kid_box[j].mx[a];
            }
        }
        k = 0;
        for (int j = 0; j < n->nkids; ++j)
            if (n->kids[j]->nkids > 0) fill(n->kids[j].get(), base + k++);
    }
};

}  // namespace

BuiltTree build_tree(const float* tri, int64_t ntri_in, const BuildParams& p) {
    if (p.width != 4 && p.width != 8) throw std::invalid_argument("width must be 4 or 8");
    if (p.max_leaf < 1 || p.max_depth < 1) throw std::invalid_argument("max_leaf and max_depth must be >= 1");
    if (p.nextra < 0 || (p.nextra > 0 && !p.extra_boxes)) throw std::invalid_argument("bad extra primitive boxes");
    const int64_t ntri = ntri_in + p.nextra;  // every primitive: triangles, then the extra ones
    if (ntri_in < 0 || ntri >= int64_t(0x7fffffff)) throw std::invalid_argument("triangle count out of range");
    BuiltTree t;
    t.width = p.width;
    const int nthreads = p.threads > 0 ? p.threads : int(std::max(1u, std::thread::hardware_concurrency()));

    // Primitive boxes (Triangle::GetBBox, shape/triangle.cpp:116-136), centroids,
    // and the scene box (core/scene.cpp:146-154).
    std::vector<Box> pbox(size_t(std::max<int64_t>(ntri, 1)));
    std::vector<Prim> prims(size_t(std::max<int64_t>(ntri, 1)));
    {
        std::vector<std::thread> pool;
        const int64_t per = (ntri + nthreads - 1) / std::max(1, nthreads);
        for (int w = 0; w < nthreads; ++w) {
            const int64_t s = w * per, e = std::min(ntri, s + per);
            if (s >= e) break;
            pool.emplace_back([&, s, e]() {
                for (int64_t i = s; i < e; ++i) {
                    Box b = empty_box();
                    if (i < ntri_in) {
                        for (int k = 0; k < 3; ++k) add_point(b, tri + i * 9 + 3 * k);
                    } else {  // Line::GetBBox (shape/line.cpp:98-106), computed by the caller
                        const float* x = p.extra_boxes + (i - ntri_in) * 6;
                        for (int k = 0; k < 3; ++k) {
                            b.mn[k] = x[k];
                            b.mx[k] = x[3 + k];
                        }
                    }
                    pbox[size_t(i)] = b;
                    Prim& pr = prims[size_t(i)];
                    for (int k = 0; k < 3; ++k) pr.c[k] = (b.mx[k] + b.mn[k]) * 0.5f;
                    pr.idx = int32_t(i);
                }
            });
        }
        for (auto& th : pool) th.join();
    }
    Box scene = empty_box();
    for (int64_t i = 0; i < ntri; ++i) add_box(scene, pbox[size_t(i)]);
    {
        const float threshold = 0.001f;
        float delta[3];
        for (int k = 0; k < 3; ++k) delta[k] = (scene.mx[k] - scene.mn[k]) * threshold;
        for (int k = 0; k < 3; ++k) {
            scene.mn[k] -= delta[k];
            scene.mx[k] += delta[k];
        }
    }
    t.scene = scene;
    if (p.nextra > 0) t.first_extra = ntri_in;
    if (ntri == 0) return t;

    Ctx c;
    c.p = p;
    c.pbox = pbox.data();
    c.prims = prims.data();
    c.free_threads = nthreads - 1;
    TNode root;
    root.off = 0;
    root.cnt = ntri;
    split_node(c, &root, scene, 1);
    t.depth = c.depth.load();

    t.order.resize(size_t(ntri));
    t.leaf_last.assign(size_t(ntri), 0);
    for (int64_t i = 0; i < ntri; ++i) {
        t.order[size_t(i)] = prims[size_t(i)].idx;
    }
    Flattener f{t, c, p.width};
    if (root.nkids == 0) {
        t.root = leaf_ref(0);
        f.leaf(&root);
    } else {
        t.root = f.alloc(1);
        f.fill(&root, t.root);
    }
    return t;
}

namespace {
void topo_rec(const BuiltTree& t, int32_t ref, std::vector<int32_t>& out) {
    if (ref_is_leaf(ref)) {
        out.push_back(0);
        const size_t cnt_pos = out.size();
        out.push_back(0);
        const int64_t b = leaf_begin(ref);
        int64_t e = b;
        while (!t.leaf_last[size_t(e)]) ++e;
        int32_t n = 0;
        auto kind = [&](int32_t p) {
            if (t.first_extra < 0 || p < t.first_extra) return 0;
            return (t.first_shape >= 0 && p >= t.first_shape) ? 2 : 1;
        };
        for (int pass = 0; pass < 3; ++pass)  // triangles, lines, area shapes
            for (int64_t i = b; i <= e; ++i) {
                if (kind(t.order[size_t(i)]) != pass) continue;
                out.push_back(t.order[size_t(i)]);
                ++n;
            }
        out[cnt_pos] = n;
        return;
    }
    const int W = t.width;
    int cnt = 0;
    while (cnt < W && t.child[size_t(ref) * W + cnt] != kEmptyRef) ++cnt;
    out.push_back(cnt);
    for (int j = 0; j < cnt; ++j) topo_rec(t, t.child[size_t(ref) * W + j], out);
}
}  // namespace

void tree_topology(const BuiltTree& t, std::vector<int32_t>& out) {
    out.clear();
    if (t.root == kEmptyRef) return;
    topo_rec(t, t.root, out);
}

}  // namespace sg
