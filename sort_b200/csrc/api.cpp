// C ABI of libsortgpu (include/sortgpu.h): scene build + upload, batched
// closest-hit / any-hit launches, host-buffer forms and error reporting.
#include "sortgpu.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "builder.h"
#include "hair.h"
#include "scene_access.h"
#include "staged_upload.h"
#include "trace_kernels.h"

namespace {

thread_local std::string g_last_error;

sg_status fail(sg_status s, const std::string& msg) {
    g_last_error = msg;
    return s;
}

sg_status cuda_fail(cudaError_t e, const char* what) {
    return fail(SG_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// Restores the caller's current device on scope exit.
struct DeviceGuard {
    int prev = -1;
    bool ok = false;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) return;
        ok = cudaSetDevice(dev) == cudaSuccess;
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

}  // namespace

struct sg_scene {
    int device = 0;
    int width = 8;
    int node_format = SG_NODES_FP32;
    int stack_need = 1;
    sg::TraceTuning tuning;
    sg::BuiltTree tree;  // host copy of the topology (slot boxes released after upload)
    float4* d_nodes = nullptr;
    float4* d_tris = nullptr;
    int* d_err = nullptr;
    unsigned long long* d_stats = nullptr;
    // Ray counters of the persistent schedule: each launch zeroes and uses the
    // next slot, so up to kCounterSlots launches on this scene may be in flight
    // on different streams at once.
    static constexpr int kCounterSlots = 64;
    unsigned long long* d_counters = nullptr;
    std::atomic<unsigned> next_counter{0};
    int64_t device_bytes = 0;
    double build_seconds = 0.0;
    // Scratch for the host-buffer entry points, grown on demand.
    std::mutex scratch_lock;
    void* d_scratch = nullptr;
    size_t scratch_bytes = 0;
    cudaStream_t stream = nullptr;  // host-buffer calls: copies in
    // Host-buffer calls pipeline chunks: copies in on `stream`, kernels on two
    // alternating streams (a chunk's tail overlaps the next chunk's start),
    // copies out on a fourth; one event per chunk and stage.
    static constexpr int kMaxChunks = 16;
    // Chunks go round these streams, so the tail of one chunk's launch overlaps
    // the next chunks' (4 measured 1% faster than 2 on 16 chunks of 262k rays).
    static constexpr int kTraceStreams = 4;
    cudaStream_t trace_stream[kTraceStreams] = {};
    cudaStream_t out_stream = nullptr;
    cudaEvent_t in_done[kMaxChunks] = {};
    cudaEvent_t trace_done[kMaxChunks] = {};
    int32_t* d_material = nullptr;  // per primitive, for sg_trace_multi_host (sg_scene_set_materials)
    float4* d_lines = nullptr;      // line records, then area-shape records (hair.h): primitives ntri ..
    int64_t n_lines = 0, n_shapes = 0;
};

namespace {

// Slot records in leaf order (layout.h); with hair lines (line_recs, 20 floats
// each, primitives ntri ..), a leaf's triangles come before its lines, each in
// leaf order, as SORT tests its triangle packs before its line packs.
sg_status upload(sg_scene* s, const float* tri, int64_t ntri, const std::vector<float>& line_recs = {},
                 int64_t nlines = 0, int64_t nshapes = 0) {
    const sg::BuiltTree& t = s->tree;
    const int W = t.width;
    const int f4 = W == 8 ? sg::NodeShape<8>::kF4 : sg::NodeShape<4>::kF4;
    const int64_t nn = t.interior();
    std::vector<float4> nodes;
    if (t.d_nodes && s->node_format != SG_NODES_FP32 && t.host_arrays()) {  // 8-bit nodes come from the host arrays
        cudaFree(t.d_nodes);
        s->tree.d_nodes = nullptr;
    }
    const bool adopt = t.d_nodes != nullptr;  // a GPU builder wrote the nodes on the device
    if (adopt) {
    } else if (s->node_format == SG_NODES_QUANT8) {
        sg::quantize_nodes(t, nodes);
    } else {
        nodes.assign(size_t(std::max<int64_t>(nn, 1)) * f4, make_float4(0.0f, 0.0f, 0.0f, 0.0f));
    }
    const int Q = W / 4;  // float4 per plane
    for (int64_t k = 0; !adopt && s->node_format == SG_NODES_FP32 && k < nn; ++k) {
        float* base = reinterpret_cast<float*>(&nodes[size_t(k) * f4]);
        for (int a = 0; a < 3; ++a)
            for (int j = 0; j < W; ++j) {
                base[(2 * a) * Q * 4 + j] = t.lo[(size_t(k) * 3 + a) * W + j];
                base[(2 * a + 1) * Q * 4 + j] = t.hi[(size_t(k) * 3 + a) * W + j];
            }
        int32_t* ch = reinterpret_cast<int32_t*>(base + 6 * Q * 4);
        for (int j = 0; j < W; ++j) ch[j] = t.child[size_t(k) * W + j];
    }
    const size_t nb = adopt ? size_t(nn) * f4 * sizeof(float4) : nodes.size() * sizeof(float4),
                 tb = size_t(ntri + nlines + nshapes + sg::kPadSlots) * 3 * sizeof(float4) +
                      size_t(nlines + nshapes) * sg::kLineF4 * sizeof(float4);
    cudaError_t e = cudaSuccess;
    if (adopt) {
        s->d_nodes = s->tree.d_nodes;
        s->tree.d_nodes = nullptr;
    } else if ((e = cudaMalloc(&s->d_nodes, nb)) != cudaSuccess) {
        return e == cudaErrorMemoryAllocation ? fail(SG_ERR_OUT_OF_MEMORY, "cudaMalloc(nodes) failed")
                                              : cuda_fail(e, "cudaMalloc(nodes)");
    }
    if ((e = cudaMalloc(&s->d_err, sizeof(int))) != cudaSuccess) return cuda_fail(e, "cudaMalloc(status)");
    if ((e = cudaMalloc(&s->d_counters, sg_scene::kCounterSlots * sizeof(unsigned long long))) != cudaSuccess)
        return cuda_fail(e, "cudaMalloc(counters)");
    if (!adopt && ((e = sg::upload_host(s->d_nodes, nodes.data(), nb, nullptr)) != cudaSuccess ||
                   (e = cudaStreamSynchronize(nullptr)) != cudaSuccess))
        return cuda_fail(e, "upload nodes");
    if ((e = cudaMemset(s->d_err, 0, sizeof(int))) != cudaSuccess) return cuda_fail(e, "clear status");
    if (s->tree.d_tris) {  // the GPU builder wrote the records on the device
        s->d_tris = s->tree.d_tris;
        s->tree.d_tris = nullptr;
    } else {
        const int64_t nextra = nlines + nshapes, nall = ntri + nextra;
        std::vector<float4> tris(size_t(nall + sg::kPadSlots) * 3);
        std::memset(tris.data(), 0, tris.size() * sizeof(float4));
        auto put = [&](int64_t slot, int32_t p, int32_t last) {
            float4* dst = &tris[size_t(slot) * 3];
            if (p < ntri) {
                const float* v = tri + int64_t(p) * 9;
                dst[0] = make_float4(v[0], v[1], v[2], 0.0f);
                dst[1] = make_float4(v[3], v[4], v[5], 0.0f);
                dst[2] = make_float4(v[6], v[7], v[8], 0.0f);
            } else {  // a line's or an area shape's record, lines first
                const int32_t rec = int32_t(p - ntri), kind = rec < nlines ? sg::kLineSlot : sg::kShapeSlot;
                std::memcpy(&dst[2].x, &rec, 4);
                std::memcpy(&dst[2].w, &kind, 4);
            }
            std::memcpy(&dst[0].w, &p, 4);
            std::memcpy(&dst[1].w, &last, 4);
        };
        if (nextra == 0) {
            for (int64_t i = 0; i < ntri; ++i) put(i, t.order[size_t(i)], t.leaf_last[size_t(i)]);
        } else {
            // A leaf's triangles, then its lines, then its area shapes, each in
            // leaf order: SORT's leaf tests its triangle packs, its line packs,
            // then its other_list (accel/fast_bvh.hpp:346-406).
            auto kind = [&](int32_t p) { return p < ntri ? 0 : (p < ntri + nlines ? 1 : 2); };
            for (int64_t b = 0; b < nall;) {  // one leaf: slots b .. e
                int64_t e = b;
                while (!t.leaf_last[size_t(e)]) ++e;
                int64_t k = b;
                for (int pass = 0; pass < 3; ++pass)
                    for (int64_t i = b; i <= e; ++i) {
                        const int32_t p = t.order[size_t(i)];
                        if (kind(p) != pass) continue;
                        const int64_t slot = k++;
                        put(slot, p, slot == e ? 1 : 0);
                    }
                b = e + 1;
            }
        }
        const size_t tbytes = tris.size() * sizeof(float4);
        e = cudaMalloc(&s->d_tris, tbytes);
        if (e != cudaSuccess)
            return e == cudaErrorMemoryAllocation ? fail(SG_ERR_OUT_OF_MEMORY, "cudaMalloc(triangles) failed")
                                                  : cuda_fail(e, "cudaMalloc(triangles)");
        if ((e = sg::upload_host(s->d_tris, tris.data(), tbytes, nullptr)) != cudaSuccess ||
            (e = cudaStreamSynchronize(nullptr)) != cudaSuccess)
            return cuda_fail(e, "upload triangles");
        if (nextra > 0) {
            if ((e = cudaMalloc(&s->d_lines, line_recs.size() * sizeof(float))) != cudaSuccess)
                return cuda_fail(e, "cudaMalloc(lines)");
            if ((e = cudaMemcpy(s->d_lines, line_recs.data(), line_recs.size() * sizeof(float),
                                cudaMemcpyHostToDevice)) != cudaSuccess)
                return cuda_fail(e, "upload lines");
            s->n_lines = nlines;
            s->n_shapes = nshapes;
        }
    }
    s->device_bytes = int64_t(nb + tb);
    return SG_OK;
}

void release(sg_scene* s) {
    if (!s) return;
    DeviceGuard g(s->device);
    if (s->d_nodes) cudaFree(s->d_nodes);
    if (s->d_tris) cudaFree(s->d_tris);
    if (s->tree.d_tris) cudaFree(s->tree.d_tris);  // a GPU build that was not adopted
    if (s->tree.d_nodes) cudaFree(s->tree.d_nodes);
    if (s->d_lines) cudaFree(s->d_lines);
    if (s->d_err) cudaFree(s->d_err);
    if (s->d_stats) cudaFree(s->d_stats);
    if (s->d_counters) cudaFree(s->d_counters);
    if (s->d_scratch) cudaFree(s->d_scratch);
    if (s->d_material) cudaFree(s->d_material);
    if (s->stream) cudaStreamDestroy(s->stream);
    for (cudaStream_t& x : s->trace_stream)
        if (x) cudaStreamDestroy(x);
    if (s->out_stream) cudaStreamDestroy(s->out_stream);
    for (int k = 0; k < sg_scene::kMaxChunks; ++k) {
        if (s->in_done[k]) cudaEventDestroy(s->in_done[k]);
        if (s->trace_done[k]) cudaEventDestroy(s->trace_done[k]);
    }
    delete s;
}

sg::DevTree dev_tree(const sg_scene* s) {
    sg::DevTree d;
    d.nodes = s->d_nodes;
    d.tris = s->d_tris;
    d.root = s->tree.root;
    for (int k = 0; k < 3; ++k) {
        d.box_lo[k] = s->tree.scene.mn[k];
        d.box_hi[k] = s->tree.scene.mx[k];
    }
    return d;
}

unsigned long long* next_counter(const sg_scene* cs) {
    sg_scene* s = const_cast<sg_scene*>(cs);
    const unsigned k = s->next_counter.fetch_add(1, std::memory_order_relaxed) % sg_scene::kCounterSlots;
    return s->d_counters + k;
}

// Status word bits: 1 traversal stack bound (cannot happen when the stack
// holds depth*(W-1)+1 entries), 2 attenuation layer limit, 4 primitive
// material id outside the caller's table. Reading a set word clears it.
sg_status check_status_word(const sg_scene* s, cudaStream_t st) {
    int h = 0;
    cudaError_t e = cudaMemcpyAsync(&h, s->d_err, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(e, "read traversal status");
    if (h == 0) return SG_OK;
    if ((e = cudaMemsetAsync(s->d_err, 0, sizeof(int), st)) == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(e, "clear traversal status");
    if (h & 1) return fail(SG_ERR_INTERNAL, "traversal stack bound exceeded");
    if (h & 4) return fail(SG_ERR_INVALID_ARGUMENT, "primitive material id outside the material table");
    return fail(SG_ERR_LIMIT, "a ray crossed more than 4096 transparent surfaces");
}

}  // namespace

namespace sg {

sg_status set_error(sg_status s, const char* msg) { return fail(s, msg); }

const int32_t* scene_materials(const sg_scene* s) { return s ? s->d_material : nullptr; }

sg_status scene_launch(const sg_scene* s, bool any, TraceLaunch* L, DevTree* tree, int* device) {
    if (!s || !L || !tree || !device) return fail(SG_ERR_INVALID_ARGUMENT, "NULL argument");
    if (s->d_lines)
        return fail(SG_ERR_UNSUPPORTED,
                    "a scene with hair lines or area shapes answers the closest-hit and any-hit queries only");
    L->width = s->width;
    L->any = any;
    L->stack_need = s->stack_need;
    L->tuning = s->tuning;
    L->q8 = s->node_format == SG_NODES_QUANT8;
    L->err = s->d_err;
    L->counter = next_counter(s);
    *tree = dev_tree(s);
    *device = s->device;
    return SG_OK;
}

sg_status scene_status(const sg_scene* s, cudaStream_t st) { return check_status_word(s, st); }

}  // namespace sg

extern "C" {

void sg_default_build_opts(sg_build_opts* o) {
    if (!o) return;
    o->width = 8;
    o->max_depth = 16;
    o->max_leaf = 8;
    o->node_format = SG_NODES_FP32;
    o->device = 0;
    o->build_threads = 0;
    o->builder = SG_BUILDER_HOST;
}

}  // extern "C"

namespace sg {

// The non-triangle primitives' records (20 floats each: the lines, then the
// area shapes) and SORT's tree over every primitive, seen in `order` (NULL:
// triangles, lines, shapes). Throws as build_tree does.
BuiltTree build_mixed(const MixedInput& in, BuildParams bp, int builder, int device, std::vector<float>& recs) {
    const int64_t nextra = in.nlines + in.nshapes, nall = in.ntri + nextra;
    recs.assign(size_t(nextra) * 20, 0.0f);
    std::vector<float> boxes(size_t(nextra) * 6);
    for (int64_t k = 0; k < in.nlines; ++k)  // Line::SetTransform / GetBBox (hair_setup.cpp)
        line_setup(in.lines + k * 10, &recs[size_t(k) * 20], &boxes[size_t(k) * 6],
                   in.transforms ? in.transforms + size_t(in.line_transform[k]) * 16 : nullptr);
    for (int64_t k = 0; k < in.nshapes; ++k)  // Quad / Disk: record and GetBBox
        shape_setup(in.shapes[k], &recs[size_t(in.nlines + k) * 20], &boxes[size_t(in.nlines + k) * 6]);
    auto run = [&](const float* tri, int64_t ntri) {
        if (builder == SG_BUILDER_GPU) return build_tree_gpu(tri, ntri, bp, device);
        if (builder == SG_BUILDER_LBVH) return build_tree_lbvh(tri, ntri, bp, device);
        if (builder == SG_BUILDER_PLOC) return build_tree_ploc(tri, ntri, bp, device);
        return build_tree(tri, ntri, bp);
    };
    BuiltTree t;
    if (!in.order) {
        bp.extra_boxes = boxes.data();
        bp.nextra = nextra;
        t = run(in.triangles, in.ntri);
    } else {
        // Every primitive's box in SORT's primitive order: the split rules see a
        // primitive only as its box and box centre, so this builds SORT's tree.
        std::vector<uint8_t> seen(size_t(nall), 0);
        std::vector<float> all(size_t(std::max<int64_t>(nall, 1)) * 6);
        for (int64_t k = 0; k < nall; ++k) {
            const int32_t id = in.order[k];
            if (id < 0 || id >= nall || seen[size_t(id)]) throw std::invalid_argument("order is not a permutation");
            seen[size_t(id)] = 1;
            float* b = &all[size_t(k) * 6];
            if (id < in.ntri) {  // Triangle::GetBBox: BBox() then Union of the three vertices
                for (int a = 0; a < 3; ++a) {
                    b[a] = 3.402823466e+38f;
                    b[3 + a] = -3.402823466e+38f;
                }
                for (int v = 0; v < 3; ++v)
                    for (int a = 0; a < 3; ++a) {
                        const float x = in.triangles[int64_t(id) * 9 + 3 * v + a];
                        if (x < b[a]) b[a] = x;
                        if (x > b[3 + a]) b[3 + a] = x;
                    }
            } else {
                std::memcpy(b, &boxes[size_t(id - in.ntri) * 6], 6 * sizeof(float));
            }
        }
        bp.extra_boxes = all.data();
        bp.nextra = nall;
        t = run(nullptr, 0);
        for (int32_t& p : t.order) p = in.order[p];
    }
    t.first_extra = nextra > 0 ? in.ntri : -1;
    t.first_shape = in.nshapes > 0 ? in.ntri + in.nlines : -1;
    return t;
}

sg_status scene_create_mixed(const MixedInput& in, const sg_build_opts* opts, sg_scene** out) {
    if (!out) return fail(SG_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (!opts) return fail(SG_ERR_INVALID_ARGUMENT, "opts is NULL");
    const int64_t ntri = in.ntri, nlines = in.nlines, nshapes = in.nshapes;
    if (ntri < 0 || (ntri > 0 && !in.triangles)) return fail(SG_ERR_INVALID_ARGUMENT, "bad triangle buffer");
    if (nlines < 0 || (nlines > 0 && !in.lines)) return fail(SG_ERR_INVALID_ARGUMENT, "bad line buffer");
    if (nshapes < 0 || (nshapes > 0 && !in.shapes)) return fail(SG_ERR_INVALID_ARGUMENT, "bad area shape buffer");
    for (int64_t k = 0; k < nshapes; ++k)
        if (in.shapes[k].kind != SG_SHAPE_QUAD && in.shapes[k].kind != SG_SHAPE_DISK)
            return fail(SG_ERR_INVALID_ARGUMENT, "unknown area shape kind");
    const bool morton = opts->builder == SG_BUILDER_LBVH || opts->builder == SG_BUILDER_PLOC;
    if ((nlines > 0 || nshapes > 0 || in.order) && morton)
        return fail(SG_ERR_UNSUPPORTED, "SG_BUILDER_LBVH / SG_BUILDER_PLOC build triangle scenes only");
    if (ntri + nlines + nshapes >= int64_t(0x7fffffff)) return fail(SG_ERR_LIMIT, "more than 2^31-2 primitives");
    if (opts->width != 4 && opts->width != 8) return fail(SG_ERR_INVALID_ARGUMENT, "width must be 4 or 8");
    if (opts->max_leaf < 1 || opts->max_depth < 1) return fail(SG_ERR_INVALID_ARGUMENT, "max_leaf/max_depth < 1");
    if (opts->node_format != SG_NODES_FP32 && opts->node_format != SG_NODES_QUANT8)
        return fail(SG_ERR_UNSUPPORTED, "unknown node format");
    if (opts->builder != SG_BUILDER_HOST && opts->builder != SG_BUILDER_GPU && !morton)
        return fail(SG_ERR_INVALID_ARGUMENT, "unknown builder");
    if (morton && opts->node_format != SG_NODES_FP32)
        return fail(SG_ERR_UNSUPPORTED, "SG_BUILDER_LBVH / SG_BUILDER_PLOC write FP32 nodes only");
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDeviceCount");
    if (opts->device < 0 || opts->device >= ndev) return fail(SG_ERR_INVALID_ARGUMENT, "no such CUDA device");

    sg_scene* s = new (std::nothrow) sg_scene();
    if (!s) return fail(SG_ERR_OUT_OF_MEMORY, "host allocation failed");
    s->device = opts->device;
    s->width = opts->width;
    s->node_format = opts->node_format;
    sg::BuildParams bp;
    bp.width = opts->width;
    bp.max_depth = opts->max_depth;
    bp.max_leaf = opts->max_leaf;
    bp.threads = opts->build_threads;
    bp.host_boxes = opts->node_format != SG_NODES_FP32;
    std::vector<float> recs;
    const auto t0 = std::chrono::steady_clock::now();
    try {
        s->tree = build_mixed(in, bp, opts->builder, opts->device, recs);
    } catch (const std::bad_alloc&) {
        delete s;
        return fail(SG_ERR_OUT_OF_MEMORY, "host memory exhausted during build");
    } catch (const std::runtime_error& ex) {
        delete s;
        return fail(SG_ERR_CUDA, ex.what());
    } catch (const std::exception& ex) {
        delete s;
        return fail(SG_ERR_INVALID_ARGUMENT, ex.what());
    }
    s->build_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    s->stack_need = std::max(1, s->tree.depth * (s->width - 1) + 1);
    if (s->stack_need > 256) {
        release(s);
        return fail(SG_ERR_LIMIT, "tree too deep for the traversal stack (depth*(width-1)+1 > 256)");
    }
    DeviceGuard g(s->device);
    if (!g.ok) {
        delete s;
        return fail(SG_ERR_CUDA, "cudaSetDevice failed");
    }
    sg_status st;
    try {
        st = upload(s, in.triangles, ntri, recs, nlines, nshapes);
    } catch (const std::bad_alloc&) {
        st = fail(SG_ERR_OUT_OF_MEMORY, "host memory exhausted during upload");
    }
    if (st != SG_OK) {
        release(s);
        return st;
    }
    std::vector<float>().swap(s->tree.lo);
    std::vector<float>().swap(s->tree.hi);
    *out = s;
    return SG_OK;
}

}  // namespace sg

namespace {

// The child references, leaf order and leaf flags of a tree that has no host
// arrays (built on the device), read back from its FP32 nodes and slot
// records (layout.h): enough for tree_topology.
sg_status device_topology_tree(const sg_scene* s, sg::BuiltTree& h) {
    const sg::BuiltTree& t = s->tree;
    if (s->node_format != SG_NODES_FP32) return fail(SG_ERR_UNSUPPORTED, "topology of a device-built 8-bit tree");
    h.width = t.width;
    h.root = t.root;
    h.depth = t.depth;
    h.first_extra = t.first_extra;
    h.first_shape = t.first_shape;
    const int W = t.width;
    const int f4 = W == 8 ? sg::NodeShape<8>::kF4 : sg::NodeShape<4>::kF4;
    const int64_t nn = t.interior(), nall = t.triangles() + s->n_lines + s->n_shapes;
    std::vector<float4> nodes(size_t(std::max<int64_t>(nn, 0)) * f4), tris(size_t(nall) * 3);
    DeviceGuard g(s->device);
    if (!g.ok) return fail(SG_ERR_CUDA, "cudaSetDevice failed");
    cudaError_t e = cudaSuccess;
    if (nn > 0) e = cudaMemcpy(nodes.data(), s->d_nodes, nodes.size() * sizeof(float4), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && nall > 0)
        e = cudaMemcpy(tris.data(), s->d_tris, tris.size() * sizeof(float4), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "read the tree back");
    h.child.resize(size_t(nn) * W);
    for (int64_t k = 0; k < nn; ++k)  // the child references follow the 6 planes of W boxes
        std::memcpy(&h.child[size_t(k) * W], reinterpret_cast<const float*>(&nodes[size_t(k) * f4]) + 6 * W,
                    size_t(W) * sizeof(int32_t));
    h.order.resize(size_t(nall));
    h.leaf_last.resize(size_t(nall));
    for (int64_t i = 0; i < nall; ++i) {
        int32_t last = 0;
        std::memcpy(&h.order[size_t(i)], &tris[size_t(i) * 3].w, 4);
        std::memcpy(&last, &tris[size_t(i) * 3 + 1].w, 4);
        h.leaf_last[size_t(i)] = last ? 1 : 0;
    }
    return SG_OK;
}

}  // namespace

extern "C" {

sg_status sg_scene_create(const float* triangles, int64_t ntri, const sg_build_opts* opts, sg_scene** out) {
    sg::MixedInput in;
    in.triangles = triangles;
    in.ntri = ntri;
    return sg::scene_create_mixed(in, opts, out);
}

sg_status sg_scene_create_hair(const float* triangles, int64_t ntri, const float* lines, int64_t nlines,
                               const sg_build_opts* opts, sg_scene** out) {
    sg::MixedInput in;
    in.triangles = triangles;
    in.ntri = ntri;
    in.lines = lines;
    in.nlines = nlines;
    return sg::scene_create_mixed(in, opts, out);
}

sg_status sg_scene_create_shapes(const sg_shapes* shapes, const sg_build_opts* opts, sg_scene** out) {
    if (!shapes) return fail(SG_ERR_INVALID_ARGUMENT, "shapes is NULL");
    sg::MixedInput in;
    in.triangles = shapes->triangles;
    in.ntri = shapes->ntri;
    in.lines = shapes->lines;
    in.nlines = shapes->nlines;
    in.shapes = shapes->shapes;
    in.nshapes = shapes->nshapes;
    in.order = shapes->order;
    return sg::scene_create_mixed(in, opts, out);
}

sg_status sg_scene_destroy(sg_scene* s) {
    release(s);
    return SG_OK;
}

sg_status sg_scene_info_get(const sg_scene* s, sg_scene_info* info) {
    if (!s || !info) return fail(SG_ERR_INVALID_ARGUMENT, "NULL argument");
    std::memset(info, 0, sizeof(*info));
    info->triangles = s->tree.triangles();
    info->interior_nodes = s->tree.interior();
    info->leaves = s->tree.leaves;
    info->depth = s->tree.depth;
    info->width = s->width;
    info->node_format = s->node_format;
    info->valid = s->tree.root != sg::kEmptyRef ? 1 : 0;
    for (int k = 0; k < 3; ++k) {
        info->bbox[k] = s->tree.scene.mn[k];
        info->bbox[3 + k] = s->tree.scene.mx[k];
    }
    info->device_bytes = s->device_bytes;
    info->build_seconds = s->build_seconds;
    info->build_rounds = s->tree.rounds;
    info->build_launches = s->tree.launches;
    return SG_OK;
}

sg_status sg_scene_topology(const sg_scene* s, int32_t* out, int64_t cap, int64_t* written) {
    if (!s || !written) return fail(SG_ERR_INVALID_ARGUMENT, "NULL argument");
    std::vector<int32_t> v;
    if (s->tree.host_arrays()) {
        sg::tree_topology(s->tree, v);
    } else {  // built on the device: read the topology back from the device layout
        sg::BuiltTree h;
        const sg_status st = device_topology_tree(s, h);
        if (st != SG_OK) return st;
        sg::tree_topology(h, v);
    }
    *written = int64_t(v.size());
    if (int64_t(v.size()) > cap || (!out && !v.empty())) return fail(SG_ERR_LIMIT, "topology buffer too small");
    if (!v.empty()) std::memcpy(out, v.data(), v.size() * sizeof(int32_t));
    return SG_OK;
}

sg_status sg_build_topology_host(const float* triangles, int64_t ntri, const sg_build_opts* opts, int32_t* out,
                                 int64_t cap, int64_t* written, int32_t* depth) {
    return sg_build_topology_host_hair(triangles, ntri, nullptr, 0, opts, out, cap, written, depth);
}

sg_status sg_build_topology_host_hair(const float* triangles, int64_t ntri, const float* lines, int64_t nlines,
                                      const sg_build_opts* opts, int32_t* out, int64_t cap, int64_t* written,
                                      int32_t* depth) {
    sg_shapes sh{triangles, ntri, lines, nlines, nullptr, 0, nullptr};
    return sg_build_topology_host_shapes(&sh, opts, out, cap, written, depth);
}

sg_status sg_build_topology_host_shapes(const sg_shapes* sh, const sg_build_opts* opts, int32_t* out, int64_t cap,
                                        int64_t* written, int32_t* depth) {
    if (!sh || !opts || !written) return fail(SG_ERR_INVALID_ARGUMENT, "NULL argument");
    if (sh->ntri < 0 || (sh->ntri > 0 && !sh->triangles)) return fail(SG_ERR_INVALID_ARGUMENT, "bad triangle buffer");
    if (sh->nlines < 0 || (sh->nlines > 0 && !sh->lines)) return fail(SG_ERR_INVALID_ARGUMENT, "bad line buffer");
    if (sh->nshapes < 0 || (sh->nshapes > 0 && !sh->shapes))
        return fail(SG_ERR_INVALID_ARGUMENT, "bad area shape buffer");
    sg::BuildParams bp;
    bp.width = opts->width;
    bp.max_depth = opts->max_depth;
    bp.max_leaf = opts->max_leaf;
    bp.threads = opts->build_threads;
    sg::MixedInput in;
    in.triangles = sh->triangles;
    in.ntri = sh->ntri;
    in.lines = sh->lines;
    in.nlines = sh->nlines;
    in.shapes = sh->shapes;
    in.nshapes = sh->nshapes;
    in.order = sh->order;
    std::vector<int32_t> v;
    try {
        std::vector<float> recs;
        const sg::BuiltTree t = sg::build_mixed(in, bp, SG_BUILDER_HOST, 0, recs);
        sg::tree_topology(t, v);
        if (depth) *depth = t.depth;
    } catch (const std::bad_alloc&) {
        return fail(SG_ERR_OUT_OF_MEMORY, "host memory exhausted during build");
    } catch (const std::exception& ex) {
        return fail(SG_ERR_INVALID_ARGUMENT, ex.what());
    }
    *written = int64_t(v.size());
    if (int64_t(v.size()) > cap || (!out && !v.empty())) return fail(SG_ERR_LIMIT, "topology buffer too small");
    if (!v.empty()) std::memcpy(out, v.data(), v.size() * sizeof(int32_t));
    return SG_OK;
}

static sg_status trace_common(const sg_scene* s, const sg_rays* rays, int64_t n, const sg_hits* hits, uint8_t* occ,
                              bool any, cudaStream_t st) {
    if (!s || !rays) return fail(SG_ERR_INVALID_ARGUMENT, "NULL scene or rays");
    if (n < 0) return fail(SG_ERR_INVALID_ARGUMENT, "negative ray count");
    if (n == 0) return SG_OK;
    if (!rays->ox || !rays->oy || !rays->oz || !rays->dx || !rays->dy || !rays->dz || !rays->tmin || !rays->tmax)
        return fail(SG_ERR_INVALID_ARGUMENT, "NULL ray array");
    if (any ? !occ : (!hits || !hits->prim || !hits->t)) return fail(SG_ERR_INVALID_ARGUMENT, "NULL output array");
    if (n > int64_t(0x7fffffff) * 128) return fail(SG_ERR_LIMIT, "batch too large");
    DeviceGuard g(s->device);
    if (!g.ok) return fail(SG_ERR_CUDA, "cudaSetDevice failed");
    sg::DevRays r{rays->ox, rays->oy, rays->oz, rays->dx, rays->dy, rays->dz, rays->tmin, rays->tmax};
    sg::TraceLaunch L;
    L.width = s->width;
    L.any = any;
    L.stack_need = s->stack_need;
    L.tuning = s->tuning;
    L.q8 = s->node_format == SG_NODES_QUANT8;
    if (any) {
        L.occ = occ;
    } else {
        L.prim = hits->prim;
        L.t = hits->t;
        L.u = hits->u;
        L.v = hits->v;
    }
    L.err = s->d_err;
    L.counter = next_counter(s);
    const cudaError_t e = s->d_lines ? sg::launch_trace_hair(L, dev_tree(s), s->d_lines, r, n, st)
                                     : sg::launch_trace_fp32(L, dev_tree(s), r, n, st);
    if (e != cudaSuccess) return cuda_fail(e, "traversal launch");
    return SG_OK;
}

sg_status sg_trace_closest(const sg_scene* s, const sg_rays* rays, int64_t n, const sg_hits* hits, void* stream) {
    return trace_common(s, rays, n, hits, nullptr, false, (cudaStream_t)stream);
}

sg_status sg_trace_any(const sg_scene* s, const sg_rays* rays, int64_t n, uint8_t* occluded, void* stream) {
    return trace_common(s, rays, n, nullptr, occluded, true, (cudaStream_t)stream);
}

static sg_status host_trace(const sg_scene* cs, const float* rays8, int64_t n, int32_t* prim, float* t, float* u,
                            float* v, uint8_t* occ, bool any) {
    if (!cs || !rays8) return fail(SG_ERR_INVALID_ARGUMENT, "NULL scene or rays");
    if (n < 0) return fail(SG_ERR_INVALID_ARGUMENT, "negative ray count");
    if (n == 0) return SG_OK;
    if (any ? !occ : (!prim || !t)) return fail(SG_ERR_INVALID_ARGUMENT, "NULL output array");
    sg_scene* s = const_cast<sg_scene*>(cs);
    std::lock_guard<std::mutex> lock(s->scratch_lock);
    DeviceGuard g(s->device);
    if (!g.ok) return fail(SG_ERR_CUDA, "cudaSetDevice failed");
    cudaError_t e;
    if (!s->stream) {
        if ((e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking)) != cudaSuccess ||
            (e = cudaStreamCreateWithFlags(&s->out_stream, cudaStreamNonBlocking)) != cudaSuccess)
            return cuda_fail(e, "cudaStreamCreate");
        for (cudaStream_t& x : s->trace_stream)
            if ((e = cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking)) != cudaSuccess)
                return cuda_fail(e, "cudaStreamCreate");
        for (int k = 0; k < sg_scene::kMaxChunks; ++k)
            if ((e = cudaEventCreateWithFlags(&s->in_done[k], cudaEventDisableTiming)) != cudaSuccess ||
                (e = cudaEventCreateWithFlags(&s->trace_done[k], cudaEventDisableTiming)) != cudaSuccess)
                return cuda_fail(e, "cudaEventCreate");
    }
    const size_t in_bytes = size_t(n) * 8 * sizeof(float);
    const size_t out_bytes = any ? size_t(n) : size_t(n) * 16;
    const size_t need = in_bytes + out_bytes + 256;
    if (s->scratch_bytes < need) {
        if (s->d_scratch) cudaFree(s->d_scratch);
        s->d_scratch = nullptr;
        s->scratch_bytes = 0;
        if ((e = cudaMalloc(&s->d_scratch, need)) != cudaSuccess)
            return e == cudaErrorMemoryAllocation ? fail(SG_ERR_OUT_OF_MEMORY, "scratch allocation failed")
                                                  : cuda_fail(e, "cudaMalloc(scratch)");
        s->scratch_bytes = need;
    }
    float* d_rays = static_cast<float*>(s->d_scratch);
    char* d_out = static_cast<char*>(s->d_scratch) + ((in_bytes + 255) & ~size_t(255));
    int32_t* dp = reinterpret_cast<int32_t*>(d_out);
    float* dt = reinterpret_cast<float*>(d_out + size_t(n) * 4);
    float* du = reinterpret_cast<float*>(d_out + size_t(n) * 8);
    float* dv = reinterpret_cast<float*>(d_out + size_t(n) * 12);
    uint8_t* docc = reinterpret_cast<uint8_t*>(d_out);
    // Chunks of at least 256k rays (one chunk below 512k), at most kMaxChunks:
    // chunk k's rays go in while chunk k-1 is traced and chunk k-2's hits come out.
    const int64_t min_chunk = int64_t(1) << 18;
    const int chunks = int(std::min<int64_t>(sg_scene::kMaxChunks, std::max<int64_t>(1, n / min_chunk / 2 * 2)));
    const int64_t per = (n + chunks - 1) / chunks;
    sg_status status = SG_OK;
    for (int k = 0; k < chunks; ++k) {
        const int64_t a = int64_t(k) * per;
        const int64_t m = std::min(per, n - a);
        if (m <= 0) break;
        cudaStream_t tr = s->trace_stream[k % sg_scene::kTraceStreams];
        // Ray planes [a, a + m) of all eight arrays: one pitched copy.
        if ((e = cudaMemcpy2DAsync(d_rays + a, size_t(n) * 4, rays8 + a, size_t(n) * 4, size_t(m) * 4, 8,
                                   cudaMemcpyHostToDevice, s->stream)) != cudaSuccess ||
            (e = cudaEventRecord(s->in_done[k], s->stream)) != cudaSuccess ||
            (e = cudaStreamWaitEvent(tr, s->in_done[k], 0)) != cudaSuccess)
            return cuda_fail(e, "copy rays to device");
        const float* b = d_rays + a;
        sg_rays r{b, b + n, b + 2 * n, b + 3 * n, b + 4 * n, b + 5 * n, b + 6 * n, b + 7 * n};
        if (any) {
            status = trace_common(s, &r, m, nullptr, docc + a, true, tr);
        } else {
            sg_hits h{dp + a, dt + a, u ? du + a : nullptr, v ? dv + a : nullptr};
            status = trace_common(s, &r, m, &h, nullptr, false, tr);
        }
        if (status != SG_OK) break;
        if ((e = cudaEventRecord(s->trace_done[k], tr)) != cudaSuccess ||
            (e = cudaStreamWaitEvent(s->out_stream, s->trace_done[k], 0)) != cudaSuccess)
            return cuda_fail(e, "order chunk copies");
        cudaStream_t o = s->out_stream;
        if (any) {
            e = cudaMemcpyAsync(occ + a, docc + a, size_t(m), cudaMemcpyDeviceToHost, o);
        } else {
            e = cudaMemcpyAsync(prim + a, dp + a, size_t(m) * 4, cudaMemcpyDeviceToHost, o);
            if (e == cudaSuccess) e = cudaMemcpyAsync(t + a, dt + a, size_t(m) * 4, cudaMemcpyDeviceToHost, o);
            if (e == cudaSuccess && u) e = cudaMemcpyAsync(u + a, du + a, size_t(m) * 4, cudaMemcpyDeviceToHost, o);
            if (e == cudaSuccess && v) e = cudaMemcpyAsync(v + a, dv + a, size_t(m) * 4, cudaMemcpyDeviceToHost, o);
        }
        if (e != cudaSuccess) return cuda_fail(e, "copy results to host");
    }
    // Everything enqueued so far completes before returning, even after an error.
    for (cudaStream_t x : s->trace_stream)
        if ((e = cudaStreamSynchronize(x)) != cudaSuccess) return cuda_fail(e, "synchronize");
    for (cudaStream_t x : {s->stream, s->out_stream})
        if ((e = cudaStreamSynchronize(x)) != cudaSuccess) return cuda_fail(e, "synchronize");
    if (status != SG_OK) return status;
    return check_status_word(s, s->out_stream);
}

sg_status sg_scene_set_materials(sg_scene* s, const int32_t* material, int64_t n) {
    if (!s || (n > 0 && !material)) return fail(SG_ERR_INVALID_ARGUMENT, "NULL argument");
    if (n != s->tree.triangles()) return fail(SG_ERR_INVALID_ARGUMENT, "one material per primitive");
    std::lock_guard<std::mutex> lock(s->scratch_lock);
    DeviceGuard g(s->device);
    if (!g.ok) return fail(SG_ERR_CUDA, "cudaSetDevice failed");
    cudaError_t e;
    if (!s->d_material && (e = cudaMalloc(&s->d_material, size_t(std::max<int64_t>(n, 1)) * 4)) != cudaSuccess)
        return cuda_fail(e, "cudaMalloc(materials)");
    if (n > 0 && (e = cudaMemcpy(s->d_material, material, size_t(n) * 4, cudaMemcpyHostToDevice)) != cudaSuccess)
        return cuda_fail(e, "upload materials");
    return SG_OK;
}

sg_status sg_trace_multi_host(const sg_scene* cs, const float* rays8, int64_t n, const int32_t* ray_material,
                              int32_t* count, int32_t* prim, float* t, float* u, float* v) {
    if (!cs || !rays8 || !ray_material || !count || !prim || !t) return fail(SG_ERR_INVALID_ARGUMENT, "NULL argument");
    if (n < 0) return fail(SG_ERR_INVALID_ARGUMENT, "negative ray count");
    if (n == 0) return SG_OK;
    sg_scene* s = const_cast<sg_scene*>(cs);
    if (!s->d_material) return fail(SG_ERR_INVALID_ARGUMENT, "no primitive materials (sg_scene_set_materials)");
    std::lock_guard<std::mutex> lock(s->scratch_lock);
    DeviceGuard g(s->device);
    if (!g.ok) return fail(SG_ERR_CUDA, "cudaSetDevice failed");
    cudaError_t e;
    if (!s->stream && (e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking)) != cudaSuccess)
        return cuda_fail(e, "cudaStreamCreate");
    // rays 32 B, ray material 4, count 4, four (prim, t, u, v) 64 per ray
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t N = size_t(n);
    const size_t need = al(N * 32) + al(N * 4) + al(N * 4) + 4 * al(N * 16);
    if (s->scratch_bytes < need) {
        if (s->d_scratch) cudaFree(s->d_scratch);
        s->d_scratch = nullptr;
        s->scratch_bytes = 0;
        if ((e = cudaMalloc(&s->d_scratch, need)) != cudaSuccess) return cuda_fail(e, "cudaMalloc(scratch)");
        s->scratch_bytes = need;
    }
    char* b = static_cast<char*>(s->d_scratch);
    float* d_rays = reinterpret_cast<float*>(b);
    b += al(N * 32);
    int32_t* d_rm = reinterpret_cast<int32_t*>(b);
    b += al(N * 4);
    sg_multi_hits h;
    h.count = reinterpret_cast<int32_t*>(b);
    b += al(N * 4);
    h.prim = reinterpret_cast<int32_t*>(b);
    b += al(N * 16);
    h.t = reinterpret_cast<float*>(b);
    b += al(N * 16);
    h.u = u ? reinterpret_cast<float*>(b) : nullptr;
    b += al(N * 16);
    h.v = v ? reinterpret_cast<float*>(b) : nullptr;
    cudaStream_t st = s->stream;
    if ((e = cudaMemcpyAsync(d_rays, rays8, N * 32, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(d_rm, ray_material, N * 4, cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return cuda_fail(e, "copy rays to device");
    const sg_rays r{d_rays, d_rays + n, d_rays + 2 * n, d_rays + 3 * n, d_rays + 4 * n, d_rays + 5 * n, d_rays + 6 * n,
                    d_rays + 7 * n};
    sg_status status = sg_trace_multi(s, &r, n, s->d_material, d_rm, &h, st);
    if (status != SG_OK) return status;
    if ((e = cudaMemcpyAsync(count, h.count, N * 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(prim, h.prim, N * 16, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(t, h.t, N * 16, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (u && (e = cudaMemcpyAsync(u, h.u, N * 16, cudaMemcpyDeviceToHost, st)) != cudaSuccess) ||
        (v && (e = cudaMemcpyAsync(v, h.v, N * 16, cudaMemcpyDeviceToHost, st)) != cudaSuccess))
        return cuda_fail(e, "copy results to host");
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(e, "synchronize");
    return check_status_word(s, st);
}

sg_status sg_trace_attenuation_host(const sg_scene* cs, const float* rays8, int64_t n,
                                    const sg_transparency* materials, int32_t nmat, float* attenuation) {
    if (!cs || !rays8 || !attenuation) return fail(SG_ERR_INVALID_ARGUMENT, "NULL argument");
    if (n < 0 || nmat < 0) return fail(SG_ERR_INVALID_ARGUMENT, "negative count");
    if (nmat > 0 && !materials) return fail(SG_ERR_INVALID_ARGUMENT, "NULL material table");
    if (n == 0) return SG_OK;
    sg_scene* s = const_cast<sg_scene*>(cs);
    if (!s->d_material) return fail(SG_ERR_INVALID_ARGUMENT, "no primitive materials (sg_scene_set_materials)");
    std::lock_guard<std::mutex> lock(s->scratch_lock);
    DeviceGuard g(s->device);
    if (!g.ok) return fail(SG_ERR_CUDA, "cudaSetDevice failed");
    cudaError_t e;
    if (!s->stream && (e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking)) != cudaSuccess)
        return cuda_fail(e, "cudaStreamCreate");
    // rays 32 B and attenuation 12 B per ray, then the material table
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t N = size_t(n), M = size_t(nmat);
    const size_t need = al(N * 32) + al(N * 12) + al(std::max<size_t>(M, 1) * sizeof(sg_transparency));
    if (s->scratch_bytes < need) {
        if (s->d_scratch) cudaFree(s->d_scratch);
        s->d_scratch = nullptr;
        s->scratch_bytes = 0;
        if ((e = cudaMalloc(&s->d_scratch, need)) != cudaSuccess) return cuda_fail(e, "cudaMalloc(scratch)");
        s->scratch_bytes = need;
    }
    char* b = static_cast<char*>(s->d_scratch);
    float* d_rays = reinterpret_cast<float*>(b);
    b += al(N * 32);
    float* d_att = reinterpret_cast<float*>(b);
    b += al(N * 12);
    sg_transparency* d_mats = reinterpret_cast<sg_transparency*>(b);
    cudaStream_t st = s->stream;
    if ((e = cudaMemcpyAsync(d_rays, rays8, N * 32, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (M && (e = cudaMemcpyAsync(d_mats, materials, M * sizeof(sg_transparency), cudaMemcpyHostToDevice, st)) !=
                  cudaSuccess))
        return cuda_fail(e, "copy rays to device");
    const sg_rays r{d_rays, d_rays + n, d_rays + 2 * n, d_rays + 3 * n, d_rays + 4 * n, d_rays + 5 * n, d_rays + 6 * n,
                    d_rays + 7 * n};
    sg_status status = sg_trace_attenuation(s, &r, n, d_mats, nmat, d_att, st);
    if (status != SG_OK) return status;
    if ((e = cudaMemcpyAsync(attenuation, d_att, N * 12, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return cuda_fail(e, "copy results to host");
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(e, "synchronize");
    return check_status_word(s, st);
}

sg_status sg_trace_stats(const sg_scene* cs, const sg_rays* rays, int64_t n, int32_t any, int64_t* node_tests,
                         int64_t* prim_tests, void* stream) {
    if (!cs || !rays || !node_tests || !prim_tests) return fail(SG_ERR_INVALID_ARGUMENT, "NULL argument");
    if (n < 0) return fail(SG_ERR_INVALID_ARGUMENT, "negative ray count");
    if (!rays->ox || !rays->oy || !rays->oz || !rays->dx || !rays->dy || !rays->dz || !rays->tmin || !rays->tmax)
        return fail(SG_ERR_INVALID_ARGUMENT, "NULL ray array");
    *node_tests = *prim_tests = 0;
    if (cs->d_lines) return fail(SG_ERR_UNSUPPORTED, "traversal statistics cover triangle scenes only");
    if (n == 0) return SG_OK;
    sg_scene* s = const_cast<sg_scene*>(cs);
    std::lock_guard<std::mutex> lock(s->scratch_lock);
    DeviceGuard g(s->device);
    if (!g.ok) return fail(SG_ERR_CUDA, "cudaSetDevice failed");
    cudaError_t e;
    cudaStream_t st = (cudaStream_t)stream;
    if (!s->d_stats && (e = cudaMalloc(&s->d_stats, 2 * sizeof(unsigned long long))) != cudaSuccess)
        return cuda_fail(e, "cudaMalloc(stats)");
    const size_t need = size_t(n) * 16 + 256;
    if (s->scratch_bytes < need) {
        if (s->d_scratch) cudaFree(s->d_scratch);
        s->d_scratch = nullptr;
        s->scratch_bytes = 0;
        if ((e = cudaMalloc(&s->d_scratch, need)) != cudaSuccess) return cuda_fail(e, "cudaMalloc(scratch)");
        s->scratch_bytes = need;
    }
    char* out = static_cast<char*>(s->d_scratch);
    if ((e = cudaMemsetAsync(s->d_stats, 0, 2 * sizeof(unsigned long long), st)) != cudaSuccess)
        return cuda_fail(e, "clear stats");
    sg::DevRays r{rays->ox, rays->oy, rays->oz, rays->dx, rays->dy, rays->dz, rays->tmin, rays->tmax};
    sg::TraceLaunch L;
    L.width = s->width;
    L.any = any != 0;
    L.stack_need = s->stack_need;
    L.tuning = s->tuning;
    L.q8 = s->node_format == SG_NODES_QUANT8;
    L.prim = reinterpret_cast<int32_t*>(out);
    L.t = reinterpret_cast<float*>(out + size_t(n) * 4);
    L.occ = reinterpret_cast<uint8_t*>(out);
    L.err = s->d_err;
    L.stats = s->d_stats;
    L.counter = next_counter(s);
    e = sg::launch_trace_fp32(L, dev_tree(s), r, n, st);
    if (e != cudaSuccess) return cuda_fail(e, "stats launch");
    unsigned long long h[2] = {0, 0};
    if ((e = cudaMemcpyAsync(h, s->d_stats, sizeof(h), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return cuda_fail(e, "read stats");
    *node_tests = int64_t(h[0]);
    *prim_tests = int64_t(h[1]);
    return check_status_word(s, st);
}

sg_status sg_trace_closest_host(const sg_scene* s, const float* rays8, int64_t n, int32_t* prim, float* t, float* u,
                                float* v) {
    return host_trace(s, rays8, n, prim, t, u, v, nullptr, false);
}

sg_status sg_trace_any_host(const sg_scene* s, const float* rays8, int64_t n, uint8_t* occluded) {
    return host_trace(s, rays8, n, nullptr, nullptr, nullptr, nullptr, occluded, true);
}

sg_status sg_scene_set_tuning(sg_scene* s, const sg_trace_tuning* t) {
    if (!s || !t) return fail(SG_ERR_INVALID_ARGUMENT, "NULL argument");
    if (t->schedule < SG_SCHEDULE_THREAD_PER_RAY || t->schedule > SG_SCHEDULE_AUTO)
        return fail(SG_ERR_INVALID_ARGUMENT, "unknown schedule");
    if (t->refill_threshold < 1 || t->refill_threshold > 32)
        return fail(SG_ERR_INVALID_ARGUMENT, "refill_threshold must be 1..32");
    s->tuning.schedule = t->schedule;
    s->tuning.refill_threshold = t->refill_threshold;
    return SG_OK;
}

sg_status sg_scene_get_tuning(const sg_scene* s, sg_trace_tuning* t) {
    if (!s || !t) return fail(SG_ERR_INVALID_ARGUMENT, "NULL argument");
    t->schedule = s->tuning.schedule;
    t->refill_threshold = s->tuning.refill_threshold;
    return SG_OK;
}

const char* sg_last_error(void) { return g_last_error.c_str(); }

const char* sg_version(void) { return "sortgpu 0.1 (sm_100a)"; }

}  // extern "C"
