// sg_batcher (include/sortgpu.h): multi-scene batch runs replayed from
// captured CUDA graphs, and the autotuner that picks their launch shape.
//
// A run's variable part (batches, trees, refill threshold, time budget) lives
// in device tables that are copied in stream order before each replay, so the
// graph depends only on the kernel configurations of its groups: one graph per
// distinct list of (width, query, node format, stack, block, grid), cached.
// Graph: a begin kernel (run clock, counters) and then one persistent kernel
// per group, the groups forked onto side streams so their blocks share the GPU.
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "batch_kernels.h"
#include "scene_access.h"
#include "sortgpu.h"

namespace {

constexpr int kSlots = 4;         // host staging buffers in flight
constexpr size_t kMaxGraphs = 64;  // cached executable graphs per batcher

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

struct Layout {
    size_t batches = 0, trees = 0, state = 0, remaining = 0, done = 0, total = 0;
    size_t stage = 0;  // bytes of header + batches + trees (the staged part)
    explicit Layout(int max_batches) {
        size_t o = align_up(sizeof(sg::RunHeader), 256);
        batches = o;
        o = align_up(o + size_t(max_batches) * sizeof(sg::BatchDesc), 256);
        trees = o;
        o = align_up(o + size_t(max_batches) * sizeof(sg::DevTree), 256);
        stage = o;
        state = o;
        o = align_up(o + sizeof(sg::RunState), 256);
        remaining = o;
        o = align_up(o + size_t(max_batches) * sizeof(unsigned long long), 256);
        done = o;
        o = align_up(o + size_t(max_batches) * sizeof(long long), 256);
        total = o;
    }
};

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

sg_status fail(sg_status s, const std::string& msg) { return sg::set_error(s, msg.c_str()); }
sg_status cuda_fail(cudaError_t e, const char* what) {
    return fail(SG_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

int stack_fit(int need) {
    for (int s : {64, 128, 256})
        if (need <= s) return s;
    return 0;
}

}  // namespace

struct sg_batcher {
    int device = 0;
    int max_batches = 0;
    int sms = 1;
    sg_batch_tuning tuning{128, 0, 8, 0};
    std::mutex lock;
    char* d_mem = nullptr;
    char* h_stage[kSlots] = {};
    cudaEvent_t stage_done[kSlots] = {};
    int slot = 0;
    cudaStream_t cap = nullptr;
    cudaStream_t side[sg::kMaxBatchGroups] = {};
    cudaEvent_t fork = nullptr;
    cudaEvent_t join[sg::kMaxBatchGroups] = {};
    std::map<std::vector<int>, cudaGraphExec_t> graphs;
    std::vector<int> perm;  // table position -> caller index, of the last run
    Layout lay{1};
};

namespace {

void release(sg_batcher* b) {
    if (!b) return;
    DeviceGuard g(b->device);
    for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
    for (int k = 0; k < kSlots; ++k) {
        if (b->stage_done[k]) {
            cudaEventSynchronize(b->stage_done[k]);
            cudaEventDestroy(b->stage_done[k]);
        }
        if (b->h_stage[k]) cudaFreeHost(b->h_stage[k]);
    }
    for (int k = 0; k < sg::kMaxBatchGroups; ++k) {
        if (b->side[k]) cudaStreamDestroy(b->side[k]);
        if (b->join[k]) cudaEventDestroy(b->join[k]);
    }
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->cap) cudaStreamDestroy(b->cap);
    if (b->d_mem) cudaFree(b->d_mem);
    delete b;
}

struct GroupPlan {
    int width = 8;
    bool any = false;
    bool q8 = false;
    int stack_need = 1;
    std::vector<int> members;  // caller indices
};

struct RunPlan {
    std::vector<GroupPlan> groups;
    std::vector<const sg_scene*> scenes;
    std::vector<sg::DevTree> trees;
    std::vector<int> tree_of;  // per caller index
};

sg_status plan_run(const sg_batcher* b, const sg_batch* batches, const sg_scene* const* scene_of, int count,
                   RunPlan& p) {
    std::map<const sg_scene*, int> tree_index;
    p.tree_of.assign(size_t(count), 0);
    for (int i = 0; i < count; ++i) {
        const sg_batch& x = batches[i];
        const sg_scene* s = scene_of ? scene_of[i] : x.scene;
        if (!s) return fail(SG_ERR_INVALID_ARGUMENT, "batch " + std::to_string(i) + ": NULL scene");
        if (x.n < 0) return fail(SG_ERR_INVALID_ARGUMENT, "batch " + std::to_string(i) + ": negative ray count");
        if (x.stride != 0 && x.stride < x.n)
            return fail(SG_ERR_INVALID_ARGUMENT, "batch " + std::to_string(i) + ": stride below n");
        if (x.any != 0 && x.any != 1) return fail(SG_ERR_INVALID_ARGUMENT, "batch " + std::to_string(i) + ": any");
        if (x.n > 0) {
            if (!x.rays) return fail(SG_ERR_INVALID_ARGUMENT, "batch " + std::to_string(i) + ": NULL rays");
            if (x.any ? !x.occluded : (!x.hits.prim || !x.hits.t))
                return fail(SG_ERR_INVALID_ARGUMENT, "batch " + std::to_string(i) + ": NULL output");
        }
        sg::TraceLaunch L;
        sg::DevTree tree;
        int dev = 0;
        sg_status st = sg::scene_launch(s, x.any != 0, &L, &tree, &dev);
        if (st != SG_OK) return st;
        if (dev != b->device)
            return fail(SG_ERR_INVALID_ARGUMENT, "batch " + std::to_string(i) + ": scene on another device");
        auto it = tree_index.find(s);
        if (it == tree_index.end()) {
            it = tree_index.emplace(s, int(p.trees.size())).first;
            p.trees.push_back(tree);
            p.scenes.push_back(s);
        }
        p.tree_of[size_t(i)] = it->second;
        int gi = -1;
        for (size_t g = 0; g < p.groups.size(); ++g)
            if (p.groups[g].width == L.width && p.groups[g].any == L.any && p.groups[g].q8 == L.q8) gi = int(g);
        if (gi < 0) {
            GroupPlan gp;
            gp.width = L.width;
            gp.any = L.any;
            gp.q8 = L.q8;
            p.groups.push_back(gp);
            gi = int(p.groups.size()) - 1;
        }
        GroupPlan& gp = p.groups[size_t(gi)];
        gp.stack_need = std::max(gp.stack_need, L.stack_need);
        gp.members.push_back(i);
    }
    if (int(p.groups.size()) > sg::kMaxBatchGroups) return fail(SG_ERR_LIMIT, "too many kernel groups");
    return SG_OK;
}

sg_status graph_for(sg_batcher* b, const std::vector<std::pair<sg::BatchKernel, int>>& kernels,
                    const std::vector<int>& key, cudaGraphExec_t* out) {
    auto it = b->graphs.find(key);
    if (it != b->graphs.end()) {
        *out = it->second;
        return SG_OK;
    }
    cudaError_t e;
    if (!b->cap) {
        if ((e = cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking)) != cudaSuccess)
            return cuda_fail(e, "cudaStreamCreate");
        if ((e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming)) != cudaSuccess)
            return cuda_fail(e, "cudaEventCreate");
        for (int k = 0; k < sg::kMaxBatchGroups; ++k) {
            if ((e = cudaStreamCreateWithFlags(&b->side[k], cudaStreamNonBlocking)) != cudaSuccess)
                return cuda_fail(e, "cudaStreamCreate");
            if ((e = cudaEventCreateWithFlags(&b->join[k], cudaEventDisableTiming)) != cudaSuccess)
                return cuda_fail(e, "cudaEventCreate");
        }
    }
    const Layout& L = b->lay;
    sg::BatchArgs a;
    a.header = reinterpret_cast<const sg::RunHeader*>(b->d_mem);
    a.batches = reinterpret_cast<const sg::BatchDesc*>(b->d_mem + L.batches);
    a.trees = reinterpret_cast<const sg::DevTree*>(b->d_mem + L.trees);
    a.state = reinterpret_cast<sg::RunState*>(b->d_mem + L.state);
    a.remaining = reinterpret_cast<unsigned long long*>(b->d_mem + L.remaining);
    a.done_ns = reinterpret_cast<long long*>(b->d_mem + L.done);
    if ((e = cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
        return cuda_fail(e, "cudaStreamBeginCapture");
    cudaError_t le = sg::launch_batch_begin(a.header, a.batches, a.state, a.remaining, a.done_ns, b->max_batches,
                                            b->cap);
    if (le == cudaSuccess) le = cudaEventRecord(b->fork, b->cap);
    for (size_t g = 1; g < kernels.size() && le == cudaSuccess; ++g) {
        le = cudaStreamWaitEvent(b->side[g], b->fork, 0);
        a.group = int(g);
        if (le == cudaSuccess) le = kernels[g].first.launch(a, kernels[g].second, b->side[g]);
        if (le == cudaSuccess) le = cudaEventRecord(b->join[g], b->side[g]);
    }
    if (le == cudaSuccess && !kernels.empty()) {
        a.group = 0;
        le = kernels[0].first.launch(a, kernels[0].second, b->cap);
    }
    for (size_t g = 1; g < kernels.size() && le == cudaSuccess; ++g) le = cudaStreamWaitEvent(b->cap, b->join[g], 0);
    cudaGraph_t graph = nullptr;
    e = cudaStreamEndCapture(b->cap, &graph);
    if (le != cudaSuccess || e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return cuda_fail(le != cudaSuccess ? le : e, "capture batch graph");
    }
    cudaGraphExec_t exec = nullptr;
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
    if (b->graphs.size() >= kMaxGraphs) {  // an in-flight executable is freed when it completes
        for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
        b->graphs.clear();
    }
    b->graphs.emplace(key, exec);
    *out = exec;
    return SG_OK;
}

// Plans, stages and enqueues one run. scene_of overrides the batches' scenes
// (the autotuner's width trials); caller holds b->lock and the device.
sg_status enqueue(sg_batcher* b, const sg_batch* batches, const sg_scene* const* scene_of, int count,
                  int64_t budget_ns, const sg_batch_tuning& tun, cudaStream_t stream) {
    if (count < 0 || (count > 0 && !batches)) return fail(SG_ERR_INVALID_ARGUMENT, "bad batch list");
    if (count > b->max_batches) return fail(SG_ERR_LIMIT, "more batches than the batcher was created for");
    if (tun.block_threads != 64 && tun.block_threads != 128 && tun.block_threads != 256)
        return fail(SG_ERR_INVALID_ARGUMENT, "block_threads must be 64, 128 or 256");
    RunPlan p;
    sg_status st = plan_run(b, batches, scene_of, count, p);
    if (st != SG_OK) return st;

    std::vector<std::pair<sg::BatchKernel, int>> kernels;
    std::vector<int> key;
    for (const GroupPlan& gp : p.groups) {
        const int fit = stack_fit(gp.stack_need);
        if (fit == 0) return fail(SG_ERR_LIMIT, "tree too deep for the traversal stack");
        const int stack = std::max(fit, stack_fit(std::max(tun.stack, 1)));
        sg::BatchKernel k = sg::batch_kernel(gp.width, gp.any, stack, tun.block_threads, gp.q8);
        if (!k.launch) return fail(SG_ERR_INTERNAL, "no kernel for this configuration");
        int bps = k.blocks_per_sm();
        if (bps < 1) return fail(SG_ERR_CUDA, "occupancy query failed");
        if (tun.blocks_per_sm > 0) bps = std::min(bps, int(tun.blocks_per_sm));
        const int grid = b->sms * bps;
        kernels.emplace_back(k, grid);
        key.insert(key.end(), {gp.width, int(gp.any), int(gp.q8), stack, int(tun.block_threads), grid});
    }
    cudaGraphExec_t exec = nullptr;
    if ((st = graph_for(b, kernels, key, &exec)) != SG_OK) return st;

    // Stage the tables: wait until the run that last used this buffer has consumed it.
    const int k = b->slot;
    b->slot = (b->slot + 1) % kSlots;
    cudaError_t e = cudaEventSynchronize(b->stage_done[k]);
    if (e != cudaSuccess) return cuda_fail(e, "wait for staging buffer");
    const Layout& L = b->lay;
    char* h = b->h_stage[k];
    sg::RunHeader* hdr = reinterpret_cast<sg::RunHeader*>(h);
    *hdr = sg::RunHeader{};
    hdr->nbatches = count;
    hdr->refill = std::min(32, std::max(1, int(tun.refill_threshold)));
    hdr->budget_ns = budget_ns > 0 ? budget_ns : 0;
    sg::BatchDesc* bd = reinterpret_cast<sg::BatchDesc*>(h + L.batches);
    b->perm.clear();
    int pos = 0;
    for (size_t g = 0; g < p.groups.size(); ++g) {
        const GroupPlan& gp = p.groups[g];
        hdr->groups[g].first = pos;
        hdr->groups[g].count = int(gp.members.size());
        int64_t start = 0;
        for (int i : gp.members) {
            const sg_batch& x = batches[i];
            sg::BatchDesc& d = bd[pos++];
            d = sg::BatchDesc{};
            d.rays = x.rays;
            d.stride = x.stride ? x.stride : x.n;
            d.start = start;
            d.n = x.n;
            d.prim = x.hits.prim;
            d.t = x.hits.t;
            d.u = x.hits.u;
            d.v = x.hits.v;
            d.occ = x.occluded;
            d.tree = p.tree_of[size_t(i)];
            start += x.n;
            b->perm.push_back(i);
        }
        hdr->groups[g].total = start;
    }
    std::copy(p.trees.begin(), p.trees.end(), reinterpret_cast<sg::DevTree*>(h + L.trees));
    const size_t head_bytes = L.batches + size_t(count) * sizeof(sg::BatchDesc);
    if ((e = cudaMemcpyAsync(b->d_mem, h, head_bytes, cudaMemcpyHostToDevice, stream)) != cudaSuccess)
        return cuda_fail(e, "stage batch table");
    if (!p.trees.empty() &&
        (e = cudaMemcpyAsync(b->d_mem + L.trees, h + L.trees, p.trees.size() * sizeof(sg::DevTree),
                             cudaMemcpyHostToDevice, stream)) != cudaSuccess)
        return cuda_fail(e, "stage tree table");
    if ((e = cudaGraphLaunch(exec, stream)) != cudaSuccess) return cuda_fail(e, "cudaGraphLaunch");
    if ((e = cudaEventRecord(b->stage_done[k], stream)) != cudaSuccess) return cuda_fail(e, "cudaEventRecord");
    return SG_OK;
}

// Median device time (ms) of `reps` runs after one untimed run.
sg_status time_runs(sg_batcher* b, const sg_batch* batches, const sg_scene* const* scene_of, int count,
                    const sg_batch_tuning& tun, int reps, cudaStream_t s, float* ms) {
    cudaEvent_t e0, e1;
    cudaError_t e;
    if ((e = cudaEventCreate(&e0)) != cudaSuccess) return cuda_fail(e, "cudaEventCreate");
    if ((e = cudaEventCreate(&e1)) != cudaSuccess) {
        cudaEventDestroy(e0);
        return cuda_fail(e, "cudaEventCreate");
    }
    std::vector<float> t;
    sg_status st = enqueue(b, batches, scene_of, count, 0, tun, s);
    for (int r = 0; r < reps && st == SG_OK; ++r) {
        cudaEventRecord(e0, s);
        st = enqueue(b, batches, scene_of, count, 0, tun, s);
        cudaEventRecord(e1, s);
        if (st != SG_OK) break;
        if ((e = cudaEventSynchronize(e1)) != cudaSuccess) {
            st = cuda_fail(e, "time batch run");
            break;
        }
        float x = 0.0f;
        cudaEventElapsedTime(&x, e0, e1);
        t.push_back(x);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != SG_OK) return st;
    std::sort(t.begin(), t.end());
    *ms = t[t.size() / 2];
    return SG_OK;
}

}  // namespace

extern "C" {

sg_status sg_batcher_create(int32_t device, int32_t max_batches, sg_batcher** out) {
    if (!out) return fail(SG_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (max_batches < 1 || max_batches > (1 << 20)) return fail(SG_ERR_INVALID_ARGUMENT, "max_batches out of range");
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDeviceCount");
    if (device < 0 || device >= ndev) return fail(SG_ERR_INVALID_ARGUMENT, "no such CUDA device");
    DeviceGuard g(device);
    if (!g.ok) return fail(SG_ERR_CUDA, "cudaSetDevice failed");
    sg_batcher* b = new (std::nothrow) sg_batcher;
    if (!b) return fail(SG_ERR_OUT_OF_MEMORY, "host allocation failed");
    b->device = device;
    b->max_batches = max_batches;
    b->lay = Layout(max_batches);
    if ((e = cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess) {
        release(b);
        return cuda_fail(e, "cudaDeviceGetAttribute");
    }
    if ((e = cudaMalloc(&b->d_mem, b->lay.total)) != cudaSuccess) {
        release(b);
        return e == cudaErrorMemoryAllocation ? fail(SG_ERR_OUT_OF_MEMORY, "batcher tables") : cuda_fail(e, "cudaMalloc");
    }
    for (int k = 0; k < kSlots; ++k) {
        if ((e = cudaMallocHost(&b->h_stage[k], b->lay.stage)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&b->stage_done[k], cudaEventDisableTiming)) != cudaSuccess) {
            release(b);
            return cuda_fail(e, "batcher staging");
        }
    }
    *out = b;
    return SG_OK;
}

sg_status sg_batcher_destroy(sg_batcher* b) {
    if (!b) return fail(SG_ERR_INVALID_ARGUMENT, "NULL batcher");
    release(b);
    return SG_OK;
}

sg_status sg_batcher_set_tuning(sg_batcher* b, const sg_batch_tuning* t) {
    if (!b || !t) return fail(SG_ERR_INVALID_ARGUMENT, "NULL argument");
    if (t->block_threads != 64 && t->block_threads != 128 && t->block_threads != 256)
        return fail(SG_ERR_INVALID_ARGUMENT, "block_threads must be 64, 128 or 256");
    if (t->stack != 0 && t->stack != 64 && t->stack != 128 && t->stack != 256)
        return fail(SG_ERR_INVALID_ARGUMENT, "stack must be 0, 64, 128 or 256");
    if (t->refill_threshold < 1 || t->refill_threshold > 32)
        return fail(SG_ERR_INVALID_ARGUMENT, "refill_threshold must be in 1..32");
    if (t->blocks_per_sm < 0) return fail(SG_ERR_INVALID_ARGUMENT, "blocks_per_sm < 0");
    std::lock_guard<std::mutex> lk(b->lock);
    b->tuning = *t;
    return SG_OK;
}

sg_status sg_batcher_get_tuning(const sg_batcher* b, sg_batch_tuning* t) {
    if (!b || !t) return fail(SG_ERR_INVALID_ARGUMENT, "NULL argument");
    *t = b->tuning;
    return SG_OK;
}

sg_status sg_batcher_run(sg_batcher* b, const sg_batch* batches, int32_t count, int64_t budget_ns, void* stream) {
    if (!b) return fail(SG_ERR_INVALID_ARGUMENT, "NULL batcher");
    std::lock_guard<std::mutex> lk(b->lock);
    DeviceGuard g(b->device);
    if (!g.ok) return fail(SG_ERR_CUDA, "cudaSetDevice failed");
    return enqueue(b, batches, nullptr, count, budget_ns, b->tuning, (cudaStream_t)stream);
}

sg_status sg_batcher_wait(sg_batcher* b, int64_t* done_ns, int32_t count, void* stream) {
    if (!b) return fail(SG_ERR_INVALID_ARGUMENT, "NULL batcher");
    std::lock_guard<std::mutex> lk(b->lock);
    if (count != int(b->perm.size())) return fail(SG_ERR_INVALID_ARGUMENT, "count differs from the last run's");
    if (count > 0 && !done_ns) return fail(SG_ERR_INVALID_ARGUMENT, "NULL done_ns");
    DeviceGuard g(b->device);
    if (!g.ok) return fail(SG_ERR_CUDA, "cudaSetDevice failed");
    cudaStream_t s = (cudaStream_t)stream;
    std::vector<long long> d(size_t(count) + 1);
    sg::RunState rs{};
    cudaError_t e = cudaSuccess;
    if (count > 0)
        e = cudaMemcpyAsync(d.data(), b->d_mem + b->lay.done, size_t(count) * sizeof(long long),
                            cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&rs, b->d_mem + b->lay.state, sizeof(rs), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, "read batch completion");
    for (int k = 0; k < count; ++k) done_ns[b->perm[size_t(k)]] = d[size_t(k)];
    if (rs.status & sg::kBatchStackOverflow) return fail(SG_ERR_INTERNAL, "traversal stack bound exceeded");
    if (rs.status & sg::kBatchBudgetCut) return fail(SG_ERR_LIMIT, "time budget ended the run early");
    return SG_OK;
}

sg_status sg_batcher_autotune(sg_batcher* b, const sg_batch* batches, const sg_scene* const* alternatives,
                              int32_t count, int32_t reps, int32_t* use_alternative, sg_batch_tuning* best,
                              void* stream) {
    if (!b || (count > 0 && !batches)) return fail(SG_ERR_INVALID_ARGUMENT, "NULL argument");
    if (alternatives && !use_alternative) return fail(SG_ERR_INVALID_ARGUMENT, "NULL use_alternative");
    if (count < 1) return fail(SG_ERR_INVALID_ARGUMENT, "nothing to tune on");
    if (reps <= 0) reps = 3;
    std::lock_guard<std::mutex> lk(b->lock);
    DeviceGuard g(b->device);
    if (!g.ok) return fail(SG_ERR_CUDA, "cudaSetDevice failed");
    cudaStream_t s = (cudaStream_t)stream;
    sg_batch_tuning cur = b->tuning;
    std::vector<const sg_scene*> scene_of(static_cast<size_t>(count));
    for (int i = 0; i < count; ++i) scene_of[size_t(i)] = batches[i].scene;

    // 1. Tree width per scene: time the scene's batches alone with each tree.
    if (alternatives) {
        std::map<const sg_scene*, const sg_scene*> alt;
        for (int i = 0; i < count; ++i) {
            use_alternative[i] = 0;
            const sg_scene* a = alternatives[i];
            if (!a) continue;
            auto it = alt.find(batches[i].scene);
            if (it != alt.end() && it->second != a)
                return fail(SG_ERR_INVALID_ARGUMENT, "batches of one scene name different alternatives");
            sg_scene_info ia, ib;
            if (sg_scene_info_get(batches[i].scene, &ia) != SG_OK || sg_scene_info_get(a, &ib) != SG_OK)
                return fail(SG_ERR_INVALID_ARGUMENT, "bad scene");
            if (ia.triangles != ib.triangles)
                return fail(SG_ERR_INVALID_ARGUMENT, "alternative scene has a different triangle count");
            alt[batches[i].scene] = a;
        }
        for (const auto& kv : alt) {
            std::vector<sg_batch> sub;
            std::vector<int> idx;
            for (int i = 0; i < count; ++i)
                if (batches[i].scene == kv.first) {
                    sub.push_back(batches[i]);
                    idx.push_back(i);
                }
            std::vector<const sg_scene*> with_alt(sub.size(), kv.second);
            float t0 = 0.0f, t1 = 0.0f;
            sg_status st = time_runs(b, sub.data(), nullptr, int(sub.size()), cur, reps, s, &t0);
            if (st == SG_OK) st = time_runs(b, sub.data(), with_alt.data(), int(sub.size()), cur, reps, s, &t1);
            if (st != SG_OK) return st;
            if (t1 < t0)
                for (int i : idx) {
                    use_alternative[i] = 1;
                    scene_of[size_t(i)] = kv.second;
                }
        }
    }

    // 2. Kernel shape: coordinate descent over block threads, refill threshold
    //    and stack size, two passes at most.
    float cur_ms = 0.0f;
    sg_status st = time_runs(b, batches, scene_of.data(), count, cur, reps, s, &cur_ms);
    if (st != SG_OK) return st;
    const std::vector<int> blocks = {64, 128, 256};
    const std::vector<int> refills = {1, 2, 4, 8, 16, 24, 32};
    const std::vector<int> stacks = {0, 128, 256};
    for (int pass = 0; pass < 2; ++pass) {
        bool changed = false;
        for (int param = 0; param < 3; ++param) {
            const std::vector<int>& vals = param == 0 ? blocks : param == 1 ? refills : stacks;
            for (int v : vals) {
                sg_batch_tuning t = cur;
                int& field = param == 0 ? t.block_threads : param == 1 ? t.refill_threshold : t.stack;
                if (field == v) continue;
                field = v;
                float ms = 0.0f;
                if ((st = time_runs(b, batches, scene_of.data(), count, t, reps, s, &ms)) != SG_OK) return st;
                if (ms < cur_ms * 0.99f) {
                    cur = t;
                    cur_ms = ms;
                    changed = true;
                }
            }
        }
        if (!changed) break;
    }
    b->tuning = cur;
    if (best) *best = cur;
    return SG_OK;
}

}  // extern "C"
