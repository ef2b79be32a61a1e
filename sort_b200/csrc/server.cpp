// sg_server (include/sortgpu.h): the host side of the render server.
//
// One loop thread per server owns the GPU work: it admits the queued
// requests the solo lanes do not take (in queue order) while a request-table
// slot and a contiguous image range of the pixel budget are free, stages the
// admissions, replays the captured bounce-step graph, and reads the
// per-request completion flags of the previous replay while the next one
// runs (two replays in flight). A completed request's image is copied to its
// host buffer on a second stream, then its slot and image range are released
// and its waiters are woken.
//
// Solo lanes: a multi-sample request of at least solo_pixels pixels waits for
// one of the lanes (oldest first) and is rendered the way sg_pt_render
// renders a frame, one wave per sample (pt_wave, on the lane's own buffers),
// two samples in flight on the lane's streams, while the pool serves the
// other requests; the lane holding the oldest request uses the high-priority
// streams. After its last wave the lane scales the image and the request
// completes like a pool request. In the pool a pixel's samples run one after
// another in one slot, so a request there finishes with its slowest pixel's
// chain; the waves have no such tail. Each pixel's samples are added in sample
// order either way, so the image is sg_pt_render's.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "pt_wave.h"
#include "scene_access.h"
#include "serve_kernels.h"
#include "sortgpu.h"
#include "trace_kernels.h"

namespace {

constexpr int kMaxScenes = 64;
constexpr int kSoloLanes = 2;  // large requests rendered as whole-frame waves at once

int64_t now_ns() {
    return std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

size_t align_up(size_t x) { return (x + 255) & ~size_t(255); }

sg_status fail(sg_status s, const std::string& msg) { return sg::set_error(s, msg.c_str()); }

// First-fit allocator of pixel ranges of the image arena.
class Arena {
public:
    explicit Arena(int64_t n) {
        if (n > 0) free_[0] = n;
    }
    int64_t alloc(int64_t n) {
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < n) continue;
            const int64_t off = it->first, len = it->second;
            free_.erase(it);
            if (len > n) free_[off + n] = len - n;
            return off;
        }
        return -1;
    }
    void release(int64_t off, int64_t n) {
        auto it = free_.emplace(off, n).first;
        auto next = std::next(it);
        if (next != free_.end() && it->first + it->second == next->first) {
            it->second += next->second;
            free_.erase(next);
        }
        if (it != free_.begin()) {
            auto prev = std::prev(it);
            if (prev->first + prev->second == it->first) {
                prev->second += it->second;
                free_.erase(it);
            }
        }
    }

private:
    std::map<int64_t, int64_t> free_;
};

struct Ticket {
    sg_request req{};
    int64_t submit_ns = 0, admit_ns = 0, done_ns = 0;
    int status = SG_OK;
    int slot = -1;         // request-table index while admitted
    int64_t arena = -1;    // first pixel of its image range
    int64_t replay = -1;   // first replay that sees it admitted
    bool cancel = false;
    bool complete = false;
};

}  // namespace

struct sg_server {
    sg_server_opts opts{};
    int width = 0;
    int node_format = -1;
    int stack_need = 1;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::thread loop;
    bool stop = false;
    sg_status loop_status = SG_OK;
    std::string loop_msg;
    int64_t next_ticket = 1;
    std::deque<int64_t> pending;
    std::unordered_map<int64_t, Ticket> tickets;
    std::vector<int64_t> slot_ticket;
    std::vector<int> free_slots;
    std::vector<int> to_cancel;
    Arena arena{0};
    int64_t admitted = 0;
    std::vector<sg::SrvScene> scenes;
    std::vector<sg::TraceLaunch> launches;  // per scene, for the solo waves
    int64_t solo_pixels = 0;                // 0: no solo phase
    // Solo lanes: each renders one large request as whole-frame waves
    // (pt_wave), two samples in flight on its own buffer sets and stream
    // pairs (sample k on [k % 2]), beside the pool's `stream`.
    struct Lane {
        int64_t id = -1;  // ticket in its solo phase
        int next = 0;     // next sample to queue a wave for
        int done = 0;     // waves finished
        int last = 0;     // waves to run (spp)
        bool finishing = false;  // every wave queued (and the scale), or cancelled: waiting for `end`
        sg::PtWave w[2] = {};
        // The waves and their shadow rays (pt_wave.h), [priority][sample % 2]:
        // the lane holding the oldest request queues its waves on the
        // high-priority streams, the others (and the pool) on normal ones.
        cudaStream_t stream[2][2] = {};
        cudaStream_t side[2][2] = {};
        cudaStream_t last_on = nullptr;  // the stream of the newest wave
        cudaEvent_t flushed[2] = {};   // image additions, chained in sample order
        cudaEvent_t wave_done[2] = {};
        cudaEvent_t ready = nullptr;   // the ticket's image is zeroed
        cudaEvent_t end = nullptr;     // its last wave (and the scale) is done
    };
    std::vector<Lane> lanes;
    char* d_solo = nullptr;
    // The bounce steps' side stream (continuation rays beside shadow rays,
    // serve_kernels.h) and its events; captured into the graph.
    cudaStream_t pool_side = nullptr;
    cudaEvent_t pool_forked = nullptr, pool_joined = nullptr;
    sg_server_stats stats{};
    // device
    char* d_mem = nullptr;
    sg::SrvBuffers b{};
    sg::SrvRequest* d_requests = nullptr;
    sg::SrvScene* d_scenes = nullptr;
    sg::SrvControl* d_control = nullptr;
    sg::SrvCounters* d_counters = nullptr;
    float* d_images = nullptr;
    // host (pinned)
    sg::SrvRequest* h_requests = nullptr;
    unsigned* h_units = nullptr;
    sg::SrvControl* h_control[2] = {};
    int* h_done[2] = {};
    sg::SrvCounters* h_counters[2] = {};
    cudaStream_t stream = nullptr, copy_stream = nullptr;
    cudaEvent_t replay_done[2] = {}, copy_done = nullptr;
    cudaGraphExec_t graph = nullptr;
    int graph_stack = 0;
};

namespace {

void free_server(sg_server* S) {
    cudaSetDevice(S->opts.device);
    if (S->stream) cudaStreamSynchronize(S->stream);
    if (S->copy_stream) cudaStreamSynchronize(S->copy_stream);
    if (S->graph) cudaGraphExecDestroy(S->graph);
    for (int k = 0; k < 2; ++k) {
        if (S->h_control[k]) cudaFreeHost(S->h_control[k]);
        if (S->h_done[k]) cudaFreeHost(S->h_done[k]);
        if (S->h_counters[k]) cudaFreeHost(S->h_counters[k]);
        if (S->replay_done[k]) cudaEventDestroy(S->replay_done[k]);
    }
    if (S->copy_done) cudaEventDestroy(S->copy_done);
    for (sg_server::Lane& L : S->lanes) {
        for (int k = 0; k < 2; ++k) {
            for (cudaStream_t t : {L.stream[0][k], L.stream[1][k], L.side[0][k], L.side[1][k]})
                if (t) {
                    cudaStreamSynchronize(t);
                    cudaStreamDestroy(t);
                }
            for (cudaEvent_t ev : {L.w[k].shaded, L.w[k].shadowed, L.flushed[k], L.wave_done[k]})
                if (ev) cudaEventDestroy(ev);
        }
        for (cudaEvent_t ev : {L.ready, L.end})
            if (ev) cudaEventDestroy(ev);
    }
    if (S->pool_side) cudaStreamDestroy(S->pool_side);
    if (S->pool_forked) cudaEventDestroy(S->pool_forked);
    if (S->pool_joined) cudaEventDestroy(S->pool_joined);

    if (S->d_solo) cudaFree(S->d_solo);
    if (S->h_requests) cudaFreeHost(S->h_requests);
    if (S->h_units) cudaFreeHost(S->h_units);
    if (S->stream) cudaStreamDestroy(S->stream);
    if (S->copy_stream) cudaStreamDestroy(S->copy_stream);
    if (S->d_mem) cudaFree(S->d_mem);
    delete S;
}

// Called with S->mu held: ends a ticket and wakes its waiters.
void complete(sg_server* S, Ticket& t, int status) {
    t.status = status;
    t.done_ns = now_ns();
    t.complete = true;
    S->cv_done.notify_all();
}

sg_status capture(sg_server* S) {
    const int stack = S->stack_need <= 64 ? 64 : S->stack_need <= 128 ? 128 : 256;
    if (S->graph && S->graph_stack == stack) return SG_OK;
    if (S->graph) {
        cudaGraphExecDestroy(S->graph);
        S->graph = nullptr;
    }
    cudaError_t e = cudaStreamBeginCapture(S->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return fail(SG_ERR_CUDA, std::string("begin capture: ") + cudaGetErrorString(e));
    const sg::SrvStreams streams{S->stream, S->pool_side, S->pool_forked, S->pool_joined};
    cudaError_t le = sg::srv_enqueue_steps(S->b, S->opts.steps_per_poll, S->width, stack,
                                           S->node_format == SG_NODES_QUANT8, streams);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(S->stream, &g);
    if (le != cudaSuccess || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return fail(SG_ERR_CUDA, std::string("capture bounce steps: ") + cudaGetErrorString(le != cudaSuccess ? le : e));
    }
    e = cudaGraphInstantiate(&S->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(SG_ERR_CUDA, std::string("instantiate: ") + cudaGetErrorString(e));
    S->graph_stack = stack;
    return SG_OK;
}

// Gives ticket id a request-table slot and an image range, stages its table
// entry and zeroes its image (S->mu held). False when either is not free.
bool reserve(sg_server* S, int64_t id) {
    if (S->free_slots.empty()) return false;
    Ticket& t = S->tickets[id];
    const int64_t P = int64_t(t.req.width) * t.req.height;
    const int64_t off = S->arena.alloc(P);
    if (off < 0) return false;  // FIFO: wait for image memory
    const int r = S->free_slots.back();
    S->free_slots.pop_back();
    sg::SrvRequest& q = S->h_requests[r];
    q = sg::SrvRequest{};
    q.cam = sg::make_camera(t.req.camera, t.req.width, t.req.height);
    q.key = make_uint2((uint32_t)t.req.seed, (uint32_t)(t.req.seed >> 32));
    q.image = S->d_images + 3 * off;
    q.scene = t.req.scene;
    q.width = t.req.width;
    q.height = t.req.height;
    q.spp = t.req.spp;
    q.max_depth = t.req.max_depth;
    q.inv_spp = 1.0f / (float)t.req.spp;
    q.cancelled = 0;
    S->h_units[r] = (unsigned)P;
    cudaMemcpyAsync(S->d_requests + r, &q, sizeof(q), cudaMemcpyHostToDevice, S->stream);
    cudaMemsetAsync(q.image, 0, size_t(P) * 3 * sizeof(float), S->stream);
    cudaMemcpyAsync(S->b.units_left + r, &S->h_units[r], sizeof(unsigned), cudaMemcpyHostToDevice, S->stream);
    cudaMemsetAsync(S->b.done + r, 0, sizeof(int), S->stream);
    t.slot = r;
    t.arena = off;
    t.admit_ns = now_ns();
    S->slot_ticket[size_t(r)] = id;
    return true;
}

// Enters a reserved ticket's pixels, from sample0 on, into the next replay's
// admissions (S->mu held).
void enter_pool(sg_server* S, sg::SrvControl& ctl, int64_t id, int sample0, int64_t replay) {
    Ticket& t = S->tickets[id];
    const int64_t P = int64_t(t.req.width) * t.req.height;
    ctl.admit[ctl.nadmit].request = t.slot;
    ctl.admit[ctl.nadmit].pixels = (int32_t)P;
    ctl.admit[ctl.nadmit].first = ctl.admit_total;
    ctl.admit[ctl.nadmit].sample0 = sample0;
    ctl.admit[ctl.nadmit].pad = 0;
    ctl.nadmit++;
    ctl.admit_total += P;
    t.replay = replay;
    S->admitted++;
}

// A request the solo lanes take (large, two or more samples); it waits in the
// queue for a free lane rather than entering the pool.
bool solo_kind(const sg_server* S, const Ticket& t) {
    return S->solo_pixels > 0 && int64_t(t.req.width) * t.req.height >= S->solo_pixels && t.req.spp >= 2;
}

// Admits into the control block of the next replay (S->mu held): first the
// requests whose solo phase ended, then the queued requests the lanes do not
// take, in queue order.
void admit(sg_server* S, sg::SrvControl& ctl, int64_t replay) {
    ctl.nadmit = 0;
    ctl.admit_total = 0;
    for (auto it = S->pending.begin(); it != S->pending.end() && ctl.nadmit < sg::kSrvMaxAdmit;) {
        const int64_t id = *it;
        if (solo_kind(S, S->tickets[id])) {
            ++it;
            continue;
        }
        if (!reserve(S, id)) break;  // FIFO: wait for image memory
        it = S->pending.erase(it);
        enter_pool(S, ctl, id, 0, replay);
    }
    for (int r : S->to_cancel) {
        S->h_requests[r].cancelled = 1;
        cudaMemcpyAsync(&S->d_requests[r].cancelled, &S->h_requests[r].cancelled, sizeof(int32_t),
                        cudaMemcpyHostToDevice, S->stream);
    }
    S->to_cancel.clear();
}

// Gives each free lane the oldest queued request it takes (S->mu held):
// reserves it and makes the lane's streams wait for its zeroed image.
void start_solo(sg_server* S) {
    for (size_t l = 0; l < S->lanes.size(); ++l) {
        sg_server::Lane& L = S->lanes[l];
        if (L.id >= 0) continue;
        auto it = std::find_if(S->pending.begin(), S->pending.end(),
                               [&](int64_t id) { return solo_kind(S, S->tickets[id]); });
        if (it == S->pending.end()) return;
        const int64_t id = *it;
        if (!reserve(S, id)) return;
        S->pending.erase(it);
        Ticket& t = S->tickets[id];
        // Never in a replay: a completion flag read back for its table slot
        // belongs to the slot's previous request.
        t.replay = INT64_MAX;
        cudaEventRecord(L.ready, S->stream);
        for (auto& pair : L.stream)
            for (cudaStream_t t : pair) cudaStreamWaitEvent(t, L.ready, 0);
        L.id = id;
        L.next = L.done = 0;
        L.last = t.req.spp;
        L.finishing = false;
    }
}

bool lanes_busy(const sg_server* S) {
    for (const sg_server::Lane& L : S->lanes)
        if (L.id >= 0) return true;
    return false;
}

// Completes a lane's request once its last wave (and the scale) is done:
// copies the image out (unless cancelled), frees its table slot and image
// range, wakes its waiters, frees the lane.
sg_status finish_lane(sg_server* S, sg_server::Lane& L) {
    cudaError_t e = cudaSuccess;
    int64_t id;
    bool cancelled;
    void* dst;
    const float* src;
    size_t bytes;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        id = L.id;
        Ticket& t = S->tickets[id];
        cancelled = t.cancel;
        dst = t.req.image;
        src = S->d_images + 3 * t.arena;
        bytes = size_t(t.req.width) * t.req.height * 3 * sizeof(float);
    }
    if (!cancelled) {
        if ((e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, S->copy_stream)) != cudaSuccess ||
            (e = cudaStreamSynchronize(S->copy_stream)) != cudaSuccess)
            return fail(SG_ERR_CUDA, std::string("copy image: ") + cudaGetErrorString(e));
    }
    std::lock_guard<std::mutex> lk(S->mu);
    Ticket& t = S->tickets[id];
    const int64_t P = int64_t(t.req.width) * t.req.height;
    S->arena.release(t.arena, P);
    S->slot_ticket[size_t(t.slot)] = -1;
    S->free_slots.push_back(t.slot);
    t.slot = -1;
    S->stats.requests_done++;
    if (!cancelled) S->stats.samples_done += P * t.req.spp;
    complete(S, t, cancelled ? SG_ERR_CANCELLED : SG_OK);
    L.id = -1;
    L.finishing = false;
    S->cv_work.notify_all();
    return SG_OK;
}

// Keeps two waves of a lane's request queued; after the last one (or a
// cancellation, or the server's stop) scales the image and, once that is
// done, completes the request.
sg_status pump_lane(sg_server* S, int l) {
    sg_server::Lane& L = S->lanes[size_t(l)];
    if (L.id < 0) return SG_OK;
    cudaError_t e = cudaSuccess;
    if (L.finishing) {
        e = cudaEventQuery(L.end);
        if (e == cudaErrorNotReady) {
            cudaGetLastError();  // not an error (see below)
            return SG_OK;
        }
        if (e != cudaSuccess) return fail(SG_ERR_CUDA, std::string("solo wave: ") + cudaGetErrorString(e));
        return finish_lane(S, L);
    }
    while (L.done < L.next) {  // retire finished waves
        e = cudaEventQuery(L.wave_done[L.done % 2]);
        if (e == cudaErrorNotReady) {
            // Not an error, but the runtime keeps it as the last error, which
            // the next launch check (cudaGetLastError) would report.
            cudaGetLastError();
            e = cudaSuccess;
            break;
        }
        if (e != cudaSuccess) return fail(SG_ERR_CUDA, std::string("solo wave: ") + cudaGetErrorString(e));
        L.done++;
    }
    sg::SrvRequest q;
    sg::SrvScene sc;
    sg::TraceLaunch base;
    bool end = false, oldest = true;
    {
        std::lock_guard<std::mutex> lk(S->mu);  // add_scene may grow the scene tables meanwhile
        const Ticket& t = S->tickets[L.id];
        q = S->h_requests[t.slot];
        sc = S->scenes[size_t(q.scene)];
        base = S->launches[size_t(q.scene)];
        end = S->stop || t.cancel;
        for (const sg_server::Lane& o : S->lanes)  // an older request in another lane
            if (o.id >= 0 && o.id != L.id) {
                const Ticket& u = S->tickets[o.id];
                if (u.submit_ns < t.submit_ns || (u.submit_ns == t.submit_ns && o.id < L.id)) oldest = false;
            }
    }
    const int rows = std::max(1, L.w[0].cap / q.width);  // rows per band: a band fits the wave buffers
    while (!end && L.next < L.last && L.next - L.done < 2) {
        // Sample k on buffer set and stream pair k % 2; its image additions
        // wait for sample k - 1's.
        const int k = L.next;
        sg::PtWave w = L.w[k % 2];
        w.flush_after = k > 0 ? L.flushed[(k - 1) % 2] : nullptr;
        w.flush_done = L.flushed[k % 2];
        const int prio = oldest ? 0 : 1;
        const cudaStream_t on = L.stream[prio][k % 2];
        w.side = L.side[prio][k % 2];
        for (int y = 0; y < q.height && e == cudaSuccess; y += rows) {
            const int y1 = std::min(q.height, y + rows);
            const int p0 = y * q.width;
            e = sg::pt_wave(sc.pt, base, sc.tree, q.cam, q.width, q.height, p0, (y1 - y) * q.width, q.key, k,
                            q.max_depth, w, q.image + 3 * int64_t(p0), on);
        }
        if (e == cudaSuccess) e = cudaEventRecord(L.wave_done[k % 2], on);
        if (e != cudaSuccess) return fail(SG_ERR_CUDA, std::string("solo wave: ") + cudaGetErrorString(e));
        L.last_on = on;
        L.next++;
        std::lock_guard<std::mutex> lk(S->mu);
        S->stats.solo_waves++;
    }
    if (end || L.next == L.last) {
        // After the last wave, whose additions came after every earlier one's:
        // the 1/spp scale (as sg_pt_render's), then `end`.
        const cudaStream_t last = L.next > 0 ? L.last_on : L.stream[1][0];
        if (!end && (e = sg::pt_scale(q.image, 3 * int64_t(q.width) * q.height, q.inv_spp, last)) != cudaSuccess)
            return fail(SG_ERR_CUDA, std::string("solo scale: ") + cudaGetErrorString(e));
        if ((e = cudaEventRecord(L.end, last)) != cudaSuccess)
            return fail(SG_ERR_CUDA, std::string("solo end: ") + cudaGetErrorString(e));
        L.finishing = true;
    }
    return SG_OK;
}

// Blocks until the oldest queued wave of a busy lane has finished, or a
// finishing lane's end.
sg_status wait_solo(sg_server* S) {
    for (sg_server::Lane& L : S->lanes) {
        if (L.id < 0) continue;
        if (L.finishing) {
            const cudaError_t e = cudaEventSynchronize(L.end);
            if (e != cudaSuccess) return fail(SG_ERR_CUDA, std::string("solo wave: ") + cudaGetErrorString(e));
            return SG_OK;
        }
        if (L.done >= L.next) continue;
        const cudaError_t e = cudaEventSynchronize(L.wave_done[L.done % 2]);
        if (e != cudaSuccess) return fail(SG_ERR_CUDA, std::string("solo wave: ") + cudaGetErrorString(e));
        L.done++;
        return SG_OK;
    }
    return SG_OK;
}

// Reads the completion flags of replay k and hands out finished requests.
sg_status collect(sg_server* S, int k, int64_t replay) {
    cudaError_t e = cudaEventSynchronize(S->replay_done[k]);
    if (e != cudaSuccess) return fail(SG_ERR_CUDA, std::string("bounce steps: ") + cudaGetErrorString(e));
    std::vector<int64_t> done;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        for (size_t r = 0; r < S->slot_ticket.size(); ++r) {
            const int64_t id = S->slot_ticket[r];
            if (id < 0 || !S->h_done[k][r]) continue;
            Ticket& t = S->tickets[id];
            if (t.replay > replay) continue;  // admitted after this replay
            done.push_back(id);
        }
        const sg::SrvCounters& c = *S->h_counters[k];
        S->stats.extension_rays = (int64_t)c.ext_rays;
        S->stats.shadow_rays = (int64_t)c.shadow_rays;
    }
    if (done.empty()) return SG_OK;
    if ((e = cudaStreamWaitEvent(S->copy_stream, S->replay_done[k], 0)) != cudaSuccess)
        return fail(SG_ERR_CUDA, cudaGetErrorString(e));
    {
        std::lock_guard<std::mutex> lk(S->mu);
        for (int64_t id : done) {
            Ticket& t = S->tickets[id];
            if (t.cancel) continue;
            const size_t bytes = size_t(t.req.width) * t.req.height * 3 * sizeof(float);
            if ((e = cudaMemcpyAsync(t.req.image, S->d_images + 3 * t.arena, bytes, cudaMemcpyDeviceToHost,
                                     S->copy_stream)) != cudaSuccess)
                return fail(SG_ERR_CUDA, std::string("copy image: ") + cudaGetErrorString(e));
        }
    }
    if ((e = cudaEventRecord(S->copy_done, S->copy_stream)) != cudaSuccess ||
        (e = cudaEventSynchronize(S->copy_done)) != cudaSuccess)
        return fail(SG_ERR_CUDA, std::string("copy image: ") + cudaGetErrorString(e));
    std::lock_guard<std::mutex> lk(S->mu);
    for (int64_t id : done) {
        Ticket& t = S->tickets[id];
        const int64_t P = int64_t(t.req.width) * t.req.height;
        S->arena.release(t.arena, P);
        S->slot_ticket[size_t(t.slot)] = -1;
        S->free_slots.push_back(t.slot);
        t.slot = -1;
        S->admitted--;
        S->stats.requests_done++;
        if (!t.cancel) S->stats.samples_done += P * t.req.spp;
        complete(S, t, t.cancel ? SG_ERR_CANCELLED : SG_OK);
    }
    S->cv_work.notify_all();
    return SG_OK;
}

void serve_loop(sg_server* S) {
    cudaSetDevice(S->opts.device);
    int64_t j = 0;
    bool inflight = false;
    sg_status st = SG_OK;
    for (;;) {
        bool launch = false;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            if (!inflight && !lanes_busy(S))
                S->cv_work.wait(lk, [&] {
                    return S->stop || !S->pending.empty() || S->admitted > 0;
                });
            if (S->stop) break;
            admit(S, *S->h_control[j % 2], j);
            start_solo(S);
            launch = S->admitted > 0;
        }
        for (int l = 0; l < int(S->lanes.size()) && st == SG_OK; ++l) st = pump_lane(S, l);
        if (st != SG_OK) break;
        if (launch) {
            cudaError_t e = cudaSuccess;
            if ((st = capture(S)) != SG_OK) break;
            e = cudaMemcpyAsync(S->d_control, S->h_control[j % 2], sizeof(sg::SrvControl), cudaMemcpyHostToDevice,
                                S->stream);
            if (e == cudaSuccess) e = cudaGraphLaunch(S->graph, S->stream);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(S->h_done[j % 2], S->b.done, sizeof(int) * size_t(S->opts.max_requests),
                                    cudaMemcpyDeviceToHost, S->stream);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(S->h_counters[j % 2], S->d_counters, sizeof(sg::SrvCounters),
                                    cudaMemcpyDeviceToHost, S->stream);
            if (e == cudaSuccess) e = cudaEventRecord(S->replay_done[j % 2], S->stream);
            if (e != cudaSuccess) {
                st = fail(SG_ERR_CUDA, std::string("replay: ") + cudaGetErrorString(e));
                break;
            }
            std::lock_guard<std::mutex> lk(S->mu);
            S->stats.graph_replays++;
        }
        if (inflight && (st = collect(S, int((j - 1) % 2), j - 1)) != SG_OK) break;
        if (!inflight && !launch && (st = wait_solo(S)) != SG_OK) break;  // only the solo waves run
        inflight = launch;
        if (launch) ++j;
    }
    if (st == SG_OK && inflight) st = collect(S, int((j - 1) % 2), j - 1);
    for (const sg_server::Lane& L : S->lanes)
        for (const auto& pair : L.stream)
            for (cudaStream_t t : pair) cudaStreamSynchronize(t);
    cudaStreamSynchronize(S->stream);
    std::lock_guard<std::mutex> lk(S->mu);
    if (st != SG_OK) {
        S->loop_status = st;
        S->loop_msg = sg_last_error();
    }
    for (auto& kv : S->tickets)
        if (!kv.second.complete) complete(S, kv.second, st != SG_OK ? int(st) : int(SG_ERR_CANCELLED));
    S->pending.clear();
    S->stop = true;
}

}  // namespace

extern "C" {

void sg_default_server_opts(sg_server_opts* o) {
    if (!o) return;
    o->device = 0;
    o->max_requests = 1024;
    o->path_slots = int64_t(1) << 20;
    o->pixel_budget = int64_t(1) << 24;
    o->steps_per_poll = 4;
    o->samples_per_claim = 1;
    o->solo_pixels = 0;
}

sg_status sg_server_create(const sg_server_opts* opts, sg_server** out) {
    if (!opts || !out) return fail(SG_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = nullptr;
    const sg_server_opts& o = *opts;
    if (o.max_requests < 1 || o.max_requests > 65535) return fail(SG_ERR_INVALID_ARGUMENT, "max_requests out of range");
    if (o.path_slots < 32 || o.path_slots > (int64_t(1) << 28))
        return fail(SG_ERR_INVALID_ARGUMENT, "path_slots out of range");
    if (o.pixel_budget < 1 || o.pixel_budget > (int64_t(1) << 31))
        return fail(SG_ERR_INVALID_ARGUMENT, "pixel_budget out of range");
    if (o.steps_per_poll < 2 || o.steps_per_poll % 2 != 0 || o.steps_per_poll > 64)
        return fail(SG_ERR_INVALID_ARGUMENT, "steps_per_poll must be even, 2..64");
    if (o.samples_per_claim < 1 || o.samples_per_claim > 65535)
        return fail(SG_ERR_INVALID_ARGUMENT, "samples_per_claim must be in 1..65535");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || o.device < 0 || o.device >= ndev)
        return fail(SG_ERR_INVALID_ARGUMENT, "no such CUDA device");
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(o.device);
    sg_server* S = new (std::nothrow) sg_server;
    if (!S) return fail(SG_ERR_OUT_OF_MEMORY, "host allocation failed");
    S->opts = o;
    S->solo_pixels = o.solo_pixels < 0 ? 0 : o.solo_pixels > 0 ? o.solo_pixels : int64_t(1);
    S->arena = Arena(o.pixel_budget);
    S->slot_ticket.assign(size_t(o.max_requests), -1);
    for (int r = o.max_requests - 1; r >= 0; --r) S->free_slots.push_back(r);
    const size_t C = size_t(o.path_slots), R = size_t(o.max_requests), P = size_t(o.pixel_budget);
    // Device layout.
    sg::SrvBuffers& b = S->b;
    int* st_arrays[5];
    float* ray_q[3];
    int* slot_q[3];
    int* scene_q[3];
    size_t total = 0;
    std::vector<size_t> offs;
    auto add = [&](size_t bytes) {
        offs.push_back(total);
        total += align_up(bytes);
    };
    add(R * sizeof(sg::SrvRequest));          // 0 requests
    add(kMaxScenes * sizeof(sg::SrvScene));  // 1 scenes
    add(sizeof(sg::SrvControl));             // 2 control
    add(sizeof(sg::SrvCounters));            // 3 counters
    add(R * sizeof(unsigned));               // 4 units_left
    add(R * sizeof(int));                    // 5 done
    add(P * sizeof(unsigned long long));     // 6 ring
    add(P * 3 * sizeof(float));              // 7 images
    for (int k = 0; k < 5; ++k) add(C * sizeof(int));  // 8..12 slot state
    add(C * 6 * sizeof(float));              // 13 thr
    add(C * 6 * sizeof(float));              // 14 vis
    for (int k = 0; k < 2; ++k) {            // 15..20 extension queues
        add(C * 8 * sizeof(float));
        add(C * sizeof(int));
        add(C * sizeof(int));
    }
    add(C * sizeof(int32_t));                // 21 hit prim
    add(C * sizeof(float));                  // 22 hit t
    add(2 * C * 8 * sizeof(float));          // 23 shadow rays
    add(2 * C * sizeof(int));                // 24 shadow slots
    add(2 * C * sizeof(int));                // 25 shadow scenes
    add(2 * C * 3 * sizeof(float));          // 26 contributions
    add(2 * C);                              // 27 occlusion
    add(sizeof(int));                        // 28 status
    cudaError_t e = cudaMalloc(&S->d_mem, total);
    if (e != cudaSuccess) {
        free_server(S);
        if (prev >= 0) cudaSetDevice(prev);
        return fail(e == cudaErrorMemoryAllocation ? SG_ERR_OUT_OF_MEMORY : SG_ERR_CUDA, "server buffers");
    }
    char* m = S->d_mem;
    S->d_requests = reinterpret_cast<sg::SrvRequest*>(m + offs[0]);
    S->d_scenes = reinterpret_cast<sg::SrvScene*>(m + offs[1]);
    S->d_control = reinterpret_cast<sg::SrvControl*>(m + offs[2]);
    S->d_counters = reinterpret_cast<sg::SrvCounters*>(m + offs[3]);
    S->d_images = reinterpret_cast<float*>(m + offs[7]);
    for (int k = 0; k < 5; ++k) st_arrays[k] = reinterpret_cast<int*>(m + offs[8 + k]);
    for (int k = 0; k < 2; ++k) {
        ray_q[k] = reinterpret_cast<float*>(m + offs[15 + 3 * k]);
        slot_q[k] = reinterpret_cast<int*>(m + offs[16 + 3 * k]);
        scene_q[k] = reinterpret_cast<int*>(m + offs[17 + 3 * k]);
    }
    b.requests = S->d_requests;
    b.scenes = S->d_scenes;
    b.control = S->d_control;
    b.counters = S->d_counters;
    b.units_left = reinterpret_cast<unsigned*>(m + offs[4]);
    b.done = reinterpret_cast<int*>(m + offs[5]);
    b.ring = reinterpret_cast<unsigned long long*>(m + offs[6]);
    b.ring_cap = int64_t(P);
    b.slots = int64_t(C);
    b.samples_per_claim = o.samples_per_claim;
    b.st_req = st_arrays[0];
    b.st_pix = st_arrays[1];
    b.st_sample = st_arrays[2];
    b.st_bounce = st_arrays[3];
    b.st_state = st_arrays[4];
    b.thr = reinterpret_cast<float*>(m + offs[13]);
    b.vis = reinterpret_cast<float*>(m + offs[14]);
    b.qa_ray = ray_q[0];
    b.qa_slot = slot_q[0];
    b.qa_scene = scene_q[0];
    b.qb_ray = ray_q[1];
    b.qb_slot = slot_q[1];
    b.qb_scene = scene_q[1];
    b.hit_prim = reinterpret_cast<int32_t*>(m + offs[21]);
    b.hit_t = reinterpret_cast<float*>(m + offs[22]);
    b.sq_ray = reinterpret_cast<float*>(m + offs[23]);
    b.sq_slot = reinterpret_cast<int*>(m + offs[24]);
    b.sq_scene = reinterpret_cast<int*>(m + offs[25]);
    b.sq_contrib = reinterpret_cast<float*>(m + offs[26]);
    b.occ = reinterpret_cast<uint8_t*>(m + offs[27]);
    b.err = reinterpret_cast<int*>(m + offs[28]);
    // Zeroed state: counters, idle slots (kSlotIdle == 0), flags, status.
    e = cudaMemset(S->d_mem, 0, offs[6]);
    if (e == cudaSuccess) e = cudaMemset(m + offs[8], 0, offs[13] - offs[8]);
    if (e == cudaSuccess) e = cudaMemset(b.err, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaMallocHost(&S->h_requests, R * sizeof(sg::SrvRequest));
    if (e == cudaSuccess) e = cudaMallocHost(&S->h_units, R * sizeof(unsigned));
    for (int k = 0; k < 2 && e == cudaSuccess; ++k) {
        e = cudaMallocHost(&S->h_control[k], sizeof(sg::SrvControl));
        if (e == cudaSuccess) e = cudaMallocHost(&S->h_done[k], R * sizeof(int));
        if (e == cudaSuccess) e = cudaMallocHost(&S->h_counters[k], sizeof(sg::SrvCounters));
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&S->replay_done[k], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&S->copy_done, cudaEventDisableTiming);
    // Stream priorities: the oldest lane's waves above everything else.
    int least = 0, greatest = 0;
    if (e == cudaSuccess) e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&S->pool_side, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&S->pool_forked, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&S->pool_joined, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&S->copy_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess && S->solo_pixels > 0) {
        // Each lane's wave buffers (pt_wave.h), two sets of path_slots paths:
        // extension queues, hits, the shadow queue (2 per path), flags, path
        // state, counters; then the ray totals every set adds to.
        S->lanes.resize(kSoloLanes);
        const size_t cap = C, scap = 2 * C;
        const size_t parts[] = {cap * 32, cap * 4, cap * 32, cap * 4, cap * 4, cap * 4, scap * 32, scap * 4,
                                scap * 12, scap, cap * 24, cap * 24, 16};
        constexpr int kParts = int(sizeof(parts) / sizeof(parts[0]));
        size_t set = 0;
        for (size_t x : parts) set += align_up(x);
        const size_t bytes = 2 * kSoloLanes * set + align_up(16);
        e = cudaMalloc(&S->d_solo, bytes);
        if (e == cudaSuccess) e = cudaMemset(S->d_solo, 0, bytes);
        char* q = S->d_solo;
        for (sg_server::Lane& L : S->lanes) {
            for (int k = 0; k < 2 && e == cudaSuccess; ++k) {
                char* at[kParts];
                for (int x = 0; x < kParts; ++x) {
                    at[x] = q;
                    q += align_up(parts[x]);
                }
                sg::PtWave& w = L.w[k];
                w.qa_ray = reinterpret_cast<float*>(at[0]);
                w.qa_slot = reinterpret_cast<int*>(at[1]);
                w.qb_ray = reinterpret_cast<float*>(at[2]);
                w.qb_slot = reinterpret_cast<int*>(at[3]);
                w.hit_prim = reinterpret_cast<int32_t*>(at[4]);
                w.hit_t = reinterpret_cast<float*>(at[5]);
                w.sq_ray = reinterpret_cast<float*>(at[6]);
                w.sq_slot = reinterpret_cast<int*>(at[7]);
                w.sq_contrib = reinterpret_cast<float*>(at[8]);
                w.occ = reinterpret_cast<uint8_t*>(at[9]);
                w.thr = reinterpret_cast<float*>(at[10]);
                w.vis = reinterpret_cast<float*>(at[11]);
                w.counters = reinterpret_cast<int*>(at[12]);
                w.cap = int(cap);
                for (int pr = 0; pr < 2 && e == cudaSuccess; ++pr) {
                    const int level = pr == 0 ? greatest : least;
                    e = cudaStreamCreateWithPriority(&L.stream[pr][k], cudaStreamNonBlocking, level);
                    if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&L.side[pr][k], cudaStreamNonBlocking, level);
                }
                if (e == cudaSuccess) e = cudaEventCreateWithFlags(&w.shaded, cudaEventDisableTiming);
                if (e == cudaSuccess) e = cudaEventCreateWithFlags(&w.shadowed, cudaEventDisableTiming);
                if (e == cudaSuccess) e = cudaEventCreateWithFlags(&L.flushed[k], cudaEventDisableTiming);
                if (e == cudaSuccess) e = cudaEventCreateWithFlags(&L.wave_done[k], cudaEventDisableTiming);
                w.side = L.side[1][k];
            }
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&L.ready, cudaEventDisableTiming);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&L.end, cudaEventDisableTiming);
        }
        if (e == cudaSuccess)
            for (sg_server::Lane& L : S->lanes) L.w[0].totals = L.w[1].totals = reinterpret_cast<unsigned long long*>(q);
    }
    if (prev >= 0) cudaSetDevice(prev);
    if (e != cudaSuccess) {
        free_server(S);
        return fail(SG_ERR_CUDA, std::string("server setup: ") + cudaGetErrorString(e));
    }
    S->loop = std::thread(serve_loop, S);
    *out = S;
    return SG_OK;
}

sg_status sg_server_add_scene(sg_server* S, const sg_pt_scene* pt, int32_t* scene_id) {
    if (!S || !pt || !scene_id) return fail(SG_ERR_INVALID_ARGUMENT, "NULL argument");
    sg::SrvScene sc{};
    const sg_scene* scene = nullptr;
    sg_status st = sg::pt_scene_parts(pt, &sc.pt, &scene);
    if (st != SG_OK) return st;
    sg::TraceLaunch L;
    int device = 0;
    if ((st = sg::scene_launch(scene, false, &L, &sc.tree, &device)) != SG_OK) return st;
    if (device != S->opts.device) return fail(SG_ERR_INVALID_ARGUMENT, "scene lives on another device");
    const int fmt = L.q8 ? SG_NODES_QUANT8 : SG_NODES_FP32;
    std::lock_guard<std::mutex> lk(S->mu);
    if (int(S->scenes.size()) >= kMaxScenes) return fail(SG_ERR_LIMIT, "too many scenes");
    if (!S->scenes.empty() && (S->width != L.width || S->node_format != fmt))
        return fail(SG_ERR_UNSUPPORTED, "all scenes of a server share one tree width and node format");
    if (L.stack_need > 256) return fail(SG_ERR_LIMIT, "tree too deep for the traversal stack");
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(S->opts.device);
    const int id = int(S->scenes.size());
    cudaError_t e = cudaMemcpy(S->d_scenes + id, &sc, sizeof(sc), cudaMemcpyHostToDevice);
    if (prev >= 0) cudaSetDevice(prev);
    if (e != cudaSuccess) return fail(SG_ERR_CUDA, std::string("scene table: ") + cudaGetErrorString(e));
    S->scenes.push_back(sc);
    S->launches.push_back(L);
    S->width = L.width;
    S->node_format = fmt;
    S->stack_need = std::max(S->stack_need, L.stack_need);
    *scene_id = id;
    return SG_OK;
}

sg_status sg_server_submit(sg_server* S, const sg_request* q, int64_t* ticket) {
    if (!S || !q || !ticket) return fail(SG_ERR_INVALID_ARGUMENT, "NULL argument");
    if (q->width <= 0 || q->height <= 0 || q->spp <= 0 || q->spp > 65535 || q->max_depth <= 0 || !q->image)
        return fail(SG_ERR_INVALID_ARGUMENT, "bad request");
    const int64_t P = int64_t(q->width) * q->height;
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->stop) return S->loop_status != SG_OK ? fail(S->loop_status, S->loop_msg) : fail(SG_ERR_INVALID_ARGUMENT, "server stopped");
    if (q->scene < 0 || q->scene >= int(S->scenes.size())) return fail(SG_ERR_INVALID_ARGUMENT, "unknown scene");
    if (P > S->opts.pixel_budget) return fail(SG_ERR_LIMIT, "request larger than the pixel budget");
    const int64_t id = S->next_ticket++;
    Ticket& t = S->tickets[id];
    t.req = *q;
    t.submit_ns = now_ns();
    S->pending.push_back(id);
    S->cv_work.notify_all();
    *ticket = id;
    return SG_OK;
}

sg_status sg_server_wait(sg_server* S, int64_t ticket, int64_t timeout_ns, sg_request_result* result) {
    if (!S || !result) return fail(SG_ERR_INVALID_ARGUMENT, "NULL argument");
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->tickets.find(ticket);
    if (it == S->tickets.end()) return fail(SG_ERR_INVALID_ARGUMENT, "unknown ticket");
    auto ready = [&] {
        auto f = S->tickets.find(ticket);
        return f == S->tickets.end() || f->second.complete;
    };
    if (timeout_ns < 0) {
        S->cv_done.wait(lk, ready);
    } else if (!S->cv_done.wait_for(lk, std::chrono::nanoseconds(timeout_ns), ready)) {
        return fail(SG_ERR_LIMIT, "request still running");
    }
    it = S->tickets.find(ticket);
    if (it == S->tickets.end()) return fail(SG_ERR_INVALID_ARGUMENT, "ticket already collected");
    const Ticket& t = it->second;
    result->ticket = ticket;
    result->status = t.status;
    result->reserved = 0;
    result->submit_ns = t.submit_ns;
    result->admit_ns = t.admit_ns;
    result->done_ns = t.done_ns;
    S->tickets.erase(it);
    return SG_OK;
}

sg_status sg_server_cancel(sg_server* S, int64_t ticket) {
    if (!S) return fail(SG_ERR_INVALID_ARGUMENT, "NULL server");
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->tickets.find(ticket);
    if (it == S->tickets.end()) return fail(SG_ERR_INVALID_ARGUMENT, "unknown ticket");
    Ticket& t = it->second;
    if (t.complete || t.cancel) return SG_OK;
    t.cancel = true;
    if (t.slot < 0) {  // still queued
        S->pending.erase(std::remove(S->pending.begin(), S->pending.end(), ticket), S->pending.end());
        complete(S, t, SG_ERR_CANCELLED);
    } else {
        S->to_cancel.push_back(t.slot);
        S->cv_work.notify_all();
    }
    return SG_OK;
}

sg_status sg_server_stats_get(sg_server* S, sg_server_stats* out) {
    if (!S || !out) return fail(SG_ERR_INVALID_ARGUMENT, "NULL argument");
    std::lock_guard<std::mutex> lk(S->mu);
    *out = S->stats;
    out->queued = int64_t(S->pending.size());
    for (const sg_server::Lane& L : S->lanes) out->admitted += L.id >= 0 ? 1 : 0;
    if (!S->lanes.empty() && S->lanes[0].w[0].totals) {  // rays of the solo waves (a snapshot while they run)
        unsigned long long h[2] = {0, 0};
        int prev = -1;
        cudaGetDevice(&prev);
        cudaSetDevice(S->opts.device);
        if (cudaMemcpy(h, S->lanes[0].w[0].totals, sizeof(h), cudaMemcpyDeviceToHost) == cudaSuccess) {
            out->extension_rays += int64_t(h[0]);
            out->shadow_rays += int64_t(h[1]);
        }
        if (prev >= 0) cudaSetDevice(prev);
    }
    return SG_OK;
}

sg_status sg_server_destroy(sg_server* S) {
    if (!S) return fail(SG_ERR_INVALID_ARGUMENT, "NULL server");
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
        S->cv_work.notify_all();
    }
    if (S->loop.joinable()) S->loop.join();
    free_server(S);
    return SG_OK;
}

}  // extern "C"
