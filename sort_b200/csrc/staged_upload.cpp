// Pinned-staging upload (staged_upload.h).
//
// A pageable cudaMemcpy stages through the driver's own pinned buffers with
// one host thread, about 10 GB/s here; the 755 MB of a 21M-triangle scene took
// ~70 ms of an LBVH build. Several threads filling pinned buffers while the
// copy engines drain the previous ones keep the host memcpy off the critical
// path.
#include "staged_upload.h"

#include <algorithm>
#include <atomic>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

namespace sg {
namespace {

constexpr size_t kDirectBelow = size_t(32) << 20;
constexpr size_t kSlotBytes = size_t(4) << 20;
constexpr int kSlots = 2;
constexpr int kMaxWorkers = 8;

struct Stager {
    std::mutex lock;
    int workers = 0;
    std::vector<char*> buf;            // workers * kSlots pinned buffers
    std::vector<cudaEvent_t> done;     // per buffer: its last copy finished
    std::vector<cudaStream_t> stream;  // per worker
    cudaEvent_t entry = nullptr;       // the caller's stream at the start of a copy
};

// Per device; made on first use with that device current.
Stager* stager(int device) {
    static std::mutex lock;
    static std::map<int, std::unique_ptr<Stager>> all;
    std::lock_guard<std::mutex> g(lock);
    auto& p = all[device];
    if (!p) p.reset(new Stager());
    return p.get();
}

cudaError_t init(Stager& s) {
    if (s.workers > 0) return cudaSuccess;
    const unsigned hw = std::thread::hardware_concurrency();
    const int w = std::max(1, std::min<int>(kMaxWorkers, hw ? int(hw) : 1));
    std::vector<char*> buf(size_t(w) * kSlots, nullptr);
    std::vector<cudaEvent_t> done(size_t(w) * kSlots, nullptr);
    std::vector<cudaStream_t> stream(size_t(w), nullptr);
    cudaError_t e = cudaSuccess;
    for (size_t k = 0; k < buf.size() && e == cudaSuccess; ++k) {
        e = cudaHostAlloc(reinterpret_cast<void**>(&buf[k]), kSlotBytes, cudaHostAllocPortable);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&done[k], cudaEventDisableTiming);
    }
    for (size_t k = 0; k < stream.size() && e == cudaSuccess; ++k)
        e = cudaStreamCreateWithFlags(&stream[k], cudaStreamNonBlocking);
    cudaEvent_t entry = nullptr;
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&entry, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        if (entry) cudaEventDestroy(entry);
        for (char* b : buf)
            if (b) cudaFreeHost(b);
        for (cudaEvent_t v : done)
            if (v) cudaEventDestroy(v);
        for (cudaStream_t t : stream)
            if (t) cudaStreamDestroy(t);
        return e;
    }
    s.buf = std::move(buf);
    s.done = std::move(done);
    s.stream = std::move(stream);
    s.entry = entry;
    s.workers = w;
    return cudaSuccess;
}

}  // namespace

cudaError_t upload_host(void* dst, const void* src, size_t bytes, cudaStream_t stream) {
    if (bytes == 0) return cudaSuccess;
    cudaPointerAttributes at{};
    const cudaError_t pe = cudaPointerGetAttributes(&at, src);
    if (pe != cudaSuccess) cudaGetLastError();  // clear: treated as pageable
    if (bytes < kDirectBelow || (pe == cudaSuccess && at.type != cudaMemoryTypeUnregistered))
        return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream);

    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
    Stager& s = *stager(device);
    std::lock_guard<std::mutex> g(s.lock);
    if ((e = init(s)) != cudaSuccess) {  // no pinned memory: the driver's own staging
        cudaGetLastError();
        return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream);
    }
    const int w = s.workers;
    // The destination may have just been taken from a stream-ordered pool on
    // `stream`, or still be read by work queued there: the worker streams
    // start their copies only after everything already on `stream`.
    if ((e = cudaEventRecord(s.entry, stream)) != cudaSuccess) return e;
    // Shares in whole slots, so every copy but the last of a share is full.
    const size_t slots_total = (bytes + kSlotBytes - 1) / kSlotBytes;
    const size_t per = ((slots_total + size_t(w) - 1) / size_t(w)) * kSlotBytes;
    std::atomic<int> first_error{int(cudaSuccess)};
    auto work = [&](int k) {
        cudaError_t r = cudaSetDevice(device);
        if (r == cudaSuccess) r = cudaStreamWaitEvent(s.stream[size_t(k)], s.entry, 0);
        const size_t a = size_t(k) * per, end = std::min(bytes, a + per);
        int slot = 0;
        for (size_t off = a; off < end && r == cudaSuccess; off += kSlotBytes) {
            const size_t m = std::min(kSlotBytes, end - off);
            const size_t b = size_t(k) * kSlots + size_t(slot);
            r = cudaEventSynchronize(s.done[b]);  // the buffer's previous copy has finished
            if (r != cudaSuccess) break;
            std::memcpy(s.buf[b], static_cast<const char*>(src) + off, m);
            r = cudaMemcpyAsync(static_cast<char*>(dst) + off, s.buf[b], m, cudaMemcpyHostToDevice, s.stream[size_t(k)]);
            if (r == cudaSuccess) r = cudaEventRecord(s.done[b], s.stream[size_t(k)]);
            slot ^= 1;
        }
        if (r != cudaSuccess) {
            int expect = int(cudaSuccess);
            first_error.compare_exchange_strong(expect, int(r));
        }
    };
    const int used = int(std::min<size_t>(size_t(w), (bytes + per - 1) / per));
    std::vector<std::thread> pool;
    pool.reserve(size_t(used > 0 ? used - 1 : 0));
    for (int k = 1; k < used; ++k) pool.emplace_back(work, k);
    work(0);
    for (auto& t : pool) t.join();
    if (first_error.load() != int(cudaSuccess)) return cudaError_t(first_error.load());
    // Later work on `stream` waits for every staged copy.
    for (size_t b = 0; b < s.done.size(); ++b)
        if ((e = cudaStreamWaitEvent(stream, s.done[b], 0)) != cudaSuccess) return e;
    return cudaSuccess;
}

}  // namespace sg
