// sg_trace_closest_host_static: the host-buffer closest-hit query without any
// device allocation.
//
// Some callers cannot call cudaMalloc at query time: hosts that hand the whole
// GPU memory budget to their own allocator up front, so nothing is left for a
// library to take, or real-time loops that must not take the allocator's locks
// or trigger the implicit device synchronisation a cudaFree brings.
// sg_trace_closest_host stages rays and hits in a device buffer it grows with
// cudaMalloc on demand; this entry point stages them in a fixed array compiled
// into the library instead, so a call allocates and frees nothing.
//
// The array is kStaticBytes of device memory that every GPU which loads this
// library keeps until the process exits. One call handles at most
// kMaxStaticRays rays (48 bytes each: 32 in, 16 out); larger batches are
// rejected with SG_ERR_LIMIT and can be split by the caller.
//
// All calls share the one array: two calls whose work overlaps on the GPU
// (different streams or threads without ordering between them) race on it.
// Each call overwrites every byte it reads back, so no part of the array has to
// start at zero.
//
// Host code cannot use the array's name as a device address, so the first
// call on each device looks the address up with cudaGetSymbolAddress (with that
// device current) and caches it. Make that first call before capturing any
// stream on that device.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "scene_access.h"
#include "sortgpu.h"
#include "trace_kernels.h"

namespace {

constexpr size_t kStaticBytes = (size_t(24) << 20) + 256;  // 24 MiB + alignment slack, per device
constexpr int64_t kRayBytes = 32;                  // ox oy oz dx dy dz tmin tmax
constexpr int64_t kHitBytes = 16;                  // prim t u v
constexpr int64_t kMaxStaticRays = 524288;         // 524,288 rays * 48 B = 24 MiB
static_assert(kMaxStaticRays * (kRayBytes + kHitBytes) + 256 <= int64_t(kStaticBytes), "static scratch too small");

static __device__ __align__(256) unsigned char g_static_scratch[kStaticBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_lock;
void* g_scratch_addr[kMaxDevices] = {};

// Device address of g_static_scratch on `device` (which must be current).
sg_status static_scratch(int device, unsigned char** out) {
    if (device < 0 || device >= kMaxDevices) return sg::set_error(SG_ERR_LIMIT, "device ordinal beyond 63");
    std::lock_guard<std::mutex> lock(g_setup_lock);
    if (!g_scratch_addr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess) return sg::set_error(SG_ERR_CUDA, cudaGetErrorString(e));
        g_scratch_addr[device] = p;
    }
    *out = static_cast<unsigned char*>(g_scratch_addr[device]);
    return SG_OK;
}

}  // namespace

extern "C" sg_status sg_trace_closest_host_static(const sg_scene* scene, const float* rays8, int64_t n, int32_t* prim,
                                                  float* t, float* u, float* v, void* stream) {
    if (!scene || !rays8) return sg::set_error(SG_ERR_INVALID_ARGUMENT, "NULL scene or rays");
    if (n < 0) return sg::set_error(SG_ERR_INVALID_ARGUMENT, "negative ray count");
    if (n > kMaxStaticRays)
        return sg::set_error(SG_ERR_LIMIT, "sg_trace_closest_host_static takes at most 524288 rays per call");
    if (!prim || !t) return sg::set_error(SG_ERR_INVALID_ARGUMENT, "NULL output array");
    if (n == 0) return SG_OK;

    sg::TraceLaunch L;
    sg::DevTree tree;
    int device = 0;
    sg_status st = sg::scene_launch(scene, false, &L, &tree, &device);
    if (st != SG_OK) return st;
    // The sorted schedule takes key and permutation scratch from a pool, and the
    // automatic choice may pick it; this entry point runs every batch one ray per
    // thread instead (same results: the schedule never changes a hit). The other
    // schedules allocate nothing.
    if (L.tuning.schedule == sg::kScheduleSorted || L.tuning.schedule == sg::kScheduleAuto)
        L.tuning.schedule = sg::kScheduleThreadPerRay;
    int prev = -1;
    cudaError_t e = cudaGetDevice(&prev);
    if (e != cudaSuccess) return sg::set_error(SG_ERR_CUDA, cudaGetErrorString(e));
    if ((e = cudaSetDevice(device)) != cudaSuccess) return sg::set_error(SG_ERR_CUDA, cudaGetErrorString(e));
    struct Restore {
        int dev;
        ~Restore() {
            if (dev >= 0) cudaSetDevice(dev);
        }
    } restore{prev};

    unsigned char* base = nullptr;
    if ((st = static_scratch(device, &base)) != SG_OK) return st;
    const size_t in_bytes = size_t(n) * kRayBytes;
    float* d_rays = reinterpret_cast<float*>(base);
    unsigned char* d_out = base + ((in_bytes + 255) & ~size_t(255));
    int32_t* d_prim = reinterpret_cast<int32_t*>(d_out);
    float* d_t = reinterpret_cast<float*>(d_out + size_t(n) * 4);
    float* d_u = reinterpret_cast<float*>(d_out + size_t(n) * 8);
    float* d_v = reinterpret_cast<float*>(d_out + size_t(n) * 12);
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    if ((e = cudaMemcpyAsync(d_rays, rays8, in_bytes, cudaMemcpyHostToDevice, s)) != cudaSuccess)
        return sg::set_error(SG_ERR_CUDA, cudaGetErrorString(e));
    const sg::DevRays r{d_rays,         d_rays + n,     d_rays + 2 * n, d_rays + 3 * n,
                        d_rays + 4 * n, d_rays + 5 * n, d_rays + 6 * n, d_rays + 7 * n};
    L.prim = d_prim;
    L.t = d_t;
    L.u = u ? d_u : nullptr;
    L.v = v ? d_v : nullptr;
    if ((e = sg::launch_trace_fp32(L, tree, r, n, s)) != cudaSuccess)
        return sg::set_error(SG_ERR_CUDA, cudaGetErrorString(e));
    if ((e = cudaMemcpyAsync(prim, d_prim, size_t(n) * 4, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(t, d_t, size_t(n) * 4, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (u && (e = cudaMemcpyAsync(u, d_u, size_t(n) * 4, cudaMemcpyDeviceToHost, s)) != cudaSuccess) ||
        (v && (e = cudaMemcpyAsync(v, d_v, size_t(n) * 4, cudaMemcpyDeviceToHost, s)) != cudaSuccess))
        return sg::set_error(SG_ERR_CUDA, cudaGetErrorString(e));
    return sg::scene_status(scene, s);  // synchronises s
}
