// sg_probe_l2_read_gbs: the L2 read bandwidth a kernel reaches on this GPU.
//
// A workload whose tree fits in the 126 MB L2 (the 81,922-triangle ray-cast
// scene holds about 5 MB) is bound by L2, not HBM, bandwidth; the roofline of
// such a workload needs the L2 figure, which no vendor table gives for this
// part. The probe reads a buffer that fits in L2 over and over with 128-bit
// loads that bypass L1 (ld.global.cg), after one untimed pass that brings it
// into L2, and reports bytes read per second of CUDA-event time.
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "scene_access.h"
#include "sortgpu.h"

namespace {

__global__ void k_l2_read(const float4* __restrict__ buf, int64_t n4, int reps, float* __restrict__ sink) {
    float acc = 0.0f;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int r = 0; r < reps; ++r) {
        for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += stride) {
            const float4 v = __ldcg(buf + i);
            acc += v.x + v.y + v.z + v.w;
        }
    }
    if (acc == 1234.5f) *sink = acc;  // keeps the loads; the buffer holds zeros, so never taken
}

}  // namespace

extern "C" sg_status sg_probe_l2_read_gbs(int32_t device, int64_t bytes, int32_t reps, double* gbs) {
    if (!gbs || bytes < (int64_t(1) << 20) || bytes > (int64_t(96) << 20) || reps < 1 || reps > 1000)
        return sg::set_error(SG_ERR_INVALID_ARGUMENT, "bytes must be 1..96 MiB, reps 1..1000");
    int prev = -1;
    cudaGetDevice(&prev);
    cudaError_t e = cudaSetDevice(device);
    float4* buf = nullptr;
    float* sink = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int sms = 1;
    const int64_t n4 = bytes / 16;
    float ms = 0.0f;
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = cudaMalloc(&buf, size_t(n4) * 16);
    if (e == cudaSuccess) e = cudaMalloc(&sink, sizeof(float));
    if (e == cudaSuccess) e = cudaMemset(buf, 0, size_t(n4) * 16);
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e == cudaSuccess) {
        const int blocks = sms * 8, threads = 256;
        k_l2_read<<<blocks, threads>>>(buf, n4, 1, sink);  // brings the buffer into L2
        cudaEventRecord(e0);
        k_l2_read<<<blocks, threads>>>(buf, n4, reps, sink);
        cudaEventRecord(e1);
        e = cudaEventSynchronize(e1);
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (buf) cudaFree(buf);
    if (sink) cudaFree(sink);
    if (prev >= 0) cudaSetDevice(prev);
    if (e != cudaSuccess) return sg::set_error(SG_ERR_CUDA, (std::string("L2 probe: ") + cudaGetErrorString(e)).c_str());
    *gbs = double(n4) * 16.0 * reps / (double(ms) * 1e-3) / 1e9;
    return SG_OK;
}
