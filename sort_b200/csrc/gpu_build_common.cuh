// Helpers shared by the GPU builders (builder_gpu.cu: SORT's tree;
// builder_lbvh.cu: the Morton-order tree): float images for atomic min/max,
// the pooled stream-ordered scratch memory, device/pinned buffers, and the
// primitive set-up and triangle-record kernels.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>

#include "builder.h"

namespace sg {
namespace gpub {

// Order-preserving int image of a float (for atomicMin / atomicMax).
__host__ __device__ __forceinline__ int f2o(float f) {
    int i;
    std::memcpy(&i, &f, 4);
    return i >= 0 ? i : i ^ 0x7fffffff;
}
__host__ __device__ __forceinline__ float o2f(int i) {
    const int b = i >= 0 ? i : i ^ 0x7fffffff;
    float f;
    std::memcpy(&f, &b, 4);
    return f;
}

__host__ __device__ __forceinline__ void empty_box(int* b) {
    for (int a = 0; a < 3; ++a) {
        b[a] = f2o(FLT_MAX);
        b[3 + a] = f2o(-FLT_MAX);
    }
}

void check(cudaError_t e, const char* what);  // throws std::runtime_error

// Scratch memory: a private stream-ordered pool per device. Builds allocate
// and free on their stream without synchronising the device, and a build
// reuses the memory the previous one mapped (up to kKeepBytes stay mapped
// between builds), so back-to-back scene builds do not pay for the mapping.
constexpr uint64_t kKeepBytes = uint64_t(16) << 30;

cudaMemPool_t scratch_pool(int device);

// The pool and stream that DevBufs declared during a build allocate on.
struct Scratch {
    cudaMemPool_t pool = nullptr;
    cudaStream_t st = nullptr;
};
extern thread_local Scratch scratch;

// Binds DevBufs to (pool, stream) for its lifetime; when it ends (after the
// DevBufs declared later have freed), waits for the stream and trims the pool.
struct ScratchScope {
    Scratch saved;
    ScratchScope(cudaMemPool_t pool, cudaStream_t st) : saved(scratch) { scratch = Scratch{pool, st}; }
    ~ScratchScope() {
        cudaStreamSynchronize(scratch.st);
        cudaMemPoolTrimTo(scratch.pool, kKeepBytes);
        scratch = saved;
    }
};

template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaMemPool_t pool = scratch.pool;
    cudaStream_t st = scratch.st;
    // Grows by at least half its size; the old contents are not kept.
    void alloc(size_t count) {
        if (count <= n) return;
        count = std::max(count, n + n / 2);
        if (p) cudaFreeAsync(p, st);
        p = nullptr;
        n = 0;
        check(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&p), std::max<size_t>(count, 1) * sizeof(T), pool, st),
              "device allocation");
        n = count;
    }
    ~DevBuf() {
        if (p) cudaFreeAsync(p, st);
    }
};

template <class T>
struct PinnedBuf {
    T* p = nullptr;
    size_t n = 0;
    void alloc(size_t count) {
        if (count <= n) return;
        count = std::max<size_t>(count, 2 * n);
        if (p) cudaFreeHost(p);
        p = nullptr;
        n = 0;
        check(cudaMallocHost(&p, std::max<size_t>(count, 1) * sizeof(T)), "cudaMallocHost");
        n = count;
    }
    ~PinnedBuf() {
        if (p) cudaFreeHost(p);
    }
};

inline unsigned grid(int64_t n, int t = 256) { return (unsigned)std::max<int64_t>(1, (n + t - 1) / t); }

inline Box box_from_images(const int* o) {
    Box b;
    for (int a = 0; a < 3; ++a) {
        b.mn[a] = o2f(o[a]);
        b.mx[a] = o2f(o[3 + a]);
    }
    return b;
}

inline float host_half_area(const Box& b) {
    const float ox = b.mx[0] - b.mn[0], oy = b.mx[1] - b.mn[1], oz = b.mx[2] - b.mn[2];
    const float a = ox * oy;
    const float c = oy * oz;
    const float e = oz * ox;
    return (a + c) + e;
}

struct Stream {
    cudaStream_t s = nullptr;
    Stream() { check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate"); }
    ~Stream() {
        if (s) cudaStreamDestroy(s);
    }
};

template <class T>
void swap_bufs(DevBuf<T>& a, DevBuf<T>& b) {
    std::swap(a.p, b.p);
    std::swap(a.n, b.n);
}

}  // namespace gpub

namespace {  // kernels: one copy per file that includes this header

using gpub::empty_box;
using gpub::f2o;
using gpub::o2f;

__device__ __forceinline__ void atomic_box(int* dst, const int (&v)[6]) {
    for (int a = 0; a < 3; ++a) {
        atomicMin(&dst[a], v[a]);
        atomicMax(&dst[3 + a], v[3 + a]);
    }
}

// Boxes, centroids and identity indices of the first `count` primitives
// (triangles); box planes and centroid arrays have `stride` entries.
__global__ void k_prim_setup(const float* __restrict__ tri, int64_t count, int64_t stride, float* __restrict__ cx,
                             float* __restrict__ cy, float* __restrict__ cz, int32_t* __restrict__ idx,
                             float* __restrict__ pb) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, mx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int k = 0; k < 3; ++k)  // BBox::Union(const Point&) per vertex (math/bbox.cpp:106-113)
        for (int a = 0; a < 3; ++a) {
            const float p = tri[i * 9 + 3 * k + a];
            if (p < mn[a]) mn[a] = p;
            if (p > mx[a]) mx[a] = p;
        }
    for (int a = 0; a < 3; ++a) {
        pb[a * stride + i] = mn[a];
        pb[(3 + a) * stride + i] = mx[a];
    }
    cx[i] = __fmul_rn(__fadd_rn(mx[0], mn[0]), 0.5f);
    cy[i] = __fmul_rn(__fadd_rn(mx[1], mn[1]), 0.5f);
    cz[i] = __fmul_rn(__fadd_rn(mx[2], mn[2]), 0.5f);
    idx[i] = (int32_t)i;
}

// The same for primitives given as boxes (6 floats: min xyz, max xyz), at
// indices first .. first + count - 1.
__global__ void k_box_setup(const float* __restrict__ boxes, int64_t first, int64_t count, int64_t stride,
                            float* __restrict__ cx, float* __restrict__ cy, float* __restrict__ cz,
                            int32_t* __restrict__ idx, float* __restrict__ pb) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const int64_t i = first + k;
    float mn[3], mx[3];
    for (int a = 0; a < 3; ++a) {
        mn[a] = boxes[k * 6 + a];
        mx[a] = boxes[k * 6 + 3 + a];
        pb[a * stride + i] = mn[a];
        pb[(3 + a) * stride + i] = mx[a];
    }
    cx[i] = __fmul_rn(__fadd_rn(mx[0], mn[0]), 0.5f);
    cy[i] = __fmul_rn(__fadd_rn(mx[1], mn[1]), 0.5f);
    cz[i] = __fmul_rn(__fadd_rn(mx[2], mn[2]), 0.5f);
    idx[i] = (int32_t)i;
}

// Union of all primitive boxes (the scene box before its enlargement).
__global__ void __launch_bounds__(256) k_scene_box(int64_t n, const float* __restrict__ pb, int* __restrict__ out) {
    __shared__ int sbox[6];
    if (threadIdx.x == 0) empty_box(sbox);
    __syncthreads();
    int v[6];
    empty_box(v);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        for (int a = 0; a < 3; ++a) {
            v[a] = min(v[a], f2o(pb[a * n + i]));
            v[3 + a] = max(v[3 + a], f2o(pb[(3 + a) * n + i]));
        }
    for (int a = 0; a < 3; ++a) {
        v[a] = __reduce_min_sync(0xffffffffu, v[a]);
        v[3 + a] = __reduce_max_sync(0xffffffffu, v[3 + a]);
    }
    if ((threadIdx.x & 31) == 0) atomic_box(sbox, v);
    __syncthreads();
    if (threadIdx.x < 3) {
        atomicMin(&out[threadIdx.x], sbox[threadIdx.x]);
        atomicMax(&out[3 + threadIdx.x], sbox[3 + threadIdx.x]);
    }
}

// Slot i of the device layout: {v0, primitive index}, {v1, last-in-leaf flag}, {v2, 0}.
__global__ void k_leaf_tris(int64_t n, const float* __restrict__ tri, const int32_t* __restrict__ idx,
                            const uint8_t* __restrict__ last, float4* __restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t p = idx[i];
    const float* v = tri + int64_t(p) * 9;
    const int32_t flag = last[i];
    out[i * 3 + 0] = make_float4(v[0], v[1], v[2], __int_as_float(p));
    out[i * 3 + 1] = make_float4(v[3], v[4], v[5], __int_as_float(flag));
    out[i * 3 + 2] = make_float4(v[6], v[7], v[8], 0.0f);
}

}  // namespace
}  // namespace sg
