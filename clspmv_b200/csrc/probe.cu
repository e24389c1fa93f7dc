// spmv_all method 0 (clSpMV_NV/src/spmv_all.cpp:196 -> mem_bandwidth.cpp): the memory
// bandwidth and kernel launch overhead of the device, measured with this library's
// own probes: an empty kernel, a streaming float4 copy and a random 4-byte gather
// (the access pattern that bounds SpMV on matrices with scattered columns).
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <algorithm>
#include <functional>
#include <vector>

#include "csp/clspmv.h"
#include "internal.h"
#include "engine.h"

namespace csp {
namespace {

__global__ void empty_kernel() {}

__global__ void __launch_bounds__(256) copy_kernel(const float4* __restrict__ a, float4* __restrict__ b, size_t n4)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += (size_t)gridDim.x * blockDim.x)
        b[i] = __ldg(a + i);
}

// out[i] = x[idx[i]] for a random idx (fixed seed, generated on the device).
__global__ void __launch_bounds__(256) fill_index_kernel(int* __restrict__ idx, size_t n, int range)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        uint32_t h = (uint32_t)i * 2654435761u;
        h ^= h >> 15;
        h *= 2246822519u;
        h ^= h >> 13;
        idx[i] = (int)(h % (uint32_t)range);
    }
}

__global__ void __launch_bounds__(256) gather_kernel(const int* __restrict__ idx, const float* __restrict__ x,
                                                     float* __restrict__ out, size_t n4)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += (size_t)gridDim.x * blockDim.x) {
        const int4 c = __ldg(reinterpret_cast<const int4*>(idx) + i);
        float4 v;
        v.x = __ldg(x + c.x);
        v.y = __ldg(x + c.y);
        v.z = __ldg(x + c.z);
        v.w = __ldg(x + c.w);
        reinterpret_cast<float4*>(out)[i] = v;
    }
}

// Random 4-byte gathers with in-register hashed indices (no index stream), from three
// places: a global array kGtPer * kGtCluster floats long (L2-resident after the first
// pass), this CTA's shared memory (kGtPer floats), and the shared memory of the 8 CTAs
// of a thread-block cluster (distributed shared memory, kGtPer floats each).
constexpr int kGtPer = 49152;
constexpr int kGtCluster = 8;
constexpr int kGtThreads = 512;
constexpr int kGtIters = 256;

__device__ __forceinline__ unsigned gt_hash(unsigned a)
{
    a ^= a >> 16;
    a *= 0x7feb352dU;
    a ^= a >> 15;
    a *= 0x846ca68bU;
    a ^= a >> 16;
    return a;
}

__global__ void __launch_bounds__(kGtThreads, 1) gt_global(const float* __restrict__ src, float* __restrict__ out)
{
    unsigned h = gt_hash(blockIdx.x * kGtThreads + threadIdx.x);
    float acc = 0.0f;
#pragma unroll 8
    for (int it = 0; it < kGtIters; it++) {
        h = gt_hash(h + it);
        acc += __ldg(src + h % (kGtPer * kGtCluster));
    }
    out[blockIdx.x * kGtThreads + threadIdx.x] = acc;
}

__global__ void __launch_bounds__(kGtThreads, 1) gt_shared(const float* __restrict__ src, float* __restrict__ out)
{
    extern __shared__ float gs[];
    for (int i = threadIdx.x; i < kGtPer; i += kGtThreads) gs[i] = src[i];
    __syncthreads();
    unsigned h = gt_hash(blockIdx.x * kGtThreads + threadIdx.x);
    float acc = 0.0f;
#pragma unroll 8
    for (int it = 0; it < kGtIters; it++) {
        h = gt_hash(h + it);
        acc += gs[h % kGtPer];
    }
    out[blockIdx.x * kGtThreads + threadIdx.x] = acc;
}

__global__ void __cluster_dims__(kGtCluster, 1, 1) __launch_bounds__(kGtThreads, 1)
    gt_cluster(const float* __restrict__ src, float* __restrict__ out)
{
    namespace cg = cooperative_groups;
    extern __shared__ float gs[];
    cg::cluster_group cl = cg::this_cluster();
    const unsigned rank = cl.block_rank();
    for (int i = threadIdx.x; i < kGtPer; i += kGtThreads) gs[i] = src[rank * kGtPer + i];
    cl.sync();
    unsigned h = gt_hash(blockIdx.x * kGtThreads + threadIdx.x);
    float acc = 0.0f;
#pragma unroll 8
    for (int it = 0; it < kGtIters; it++) {
        h = gt_hash(h + it);
        const unsigned idx = h % (kGtPer * kGtCluster);
        acc += cl.map_shared_rank(gs, idx / kGtPer)[idx % kGtPer];
    }
    cl.sync();   // no CTA leaves while the others may still read its shared memory
    out[blockIdx.x * kGtThreads + threadIdx.x] = acc;
}

float time_ms(cudaStream_t st, int reps, const std::function<void()>& f)
{
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    f();
    cudaEventRecord(e0, st);
    for (int i = 0; i < reps; i++) f();
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return ms / reps;
}

}  // namespace
}  // namespace csp

extern "C" int csp_bandwidth_test(size_t bytes, int gather_range, csp_bandwidth_report* rep)
{
    using namespace csp;
    if (!rep || bytes < (1u << 20) || gather_range <= 0) return set_error(CSP_EINVAL, "bandwidth_test: bad argument");
    const size_t n4 = bytes / 16;
    float4 *a = nullptr, *b = nullptr;
    int* idx = nullptr;
    float* x = nullptr;
    cudaStream_t st = nullptr;
    int rc = CSP_OK;
    if (cudaMalloc(&a, n4 * 16) != cudaSuccess || cudaMalloc(&b, n4 * 16) != cudaSuccess ||
        cudaMalloc(&idx, n4 * 16) != cudaSuccess || cudaMalloc(&x, (size_t)gather_range * 4) != cudaSuccess) {
        rc = set_error(CSP_ENOMEM, "bandwidth_test: device allocation");
    }
    int dev = 0, sms = 148;
    if (!rc) {
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
        cudaMemsetAsync(a, 0, n4 * 16, st);
        cudaMemsetAsync(x, 0, (size_t)gather_range * 4, st);
        fill_index_kernel<<<sms * 8, 256, 0, st>>>(idx, n4 * 4, gather_range);
        const unsigned g = (unsigned)sms * 8;
        rep->launch_us = 1e3 * time_ms(st, 200, [&] { empty_kernel<<<1, 32, 0, st>>>(); });
        const float cms = time_ms(st, 10, [&] { copy_kernel<<<g, 256, 0, st>>>(a, b, n4); });
        rep->copy_gbs = 2.0 * (double)(n4 * 16) / (cms * 1e-3) / 1e9;
        const float gms = time_ms(st, 10, [&] { gather_kernel<<<g, 256, 0, st>>>(idx, x, reinterpret_cast<float*>(b), n4); });
        rep->gather_per_s = (double)(n4 * 4) / (gms * 1e-3);
        rep->gather_gbs = (double)(n4 * 4) * 8.0 / (gms * 1e-3) / 1e9;
        cudaError_t e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) rc = cuda_error(e, "bandwidth_test");
    }
    if (st) cudaStreamDestroy(st);
    cudaFree(a);
    cudaFree(b);
    cudaFree(idx);
    cudaFree(x);
    return rc;
}

extern "C" int csp_gather_test(csp_gather_report* rep)
{
    using namespace csp;
    if (!rep) return set_error(CSP_EINVAL, "gather_test: null report");
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return set_error(CSP_ENODEV, "gather_test: no device");
    const int grid = std::max(kGtCluster, sms / kGtCluster * kGtCluster);
    float *src = nullptr, *out = nullptr;
    cudaStream_t st = nullptr;
    int rc = CSP_OK;
    if (cudaMalloc(&src, sizeof(float) * kGtPer * kGtCluster) != cudaSuccess ||
        cudaMalloc(&out, sizeof(float) * grid * kGtThreads) != cudaSuccess)
        rc = set_error(CSP_ENOMEM, "gather_test: device allocation");
    const size_t smem = sizeof(float) * kGtPer;
    if (!rc) {
        cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
        cudaMemsetAsync(src, 0, sizeof(float) * kGtPer * kGtCluster, st);
        cudaFuncSetAttribute(gt_shared, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaFuncSetAttribute(gt_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        const double n = (double)grid * kGtThreads * kGtIters;
        rep->array_bytes = (double)sizeof(float) * kGtPer * kGtCluster;
        rep->l2_per_s = n / (time_ms(st, 5, [&] { gt_global<<<grid, kGtThreads, 0, st>>>(src, out); }) * 1e-3);
        rep->shared_per_s = n / (time_ms(st, 5, [&] { gt_shared<<<grid, kGtThreads, smem, st>>>(src, out); }) * 1e-3);
        cudaError_t e = cudaStreamSynchronize(st);
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e != cudaSuccess) rc = cuda_error(e, "gather_test");
        if (!rc) {
            rep->cluster_per_s = n / (time_ms(st, 5, [&] { gt_cluster<<<grid, kGtThreads, smem, st>>>(src, out); }) * 1e-3);
            e = cudaStreamSynchronize(st);
            if (e == cudaSuccess) e = cudaGetLastError();
            if (e != cudaSuccess) { rep->cluster_per_s = -1.0; clear_error(); }   // no clusters on this device
        }
    }
    if (st) cudaStreamDestroy(st);
    cudaFree(src);
    cudaFree(out);
    return rc;
}
