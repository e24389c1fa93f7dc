// spmv_all method 0 (clSpMV_NV/src/spmv_all.cpp:196 -> mem_bandwidth.cpp): the memory
// bandwidth and kernel launch overhead of the device, measured with this library's
// own probes: an empty kernel, a streaming float4 copy and a random 4-byte gather
// (the access pattern that bounds SpMV on matrices with scattered columns).
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
