// Shared device helpers for the SpMV kernels.
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>

namespace csp {
namespace dev {

constexpr int kWarp = 32;

// Matrix values are stored as FP32 or BF16; arithmetic is always FP32.
template <class V> struct Val;

template <> struct Val<float> {
    __device__ __forceinline__ static float ld(const float* p) { return __ldg(p); }
    // Four consecutive values; p must be 16-byte aligned.
    __device__ __forceinline__ static float4 ld4(const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); }
};

template <> struct Val<__nv_bfloat16> {
    __device__ __forceinline__ static float ld(const __nv_bfloat16* p)
    {
        unsigned short u = __ldg(reinterpret_cast<const unsigned short*>(p));
        return __uint_as_float(((unsigned)u) << 16);
    }
    // Four consecutive values; p must be 8-byte aligned.
    __device__ __forceinline__ static float4 ld4(const __nv_bfloat16* p)
    {
        uint2 u = __ldg(reinterpret_cast<const uint2*>(p));
        float4 f;
        f.x = __uint_as_float(u.x << 16);
        f.y = __uint_as_float(u.x & 0xffff0000u);
        f.z = __uint_as_float(u.y << 16);
        f.w = __uint_as_float(u.y & 0xffff0000u);
        return f;
    }
};

__device__ __forceinline__ int4 ld_int4(const int* p) { return __ldg(reinterpret_cast<const int4*>(p)); }
__device__ __forceinline__ float ldx(const float* x, int i) { return __ldg(x + i); }
__device__ __forceinline__ float4 ldx4(const float* x, int i) { return __ldg(reinterpret_cast<const float4*>(x + i)); }

// Sum over the G lanes of an aligned lane group (G a power of two, <= 32).
template <int G>
__device__ __forceinline__ float group_sum(float v)
{
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, G);
    return v;
}

// Block-wide sum; every thread gets the total.  `scratch` holds >= blockDim.x / 32 floats.
__device__ __forceinline__ float block_sum(float v, float* scratch)
{
    v = group_sum<kWarp>(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    __syncthreads();
    if (lane == 0) scratch[wid] = v;
    __syncthreads();
    float t = 0.0f;
    for (int i = 0; i < nw; i++) t += scratch[i];
    return t;
}

}  // namespace dev
}  // namespace csp
