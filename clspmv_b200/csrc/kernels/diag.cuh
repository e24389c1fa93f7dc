// Diagonal-format SpMV kernels: DIA and BDIA (banded DIA).
//
// Layout (matrix_storage.h:27-94): diagonal d of `len` rows at data[d*len + row],
// x index row + offset.  Out-of-range columns hold 0 in the data and are skipped
// here by a predicated load instead of the reference's zero-extended copy of x
// (spmv_cocktail.cpp:253 cpy_vec_extended), so no extended vector has to be kept
// in sync with x.
#pragma once

#include "common.cuh"

namespace csp {
namespace dev {

constexpr int kDiaThreads = 256;

__device__ __forceinline__ float ldx_guarded(const float* __restrict__ x, int c, int n)
{
    return (c >= 0 && c < n) ? __ldg(x + c) : 0.0f;
}

// DIA, ROWS rows per thread strided by the CTA width: coalesced 4-byte loads of every
// diagonal, offsets staged in shared memory (spmv_dia.cl gpu_dia).
template <class V, int ROWS>
__global__ void __launch_bounds__(kDiaThreads) dia_kernel(const int* __restrict__ offsets, const V* __restrict__ data,
                                                          const float* __restrict__ x, float* __restrict__ y,
                                                          int m, int n, int ndia, int len)
{
    extern __shared__ int s_off[];
    for (int i = threadIdx.x; i < ndia; i += kDiaThreads) s_off[i] = __ldg(offsets + i);
    __syncthreads();
    const int base = blockIdx.x * (kDiaThreads * ROWS) + threadIdx.x;
    float acc[ROWS];
#pragma unroll
    for (int q = 0; q < ROWS; q++) acc[q] = 0.0f;
    for (int d = 0; d < ndia; d++) {
        const int o = s_off[d];
        const V* dd = data + (size_t)d * len;
#pragma unroll
        for (int q = 0; q < ROWS; q++) {
            const int r = base + q * kDiaThreads;
            if (r < m) acc[q] += Val<V>::ld(dd + r) * ldx_guarded(x, r + o, n);
        }
    }
#pragma unroll
    for (int q = 0; q < ROWS; q++) {
        const int r = base + q * kDiaThreads;
        if (r < m) y[r] += acc[q];
    }
}

// DIA, four consecutive rows per thread with 128-bit loads of the diagonals
// (spmv_dia.cl gpu_dia_v4; len is a multiple of 4).
template <class V>
__global__ void __launch_bounds__(kDiaThreads) dia4_kernel(const int* __restrict__ offsets, const V* __restrict__ data,
                                                           const float* __restrict__ x, float* __restrict__ y,
                                                           int m, int n, int ndia, int len)
{
    extern __shared__ int s_off[];
    for (int i = threadIdx.x; i < ndia; i += kDiaThreads) s_off[i] = __ldg(offsets + i);
    __syncthreads();
    const int r0 = (blockIdx.x * kDiaThreads + threadIdx.x) * 4;
    if (r0 >= m) return;
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int d = 0; d < ndia; d++) {
        const int c = r0 + s_off[d];
        const float4 a = Val<V>::ld4(data + (size_t)d * len + r0);
        acc.x += a.x * ldx_guarded(x, c, n);
        acc.y += a.y * ldx_guarded(x, c + 1, n);
        acc.z += a.z * ldx_guarded(x, c + 2, n);
        acc.w += a.w * ldx_guarded(x, c + 3, n);
    }
    y[r0] += acc.x;
    if (r0 + 1 < m) y[r0 + 1] += acc.y;
    if (r0 + 2 < m) y[r0 + 2] += acc.z;
    if (r0 + 3 < m) y[r0 + 3] += acc.w;
}

// BDIA with the band's window of x staged in shared memory (spmv_bdia.cl gpu_bdia:
// one staged window per band, reused by the band's adjacent diagonals).  The CTA
// covers kDiaThreads*ROWS rows, thread t owning rows t, t+256, ... so shared-memory
// reads are conflict-free and global loads coalesced.  Dynamic shared memory holds
// kDiaThreads*ROWS + max_band_width - 1 floats.
template <class V, int ROWS>
__global__ void __launch_bounds__(kDiaThreads) bdia_staged_kernel(const int* __restrict__ offsets, const int* __restrict__ bptr,
                                                                  const V* __restrict__ data, const float* __restrict__ x,
                                                                  float* __restrict__ y, int m, int n, int nbands, int len)
{
    extern __shared__ float s_x[];
    constexpr int RB = kDiaThreads * ROWS;
    const int rbase = blockIdx.x * RB;
    float acc[ROWS];
#pragma unroll
    for (int q = 0; q < ROWS; q++) acc[q] = 0.0f;
    for (int b = 0; b < nbands; b++) {
        const int o = __ldg(offsets + b);
        const int d0 = __ldg(bptr + b), w = __ldg(bptr + b + 1) - d0;
        __syncthreads();
        for (int i = threadIdx.x; i < RB + w - 1; i += kDiaThreads) s_x[i] = ldx_guarded(x, rbase + o + i, n);
        __syncthreads();
        for (int k = 0; k < w; k++) {
            const V* dd = data + (size_t)(d0 + k) * len + rbase;
#pragma unroll
            for (int q = 0; q < ROWS; q++) {
                const int lr = threadIdx.x + q * kDiaThreads;
                if (rbase + lr < m) acc[q] += Val<V>::ld(dd + lr) * s_x[lr + k];
            }
        }
    }
#pragma unroll
    for (int q = 0; q < ROWS; q++) {
        const int r = rbase + threadIdx.x + q * kDiaThreads;
        if (r < m) y[r] += acc[q];
    }
}

// BDIA reading x directly (spmv_bdia.cl gpu_bdia_v4_nlvec): four consecutive rows per
// thread, 128-bit loads of the diagonals.
template <class V>
__global__ void __launch_bounds__(kDiaThreads) bdia4_kernel(const int* __restrict__ offsets, const int* __restrict__ bptr,
                                                            const V* __restrict__ data, const float* __restrict__ x,
                                                            float* __restrict__ y, int m, int n, int nbands, int len)
{
    const int r0 = (blockIdx.x * kDiaThreads + threadIdx.x) * 4;
    if (r0 >= m) return;
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int b = 0; b < nbands; b++) {
        const int o = __ldg(offsets + b);
        const int d0 = __ldg(bptr + b), d1 = __ldg(bptr + b + 1);
        for (int d = d0; d < d1; d++) {
            const int c = r0 + o + (d - d0);
            const float4 a = Val<V>::ld4(data + (size_t)d * len + r0);
            acc.x += a.x * ldx_guarded(x, c, n);
            acc.y += a.y * ldx_guarded(x, c + 1, n);
            acc.z += a.z * ldx_guarded(x, c + 2, n);
            acc.w += a.w * ldx_guarded(x, c + 3, n);
        }
    }
    y[r0] += acc.x;
    if (r0 + 1 < m) y[r0 + 1] += acc.y;
    if (r0 + 2 < m) y[r0 + 2] += acc.z;
    if (r0 + 3 < m) y[r0 + 3] += acc.w;
}

}  // namespace dev
}  // namespace csp
