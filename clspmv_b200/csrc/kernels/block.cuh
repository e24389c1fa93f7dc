// Block-format SpMV kernels: BELL and SBELL in the "b4" layout (float4 of four
// consecutive columns, column ids in float4 units), BCSR in the b4 layout, and
// generic row-major BCSR for arbitrary bh x bw blocks.
//
// Layouts (matrix_storage.h): b4ell :2010, sbell :2203, b4csr :1741, bcsr :1595.
// x is zero-padded on the device to a multiple of 64 entries, so the float4 of x
// at any stored block column is in bounds and padding columns multiply zeros.
#pragma once

#include "common.cuh"

namespace csp {
namespace dev {

__device__ __forceinline__ float dot4(float4 a, float4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }

// BELL (b4ell): one thread per block row (spmv_bell.cl gpu_bell<bh><bw>).
template <class V, int BH, int BW4>
__global__ void __launch_bounds__(256) bell_b4_kernel(const int* __restrict__ col, const V* __restrict__ data,
                                                      const float* __restrict__ x, float* __restrict__ y,
                                                      int nbr, int ellnum, int hal, int f4, int m)
{
    const int br = blockIdx.x * blockDim.x + threadIdx.x;
    if (br >= nbr) return;
    const size_t colsize = (size_t)f4 * BW4 * BH, w4size = (size_t)f4 * BH;
    float acc[BH];
#pragma unroll
    for (int h = 0; h < BH; h++) acc[h] = 0.0f;
    for (int k = 0; k < ellnum; k++) {
        const int c4 = __ldg(col + (size_t)k * hal + br);
        const V* dk = data + (size_t)k * colsize + (size_t)br * 4;
#pragma unroll
        for (int w4 = 0; w4 < BW4; w4++) {
            const float4 xv = ldx4(x, (c4 + w4) * 4);
#pragma unroll
            for (int h = 0; h < BH; h++) acc[h] += dot4(Val<V>::ld4(dk + (size_t)h * f4 + w4 * w4size), xv);
        }
    }
#pragma unroll
    for (int h = 0; h < BH; h++) {
        const int r = br * BH + h;
        if (r < m) y[r] += acc[h];
    }
}

// SBELL: slices of `sh` block rows, one thread per block row (spmv_sbell.cl gpu_sbell<bh><bw>).
template <class V, int BH, int BW4>
__global__ void __launch_bounds__(256) sbell_b4_kernel(const int* __restrict__ slice_ptr, const int* __restrict__ col,
                                                       const V* __restrict__ data, const float* __restrict__ x,
                                                       float* __restrict__ y, int nbr, int sh, int m)
{
    const int br = blockIdx.x * blockDim.x + threadIdx.x;
    if (br >= nbr) return;
    const int sl = br / sh, lr = br - sl * sh;
    const int cs = __ldg(slice_ptr + sl);
    const int width = (__ldg(slice_ptr + sl + 1) - cs) / sh;
    const size_t slotsize = (size_t)sh * BW4 * BH * 4, w4size = (size_t)sh * BH * 4, hsize = (size_t)sh * 4;
    const V* ds = data + (size_t)cs * (BW4 * 4 * BH) + (size_t)lr * 4;
    float acc[BH];
#pragma unroll
    for (int h = 0; h < BH; h++) acc[h] = 0.0f;
    for (int k = 0; k < width; k++) {
        const int c4 = __ldg(col + cs + lr + (size_t)k * sh);
        const V* dk = ds + (size_t)k * slotsize;
#pragma unroll
        for (int w4 = 0; w4 < BW4; w4++) {
            const float4 xv = ldx4(x, (c4 + w4) * 4);
#pragma unroll
            for (int h = 0; h < BH; h++) acc[h] += dot4(Val<V>::ld4(dk + h * hsize + w4 * w4size), xv);
        }
    }
#pragma unroll
    for (int h = 0; h < BH; h++) {
        const int r = br * BH + h;
        if (r < m) y[r] += acc[h];
    }
}

// BCSR in the b4 layout: a group of G lanes per block row, lanes striding over the
// row's blocks (spmv_bcsr.cl gpu_bcsr_red_<bh><bw>: a 128-thread group per block row
// with a shared-memory tree; here a shuffle reduction).
template <class V, int BH, int BW4, int G>
__global__ void __launch_bounds__(256) bcsr_b4_kernel(const int* __restrict__ rp, const int* __restrict__ col,
                                                      const V* __restrict__ data, const float* __restrict__ x,
                                                      float* __restrict__ y, int nbr, int al, int m)
{
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int br = (int)(gid / G), lane = (int)(gid % G);
    const bool valid = br < nbr;
    const int s = valid ? __ldg(rp + br) : 0, e = valid ? __ldg(rp + br + 1) : 0;
    const size_t rowlen = (size_t)al * BH;
    float acc[BH];
#pragma unroll
    for (int h = 0; h < BH; h++) acc[h] = 0.0f;
    for (int j = s + lane; j < e; j += G) {
        const int c4 = __ldg(col + j);
#pragma unroll
        for (int w4 = 0; w4 < BW4; w4++) {
            const float4 xv = ldx4(x, (c4 + w4) * 4);
#pragma unroll
            for (int h = 0; h < BH; h++) acc[h] += dot4(Val<V>::ld4(data + w4 * rowlen + (size_t)h * al + (size_t)j * 4), xv);
        }
    }
#pragma unroll
    for (int h = 0; h < BH; h++) {
        const float t = group_sum<G>(acc[h]);
        const int r = br * BH + h;
        if (valid && lane == 0 && r < m) y[r] += t;
    }
}

// Generic BCSR (block-element-major data[k * aligned + block]) for any block shape with
// bh <= 8: a group of G lanes per block row, consecutive lanes reading consecutive
// blocks, so every data load is coalesced.
template <class V, int BH, int BW, int G>
__global__ void __launch_bounds__(256) bcsr_generic_kernel(const int* __restrict__ rp, const int* __restrict__ col,
                                                           const V* __restrict__ data, const float* __restrict__ x,
                                                           float* __restrict__ y, int nbr, int aligned, int m, int n)
{
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int br = (int)(gid / G), lane = (int)(gid % G);
    const bool valid = br < nbr;
    const int s = valid ? __ldg(rp + br) : 0, e = valid ? __ldg(rp + br + 1) : 0;
    float acc[BH];
#pragma unroll
    for (int h = 0; h < BH; h++) acc[h] = 0.0f;
    for (int j = s + lane; j < e; j += G) {
        const int c0 = __ldg(col + j);
        float xv[BW];
#pragma unroll
        for (int w = 0; w < BW; w++) xv[w] = (c0 + w < n) ? __ldg(x + c0 + w) : 0.0f;
#pragma unroll
        for (int h = 0; h < BH; h++)
#pragma unroll
            for (int w = 0; w < BW; w++) acc[h] += Val<V>::ld(data + (size_t)(h * BW + w) * aligned + j) * xv[w];
    }
#pragma unroll
    for (int h = 0; h < BH; h++) {
        const float t = group_sum<G>(acc[h]);
        const int r = br * BH + h;
        if (valid && lane == 0 && r < m) y[r] += t;
    }
}

}  // namespace dev
}  // namespace csp
