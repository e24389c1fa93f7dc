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

// Generic BCSR, one right-hand side, for blocks of at most 16 elements.  The host cuts
// the block rows into work items of at most kGbBlocks - 3 blocks and kGbRows block rows
// and lays each item out on its own: its blocks start at a multiple of 4 (`ds`) and are
// in column order (stable), dealt to lanes so that lane t of warp w holds the column
// ranks 128w + qT + t (q < 4; T = 32, or a quarter of the item's last, shorter chunk,
// rounded up) at stored slots 128w + 4t + q.  tgt holds each block's position in the
// item's row order (0xffff for the empty slots of the last chunk).  A thread loads its
// four slots with one 128-bit load of their column ids, one of their targets and one per
// block element plane, so every matrix byte moves in a coalesced load; and one gather
// instruction of a warp reads x at 32 consecutive columns of the item (few cache lines).
// The item's y rows are read with the blocks.  Each block's BH row products go to shared
// memory at its target; then a lane group per block row adds its blocks in row order
// (fixed shuffle tree) and writes y.  Work item descriptor: {first block row,
// block rows | blocks << 16, first block in the source (row-pointer) numbering, first
// stored slot}.
constexpr int kGbThreads = 128;   // 8 CTAs per SM at 64 registers: their load and gather phases overlap
constexpr int kGbBlocks = 4 * kGbThreads;
constexpr int kGbRows = 128;

// Row sums of one item: a lane group of G lanes per block row adds the row's block
// products (prod, row order) and writes y = s_y + sum (s_y: the item's y rows).
template <int BH, int G>
__device__ __forceinline__ void gb_rows(const int* s_rp, const float* prod, const float* s_y, int br0, int nrows, int m,
                                        float* __restrict__ y)
{
    const int lane = threadIdx.x % G;
    constexpr int ngroups = kGbThreads / G;
    for (int first = 0; first < nrows; first += ngroups) {
        const int lr = first + threadIdx.x / G;
        const bool valid = lr < nrows;
        const int a = valid ? s_rp[lr] : 0, b = valid ? s_rp[lr + 1] : 0;
        float acc[BH];
#pragma unroll
        for (int h = 0; h < BH; h++) acc[h] = 0.0f;
        for (int k = a + lane; k < b; k += G)
#pragma unroll
            for (int h = 0; h < BH; h++) acc[h] += prod[k * BH + h];
#pragma unroll
        for (int h = 0; h < BH; h++) {
            const float t = group_sum<G>(acc[h]);
            const int r = (br0 + lr) * BH + h;
            if (valid && lane == 0 && r < m) y[r] = s_y[lr * BH + h] + t;
        }
    }
}

template <class V, int BH, int BW>
__global__ void __launch_bounds__(kGbThreads) bcsr_adaptive_kernel(const int* __restrict__ rp, const int* __restrict__ col,
                                                                   const V* __restrict__ data, const float* __restrict__ x,
                                                                   float* __restrict__ y, const int4* __restrict__ work,
                                                                   const unsigned short* __restrict__ tgt, int aligned, int m,
                                                                   int n)
{
    __shared__ float prod[kGbBlocks * BH];
    __shared__ float s_y[kGbRows * BH];
    __shared__ int s_rp[kGbRows + 1];
    const int4 wk = __ldg(work + blockIdx.x);
    const int br0 = wk.x, nrows = wk.y & 0xffff, cnt = wk.y >> 16, s = wk.z;
    const int tid = threadIdx.x;
    const int j = wk.w + 4 * tid;
    const bool act = 4 * tid < cnt;
    int4 c = make_int4(0, 0, 0, 0);
    uint2 tg = make_uint2(0, 0);
    float4 d[BH * BW];
    if (act) {
        c = ld_int4(col + j);
        tg = __ldg(reinterpret_cast<const uint2*>(tgt + j));
#pragma unroll
        for (int k = 0; k < BH * BW; k++) d[k] = Val<V>::ld4(data + (size_t)k * aligned + j);
    }
    // the item's row pointers and y rows, requested with the blocks so that the y update
    // does not wait on DRAM
    if (tid < nrows) s_rp[tid] = __ldg(rp + br0 + tid) - s;
    if (tid == 0) s_rp[nrows] = cnt;
    for (int i = tid; i < nrows * BH; i += kGbThreads)
        if (br0 * BH + i < m) s_y[i] = y[br0 * BH + i];
    if (act) {
        const int cc[4] = {c.x, c.y, c.z, c.w};
        const int tq[4] = {(int)(tg.x & 0xffffu), (int)(tg.x >> 16), (int)(tg.y & 0xffffu), (int)(tg.y >> 16)};
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const bool in = tq[q] != 0xffff;
            float xv[BW];
#pragma unroll
            for (int w = 0; w < BW; w++) xv[w] = (in && cc[q] + w < n) ? __ldg(x + cc[q] + w) : 0.0f;
#pragma unroll
            for (int h = 0; h < BH; h++) {
                float t = 0.0f;
#pragma unroll
                for (int w = 0; w < BW; w++) {
                    const float4 v = d[h * BW + w];
                    const float a = q == 0 ? v.x : q == 1 ? v.y : q == 2 ? v.z : v.w;
                    t += a * xv[w];
                }
                if (in) prod[tq[q] * BH + h] = t;
            }
        }
    }
    __syncthreads();
    if (nrows * 32 <= kGbThreads * 2) gb_rows<BH, 32>(s_rp, prod, s_y, br0, nrows, m, y);
    else if (nrows * 8 <= kGbThreads * 2) gb_rows<BH, 8>(s_rp, prod, s_y, br0, nrows, m, y);
    else if (nrows * 2 <= kGbThreads * 2) gb_rows<BH, 2>(s_rp, prod, s_y, br0, nrows, m, y);
    else gb_rows<BH, 1>(s_rp, prod, s_y, br0, nrows, m, y);
}

}  // namespace dev
}  // namespace csp
