// Value-gradient kernels of the adjoint: abar[slot] = ybar[row(slot)] * x[col(slot)]
// over every stored slot of a part, in the part's storage order, or -- when `prow`
// is non-null -- the (row, col) of each slot (row -1 for slots outside the matrix:
// alignment rows and out-of-range diagonal positions), so a caller can map abar back
// to matrix entries.  The transposed product itself reuses the forward kernels on
// transposed parts.
#pragma once

#include "common.cuh"

namespace csp {
namespace dev {

__device__ __forceinline__ void put_slot(size_t i, int row, int col, const float* __restrict__ ybar,
                                         const float* __restrict__ x, float* __restrict__ abar,
                                         int* __restrict__ prow, int* __restrict__ pcol)
{
    if (prow) {
        prow[i] = row;
        pcol[i] = row < 0 ? -1 : col;
    } else {
        abar[i] = row < 0 ? 0.0f : __ldg(ybar + row) * __ldg(x + col);
    }
}

// DIA-layout slots (also BDIA, whose slots carry per-slot offsets): slot (d, r)
// couples row r with column r + off[d].
__global__ void __launch_bounds__(256) abar_dia_kernel(const int* __restrict__ off, int nslots_per_row, int len,
                                                       int m, int n, const float* __restrict__ ybar,
                                                       const float* __restrict__ x, float* __restrict__ abar,
                                                       int* __restrict__ prow, int* __restrict__ pcol)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)nslots_per_row * len) return;
    const int d = (int)(i / len), r = (int)(i % len);
    const int c = r + __ldg(off + d);
    const bool in = r < m && c >= 0 && c < n;
    put_slot(i, in ? r : -1, c, ybar, x, abar, prow, pcol);
}

// Value gradients of DIA-layout slots, four rows per thread over every diagonal: the
// thread's ybar values are loaded once, x around row r + off[d] comes from two aligned
// 128-bit loads (scalar, guarded loads at the matrix edges), and each diagonal gets one
// 128-bit streaming store, so a warp writes 512 contiguous bytes per diagonal.  No
// 64-bit index division.  len is a multiple of 4, abar is 16-byte aligned (checked by
// the host) and x is the handle's padded x; the offsets (nd of them) are staged in
// shared memory.
__global__ void __launch_bounds__(256) abar_dia4_kernel(const int* __restrict__ off, int nd, int len, int m, int n,
                                                        const float* __restrict__ ybar, const float* __restrict__ x,
                                                        float* __restrict__ abar)
{
    extern __shared__ int s_off[];
    for (int i = threadIdx.x; i < nd; i += blockDim.x) s_off[i] = __ldg(off + i);
    __syncthreads();
    const int r = 4 * (blockIdx.x * blockDim.x + threadIdx.x);
    if (r >= len) return;
    float yb[4];
#pragma unroll
    for (int q = 0; q < 4; q++) yb[q] = r + q < m ? __ldg(ybar + r + q) : 0.0f;
    for (int d = 0; d < nd; d++) {
        const int base = r + s_off[d];
        float xv[4];
        if (base >= 0 && base + 3 < n) {
            // x[base .. base+3] from the two aligned float4s around it (x is 16-byte
            // aligned and zero-padded by at least 64 entries past n)
            const int b4 = base & ~3;
            const float4 lo = ldx4(x, b4), hi = ldx4(x, b4 + 4);
            switch (base - b4) {
            case 0: xv[0] = lo.x; xv[1] = lo.y; xv[2] = lo.z; xv[3] = lo.w; break;
            case 1: xv[0] = lo.y; xv[1] = lo.z; xv[2] = lo.w; xv[3] = hi.x; break;
            case 2: xv[0] = lo.z; xv[1] = lo.w; xv[2] = hi.x; xv[3] = hi.y; break;
            default: xv[0] = lo.w; xv[1] = hi.x; xv[2] = hi.y; xv[3] = hi.z; break;
            }
        } else {
#pragma unroll
            for (int q = 0; q < 4; q++) xv[q] = (base + q >= 0 && base + q < n) ? __ldg(x + base + q) : 0.0f;
        }
        __stcs(reinterpret_cast<float4*>(abar + (size_t)d * len + r),
               make_float4(yb[0] * xv[0], yb[1] * xv[1], yb[2] * xv[2], yb[3] * xv[3]));
    }
}

// Slot lists with explicit row ids (COO; CSR with its row-id array; the block layouts'
// slot maps, row -1 on padding slots).
__global__ void __launch_bounds__(256) abar_list_kernel(const int* __restrict__ rows, const int* __restrict__ cols,
                                                        size_t nslots, const float* __restrict__ ybar,
                                                        const float* __restrict__ x, float* __restrict__ abar,
                                                        int* __restrict__ prow, int* __restrict__ pcol)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nslots) return;
    put_slot(i, __ldg(rows + i), __ldg(cols + i), ybar, x, abar, prow, pcol);
}

// Generic BCSR slots data[e * aligned + j]: element e of block j couples row
// brow[j] * bh + e / bw with column col[j] + e % bw (row -1 past the blocks or the matrix).
__global__ void __launch_bounds__(256) abar_gbcsr_kernel(const int* __restrict__ brow, const int* __restrict__ col,
                                                         int aligned, int nblocks, int bh, int bw, int m, int n,
                                                         const float* __restrict__ ybar, const float* __restrict__ x,
                                                         float* __restrict__ abar, int* __restrict__ prow,
                                                         int* __restrict__ pcol)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)aligned * bh * bw) return;
    const int e = (int)(i / aligned), j = (int)(i % aligned);
    int r = -1, c = -1;
    if (j < nblocks) {
        r = __ldg(brow + j) * bh + e / bw;
        c = __ldg(col + j) + e % bw;
        if (r >= m || c >= n) r = -1;
    }
    put_slot(i, r, c, ybar, x, abar, prow, pcol);
}

// Column-major ELL slots (k, r), r < height_aligned.
__global__ void __launch_bounds__(256) abar_ell_kernel(const int* __restrict__ col, int ell_num, int hal, int m,
                                                       const float* __restrict__ ybar, const float* __restrict__ x,
                                                       float* __restrict__ abar, int* __restrict__ prow,
                                                       int* __restrict__ pcol)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)ell_num * hal) return;
    const int r = (int)(i % hal);
    put_slot(i, r < m ? r : -1, __ldg(col + i), ybar, x, abar, prow, pcol);
}

// SELL slots: one thread per slice row walks that row's slots.
__global__ void __launch_bounds__(256) abar_sell_kernel(const int* __restrict__ slice_ptr, const int* __restrict__ col,
                                                        int H, int nslices, int m, const float* __restrict__ ybar,
                                                        const float* __restrict__ x, float* __restrict__ abar,
                                                        int* __restrict__ prow, int* __restrict__ pcol)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nslices * H) return;
    const int s = t / H, lr = t % H;
    const int b = __ldg(slice_ptr + s);
    const int width = (__ldg(slice_ptr + s + 1) - b) / H;
    const int r = s * H + lr;
    for (int k = 0; k < width; k++) {
        const size_t i = (size_t)b + (size_t)k * H + lr;
        put_slot(i, r < m ? r : -1, __ldg(col + i), ybar, x, abar, prow, pcol);
    }
}

}  // namespace dev
}  // namespace csp
