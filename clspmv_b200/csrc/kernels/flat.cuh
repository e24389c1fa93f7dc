// Flat-format SpMV kernels: CSR (scalar, vector, adaptive row blocks), COO
// (segmented reduction), ELL and SELL.  All compute y += A * x with FP32
// accumulation, are deterministic (no floating-point atomics) and read matrix
// data with 128-bit loads wherever the layout allows.
//
// Semantics follow the reference kernels named beside each one
// (clSpMV_NV/kernels/*.cl); the work decomposition is this library's own.
#pragma once

#include "common.cuh"

namespace csp {
namespace dev {

// ---------------------------------------------------------------------------
// CSR scalar: one thread per row (spmv_csr_scalar.cl gpu_csr_sc_pm / _u4).
// UNROLL=4 issues four independent gathers per iteration.
// ---------------------------------------------------------------------------
template <class V, int UNROLL>
__global__ void __launch_bounds__(256) csr_scalar_kernel(const int* __restrict__ rp, const int* __restrict__ col,
                                                         const V* __restrict__ val, const float* __restrict__ x,
                                                         float* __restrict__ y, int m)
{
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= m) return;
    const int s = __ldg(rp + row), e = __ldg(rp + row + 1);
    float acc[UNROLL];
#pragma unroll
    for (int u = 0; u < UNROLL; u++) acc[u] = 0.0f;
    int j = s;
    for (; j + UNROLL <= e; j += UNROLL) {
#pragma unroll
        for (int u = 0; u < UNROLL; u++) acc[u] += Val<V>::ld(val + j + u) * ldx(x, __ldg(col + j + u));
    }
    for (; j < e; j++) acc[0] += Val<V>::ld(val + j) * ldx(x, __ldg(col + j));
    float t = 0.0f;
#pragma unroll
    for (int u = 0; u < UNROLL; u++) t += acc[u];
    y[row] += t;
}

// CSR scalar on a row-padded CSR (every row a multiple of 4 entries starting on a
// multiple of 4; util.cpp:31 pad_csr): 128-bit loads, no remainder branch
// (spmv_csr_scalar.cl gpu_csr_sc_pm_float4_noif).
template <class V>
__global__ void __launch_bounds__(256) csr_scalar4_kernel(const int* __restrict__ rp, const int* __restrict__ col,
                                                          const V* __restrict__ val, const float* __restrict__ x,
                                                          float* __restrict__ y, int m)
{
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= m) return;
    const int s = __ldg(rp + row), e = __ldg(rp + row + 1);
    float acc = 0.0f;
    for (int j = s; j < e; j += 4) {
        const int4 c = ld_int4(col + j);
        const float4 v = Val<V>::ld4(val + j);
        acc += v.x * ldx(x, c.x) + v.y * ldx(x, c.y) + v.z * ldx(x, c.z) + v.w * ldx(x, c.w);
    }
    y[row] += acc;
}

// Products of the row segment [s, e) handled by one lane group of G lanes, read as
// aligned 4-wide vectors (col/val arrays are padded to a multiple of 4 entries, so the
// aligned vector covering e-1 is always in bounds).
template <class V, int G>
__device__ __forceinline__ float segment_dot(const int* __restrict__ col, const V* __restrict__ val,
                                             const float* __restrict__ x, int s, int e, int lane)
{
    float acc = 0.0f;
    for (int j = (s & ~3) + 4 * lane; j < e; j += 4 * G) {
        const int4 c = ld_int4(col + j);
        const float4 v = Val<V>::ld4(val + j);
        if (j >= s && j + 3 < e) {
            acc += v.x * ldx(x, c.x) + v.y * ldx(x, c.y) + v.z * ldx(x, c.z) + v.w * ldx(x, c.w);
        } else {
            if (j + 0 >= s && j + 0 < e) acc += v.x * ldx(x, c.x);
            if (j + 1 >= s && j + 1 < e) acc += v.y * ldx(x, c.y);
            if (j + 2 >= s && j + 2 < e) acc += v.z * ldx(x, c.z);
            if (j + 3 >= s && j + 3 < e) acc += v.w * ldx(x, c.w);
        }
    }
    return acc;
}

// ---------------------------------------------------------------------------
// CSR vector: a group of G lanes per row (G = 32 is spmv_csr_vector.cl
// gpu_csr_ve_slm_pm: one warp per row; the reduction is shuffles, not the
// reference's barrier-free shared-memory tree, which is unsafe under independent
// thread scheduling).
// ---------------------------------------------------------------------------
template <class V, int G>
__global__ void __launch_bounds__(256) csr_vector_kernel(const int* __restrict__ rp, const int* __restrict__ col,
                                                         const V* __restrict__ val, const float* __restrict__ x,
                                                         float* __restrict__ y, int m)
{
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int row = (int)(gid / G);
    const int lane = (int)(gid % G);
    // rows past m keep their lanes in the shuffle with an empty segment
    const bool valid = row < m;
    const int s = valid ? __ldg(rp + row) : 0, e = valid ? __ldg(rp + row + 1) : 0;
    float acc = segment_dot<V, G>(col, val, x, s, e, lane);
    acc = group_sum<G>(acc);
    if (valid && lane == 0) y[row] += acc;
}

// CSR with one CTA per row (spmv_csr_vector.cl gpu_csr_ve_reduction: a 128-thread
// group per row).
template <class V, int THREADS>
__global__ void __launch_bounds__(THREADS) csr_block_row_kernel(const int* __restrict__ rp, const int* __restrict__ col,
                                                                const V* __restrict__ val, const float* __restrict__ x,
                                                                float* __restrict__ y, int m)
{
    __shared__ float red[THREADS / 32];
    const int row = blockIdx.x;
    const int s = __ldg(rp + row), e = __ldg(rp + row + 1);
    float acc = segment_dot<V, THREADS>(col, val, x, s, e, threadIdx.x);
    acc = block_sum(acc, red);
    if (threadIdx.x == 0) y[row] += acc;
}

// ---------------------------------------------------------------------------
// CSR adaptive (this library's B200 kernel for irregular rows).  The host cuts the
// rows into row blocks of at most ADAPT_NNZ entries and at most THREADS rows
// (a longer row forms a block on its own).  A CTA streams its block's entries with
// coalesced 128-bit loads into shared memory as products val*x[col], then reduces
// each row from shared memory with a lane group sized to the block's row count; a
// single long row is reduced by the whole CTA.  Every row is written by exactly one
// thread, so the result is deterministic.
// ---------------------------------------------------------------------------
constexpr int kAdaptThreads = 256;
constexpr int kAdaptNnz = 2048;

template <int G>
__device__ __forceinline__ void adaptive_rows(const int* __restrict__ rp, const float* prod, int s4, int r0, int r1,
                                              float* __restrict__ y)
{
    const int lane = threadIdx.x % G;
    const int ngroups = kAdaptThreads / G;
    // uniform trip count across the CTA so every lane takes part in the shuffles
    for (int first = r0; first < r1; first += ngroups) {
        const int r = first + threadIdx.x / G;
        const bool valid = r < r1;
        const int a = valid ? __ldg(rp + r) - s4 : 0, b = valid ? __ldg(rp + r + 1) - s4 : 0;
        float acc = 0.0f;
        for (int j = a + lane; j < b; j += G) acc += prod[j];
        acc = group_sum<G>(acc);
        if (valid && lane == 0) y[r] += acc;
    }
}

template <class V>
__global__ void __launch_bounds__(kAdaptThreads) csr_adaptive_kernel(const int* __restrict__ rp, const int* __restrict__ col,
                                                                     const V* __restrict__ val, const float* __restrict__ x,
                                                                     float* __restrict__ y, const int* __restrict__ blocks)
{
    __shared__ __align__(16) float prod[kAdaptNnz + 8];
    __shared__ float red[kAdaptThreads / 32];
    const int r0 = __ldg(blocks + blockIdx.x), r1 = __ldg(blocks + blockIdx.x + 1);
    const int s = __ldg(rp + r0), e = __ldg(rp + r1);
    if (e - s > kAdaptNnz) {
        // one long row
        float acc = segment_dot<V, kAdaptThreads>(col, val, x, s, e, threadIdx.x);
        acc = block_sum(acc, red);
        if (threadIdx.x == 0) y[r0] += acc;
        return;
    }
    const int s4 = s & ~3;
    const int nvec = (e - s4 + 3) >> 2;   // <= kAdaptNnz / 4 + 1
    for (int v = threadIdx.x; v < nvec; v += kAdaptThreads) {
        const int j = s4 + 4 * v;
        const int4 c = ld_int4(col + j);
        const float4 a = Val<V>::ld4(val + j);
        float4 p;
        p.x = (j + 0 >= s && j + 0 < e) ? a.x * ldx(x, c.x) : 0.0f;
        p.y = (j + 1 >= s && j + 1 < e) ? a.y * ldx(x, c.y) : 0.0f;
        p.z = (j + 2 >= s && j + 2 < e) ? a.z * ldx(x, c.z) : 0.0f;
        p.w = (j + 3 >= s && j + 3 < e) ? a.w * ldx(x, c.w) : 0.0f;
        reinterpret_cast<float4*>(prod)[v] = p;
    }
    __syncthreads();
    const int nrows = r1 - r0;
    // lanes per row: as many as the block's row count allows, at most a warp
    if (nrows * 32 <= kAdaptThreads) adaptive_rows<32>(rp, prod, s4, r0, r1, y);
    else if (nrows * 16 <= kAdaptThreads) adaptive_rows<16>(rp, prod, s4, r0, r1, y);
    else if (nrows * 8 <= kAdaptThreads) adaptive_rows<8>(rp, prod, s4, r0, r1, y);
    else if (nrows * 4 <= kAdaptThreads) adaptive_rows<4>(rp, prod, s4, r0, r1, y);
    else if (nrows * 2 <= kAdaptThreads) adaptive_rows<2>(rp, prod, s4, r0, r1, y);
    else adaptive_rows<1>(rp, prod, s4, r0, r1, y);
}

// ---------------------------------------------------------------------------
// COO: nnz-balanced segmented reduction (spmv_coo.cl gpu_coo_s1 / gpu_coo_s2).
// Each warp owns a chunk of kCooTiles tiles of 128 entries (4 per lane, 128-bit
// loads).  Inside a tile, lanes reduce their 4 entries, a keyed shuffle scan over
// lanes joins row segments that cross lanes, and a running carry joins segments
// that cross tiles.  Rows that begin and end inside the chunk are added to y by
// the one lane that closes them.  The chunk's first row segment ("head") and its
// still-open last segment ("tail") go to a scratch array of (row, partial) pairs;
// coo_fixup_kernel then adds every run of equal rows there in order.  No atomics:
// every y entry has a single writer per kernel and the result is deterministic.
// Requires the arrays padded to a multiple of 128 entries with (last row, last
// col, 0.0) and rows sorted.
// ---------------------------------------------------------------------------
constexpr int kCooTiles = 4;
constexpr int kCooChunk = 128 * kCooTiles;

template <class V>
__global__ void __launch_bounds__(256) coo_segment_kernel(const int* __restrict__ rowid, const int* __restrict__ colid,
                                                          const V* __restrict__ val, const float* __restrict__ x,
                                                          float* __restrict__ y, int nnz_pad, int nwarps,
                                                          int* __restrict__ part_row, float* __restrict__ part_val)
{
    const int lane = threadIdx.x & 31;
    const int w = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (w >= nwarps) return;
    const int base = w * kCooChunk;
    const int end = min(base + kCooChunk, nnz_pad);
    const int head_row = __ldg(rowid + base);
    bool head_open = true;
    int carry_row = head_row;
    float carry_val = 0.0f;

    for (int t = base; t < end; t += 128) {
        const int j = t + 4 * lane;
        const int4 r = ld_int4(rowid + j);
        const int4 c = ld_int4(colid + j);
        const float4 a = Val<V>::ld4(val + j);
        const float p0 = a.x * ldx(x, c.x), p1 = a.y * ldx(x, c.y);
        const float p2 = a.z * ldx(x, c.z), p3 = a.w * ldx(x, c.w);
        // the segment carried out of the previous tile ends if this tile starts a new row
        const int tile_first = __shfl_sync(0xffffffffu, r.x, 0);
        if (tile_first != carry_row) {
            if (lane == 0) {
                if (head_open && carry_row == head_row) {
                    part_row[2 * w] = carry_row;
                    part_val[2 * w] = carry_val;
                } else {
                    y[carry_row] += carry_val;
                }
            }
            if (head_open && carry_row == head_row) head_open = false;
            carry_row = tile_first;
            carry_val = 0.0f;
        }
        // suffix run of this lane (entries equal to its last row)
        float tail = p3;
        if (r.z == r.w) { tail += p2; if (r.y == r.w) { tail += p1; if (r.x == r.w) tail += p0; } }
        // keyed inclusive scan of the suffix runs over lanes (rows are sorted, so equal
        // keys are contiguous)
        float scan = tail;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const float o = __shfl_up_sync(0xffffffffu, scan, d);
            const int ok = __shfl_up_sync(0xffffffffu, r.w, d);
            if (lane >= d && ok == r.w) scan += o;
        }
        const float prev_scan = __shfl_up_sync(0xffffffffu, scan, 1);
        const int prev_key = __shfl_up_sync(0xffffffffu, r.w, 1);
        const int next_first = __shfl_down_sync(0xffffffffu, r.x, 1);
        float run = (lane > 0 && prev_key == r.x) ? prev_scan : 0.0f;
        if (r.x == carry_row) run += carry_val;
        bool closed_head = false;
        // walk the lane's four entries, closing segments
        const int rr[4] = {r.x, r.y, r.z, r.w};
        const float pp[4] = {p0, p1, p2, p3};
#pragma unroll
        for (int k = 0; k < 4; k++) {
            run += pp[k];
            const bool last_in_lane = (k == 3);
            const int nxt = last_in_lane ? next_first : rr[k + 1];
            const bool closes = !last_in_lane ? (nxt != rr[k]) : (lane < 31 && nxt != rr[k]);
            if (closes) {
                if (head_open && rr[k] == head_row) {
                    part_row[2 * w] = rr[k];
                    part_val[2 * w] = run;
                    closed_head = true;
                } else {
                    y[rr[k]] += run;
                }
                run = 0.0f;
            }
        }
        // the segment still open at lane 31 carries into the next tile
        carry_row = __shfl_sync(0xffffffffu, r.w, 31);
        carry_val = __shfl_sync(0xffffffffu, run, 31);
        if (__any_sync(0xffffffffu, closed_head)) head_open = false;
    }
    if (lane == 0) {
        if (head_open) {
            part_row[2 * w] = carry_row;      // == head_row: the chunk is one open segment
            part_val[2 * w] = carry_val;
            part_row[2 * w + 1] = carry_row;
            part_val[2 * w + 1] = 0.0f;
        } else {
            part_row[2 * w + 1] = carry_row;
            part_val[2 * w + 1] = carry_val;
        }
    }
}

// Adds the chunk heads/tails: the first entry of every run of equal rows sums the run.
__global__ void __launch_bounds__(256) coo_fixup_kernel(const int* __restrict__ part_row, const float* __restrict__ part_val,
                                                        int nparts, float* __restrict__ y)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nparts) return;
    const int r = part_row[i];
    if (i > 0 && part_row[i - 1] == r) return;
    float acc = 0.0f;
    for (int k = i; k < nparts && part_row[k] == r; k++) acc += part_val[k];
    y[r] += acc;
}

// ---------------------------------------------------------------------------
// ELL, column-major (spmv_ell.cl gpu_ell / gpu_ell_v4).  ROWS consecutive rows per
// thread; ROWS = 4 uses 128-bit loads (height_aligned is a multiple of 4).
// ---------------------------------------------------------------------------
template <class V, int ROWS>
__global__ void __launch_bounds__(256) ell_kernel(const int* __restrict__ col, const V* __restrict__ val,
                                                  const float* __restrict__ x, float* __restrict__ y,
                                                  int m, int ell_num, int hal)
{
    const int r0 = (blockIdx.x * blockDim.x + threadIdx.x) * ROWS;
    if (r0 >= m) return;
    if (ROWS == 4) {
        float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
        for (int k = 0; k < ell_num; k++) {
            const size_t j = (size_t)k * hal + r0;
            const int4 c = ld_int4(col + j);
            const float4 a = Val<V>::ld4(val + j);
            acc.x += a.x * ldx(x, c.x);
            acc.y += a.y * ldx(x, c.y);
            acc.z += a.z * ldx(x, c.z);
            acc.w += a.w * ldx(x, c.w);
        }
        y[r0] += acc.x;
        if (r0 + 1 < m) y[r0 + 1] += acc.y;
        if (r0 + 2 < m) y[r0 + 2] += acc.z;
        if (r0 + 3 < m) y[r0 + 3] += acc.w;
    } else {
        float acc = 0.0f;
        for (int k = 0; k < ell_num; k++) {
            const size_t j = (size_t)k * hal + r0;
            acc += Val<V>::ld(val + j) * ldx(x, __ldg(col + j));
        }
        y[r0] += acc;
    }
}

// ---------------------------------------------------------------------------
// SELL (spmv_sell.cl gpu_sell_warp / gpu_sell_group): slices of H rows, each a
// column-major ELL of its own width.  Four consecutive rows per thread with 128-bit
// loads (H is a multiple of 4).
// ---------------------------------------------------------------------------
template <class V>
__global__ void __launch_bounds__(256) sell4_kernel(const int* __restrict__ slice_ptr, const int* __restrict__ col,
                                                    const V* __restrict__ val, const float* __restrict__ x,
                                                    float* __restrict__ y, int m, int H)
{
    const int r0 = (blockIdx.x * blockDim.x + threadIdx.x) * 4;
    if (r0 >= m) return;
    const int sl = r0 / H, lr = r0 - sl * H;
    const int b = __ldg(slice_ptr + sl);
    const int width = (__ldg(slice_ptr + sl + 1) - b) / H;
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int k = 0; k < width; k++) {
        const int j = b + k * H + lr;
        const int4 c = ld_int4(col + j);
        const float4 a = Val<V>::ld4(val + j);
        acc.x += a.x * ldx(x, c.x);
        acc.y += a.y * ldx(x, c.y);
        acc.z += a.z * ldx(x, c.z);
        acc.w += a.w * ldx(x, c.w);
    }
    y[r0] += acc.x;
    if (r0 + 1 < m) y[r0 + 1] += acc.y;
    if (r0 + 2 < m) y[r0 + 2] += acc.z;
    if (r0 + 3 < m) y[r0 + 3] += acc.w;
}

template <class V>
__global__ void __launch_bounds__(256) sell1_kernel(const int* __restrict__ slice_ptr, const int* __restrict__ col,
                                                    const V* __restrict__ val, const float* __restrict__ x,
                                                    float* __restrict__ y, int m, int H)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= m) return;
    const int sl = r / H, lr = r - sl * H;
    const int b = __ldg(slice_ptr + sl);
    const int width = (__ldg(slice_ptr + sl + 1) - b) / H;
    float acc = 0.0f;
    for (int k = 0; k < width; k++) {
        const int j = b + k * H + lr;
        acc += Val<V>::ld(val + j) * ldx(x, __ldg(col + j));
    }
    y[r] += acc;
}

}  // namespace dev
}  // namespace csp
