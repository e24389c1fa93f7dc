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
// matrix into work blocks of at most kAdaptNnz entries: runs of whole rows (at most
// kAdaptThreads of them), or one chunk of a row longer than kAdaptNnz, so every CTA
// moves about the same bytes.  Each block is described by an int4
// {first row, row count, first entry, end entry}, or for a chunk
// {chunk index, -(long row id + 1), first entry, end entry}; chunk blocks come first
// in the grid.
//
// A CTA issues every independent load of its block at once -- the 128-bit column
// and value vectors (at most two per thread), the block's row pointers and its y
// values -- then the x gathers, so a block costs two dependent memory round trips.
// Products go to shared memory; each row is reduced by a lane group sized to the
// block's row count and written once (y = y + sum).  A chunk of a long row writes
// its partial sum to a scratch slot; the CTA that finishes a row's last chunk (an
// integer arrival counter, reset by that CTA for the next SpMV) adds the row's
// partials in chunk order.  Results are deterministic.
// ---------------------------------------------------------------------------
constexpr int kAdaptThreads = 256;
constexpr int kAdaptNnz = 2040;                      // <= 2 aligned 4-vectors per thread
constexpr int kAdaptVecs = (kAdaptNnz + 3) / 4 + 1;  // 511

template <int G>
__device__ __forceinline__ void adaptive_rows(const int* s_rp, const float* prod, const float* s_y, int r0, int nrows,
                                              float* __restrict__ y)
{
    const int lane = threadIdx.x % G;
    const int ngroups = kAdaptThreads / G;
    // uniform trip count across the CTA so every lane takes part in the shuffles
    for (int first = 0; first < nrows; first += ngroups) {
        const int lr = first + threadIdx.x / G;
        const bool valid = lr < nrows;
        const int a = valid ? s_rp[lr] : 0, b = valid ? s_rp[lr + 1] : 0;
        float acc = 0.0f;
        for (int j = a + lane; j < b; j += G) acc += prod[j];
        acc = group_sum<G>(acc);
        if (valid && lane == 0) y[r0 + lr] = s_y[lr] + acc;
    }
}

template <class V>
__global__ void __launch_bounds__(kAdaptThreads) csr_adaptive_kernel(const int* __restrict__ rp, const int* __restrict__ col,
                                                                     const V* __restrict__ val, const float* __restrict__ x,
                                                                     float* __restrict__ y, const int4* __restrict__ blocks,
                                                                     const int4* __restrict__ long_rows,
                                                                     float* __restrict__ partial, int* __restrict__ arrivals)
{
    __shared__ __align__(16) float prod[4 * kAdaptVecs];
    __shared__ int s_rp[kAdaptThreads + 1];
    __shared__ float s_y[kAdaptThreads];
    __shared__ float red[kAdaptThreads / 32];
    __shared__ bool s_last;
    const int4 blk = __ldg(blocks + blockIdx.x);
    const int r0 = blk.x, code = blk.y, s = blk.z, e = blk.w;
    const int s4 = s & ~3;
    const int nvec = (e - s4 + 3) >> 2;
    const int tid = threadIdx.x;

    // --- every independent load first ---
    const int v0 = tid, v1 = tid + kAdaptThreads;
    int4 c0 = make_int4(0, 0, 0, 0), c1 = c0;
    float4 a0 = make_float4(0.f, 0.f, 0.f, 0.f), a1 = a0;
    if (v0 < nvec) { c0 = ld_int4(col + s4 + 4 * v0); a0 = Val<V>::ld4(val + s4 + 4 * v0); }
    if (v1 < nvec) { c1 = ld_int4(col + s4 + 4 * v1); a1 = Val<V>::ld4(val + s4 + 4 * v1); }
    const int nrows = code > 0 ? code : 1;
    if (code > 0) {
        // nrows can equal the CTA width, so the end pointer (= e) is written separately
        if (tid < nrows) s_rp[tid] = __ldg(rp + r0 + tid) - s4;
        if (tid == 0) s_rp[nrows] = e - s4;
        if (tid < nrows) s_y[tid] = y[r0 + tid];
    }
    // --- dependent x gathers; entries outside [s, e) contribute nothing ---
    float4 p0, p1;
    {
        const int j = s4 + 4 * v0;
        p0.x = (j + 0 >= s && j + 0 < e) ? a0.x * ldx(x, c0.x) : 0.0f;
        p0.y = (j + 1 >= s && j + 1 < e) ? a0.y * ldx(x, c0.y) : 0.0f;
        p0.z = (j + 2 >= s && j + 2 < e) ? a0.z * ldx(x, c0.z) : 0.0f;
        p0.w = (j + 3 >= s && j + 3 < e) ? a0.w * ldx(x, c0.w) : 0.0f;
    }
    {
        const int j = s4 + 4 * v1;
        p1.x = (j + 0 >= s && j + 0 < e) ? a1.x * ldx(x, c1.x) : 0.0f;
        p1.y = (j + 1 >= s && j + 1 < e) ? a1.y * ldx(x, c1.y) : 0.0f;
        p1.z = (j + 2 >= s && j + 2 < e) ? a1.z * ldx(x, c1.z) : 0.0f;
        p1.w = (j + 3 >= s && j + 3 < e) ? a1.w * ldx(x, c1.w) : 0.0f;
    }
    if (code < 0) {
        // one chunk of a long row: CTA-wide sum to a scratch slot
        float t = (p0.x + p0.y) + (p0.z + p0.w) + ((p1.x + p1.y) + (p1.z + p1.w));
        t = block_sum(t, red);
        const int4 lr = __ldg(long_rows + (-code - 1));   // {row, first slot, chunks, -}
        const int chunk = r0;                              // a chunk block carries its chunk index here
        if (tid == 0) {
            partial[lr.y + chunk] = t;
            __threadfence();
            const int seen = atomicAdd(arrivals + (-code - 1), 1);
            s_last = (seen == lr.z - 1);
        }
        __syncthreads();
        if (s_last && tid == 0) {
            __threadfence();
            float tot = 0.0f;
            for (int k = 0; k < lr.z; k++) tot += __ldcg(partial + lr.y + k);
            y[lr.x] += tot;
            arrivals[-code - 1] = 0;
        }
        return;
    }
    if (v0 < nvec) reinterpret_cast<float4*>(prod)[v0] = p0;
    if (v1 < nvec) reinterpret_cast<float4*>(prod)[v1] = p1;
    __syncthreads();
    if (nrows * 32 <= kAdaptThreads) adaptive_rows<32>(s_rp, prod, s_y, r0, nrows, y);
    else if (nrows * 16 <= kAdaptThreads) adaptive_rows<16>(s_rp, prod, s_y, r0, nrows, y);
    else if (nrows * 8 <= kAdaptThreads) adaptive_rows<8>(s_rp, prod, s_y, r0, nrows, y);
    else if (nrows * 4 <= kAdaptThreads) adaptive_rows<4>(s_rp, prod, s_y, r0, nrows, y);
    else if (nrows * 2 <= kAdaptThreads) adaptive_rows<2>(s_rp, prod, s_y, r0, nrows, y);
    else adaptive_rows<1>(s_rp, prod, s_y, r0, nrows, y);
}

// ---------------------------------------------------------------------------
// COO: nnz-balanced segmented reduction (spmv_coo.cl gpu_coo_s1 / gpu_coo_s2).
// Each warp owns a chunk of kCooTiles tiles of 128 entries (4 per lane, 128-bit
// loads).  Inside a tile, lanes reduce their 4 entries, a keyed shuffle scan over
// lanes joins row segments that cross lanes, and a running carry joins segments
// that cross tiles.  Rows that lie inside one chunk are added to y by the one lane
// that closes them.  A row that crosses a chunk boundary is a "span", found by the
// host when the matrix is uploaded: spans[s] = {row, first chunk, chunks, -} and
// span_of_head[w] = the span that chunk w's first row continues, or -1.  Each chunk
// writes its share of a span to part_val (slot 2w for the chunk's first row, 2w + 1
// for its last) and counts itself on the span's arrival counter; the chunk that
// arrives last adds the shares in chunk order to y and resets the counter.  No
// atomics on y and no second pass: every y entry has a single writer per launch and
// the result is deterministic.  Requires the arrays padded to a multiple of 128
// entries with (last row, last col, 0.0) and rows sorted.
// ---------------------------------------------------------------------------
constexpr int kCooTiles = 4;
constexpr int kCooChunk = 128 * kCooTiles;

template <class V>
__global__ void __launch_bounds__(256) coo_segment_kernel(const int* __restrict__ rowid, const int* __restrict__ colid,
                                                          const V* __restrict__ val, const float* __restrict__ x,
                                                          float* __restrict__ y, int nnz_pad, int nwarps,
                                                          const int* __restrict__ span_of_head, const int4* __restrict__ spans,
                                                          int* __restrict__ span_count, float* __restrict__ part_val)
{
    const int lane = threadIdx.x & 31;
    const int w = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (w >= nwarps) return;
    const int base = w * kCooChunk;
    const int end = min(base + kCooChunk, nnz_pad);
    const int head_row = __ldg(rowid + base);
    const int head_span = __ldg(span_of_head + w);
    const int next_span = (w + 1 < nwarps) ? __ldg(span_of_head + w + 1) : -1;
    // the head segment stays open (deferred to part_val) only if the row began earlier
    bool head_open = head_span >= 0;
    int carry_row = head_row;
    float carry_val = 0.0f;

    // software pipeline: the next tile's rows, columns and values are in flight while
    // the current tile gathers x and reduces
    int4 rn = ld_int4(rowid + base + 4 * lane);
    int4 cn = ld_int4(colid + base + 4 * lane);
    float4 an = Val<V>::ld4(val + base + 4 * lane);
    for (int t = base; t < end; t += 128) {
        const int4 r = rn;
        const int4 c = cn;
        const float4 a = an;
        if (t + 128 < end) {
            const int jn = t + 128 + 4 * lane;
            rn = ld_int4(rowid + jn);
            cn = ld_int4(colid + jn);
            an = Val<V>::ld4(val + jn);
        }
        // y of the tile's rows is requested together with the x gathers, so closing a
        // segment needs no further round trip.  A row closed here is written only by the
        // lane that closes it (head and tail rows go to the scratch pairs instead), so
        // the value read is still the original y.
        const float y0 = y[r.x], y1 = y[r.y], y2 = y[r.z], y3 = y[r.w];
        const float p0 = a.x * ldx(x, c.x), p1 = a.y * ldx(x, c.y);
        const float p2 = a.z * ldx(x, c.z), p3 = a.w * ldx(x, c.w);
        // the segment carried out of the previous tile ends if this tile starts a new row
        const int tile_first = __shfl_sync(0xffffffffu, r.x, 0);
        if (tile_first != carry_row) {
            if (lane == 0) {
                if (head_open && carry_row == head_row) {
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
        const float yy[4] = {y0, y1, y2, y3};
#pragma unroll
        for (int k = 0; k < 4; k++) {
            run += pp[k];
            const bool last_in_lane = (k == 3);
            const int nxt = last_in_lane ? next_first : rr[k + 1];
            const bool closes = !last_in_lane ? (nxt != rr[k]) : (lane < 31 && nxt != rr[k]);
            if (closes) {
                if (head_open && rr[k] == head_row) {
                    part_val[2 * w] = run;
                    closed_head = true;
                } else {
                    y[rr[k]] = yy[k] + run;
                }
                run = 0.0f;
            }
        }
        // the segment still open at lane 31 carries into the next tile
        carry_row = __shfl_sync(0xffffffffu, r.w, 31);
        carry_val = __shfl_sync(0xffffffffu, run, 31);
        if (__any_sync(0xffffffffu, closed_head)) head_open = false;
    }
    // the segment still open at the end of the chunk: its row continues into the next
    // chunk exactly when that chunk's head belongs to a span
    int arrive0 = -1, arrive1 = -1;
    if (head_open) {
        // the whole chunk lies in the head row, which began in an earlier chunk
        if (lane == 0) part_val[2 * w] = carry_val;
        arrive0 = head_span;
    } else {
        if (head_span >= 0) arrive0 = head_span;   // its share was written when the head closed
        if (next_span >= 0) {
            if (lane == 0) part_val[2 * w + 1] = carry_val;
            arrive1 = next_span;
        } else if (lane == 0) {
            y[carry_row] += carry_val;
        }
    }
    if (arrive0 < 0 && arrive1 < 0) return;
    __threadfence();
    __syncwarp();
    if (lane != 0) return;
    const int arr[2] = {arrive0, arrive1};
#pragma unroll
    for (int q = 0; q < 2; q++) {
        const int sp = arr[q];
        if (sp < 0) continue;
        const int4 d = __ldg(spans + sp);   // {row, first chunk, chunks, -}
        if (atomicAdd(span_count + sp, 1) == d.z - 1) {
            __threadfence();
            float tot = __ldcg(part_val + 2 * d.y + 1);
            for (int c = d.y + 1; c < d.y + d.z; c++) tot += __ldcg(part_val + 2 * c);
            y[d.x] += tot;
            span_count[sp] = 0;
        }
    }
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
