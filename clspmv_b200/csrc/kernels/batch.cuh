// Batched execution: one persistent kernel serves a work list of (part, row-slice)
// items drawn from many matrices of uneven size.  A part is one matrix (or its
// transpose, for the adjoint) stored in one of the batch formats:
//
//   BK_CSR    CSR cut into work blocks of whole rows (<= kAdaptNnz entries) or
//             chunks of one long row, the same blocks as csr_adaptive_kernel, one
//             block per item;
//   BK_SELL   sliced ELL, slice height H (32 or 128), column-major inside a slice,
//             padding slots carry column -1;
//   BK_DIA    diagonals, data[d * stride + r] couples row r with column r + off[d];
//   BK_BCSR*  B x B blocks (B = 2, 3, 4), block-element-major data[q * aligned + j].
//
// A forward part may also write the value gradient abar[slot] = ybar[row] * x[col]
// for each stored slot, in the part's storage order: the x value is already in a
// register, so the gradient costs one coalesced store per slot.  The adjoint
// xbar += A^T ybar runs the same bodies on a part that stores A^T.
//
// Items are 32 bytes: {part, first virtual block, end virtual block, -} and, for a
// CSR item, the CSR work block itself.  CTA c runs items c, c + G, c + 2G, ... (G =
// grid size): the items are cut to about the same bytes, so a static round-robin
// balances, and every CTA knows its next items in advance.  Two items ahead it
// loads the item, one item ahead the part descriptor, both while the current item
// runs, so an item starts with its descriptor already in shared memory and its first
// loads are the matrix data.  Every output element has exactly one writer per
// launch and every sum is taken in a fixed order, so results are deterministic.
#pragma once

#include "common.cuh"
#include "flat.cuh"

namespace csp {
namespace dev {

enum BatchKind : int { BK_CSR = 0, BK_SELL = 1, BK_DIA = 2, BK_BCSR2 = 3, BK_BCSR3 = 4, BK_BCSR4 = 5 };

constexpr int kBatchThreads = 256;
constexpr int kBatchMaxDiag = 64;
constexpr int kBatchDiaRows = 2;   // rows per thread in a DIA item step
constexpr int kBatchBcsrLanes = 4; // lanes per block row

struct BatchPart {
    int kind;
    int m, n;        // rows and columns of the stored operator
    int k;           // DIA: diagonals
    int stride;      // DIA: slot stride; SELL: slice height; BCSR: aligned block count
    int nbr;         // BCSR: block rows; SELL: slices
    int grad;        // 1: write the value gradient (forward parts only)
    int pad0;
    const int* i0;   // CSR row_ptr / SELL slice_ptr / DIA offsets / BCSR block-row pointer
    const int* i1;   // CSR / SELL column ids, BCSR block columns
    const void* v;   // values (FP32 or BF16)
    const int4* long_rows;  // CSR long rows {row, first partial slot, chunks, -}
    float* partial;         // CSR long-row chunk sums
    int* arrivals;          // CSR long-row arrival counters
    const float* x;
    float* y;
    const float* ybar;
    float* abar;
};
static_assert(sizeof(BatchPart) % 8 == 0, "BatchPart layout");
constexpr int kBatchPartWords = (int)(sizeof(BatchPart) / 4);

struct BatchItem {
    int part, v0, v1, pad;
    int4 blk;   // CSR items: the work block (v1 == v0 + 1)
};
constexpr int kBatchItemWords = (int)(sizeof(BatchItem) / 4);

struct BatchSmem {
    BatchPart part[2];
    BatchItem item[2];
    float4 prod[kAdaptVecs];
    int rp[kAdaptThreads + 1];
    float ys[kAdaptThreads];
    unsigned char rowid[4 * kAdaptVecs];
    float red[kBatchThreads / 32];
    int off[kBatchMaxDiag];
    int last;
};

// one float4 of entries [j, j + 4) of a gradient array; only slots inside [s, e)
__device__ __forceinline__ void put_grad4(float* __restrict__ abar, int j, int s, int e, float4 g)
{
    if (j >= s && j + 3 < e) {
        *reinterpret_cast<float4*>(abar + j) = g;
    } else {
        if (j + 0 >= s && j + 0 < e) abar[j + 0] = g.x;
        if (j + 1 >= s && j + 1 < e) abar[j + 1] = g.y;
        if (j + 2 >= s && j + 2 < e) abar[j + 2] = g.z;
        if (j + 3 >= s && j + 3 < e) abar[j + 3] = g.w;
    }
}

template <int G, bool GRAD>
__device__ __forceinline__ void batch_rows(BatchSmem& sm, int r0, int nrows, float* __restrict__ y)
{
    const float* prod = reinterpret_cast<const float*>(sm.prod);
    const int lane = threadIdx.x % G;
    constexpr int ngroups = kBatchThreads / G;
    for (int first = 0; first < nrows; first += ngroups) {
        const int lr = first + threadIdx.x / G;
        const bool valid = lr < nrows;
        const int a = valid ? sm.rp[lr] : 0, b = valid ? sm.rp[lr + 1] : 0;
        float acc = 0.0f;
        for (int j = a + lane; j < b; j += G) {
            acc += prod[j];
            if (GRAD) sm.rowid[j] = (unsigned char)lr;
        }
        acc = group_sum<G>(acc);
        if (valid && lane == 0) y[r0 + lr] = sm.ys[lr] + acc;
    }
}

// CSR work block `vb` (see csr_adaptive_kernel for the block encoding).
template <class V, bool GRAD>
__device__ __forceinline__ void batch_csr(BatchSmem& sm, const BatchPart& P, int4 blk)
{
    const int* __restrict__ col = P.i1;
    const V* __restrict__ val = static_cast<const V*>(P.v);
    const float* __restrict__ x = P.x;
    float* __restrict__ y = P.y;
    const int r0 = blk.x, code = blk.y, s = blk.z, e = blk.w;
    const int s4 = s & ~3;
    const int nvec = (e - s4 + 3) >> 2;
    const int tid = threadIdx.x;
    const int v0 = tid, v1 = tid + kBatchThreads;
    int4 c0 = make_int4(0, 0, 0, 0), c1 = c0;
    float4 a0 = make_float4(0.f, 0.f, 0.f, 0.f), a1 = a0;
    if (v0 < nvec) { c0 = ld_int4(col + s4 + 4 * v0); a0 = Val<V>::ld4(val + s4 + 4 * v0); }
    if (v1 < nvec) { c1 = ld_int4(col + s4 + 4 * v1); a1 = Val<V>::ld4(val + s4 + 4 * v1); }
    const int nrows = code > 0 ? code : 1;
    if (code > 0) {
        if (tid < nrows) sm.rp[tid] = __ldg(P.i0 + r0 + tid) - s4;
        if (tid == 0) sm.rp[nrows] = e - s4;
        if (tid < nrows) sm.ys[tid] = y[r0 + tid];
    }
    float4 x0, x1;
    {
        const int j = s4 + 4 * v0;
        x0.x = (j + 0 >= s && j + 0 < e) ? ldx(x, c0.x) : 0.0f;
        x0.y = (j + 1 >= s && j + 1 < e) ? ldx(x, c0.y) : 0.0f;
        x0.z = (j + 2 >= s && j + 2 < e) ? ldx(x, c0.z) : 0.0f;
        x0.w = (j + 3 >= s && j + 3 < e) ? ldx(x, c0.w) : 0.0f;
    }
    {
        const int j = s4 + 4 * v1;
        x1.x = (j + 0 >= s && j + 0 < e) ? ldx(x, c1.x) : 0.0f;
        x1.y = (j + 1 >= s && j + 1 < e) ? ldx(x, c1.y) : 0.0f;
        x1.z = (j + 2 >= s && j + 2 < e) ? ldx(x, c1.z) : 0.0f;
        x1.w = (j + 3 >= s && j + 3 < e) ? ldx(x, c1.w) : 0.0f;
    }
    const float4 p0 = make_float4(a0.x * x0.x, a0.y * x0.y, a0.z * x0.z, a0.w * x0.w);
    const float4 p1 = make_float4(a1.x * x1.x, a1.y * x1.y, a1.z * x1.z, a1.w * x1.w);
    if (code < 0) {
        // one chunk of a long row
        float t = (p0.x + p0.y) + (p0.z + p0.w) + ((p1.x + p1.y) + (p1.z + p1.w));
        t = block_sum(t, sm.red);
        const int4 lr = __ldg(P.long_rows + (-code - 1));
        if (GRAD) {
            const float yb = __ldg(P.ybar + lr.x);
            if (v0 < nvec) put_grad4(P.abar, s4 + 4 * v0, s, e, make_float4(yb * x0.x, yb * x0.y, yb * x0.z, yb * x0.w));
            if (v1 < nvec) put_grad4(P.abar, s4 + 4 * v1, s, e, make_float4(yb * x1.x, yb * x1.y, yb * x1.z, yb * x1.w));
        }
        if (tid == 0) {
            P.partial[lr.y + r0] = t;
            __threadfence();
            const int seen = atomicAdd(P.arrivals + (-code - 1), 1);
            sm.last = (seen == lr.z - 1);
        }
        __syncthreads();
        if (sm.last && tid == 0) {
            __threadfence();
            float tot = 0.0f;
            for (int k = 0; k < lr.z; k++) tot += __ldcg(P.partial + lr.y + k);
            y[lr.x] += tot;
            P.arrivals[-code - 1] = 0;
        }
        return;
    }
    if (v0 < nvec) sm.prod[v0] = p0;
    if (v1 < nvec) sm.prod[v1] = p1;
    __syncthreads();
    if (nrows * 32 <= kBatchThreads) batch_rows<32, GRAD>(sm, r0, nrows, y);
    else if (nrows * 16 <= kBatchThreads) batch_rows<16, GRAD>(sm, r0, nrows, y);
    else if (nrows * 8 <= kBatchThreads) batch_rows<8, GRAD>(sm, r0, nrows, y);
    else if (nrows * 4 <= kBatchThreads) batch_rows<4, GRAD>(sm, r0, nrows, y);
    else if (nrows * 2 <= kBatchThreads) batch_rows<2, GRAD>(sm, r0, nrows, y);
    else batch_rows<1, GRAD>(sm, r0, nrows, y);
    if (GRAD) {
        __syncthreads();
        const float* __restrict__ yb = P.ybar + r0;
        if (v0 < nvec) {
            const int j = 4 * v0;
            float4 g;
            g.x = (s4 + j + 0 >= s && s4 + j + 0 < e) ? __ldg(yb + sm.rowid[j + 0]) * x0.x : 0.0f;
            g.y = (s4 + j + 1 >= s && s4 + j + 1 < e) ? __ldg(yb + sm.rowid[j + 1]) * x0.y : 0.0f;
            g.z = (s4 + j + 2 >= s && s4 + j + 2 < e) ? __ldg(yb + sm.rowid[j + 2]) * x0.z : 0.0f;
            g.w = (s4 + j + 3 >= s && s4 + j + 3 < e) ? __ldg(yb + sm.rowid[j + 3]) * x0.w : 0.0f;
            put_grad4(P.abar, s4 + j, s, e, g);
        }
        if (v1 < nvec) {
            const int j = 4 * v1;
            float4 g;
            g.x = (s4 + j + 0 >= s && s4 + j + 0 < e) ? __ldg(yb + sm.rowid[j + 0]) * x1.x : 0.0f;
            g.y = (s4 + j + 1 >= s && s4 + j + 1 < e) ? __ldg(yb + sm.rowid[j + 1]) * x1.y : 0.0f;
            g.z = (s4 + j + 2 >= s && s4 + j + 2 < e) ? __ldg(yb + sm.rowid[j + 2]) * x1.z : 0.0f;
            g.w = (s4 + j + 3 >= s && s4 + j + 3 < e) ? __ldg(yb + sm.rowid[j + 3]) * x1.w : 0.0f;
            put_grad4(P.abar, s4 + j, s, e, g);
        }
    }
}

// SELL rows [vb * 256, vb * 256 + 256): one thread per row.
template <class V, bool GRAD>
__device__ __forceinline__ void batch_sell(const BatchPart& P, int vb)
{
    const int r = vb * kBatchThreads + threadIdx.x;
    if (r >= P.m) return;
    const int H = P.stride;
    const int sl = r / H, lr = r - sl * H;
    const int b = __ldg(P.i0 + sl);
    const int width = (__ldg(P.i0 + sl + 1) - b) / H;
    const int* __restrict__ col = P.i1 + b + lr;
    const V* __restrict__ val = static_cast<const V*>(P.v) + b + lr;
    const float* __restrict__ x = P.x;
    const float yo = P.y[r];   // requested with the first slots, not after the last
    float acc = 0.0f;
    const float yb = GRAD ? __ldg(P.ybar + r) : 0.0f;
    float* __restrict__ g = GRAD ? P.abar + b + lr : nullptr;
#pragma unroll 4
    for (int k = 0; k < width; k++) {
        const int c = __ldg(col + (size_t)k * H);
        const float a = Val<V>::ld(val + (size_t)k * H);
        const float xv = c >= 0 ? ldx(x, c) : 0.0f;
        acc += a * xv;
        if (GRAD) g[(size_t)k * H] = yb * xv;
    }
    P.y[r] = yo + acc;
}

// DIA rows [vb * 512, vb * 512 + 512): kBatchDiaRows rows per thread, 256 apart.
template <class V, bool GRAD>
__device__ __forceinline__ void batch_dia(BatchSmem& sm, const BatchPart& P, int vb)
{
    const int nd = P.k;
    for (int d = threadIdx.x; d < nd; d += kBatchThreads) sm.off[d] = __ldg(P.i0 + d);
    __syncthreads();
    const V* __restrict__ val = static_cast<const V*>(P.v);
    const float* __restrict__ x = P.x;
    const int m = P.m, n = P.n;
    const size_t stride = (size_t)P.stride;
#pragma unroll
    for (int i = 0; i < kBatchDiaRows; i++) {
        const int r = (vb * kBatchDiaRows + i) * kBatchThreads + threadIdx.x;
        if (r >= m) break;
        const float yo = P.y[r];   // requested with the first diagonals, not after the last
        const float yb = GRAD ? __ldg(P.ybar + r) : 0.0f;
        float acc = 0.0f;
#pragma unroll 4
        for (int d = 0; d < nd; d++) {
            const int c = r + sm.off[d];
            const bool in = c >= 0 && c < n;
            const float xv = in ? ldx(x, c) : 0.0f;
            acc += Val<V>::ld(val + (size_t)d * stride + r) * xv;
            if (GRAD) P.abar[(size_t)d * stride + r] = yb * xv;
        }
        P.y[r] = yo + acc;
    }
}

// BCSR block rows [vb * 64, vb * 64 + 64): kBatchBcsrLanes lanes per block row.
template <class V, int B, bool GRAD>
__device__ __forceinline__ void batch_bcsr(const BatchPart& P, int vb)
{
    constexpr int G = kBatchBcsrLanes;
    const int br = vb * (kBatchThreads / G) + threadIdx.x / G, lane = threadIdx.x % G;
    const bool valid = br < P.nbr;
    const int s = valid ? __ldg(P.i0 + br) : 0, e = valid ? __ldg(P.i0 + br + 1) : 0;
    const V* __restrict__ data = static_cast<const V*>(P.v);
    const float* __restrict__ x = P.x;
    const size_t al = (size_t)P.stride;
    const int m = P.m, n = P.n;
    float yb[B];
    if (GRAD) {
#pragma unroll
        for (int h = 0; h < B; h++) yb[h] = (valid && br * B + h < m) ? __ldg(P.ybar + br * B + h) : 0.0f;
    }
    // the block row's y, requested with its first blocks, not after the last
    float yo[B];
#pragma unroll
    for (int h = 0; h < B; h++) yo[h] = (valid && lane == 0 && br * B + h < m) ? P.y[br * B + h] : 0.0f;
    float acc[B];
#pragma unroll
    for (int h = 0; h < B; h++) acc[h] = 0.0f;
    for (int j = s + lane; j < e; j += G) {
        const int c0 = __ldg(P.i1 + j);
        float a[B * B];
#pragma unroll
        for (int q = 0; q < B * B; q++) a[q] = Val<V>::ld(data + (size_t)q * al + j);
        float xv[B];
#pragma unroll
        for (int w = 0; w < B; w++) xv[w] = (c0 + w < n) ? ldx(x, c0 + w) : 0.0f;
#pragma unroll
        for (int h = 0; h < B; h++)
#pragma unroll
            for (int w = 0; w < B; w++) acc[h] += a[h * B + w] * xv[w];
        if (GRAD) {
#pragma unroll
            for (int h = 0; h < B; h++)
#pragma unroll
                for (int w = 0; w < B; w++) P.abar[(size_t)(h * B + w) * al + j] = yb[h] * xv[w];
        }
    }
#pragma unroll
    for (int h = 0; h < B; h++) {
        const float t = group_sum<G>(acc[h]);
        const int r = br * B + h;
        if (valid && lane == 0 && r < m) P.y[r] = yo[h] + t;
    }
}

template <class V, bool GRAD>
__device__ __forceinline__ void batch_item(BatchSmem& sm, const BatchPart& P, const BatchItem& it)
{
    switch (P.kind) {
    case BK_CSR: batch_csr<V, GRAD>(sm, P, it.blk); break;
    case BK_SELL:
        for (int vb = it.v0; vb < it.v1; vb++) batch_sell<V, GRAD>(P, vb);
        break;
    case BK_DIA:
        for (int vb = it.v0; vb < it.v1; vb++) {
            batch_dia<V, GRAD>(sm, P, vb);
            __syncthreads();
        }
        break;
    case BK_BCSR2:
        for (int vb = it.v0; vb < it.v1; vb++) batch_bcsr<V, 2, GRAD>(P, vb);
        break;
    case BK_BCSR3:
        for (int vb = it.v0; vb < it.v1; vb++) batch_bcsr<V, 3, GRAD>(P, vb);
        break;
    case BK_BCSR4:
        for (int vb = it.v0; vb < it.v1; vb++) batch_bcsr<V, 4, GRAD>(P, vb);
        break;
    }
}

// `cycles`, when non-null, receives per part the SM clock cycles its items held a
// CTA (the autotuner's cost).
template <class V>
__global__ void __launch_bounds__(kBatchThreads, 4) batch_kernel(const BatchPart* __restrict__ parts,
                                                                  const BatchItem* __restrict__ items, int nitems,
                                                                  unsigned long long* __restrict__ cycles)
{
    __shared__ __align__(16) BatchSmem sm;
    const int tid = threadIdx.x;
    const int G = gridDim.x;
    const int* __restrict__ iw = reinterpret_cast<const int*>(items);
    const int* __restrict__ pw = reinterpret_cast<const int*>(parts);
    int it = blockIdx.x;
    if (it >= nitems) return;
    // prologue: item `it` and its descriptor into buffer 0
    if (tid < kBatchItemWords) reinterpret_cast<int*>(&sm.item[0])[tid] = __ldg(iw + (size_t)it * kBatchItemWords + tid);
    if (tid < kBatchPartWords) {
        const int px = __ldg(iw + (size_t)it * kBatchItemWords);
        reinterpret_cast<int*>(&sm.part[0])[tid] = __ldg(pw + (size_t)px * kBatchPartWords + tid);
    }
    // registers: item words of the next item
    int nw = 0, npx = 0;
    if (it + G < nitems) {
        if (tid < kBatchItemWords) nw = __ldg(iw + (size_t)(it + G) * kBatchItemWords + tid);
        if (tid < kBatchPartWords) npx = __ldg(iw + (size_t)(it + G) * kBatchItemWords);
    }
    __syncthreads();
    int b = 0;
    while (true) {
        const int n1 = it + G, n2 = it + 2 * G;
        // one ahead: the next item's descriptor; two ahead: the item after it
        int pword = 0, nw2 = 0, npx2 = 0;
        if (n1 < nitems && tid < kBatchPartWords) pword = __ldg(pw + (size_t)npx * kBatchPartWords + tid);
        if (n2 < nitems) {
            if (tid < kBatchItemWords) nw2 = __ldg(iw + (size_t)n2 * kBatchItemWords + tid);
            if (tid < kBatchPartWords) npx2 = __ldg(iw + (size_t)n2 * kBatchItemWords);
        }
        long long t0 = 0;
        if (cycles && tid == 0) t0 = clock64();
        const BatchPart& P = sm.part[b];
        if (P.grad) batch_item<V, true>(sm, P, sm.item[b]);
        else batch_item<V, false>(sm, P, sm.item[b]);
        if (cycles && tid == 0) atomicAdd(cycles + sm.item[b].part, (unsigned long long)(clock64() - t0));
        if (n1 >= nitems) break;
        if (tid < kBatchItemWords) reinterpret_cast<int*>(&sm.item[b ^ 1])[tid] = nw;
        if (tid < kBatchPartWords) reinterpret_cast<int*>(&sm.part[b ^ 1])[tid] = pword;
        __syncthreads();
        nw = nw2;
        npx = npx2;
        it = n1;
        b ^= 1;
    }
}

// Value gradient of a plain CSR matrix, one warp per row: abar[j] = ybar[row] * x[col[j]].
__global__ void __launch_bounds__(256) csr_grad_kernel(const int* __restrict__ rp, const int* __restrict__ col,
                                                       const float* __restrict__ ybar, const float* __restrict__ x,
                                                       float* __restrict__ abar, int m)
{
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int row = (int)(gid >> 5), lane = (int)(gid & 31);
    if (row >= m) return;
    const float yb = __ldg(ybar + row);
    const int e = __ldg(rp + row + 1);
    for (int j = __ldg(rp + row) + lane; j < e; j += 32) abar[j] = yb * ldx(x, __ldg(col + j));
}

}  // namespace dev
}  // namespace csp
