// Batched execution: one persistent kernel serves a work list of (part, row-slice)
// items drawn from many matrices of uneven size.  A part is one matrix (or its
// transpose, for the adjoint) stored in one of the batch formats:
//
//   BK_CSR    CSR cut into work blocks of whole rows (<= kWarpNnz entries and
//             kWarpRows rows) or chunks of one long row, one block per item;
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
// The unit of work is a WARP: warps take the next item from a shared counter, so the
// items in flight at any time are neighbours in the list (mostly of one matrix, whose
// x stays in L2), and formats whose items cost different times per byte still balance.
// No body synchronises more than its own warp, so a warp whose gathers are slow holds
// up no other warp.  Each warp keeps its item and part descriptor in its own slice of
// shared memory, double-buffered: two items ahead it loads the item words, one item
// ahead the part descriptor, both while the current item runs.  Every output element has exactly one writer per launch and every
// sum is taken in a fixed order, so results are deterministic.
#pragma once

#include "common.cuh"
#include "flat.cuh"

namespace csp {
namespace dev {

enum BatchKind : int { BK_CSR = 0, BK_SELL = 1, BK_DIA = 2, BK_BCSR2 = 3, BK_BCSR3 = 4, BK_BCSR4 = 5 };

constexpr int kBatchThreads = 256;
constexpr int kBatchWarps = kBatchThreads / 32;
constexpr int kBatchMaxDiag = 64;
constexpr int kWarpVecs = 2;                     // CSR: aligned 4-vectors of entries per lane
constexpr int kWarpNnz = 32 * 4 * kWarpVecs - 4; // CSR item entries (room for the 4-alignment of its start)
constexpr int kWarpRows = 64;                    // CSR item rows
constexpr int kBatchDiaRows = 4 * 32;            // DIA step: four consecutive rows per lane
constexpr int kBatchSellRows = 32;               // SELL step: a row per lane
constexpr int kBatchBcsrLanes = 2;               // BCSR: lanes per block row
constexpr int kBatchBcsrRows = 32 / kBatchBcsrLanes;   // BCSR step: block rows per warp
constexpr int kBatchReserve = 4;                 // items a warp takes from the counter at once

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
static_assert(kBatchPartWords <= 32, "a descriptor is loaded by one warp, a word per lane");

struct BatchItem {
    int part, v0, v1, pad;
    int4 blk;   // CSR items: the work block {first row, rows or -(long row + 1), first entry, end entry}
};
constexpr int kBatchItemWords = (int)(sizeof(BatchItem) / 4);

// One warp's shared memory.
struct WarpSmem {
    BatchPart part[2];                     // descriptors of the current and the next item
    BatchItem item[3];                     // words of the current item and the next two
    int res_next, res_end;                 // items reserved from the counter (lane 0)
    float4 prod[32 * kWarpVecs];           // CSR: the item's products, at entry - 4-aligned start
    int rp[kWarpRows + 1];                 // CSR: the item's row pointers, relative to that start
    float ys[kWarpRows];                   // CSR: the item's y rows
    unsigned char rowid[32 * 4 * kWarpVecs];   // CSR: row of each entry (value gradients)
};
struct BatchSmem {
    WarpSmem w[kBatchWarps];
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

__device__ __forceinline__ float warp_sum(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// The item's row sums: lane groups of G lanes, one group per row, over the products
// staged in ws.prod; y[r0 + lr] = ys[lr] + sum (in a fixed order per row).
template <int G, bool GRAD>
__device__ __forceinline__ void warp_rows(WarpSmem& ws, int r0, int nrows, float* __restrict__ y, int lane)
{
    const float* prod = reinterpret_cast<const float*>(ws.prod);
    const int sub = lane % G;
    constexpr int ngroups = 32 / G;
    for (int first = 0; first < nrows; first += ngroups) {
        const int lr = first + lane / G;
        const bool valid = lr < nrows;
        const int a = valid ? ws.rp[lr] : 0, b = valid ? ws.rp[lr + 1] : 0;
        float acc = 0.0f;
        for (int j = a + sub; j < b; j += G) {
            acc += prod[j];
            if (GRAD) ws.rowid[j] = (unsigned char)lr;
        }
        acc = group_sum<G>(acc);
        if (valid && sub == 0) y[r0 + lr] = ws.ys[lr] + acc;
    }
}

// CSR work block: rows [r0, r0 + nrows) whose entries [s, e) fit the warp (or one chunk
// of a long row).  Lane l holds the aligned 4-vectors l, l + 32, ... of the entries
// from s & ~3: every load is a coalesced 512-byte segment per warp, and all 16 x
// gathers of a lane are in flight together.
template <class V, bool GRAD>
__device__ __forceinline__ void batch_csr(WarpSmem& ws, const BatchPart& P, int4 blk, int lane)
{
    const int* __restrict__ col = P.i1;
    const V* __restrict__ val = static_cast<const V*>(P.v);
    const float* __restrict__ x = P.x;
    float* __restrict__ y = P.y;
    const int r0 = blk.x, code = blk.y, s = blk.z, e = blk.w;
    const int s4 = s & ~3;
    const int nvec = (e - s4 + 3) >> 2;
    int4 c[kWarpVecs];
    float4 a[kWarpVecs];
#pragma unroll
    for (int k = 0; k < kWarpVecs; k++) {
        const int v = lane + 32 * k;
        c[k] = make_int4(0, 0, 0, 0);
        a[k] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (v < nvec) {
            c[k] = ld_int4(col + s4 + 4 * v);
            a[k] = Val<V>::ld4(val + s4 + 4 * v);
        }
    }
    const int nrows = code > 0 ? code : 1;
    if (code > 0) {
        // the item's row pointers and y rows, requested with the entries
        for (int i = lane; i <= nrows; i += 32) ws.rp[i] = (i < nrows ? __ldg(P.i0 + r0 + i) : e) - s4;
        for (int i = lane; i < nrows; i += 32) ws.ys[i] = y[r0 + i];
    }
    float4 xv[kWarpVecs];
#pragma unroll
    for (int k = 0; k < kWarpVecs; k++) {
        const int j = s4 + 4 * (lane + 32 * k);
        xv[k].x = (j + 0 >= s && j + 0 < e) ? ldx(x, c[k].x) : 0.0f;
        xv[k].y = (j + 1 >= s && j + 1 < e) ? ldx(x, c[k].y) : 0.0f;
        xv[k].z = (j + 2 >= s && j + 2 < e) ? ldx(x, c[k].z) : 0.0f;
        xv[k].w = (j + 3 >= s && j + 3 < e) ? ldx(x, c[k].w) : 0.0f;
    }
    float4 p[kWarpVecs];
#pragma unroll
    for (int k = 0; k < kWarpVecs; k++)
        p[k] = make_float4(a[k].x * xv[k].x, a[k].y * xv[k].y, a[k].z * xv[k].z, a[k].w * xv[k].w);
    if (code < 0) {
        // one chunk of a long row: the chunk's sum, and the last chunk to arrive adds
        // all of them to y in chunk order
        float t = 0.0f;
#pragma unroll
        for (int k = 0; k < kWarpVecs; k++) t += (p[k].x + p[k].y) + (p[k].z + p[k].w);
        t = warp_sum(t);
        const int4 lr = __ldg(P.long_rows + (-code - 1));
        if (GRAD) {
            const float yb = __ldg(P.ybar + lr.x);
#pragma unroll
            for (int k = 0; k < kWarpVecs; k++)
                if (lane + 32 * k < nvec)
                    put_grad4(P.abar, s4 + 4 * (lane + 32 * k), s, e,
                              make_float4(yb * xv[k].x, yb * xv[k].y, yb * xv[k].z, yb * xv[k].w));
        }
        int last = 0;
        if (lane == 0) {
            P.partial[lr.y + r0] = t;
            __threadfence();
            const int seen = atomicAdd(P.arrivals + (-code - 1), 1);
            last = (seen == lr.z - 1);
            if (last) {
                __threadfence();
                float tot = 0.0f;
                for (int k = 0; k < lr.z; k++) tot += __ldcg(P.partial + lr.y + k);
                y[lr.x] += tot;
                P.arrivals[-code - 1] = 0;
            }
        }
        return;
    }
#pragma unroll
    for (int k = 0; k < kWarpVecs; k++)
        if (lane + 32 * k < nvec) ws.prod[lane + 32 * k] = p[k];
    __syncwarp();
    if (nrows <= 1) warp_rows<32, GRAD>(ws, r0, nrows, y, lane);
    else if (nrows <= 2) warp_rows<16, GRAD>(ws, r0, nrows, y, lane);
    else if (nrows <= 4) warp_rows<8, GRAD>(ws, r0, nrows, y, lane);
    else if (nrows <= 8) warp_rows<4, GRAD>(ws, r0, nrows, y, lane);
    else if (nrows <= 16) warp_rows<2, GRAD>(ws, r0, nrows, y, lane);
    else warp_rows<1, GRAD>(ws, r0, nrows, y, lane);
    if (GRAD) {
        __syncwarp();
        const float* __restrict__ yb = P.ybar + r0;
#pragma unroll
        for (int k = 0; k < kWarpVecs; k++) {
            const int v = lane + 32 * k;
            if (v >= nvec) continue;
            const int j = 4 * v, g0 = s4 + j;
            float4 g;
            g.x = (g0 + 0 >= s && g0 + 0 < e) ? __ldg(yb + ws.rowid[j + 0]) * xv[k].x : 0.0f;
            g.y = (g0 + 1 >= s && g0 + 1 < e) ? __ldg(yb + ws.rowid[j + 1]) * xv[k].y : 0.0f;
            g.z = (g0 + 2 >= s && g0 + 2 < e) ? __ldg(yb + ws.rowid[j + 2]) * xv[k].z : 0.0f;
            g.w = (g0 + 3 >= s && g0 + 3 < e) ? __ldg(yb + ws.rowid[j + 3]) * xv[k].w : 0.0f;
            put_grad4(P.abar, g0, s, e, g);
        }
    }
}

// SELL rows [vb * 32, vb * 32 + 32): one lane per row.
template <class V, bool GRAD>
__device__ __forceinline__ void batch_sell(const BatchPart& P, int vb, int lane)
{
    const int r = vb * kBatchSellRows + lane;
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

// DIA rows [vb * 128, vb * 128 + 128): four consecutive rows per lane, so every
// diagonal is one 128-bit load of values (and, with the gradient, one 128-bit streaming
// store) per lane; the x and y entries of the four rows are consecutive 4-byte
// accesses across the warp (the batch's vectors are not 16-byte aligned per matrix).
// The slot stride is a multiple of 32 and zero-filled past the last row, so the
// vector accesses stay inside the part; padding rows get value-gradient 0.  The
// offsets are read through the read-only path (one address per warp).
template <class V, bool GRAD>
__device__ __forceinline__ void batch_dia(const BatchPart& P, int vb, int lane)
{
    const V* __restrict__ val = static_cast<const V*>(P.v);
    const float* __restrict__ x = P.x;
    const int* __restrict__ off = P.i0;
    const int m = P.m, n = P.n, nd = P.k;
    const size_t stride = (size_t)P.stride;
    const int r0 = vb * kBatchDiaRows + 4 * lane;
    if (r0 >= m) return;
    // y (and ybar) of the four rows, requested with the first diagonals
    float yo[4], yb[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        yo[q] = r0 + q < m ? P.y[r0 + q] : 0.0f;
        yb[q] = (GRAD && r0 + q < m) ? __ldg(P.ybar + r0 + q) : 0.0f;
    }
    float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll 2
    for (int d = 0; d < nd; d++) {
        const int c = r0 + __ldg(off + d);
        const float4 a = Val<V>::ld4(val + (size_t)d * stride + r0);
        float xv[4];
#pragma unroll
        for (int q = 0; q < 4; q++) xv[q] = (c + q >= 0 && c + q < n) ? ldx(x, c + q) : 0.0f;
        acc[0] += a.x * xv[0];
        acc[1] += a.y * xv[1];
        acc[2] += a.z * xv[2];
        acc[3] += a.w * xv[3];
        if (GRAD)
            __stcs(reinterpret_cast<float4*>(P.abar + (size_t)d * stride + r0),
                   make_float4(yb[0] * xv[0], yb[1] * xv[1], yb[2] * xv[2], yb[3] * xv[3]));
    }
#pragma unroll
    for (int q = 0; q < 4; q++)
        if (r0 + q < m) P.y[r0 + q] = yo[q] + acc[q];
}

// BCSR block rows [vb * 16, vb * 16 + 16): kBatchBcsrLanes (2) lanes per block row,
// each lane taking two of its row's blocks per round, whose column ids, values and x
// gathers are all requested before any is used (the batch's block rows hold a few
// blocks each: one or two rounds).
template <class V, int B, bool GRAD>
__device__ __forceinline__ void batch_bcsr(const BatchPart& P, int vb, int lane32)
{
    constexpr int G = kBatchBcsrLanes;
    constexpr int U = B <= 3 ? 2 : 1;   // two 4x4 blocks in registers would spill
    const int br = vb * kBatchBcsrRows + lane32 / G, lane = lane32 % G;
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
    for (int j0 = s + lane; j0 < e; j0 += G * U) {
        int c0[U];
        float a[U][B * B];
        float xv[U][B];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int j = j0 + u * G;
            const bool in = j < e;
            c0[u] = in ? __ldg(P.i1 + j) : 0;
#pragma unroll
            for (int q = 0; q < B * B; q++) a[u][q] = in ? Val<V>::ld(data + (size_t)q * al + j) : 0.0f;
        }
#pragma unroll
        for (int u = 0; u < U; u++)
#pragma unroll
            for (int w = 0; w < B; w++) xv[u][w] = (j0 + u * G < e && c0[u] + w < n) ? ldx(x, c0[u] + w) : 0.0f;
#pragma unroll
        for (int u = 0; u < U; u++) {
#pragma unroll
            for (int h = 0; h < B; h++)
#pragma unroll
                for (int w = 0; w < B; w++) acc[h] += a[u][h * B + w] * xv[u][w];
            if (GRAD && j0 + u * G < e) {
#pragma unroll
                for (int h = 0; h < B; h++)
#pragma unroll
                    for (int w = 0; w < B; w++) P.abar[(size_t)(h * B + w) * al + j0 + u * G] = yb[h] * xv[u][w];
            }
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
__device__ __forceinline__ void batch_item(WarpSmem& ws, const BatchPart& P, const BatchItem& it, int lane)
{
    switch (P.kind) {
    case BK_CSR: batch_csr<V, GRAD>(ws, P, it.blk, lane); break;
    case BK_SELL:
        for (int vb = it.v0; vb < it.v1; vb++) batch_sell<V, GRAD>(P, vb, lane);
        break;
    case BK_DIA:
        for (int vb = it.v0; vb < it.v1; vb++) batch_dia<V, GRAD>(P, vb, lane);
        break;
    case BK_BCSR2:
        for (int vb = it.v0; vb < it.v1; vb++) batch_bcsr<V, 2, GRAD>(P, vb, lane);
        break;
    case BK_BCSR3:
        for (int vb = it.v0; vb < it.v1; vb++) batch_bcsr<V, 3, GRAD>(P, vb, lane);
        break;
    case BK_BCSR4:
        for (int vb = it.v0; vb < it.v1; vb++) batch_bcsr<V, 4, GRAD>(P, vb, lane);
        break;
    }
}

__device__ __forceinline__ void cp_async4(void* dst, const void* src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src));
}
__device__ __forceinline__ void cp_async_commit_wait_all() { asm volatile("cp.async.commit_group;\ncp.async.wait_all;\n" ::); }
__device__ __forceinline__ void cp_async_commit_group() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::); }

// The warps take items from a shared counter (`next`, zero at launch), kBatchReserve
// consecutive items per atomic: a warp reserves the item after its next one while it
// runs the current item, so the items a warp gets follow how long its earlier ones
// took, and a warp holds at most kBatchReserve + 1 items it has not started.  The next
// item's descriptor and the words of the item after it are copied into the warp's
// shared memory asynchronously (cp.async) while the current item runs, so no register
// holds them across the item.  Which warp runs an item does not change any result.
// `cycles`, when non-null, receives per part the SM clock cycles its items held a warp
// (the autotuner's cost).
template <class V>
__global__ void __launch_bounds__(kBatchThreads, 4) batch_kernel(const BatchPart* __restrict__ parts,
                                                                  const BatchItem* __restrict__ items, int nitems,
                                                                  int* __restrict__ next,
                                                                  unsigned long long* __restrict__ cycles)
{
    __shared__ __align__(16) BatchSmem sm;
    const int lane = threadIdx.x & 31;
    WarpSmem& ws = sm.w[threadIdx.x >> 5];
    const int* __restrict__ iw = reinterpret_cast<const int*>(items);
    const int* __restrict__ pw = reinterpret_cast<const int*>(parts);
    auto reserve = [&]() {
        int v = 0;
        if (lane == 0) {
            if (ws.res_next == ws.res_end) {
                ws.res_next = atomicAdd(next, kBatchReserve);
                ws.res_end = ws.res_next + kBatchReserve;
            }
            v = ws.res_next++;
        }
        return __shfl_sync(0xffffffffu, v, 0);
    };
    if (lane == 0) ws.res_next = ws.res_end = 0;
    __syncwarp();
    int it = reserve();
    if (it >= nitems) return;   // the whole warp leaves together
    // prologue: item `it` and its descriptor into slots 0, the next item's words in flight
    if (lane < kBatchItemWords) reinterpret_cast<int*>(&ws.item[0])[lane] = __ldg(iw + (size_t)it * kBatchItemWords + lane);
    if (lane < kBatchPartWords) {
        const int px = __ldg(iw + (size_t)it * kBatchItemWords);
        reinterpret_cast<int*>(&ws.part[0])[lane] = __ldg(pw + (size_t)px * kBatchPartWords + lane);
    }
    int n1 = reserve();
    if (n1 < nitems && lane < kBatchItemWords)
        cp_async4(reinterpret_cast<int*>(&ws.item[1]) + lane, iw + (size_t)n1 * kBatchItemWords + lane);
    cp_async_commit_wait_all();
    __syncwarp();
    int ib = 0, pb = 0;
    while (true) {
        // the next item's words have landed: its descriptor, and the words of the one after
        const int ib1 = ib == 2 ? 0 : ib + 1, ib2 = ib1 == 2 ? 0 : ib1 + 1;
        const int n2 = n1 < nitems ? reserve() : nitems;
        if (n1 < nitems && lane < kBatchPartWords)
            cp_async4(reinterpret_cast<int*>(&ws.part[pb ^ 1]) + lane, pw + (size_t)ws.item[ib1].part * kBatchPartWords + lane);
        if (n2 < nitems && lane < kBatchItemWords)
            cp_async4(reinterpret_cast<int*>(&ws.item[ib2]) + lane, iw + (size_t)n2 * kBatchItemWords + lane);
        cp_async_commit_group();
        long long t0 = 0;
        if (cycles && lane == 0) t0 = clock64();
        const BatchPart& P = ws.part[pb];
        if (P.grad) batch_item<V, true>(ws, P, ws.item[ib], lane);
        else batch_item<V, false>(ws, P, ws.item[ib], lane);
        if (cycles && lane == 0) atomicAdd(cycles + ws.item[ib].part, (unsigned long long)(clock64() - t0));
        if (n1 >= nitems) break;
        cp_async_wait_all();
        __syncwarp();
        n1 = n2;
        ib = ib1;
        pb ^= 1;
    }
    cp_async_wait_all();   // no copy is left in flight when the warp leaves
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
