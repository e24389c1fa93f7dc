// x staged in shared memory by column panels: the layout for sparse parts whose
// column accesses have no locality (random graphs, Zipf rows), where the x gathers of
// the reference-style COO/CSR kernels (clSpMV_NV/kernels/spmv_coo.cl,
// spmv_csr_vector.cl) are limited by L2 request throughput, not by HBM.
//
// Layout (built once by the host):
//   * columns are cut into panels of `panel_w` columns (panel_w * 4 bytes of shared
//     memory); the part's nonzeros are regrouped by panel, keeping row order inside
//     each panel, and every panel is padded to whole tiles of kXpTile entries;
//   * inside one tile, a "run" is a maximal group of consecutive entries of one row.
//     A row with one run in all adds that run to y[row] directly (its entries carry
//     the code -(row + 1)): it is the row's only writer in the launch.  Every run of
//     the other rows owns one slot of a partial-sum array; slots are numbered row by
//     row and, inside a row, in panel order.  Pad entries extend the panel's last run
//     (value 0, column 0);
//   * per entry: the slot id of its run, or the direct-row code (int32), the column
//     inside its panel (uint16) and the value (FP32 or BF16);
//   * run_ptr[i]..run_ptr[i+1] are the slots of the i-th listed row: every row with
//     two or more runs, in order (run_rows[i] is that row, or i itself when every row
//     is listed).  long_list holds the listed rows with more than kXpShortRuns slots.
//
// xpanel_kernel: each CTA takes an equal share of the tiles (tiles are ordered panel
// by panel); for each panel its share touches it copies that panel of x into shared
// memory with cp.async, then every warp streams whole tiles through a per-warp ring
// of kXpStages tiles (cp.async, so several tiles per warp are in flight): four entries
// per lane, products from shared-memory x, a keyed shuffle scan over the lanes joins
// runs that cross lanes, and the lane holding the last entry of a run stores the run's
// sum to its slot.  Runs never cross tiles: no carry and no atomic.
// xpanel_merge_kernel: y[row] += the row's slots in order; a thread per listed row
// (in order) with at most kXpShortRuns slots, a lane group per longer row.  Both
// kernels are deterministic.
#pragma once

#include "common.cuh"

namespace csp {
namespace dev {

constexpr int kXpThreads = 512;
constexpr int kXpWarps = kXpThreads / 32;
constexpr int kXpTile = 128;                // entries per tile: 4 per lane
constexpr int kXpPanelMax = 65536;          // panel-local columns are 16-bit
constexpr int kXpStages = 4;                // tiles in flight per warp
constexpr int kXpShortRuns = 8;             // rows with at most this many slots: a thread each
constexpr int kXpMergeLanes = 8;            // lanes per longer row in the merge

// One tile as staged in shared memory.  Lane l copies and later reads back only its
// own four entries, so no barrier orders the ring: cp.async.wait_group suffices.
template <class V>
struct XpStage {
    int slot[kXpTile];
    V val[kXpTile];
    unsigned short lcol[kXpTile];
};

// Dynamic shared memory of one CTA: the per-warp tile rings, then the x panel.
template <class V>
__host__ __device__ constexpr size_t xpanel_ring_bytes() { return sizeof(XpStage<V>) * kXpWarps * kXpStages; }

__device__ __forceinline__ void cp_async16(void* dst, const void* src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src));
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

template <class V>
__device__ __forceinline__ void xpanel_issue(XpStage<V>& st, int tile, int seg_end, int lane, const int* __restrict__ slot,
                                             const unsigned short* __restrict__ lcol, const V* __restrict__ val)
{
    if (tile < seg_end) {
        const size_t b = (size_t)tile * kXpTile + 4 * lane;
        cp_async16(&st.slot[4 * lane], slot + b);
        if (sizeof(V) == 4) cp_async16(&st.val[4 * lane], val + b);
        else cp_async8(&st.val[4 * lane], val + b);
        cp_async8(&st.lcol[4 * lane], lcol + b);
    }
    cp_async_commit();   // possibly empty: keeps the group count uniform
}

template <class V> __device__ __forceinline__ float4 xp_vals(const XpStage<V>& st, int lane);
template <> __device__ __forceinline__ float4 xp_vals<float>(const XpStage<float>& st, int lane)
{
    return *reinterpret_cast<const float4*>(&st.val[4 * lane]);
}
template <> __device__ __forceinline__ float4 xp_vals<__nv_bfloat16>(const XpStage<__nv_bfloat16>& st, int lane)
{
    const uint2 u = *reinterpret_cast<const uint2*>(&st.val[4 * lane]);
    return make_float4(__uint_as_float(u.x << 16), __uint_as_float(u.x & 0xffff0000u), __uint_as_float(u.y << 16),
                       __uint_as_float(u.y & 0xffff0000u));
}

// The sum of a closed run: to its slot, or added to y for a one-run row (code
// -(row + 1)).  The add is a reduction store (no value returned, so the warp does not
// wait on y); the row has no other writer in the launch, so y_row + v is exact and
// deterministic.
__device__ __forceinline__ void xp_close(int key, float v, float* __restrict__ partial, float* __restrict__ y)
{
    if (key >= 0) partial[key] = v;
    else atomicAdd(y + (-key - 1), v);
}

template <class V>
__global__ void __launch_bounds__(kXpThreads, 1) xpanel_kernel(const int* __restrict__ tile0, int ntiles, int npanels,
                                                               const int* __restrict__ slot,
                                                               const unsigned short* __restrict__ lcol,
                                                               const V* __restrict__ val, const float* __restrict__ x,
                                                               int n, int panel_w, float* __restrict__ partial,
                                                               float* __restrict__ y)
{
    extern __shared__ __align__(16) unsigned char xp_smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    XpStage<V>* ring = reinterpret_cast<XpStage<V>*>(xp_smem) + warp * kXpStages;
    float* xs = reinterpret_cast<float*>(xp_smem + xpanel_ring_bytes<V>());
    const int t_begin = (int)((long long)blockIdx.x * ntiles / gridDim.x);
    const int t_end = (int)((long long)(blockIdx.x + 1) * ntiles / gridDim.x);
    if (t_begin >= t_end) return;
    // panel holding t_begin: the last p with tile0[p] <= t_begin
    int lo = 0, hi = npanels - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(tile0 + mid) <= t_begin) lo = mid; else hi = mid - 1;
    }
    int p = lo;
    int t = t_begin;
    while (t < t_end) {
        const int seg_end = min(t_end, __ldg(tile0 + p + 1));
        if (seg_end > t) {
            // --- this panel of x into shared memory (x is zero-padded past n to a multiple of 64) ---
            const int c0 = p * panel_w;
            const int nv4 = (min(panel_w, n - c0) + 3) >> 2;
            const float4* __restrict__ xg = reinterpret_cast<const float4*>(x + c0);
            for (int i = threadIdx.x; i < nv4; i += kXpThreads) cp_async16(reinterpret_cast<float4*>(xs) + i, xg + i);
            cp_async_commit();
            // the first kXpStages - 1 tiles of this warp
            const int first = t + warp;
#pragma unroll
            for (int q = 0; q < kXpStages - 1; q++) xpanel_issue<V>(ring[q], first + q * kXpWarps, seg_end, lane, slot, lcol, val);
            cp_async_wait<kXpStages - 1>();   // the x group (the oldest) has landed
            __syncthreads();
            int stage = 0;
            for (int tt = first; tt < seg_end; tt += kXpWarps) {
                xpanel_issue<V>(ring[(stage + kXpStages - 1) % kXpStages], tt + (kXpStages - 1) * kXpWarps, seg_end, lane,
                                slot, lcol, val);
                cp_async_wait<kXpStages - 1>();   // tile tt has landed
                const XpStage<V>& st = ring[stage];
                stage = (stage + 1) % kXpStages;
                const int4 s = *reinterpret_cast<const int4*>(&st.slot[4 * lane]);
                const uint2 cc = *reinterpret_cast<const uint2*>(&st.lcol[4 * lane]);
                const float4 a = xp_vals<V>(st, lane);
                const float p0 = a.x * xs[cc.x & 0xffffu], p1 = a.y * xs[cc.x >> 16];
                const float p2 = a.z * xs[cc.y & 0xffffu], p3 = a.w * xs[cc.y >> 16];
                // the lane's suffix run (entries of its last slot; slots are sorted)
                float tail = p3;
                if (s.z == s.w) { tail += p2; if (s.y == s.w) { tail += p1; if (s.x == s.w) tail += p0; } }
                // keyed inclusive scan of the suffix runs over lanes; the key comparisons
                // do not depend on the values and are made first
                unsigned same = 0u;
#pragma unroll
                for (int b = 0; b < 5; b++) {
                    const int ok = __shfl_up_sync(0xffffffffu, s.w, 1 << b);
                    if (lane >= (1 << b) && ok == s.w) same |= 1u << b;
                }
                float scan = tail;
#pragma unroll
                for (int b = 0; b < 5; b++) {
                    const float o = __shfl_up_sync(0xffffffffu, scan, 1 << b);
                    if (same & (1u << b)) scan += o;
                }
                const float prev_scan = __shfl_up_sync(0xffffffffu, scan, 1);
                const int next_first = __shfl_down_sync(0xffffffffu, s.x, 1);
                // the previous lane's last key equals this lane's first exactly when bit 0
                // of its own comparison chain would say so for key s.x
                const int prev_key = __shfl_up_sync(0xffffffffu, s.w, 1);
                float run = (lane > 0 && prev_key == s.x) ? prev_scan : 0.0f;
                run += p0;
                if (s.y != s.x) { xp_close(s.x, run, partial, y); run = 0.0f; }
                run += p1;
                if (s.z != s.y) { xp_close(s.y, run, partial, y); run = 0.0f; }
                run += p2;
                if (s.w != s.z) { xp_close(s.z, run, partial, y); run = 0.0f; }
                run += p3;
                if (lane == 31 || next_first != s.w) xp_close(s.w, run, partial, y);
            }
            cp_async_wait<0>();   // only empty groups remain; keeps the accounting clean per panel
            __syncthreads();      // every warp is done with this panel before the next overwrites it
        }
        t = max(t, seg_end);
        p++;
    }
}

// y[row] += sum of the row's slots, in slot order.  Threads [0, nrows): listed row
// gid, if it has at most kXpShortRuns slots (independent, predicated loads).  The
// rest of the grid: a group of kXpMergeLanes lanes per entry of long_list, striding
// over that row's slots and reducing with a fixed shuffle tree.
__global__ void __launch_bounds__(256) xpanel_merge_kernel(const int* __restrict__ run_ptr, const int* __restrict__ run_rows,
                                                           int nrows, const int* __restrict__ long_list, int nlong,
                                                           const float* __restrict__ partial, float* __restrict__ y)
{
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long short_threads = (long long)(nrows + 255) / 256 * 256;
    if (gid < short_threads) {
        if (gid >= nrows) return;
        const int i = (int)gid;
        const int a = __ldg(run_ptr + i), b = __ldg(run_ptr + i + 1);
        if (b - a > kXpShortRuns) return;
        const int r = run_rows ? __ldg(run_rows + i) : i;
        const float yv = y[r];
        float q[kXpShortRuns];
#pragma unroll
        for (int k = 0; k < kXpShortRuns; k++) q[k] = a + k < b ? partial[a + k] : 0.0f;
        float s = q[0];
#pragma unroll
        for (int k = 1; k < kXpShortRuns; k++) s += q[k];
        y[r] = yv + s;
        return;
    }
    const long long g = (gid - short_threads) / kXpMergeLanes;
    const int lane = (int)((gid - short_threads) % kXpMergeLanes);
    const bool valid = g < nlong;
    // groups past the list keep their lanes in the shuffle with an empty range
    const int i = valid ? __ldg(long_list + g) : 0;
    const int a = valid ? __ldg(run_ptr + i) : 0, b = valid ? __ldg(run_ptr + i + 1) : 0;
    float s = 0.0f;
#pragma unroll 4
    for (int j = a + lane; j < b; j += kXpMergeLanes) s += partial[j];
    s = group_sum<kXpMergeLanes>(s);
    if (valid && lane == 0) {
        const int r = run_rows ? __ldg(run_rows + i) : i;
        y[r] += s;
    }
}

}  // namespace dev
}  // namespace csp
