// COO SpMV for callers that cannot allocate device memory.
//
// Some callers of this library must not call the CUDA allocator at all: code that
// runs inside a framework whose caching allocator has already reserved the device's
// memory, real-time solver loops where cudaMalloc/cudaFree (which can synchronize the
// whole device and take milliseconds) are forbidden, and embedders that hand the
// library only the buffers they own.  csp_coo_spmv_noalloc serves them: it computes
// y += A*x for a row-sorted COO matrix whose arrays the caller already holds in device
// memory, and allocates nothing.  The per-warp partial sums that the segmented
// reduction needs live in g_noalloc_scratch, a fixed array in this library's device
// image (CSP_NOALLOC_SCRATCH_BYTES = 1 MiB): every GPU that loads the library holds it
// until the process exits.  It bounds the matrix to CSP_NOALLOC_MAX_NNZ entries.
//
// The kernels restate the COO segmented reduction of kernels/flat.cuh
// (coo_segment_kernel + coo_fixup_kernel) for unpadded caller arrays: the last tile
// is read with masked scalar loads, and every row/column index is range-checked so a
// malformed matrix gives a wrong result instead of an out-of-bounds access.
#include <cuda_runtime.h>
#include <mutex>

#include "csp/clspmv.h"
#include "internal.h"
#include "engine.h"
#include "kernels/common.cuh"

namespace csp {

constexpr int kNoAllocChunk = 512;                                        // entries per warp
constexpr int kNoAllocMaxWarps = CSP_NOALLOC_MAX_NNZ / kNoAllocChunk;     // 65,536
static_assert(CSP_NOALLOC_SCRATCH_BYTES == 2 * kNoAllocMaxWarps * (4 + 4), "scratch holds 2 (row, sum) pairs per warp");

// Scratch of the no-allocation entry point: rows of the 2 * warps (row, partial) pairs,
// then their partial sums.  Shared by every call on a device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[CSP_NOALLOC_SCRATCH_BYTES];

namespace {

__device__ __forceinline__ void load_entry(const int* __restrict__ rowid, const int* __restrict__ colid,
                                           const float* __restrict__ val, int j, int nnz, int last_row,
                                           int& r, int& c, float& v)
{
    if (j < nnz) {
        r = __ldg(rowid + j);
        c = __ldg(colid + j);
        v = __ldg(val + j);
    } else {   // padding past the caller's arrays: extends the last row by zeros
        r = last_row;
        c = 0;
        v = 0.0f;
    }
}

__device__ __forceinline__ float x_at(const float* __restrict__ x, int c, int width)
{
    return (c >= 0 && c < width) ? __ldg(x + c) : 0.0f;
}

__device__ __forceinline__ float y_at(const float* y, int r, int height)
{
    return (r >= 0 && r < height) ? y[r] : 0.0f;
}

__global__ void __launch_bounds__(256) coo_noalloc_segment(const int* __restrict__ rowid, const int* __restrict__ colid,
                                                           const float* __restrict__ val, const float* __restrict__ x,
                                                           float* __restrict__ y, int nnz, int height, int width, int nwarps,
                                                           int* __restrict__ part_row, float* __restrict__ part_val)
{
    const int lane = threadIdx.x & 31;
    const int w = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (w >= nwarps) return;
    const int last_row = __ldg(rowid + nnz - 1);
    const int nnz_tiles = (nnz + 127) / 128 * 128;
    const int base = w * kNoAllocChunk;
    const int end = min(base + kNoAllocChunk, nnz_tiles);
    const int head_row = __ldg(rowid + base);
    bool head_open = true;
    int carry_row = head_row;
    float carry_val = 0.0f;
    for (int t = base; t < end; t += 128) {
        const int j = t + 4 * lane;
        int4 r;
        int4 c;
        float4 a;
        if (t + 128 <= nnz) {
            r = dev::ld_int4(rowid + j);
            c = dev::ld_int4(colid + j);
            a = dev::Val<float>::ld4(val + j);
        } else {
            load_entry(rowid, colid, val, j + 0, nnz, last_row, r.x, c.x, a.x);
            load_entry(rowid, colid, val, j + 1, nnz, last_row, r.y, c.y, a.y);
            load_entry(rowid, colid, val, j + 2, nnz, last_row, r.z, c.z, a.z);
            load_entry(rowid, colid, val, j + 3, nnz, last_row, r.w, c.w, a.w);
        }
        const float y0 = y_at(y, r.x, height), y1 = y_at(y, r.y, height), y2 = y_at(y, r.z, height), y3 = y_at(y, r.w, height);
        const float p0 = a.x * x_at(x, c.x, width), p1 = a.y * x_at(x, c.y, width);
        const float p2 = a.z * x_at(x, c.z, width), p3 = a.w * x_at(x, c.w, width);
        const int tile_first = __shfl_sync(0xffffffffu, r.x, 0);
        if (tile_first != carry_row) {
            if (lane == 0) {
                if (head_open && carry_row == head_row) {
                    part_row[2 * w] = carry_row;
                    part_val[2 * w] = carry_val;
                } else if (carry_row >= 0 && carry_row < height) {
                    y[carry_row] += carry_val;
                }
            }
            if (head_open && carry_row == head_row) head_open = false;
            carry_row = tile_first;
            carry_val = 0.0f;
        }
        float tail = p3;
        if (r.z == r.w) { tail += p2; if (r.y == r.w) { tail += p1; if (r.x == r.w) tail += p0; } }
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
        const int rr[4] = {r.x, r.y, r.z, r.w};
        const float pp[4] = {p0, p1, p2, p3};
        const float yy[4] = {y0, y1, y2, y3};
#pragma unroll
        for (int k = 0; k < 4; k++) {
            run += pp[k];
            const int nxt = (k == 3) ? next_first : rr[k + 1];
            const bool closes = (k < 3) ? (nxt != rr[k]) : (lane < 31 && nxt != rr[k]);
            if (closes) {
                if (head_open && rr[k] == head_row) {
                    part_row[2 * w] = rr[k];
                    part_val[2 * w] = run;
                    closed_head = true;
                } else if (rr[k] >= 0 && rr[k] < height) {
                    y[rr[k]] = yy[k] + run;
                }
                run = 0.0f;
            }
        }
        carry_row = __shfl_sync(0xffffffffu, r.w, 31);
        carry_val = __shfl_sync(0xffffffffu, run, 31);
        if (__any_sync(0xffffffffu, closed_head)) head_open = false;
    }
    if (lane == 0) {
        if (head_open) {
            part_row[2 * w] = carry_row;
            part_val[2 * w] = carry_val;
            part_row[2 * w + 1] = carry_row;
            part_val[2 * w + 1] = 0.0f;
        } else {
            part_row[2 * w + 1] = carry_row;
            part_val[2 * w + 1] = carry_val;
        }
    }
}

__global__ void __launch_bounds__(256) coo_noalloc_fixup(const int* __restrict__ part_row, const float* __restrict__ part_val,
                                                         int nparts, int height, float* __restrict__ y)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nparts) return;
    const int r = part_row[i];
    if (i > 0 && part_row[i - 1] == r) return;
    float acc = 0.0f;
    for (int k = i; k < nparts && part_row[k] == r; k++) acc += part_val[k];
    if (r >= 0 && r < height) y[r] += acc;
}

// Device address of g_noalloc_scratch, looked up once per device with that device
// current and kept for the process (a cudaDeviceReset afterwards is not supported).
constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
void* g_scratch_addr[kMaxDevices];

int scratch_for_current_device(void** out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_error(e, "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) return set_error(CSP_EUNSUP, "device %d beyond the %d the no-allocation path tracks", dev, kMaxDevices);
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_error(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return CSP_OK;
}

}  // namespace
}  // namespace csp

extern "C" int csp_coo_spmv_noalloc(int height, int width, int nnz, const int* d_row, const int* d_col, const float* d_val,
                                    const float* d_x, float* d_y, void* stream)
{
    using namespace csp;
    if (height < 0 || width < 0 || nnz < 0) return set_error(CSP_EINVAL, "coo_spmv_noalloc: negative size");
    if (nnz > CSP_NOALLOC_MAX_NNZ)
        return set_error(CSP_EINVAL, "coo_spmv_noalloc: %d entries exceed the no-allocation limit of %d (use csp_init_mat_kernels)",
                         nnz, CSP_NOALLOC_MAX_NNZ);
    if (nnz == 0) return CSP_OK;
    if (!d_row || !d_col || !d_val || !d_x || !d_y) return set_error(CSP_EINVAL, "coo_spmv_noalloc: null device pointer");
    {
        // x is read while y is written: the arrays must not overlap
        const uintptr_t x0 = (uintptr_t)d_x, x1 = x0 + sizeof(float) * (size_t)width;
        const uintptr_t y0 = (uintptr_t)d_y, y1 = y0 + sizeof(float) * (size_t)height;
        if (x0 < y1 && y0 < x1 && width > 0 && height > 0)
            return set_error(CSP_EINVAL, "coo_spmv_noalloc: x and y overlap");
    }
    if (((uintptr_t)d_row | (uintptr_t)d_col | (uintptr_t)d_val) & 15)
        return set_error(CSP_EINVAL, "coo_spmv_noalloc: row, column and value arrays must be 16-byte aligned");
    void* scratch = nullptr;
    int rc = scratch_for_current_device(&scratch);
    if (rc) return rc;
    int* part_row = static_cast<int*>(scratch);
    float* part_val = reinterpret_cast<float*>(static_cast<char*>(scratch) + CSP_NOALLOC_SCRATCH_BYTES / 2);
    const int nwarps = (nnz + kNoAllocChunk - 1) / kNoAllocChunk;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    coo_noalloc_segment<<<(nwarps * 32 + 255) / 256, 256, 0, st>>>(d_row, d_col, d_val, d_x, d_y, nnz, height, width, nwarps,
                                                                   part_row, part_val);
    coo_noalloc_fixup<<<(2 * nwarps + 255) / 256, 256, 0, st>>>(part_row, part_val, 2 * nwarps, height, d_y);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? CSP_OK : cuda_error(e, "coo_spmv_noalloc launch");
}
