// COO sort by (row, column) on the device: the sort step of MatrixMarket ingestion
// (clSpMV_NV/src/fileio.cpp:10 ReadMMF sorts with sort_coo, matrix_storage.h:745).
//
// A stable least-significant-digit radix sort of 64-bit keys row << cb | col (cb =
// the bits of the largest column), 8-bit digits, only as many passes as the keys have
// significant bits.  One pass:
//   * radix_hist_kernel: each tile of kSortTile keys counts its digits (shared-memory
//     histogram), written digit-major, hist[d * ntiles + tile];
//   * an exclusive scan of the histogram gives every (digit, tile) its first output slot;
//   * radix_scatter_kernel: each tile walks its keys in order, kSortThreads at a time,
//     ranking each key among the equal digits before it (warp __match_any_sync, then
//     per-warp counts in shared memory), and writes key and payload to their slot.
// Stability makes keys that compare equal keep their input order; when no two entries
// share (row, col) the result is the unique (row, col) order, the one the reference's
// quicksort produces.
#include <cuda_runtime.h>
#include <stdint.h>
#include <algorithm>
#include <vector>

#include "csp/clspmv.h"
#include "internal.h"
#include "engine.h"

namespace csp {
namespace {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;
constexpr int kScanThreads = 1024;

__global__ void __launch_bounds__(kSortThreads) radix_hist_kernel(const uint64_t* __restrict__ keys, long long n,
                                                                  int shift, int ntiles, unsigned* __restrict__ hist)
{
    __shared__ unsigned h[256];
    for (int d = threadIdx.x; d < 256; d += kSortThreads) h[d] = 0;
    __syncthreads();
    const long long base = (long long)blockIdx.x * kSortTile;
#pragma unroll 4
    for (int k = 0; k < kSortItems; k++) {
        const long long i = base + (long long)k * kSortThreads + threadIdx.x;
        if (i < n) atomicAdd(&h[(unsigned)(keys[i] >> shift) & 255u], 1u);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < 256; d += kSortThreads) hist[(size_t)d * ntiles + blockIdx.x] = h[d];
}

__global__ void __launch_bounds__(kSortThreads) radix_scatter_kernel(const uint64_t* __restrict__ kin,
                                                                     const unsigned* __restrict__ vin, long long n,
                                                                     int shift, int ntiles, const unsigned* __restrict__ offs,
                                                                     uint64_t* __restrict__ kout, unsigned* __restrict__ vout)
{
    __shared__ unsigned run[256];                 // next free slot per digit for this tile
    __shared__ unsigned wcnt[kSortWarps][256];    // keys per digit of each warp in this step
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    for (int d = t; d < 256; d += kSortThreads) run[d] = offs[(size_t)d * ntiles + blockIdx.x];
    const long long base = (long long)blockIdx.x * kSortTile;
    const unsigned lt = (1u << lane) - 1u;
    for (int k = 0; k < kSortItems; k++) {
        for (int q = t; q < kSortWarps * 256; q += kSortThreads) (&wcnt[0][0])[q] = 0;
        __syncthreads();
        const long long i = base + (long long)k * kSortThreads + t;
        const bool valid = i < n;
        const uint64_t key = valid ? kin[i] : 0;
        const unsigned val = valid ? vin[i] : 0;
        const unsigned dg = valid ? ((unsigned)(key >> shift) & 255u) : 256u;   // 256: no key
        const unsigned peers = __match_any_sync(0xffffffffu, dg);
        const unsigned rank = __popc(peers & lt);
        if (valid && rank == 0) wcnt[warp][dg] = __popc(peers);
        __syncthreads();
        unsigned pos = 0;
        if (valid) {
            pos = run[dg] + rank;
            for (int w = 0; w < warp; w++) pos += wcnt[w][dg];
        }
        __syncthreads();   // every key has read run[] and wcnt[] for this step
        for (int d = t; d < 256; d += kSortThreads) {
            unsigned s = 0;
#pragma unroll
            for (int w = 0; w < kSortWarps; w++) s += wcnt[w][d];
            run[d] += s;
        }
        if (valid) {
            kout[pos] = key;
            vout[pos] = val;
        }
        __syncthreads();   // run[] is updated and wcnt[] read before the next step clears it
    }
}

// Exclusive scan of each kScanThreads-element chunk of `a` in place; chunk totals to `sums`.
__global__ void __launch_bounds__(kScanThreads) scan_chunks_kernel(unsigned* __restrict__ a, size_t n,
                                                                   unsigned* __restrict__ sums)
{
    __shared__ unsigned s[kScanThreads];
    const size_t i = (size_t)blockIdx.x * kScanThreads + threadIdx.x;
    const unsigned v = i < n ? a[i] : 0u;
    s[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < kScanThreads; o <<= 1) {
        const unsigned add = threadIdx.x >= (unsigned)o ? s[threadIdx.x - o] : 0u;
        __syncthreads();
        s[threadIdx.x] += add;
        __syncthreads();
    }
    if (i < n) a[i] = s[threadIdx.x] - v;
    if (threadIdx.x == kScanThreads - 1) sums[blockIdx.x] = s[threadIdx.x];
}

__global__ void __launch_bounds__(kScanThreads) add_chunk_offsets_kernel(unsigned* __restrict__ a, size_t n,
                                                                         const unsigned* __restrict__ sums)
{
    const size_t i = (size_t)blockIdx.x * kScanThreads + threadIdx.x;
    if (i < n) a[i] += sums[blockIdx.x];
}

__global__ void __launch_bounds__(256) pack_keys_kernel(const int* __restrict__ row, const int* __restrict__ col, long long n,
                                                        int cb, uint64_t* __restrict__ keys, unsigned* __restrict__ idx)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    keys[i] = ((uint64_t)(uint32_t)row[i] << cb) | (uint32_t)col[i];
    idx[i] = (unsigned)i;
}

__global__ void __launch_bounds__(256) unpack_kernel(const uint64_t* __restrict__ keys, const unsigned* __restrict__ idx,
                                                     const float* __restrict__ vin, long long n, int cb,
                                                     int* __restrict__ row, int* __restrict__ col, float* __restrict__ vout)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t k = keys[i];
    row[i] = (int)(k >> cb);
    col[i] = (int)(k & ((1ull << cb) - 1ull));
    vout[i] = vin[idx[i]];
}

struct DBuf {
    void* p = nullptr;
    ~DBuf() { if (p) cudaFree(p); }
};

#define SCUDA(call)                                                 \
    do {                                                            \
        cudaError_t _e = (call);                                    \
        if (_e != cudaSuccess) return cuda_error(_e, #call);        \
    } while (0)

int bits_of(long long v)
{
    int b = 0;
    while (v > 0) { b++; v >>= 1; }
    return b;
}

}  // namespace

// Exclusive scan of a[0, n) on the device (chunk scans, then the chunk totals, recursively).
int device_exclusive_scan(unsigned* a, size_t n, cudaStream_t st)
{
    if (n == 0) return CSP_OK;
    const size_t chunks = (n + kScanThreads - 1) / kScanThreads;
    DBuf sums;
    SCUDA(cudaMalloc(&sums.p, std::max<size_t>(chunks, 1) * sizeof(unsigned)));
    scan_chunks_kernel<<<(unsigned)chunks, kScanThreads, 0, st>>>(a, n, static_cast<unsigned*>(sums.p));
    SCUDA(cudaGetLastError());
    if (chunks > 1) {
        int rc = device_exclusive_scan(static_cast<unsigned*>(sums.p), chunks, st);
        if (rc) return rc;
        add_chunk_offsets_kernel<<<(unsigned)chunks, kScanThreads, 0, st>>>(a, n, static_cast<unsigned*>(sums.p));
        SCUDA(cudaGetLastError());
    }
    return CSP_OK;
}


// Stable LSD radix sort of n 64-bit keys with 32-bit payloads over the low `bits` bits
// of the keys; k0/v0 hold the input, k1/v1 are scratch of the same sizes; *kres/*vres
// receive whichever pair of buffers holds the result.
int device_radix_sort_pairs(uint64_t* k0, uint64_t* k1, unsigned* v0, unsigned* v1, long long n, int bits,
                            cudaStream_t st, uint64_t** kres, unsigned** vres)
{
    *kres = k0;
    *vres = v0;
    if (n <= 1) return CSP_OK;
    const int passes = (std::max(bits, 1) + 7) / 8;
    const int ntiles = (int)((n + kSortTile - 1) / kSortTile);
    DBuf hist;
    SCUDA(cudaMalloc(&hist.p, (size_t)256 * ntiles * sizeof(unsigned)));
    unsigned* hs = static_cast<unsigned*>(hist.p);
    uint64_t* kin = k0;
    uint64_t* kout = k1;
    unsigned* vin = v0;
    unsigned* vout = v1;
    for (int p = 0; p < passes; p++) {
        const int shift = 8 * p;
        radix_hist_kernel<<<ntiles, kSortThreads, 0, st>>>(kin, n, shift, ntiles, hs);
        SCUDA(cudaGetLastError());
        int rc = device_exclusive_scan(hs, (size_t)256 * ntiles, st);
        if (rc) return rc;
        radix_scatter_kernel<<<ntiles, kSortThreads, 0, st>>>(kin, vin, n, shift, ntiles, hs, kout, vout);
        SCUDA(cudaGetLastError());
        std::swap(kin, kout);
        std::swap(vin, vout);
    }
    *kres = kin;
    *vres = vin;
    return CSP_OK;
}

int device_sort_coo(coo_matrix_if* m)
{
    const long long n = m->matinfo.nnz;
    if (n <= 1) return CSP_OK;
    if (n > (long long)UINT32_MAX) return set_error(CSP_EUNSUP, "device sort: more than 2^32 entries");
    const int cb = std::max(1, bits_of(std::max(m->matinfo.width, 1) - 1));
    const int rb = std::max(1, bits_of(std::max(m->matinfo.height, 1) - 1));
    DBuf drow, dcol, dval, dval2, k0, k1, v0, v1;
    SCUDA(cudaMalloc(&drow.p, n * 4));
    SCUDA(cudaMalloc(&dcol.p, n * 4));
    SCUDA(cudaMalloc(&dval.p, n * 4));
    SCUDA(cudaMalloc(&dval2.p, n * 4));
    SCUDA(cudaMalloc(&k0.p, n * 8));
    SCUDA(cudaMalloc(&k1.p, n * 8));
    SCUDA(cudaMalloc(&v0.p, n * 4));
    SCUDA(cudaMalloc(&v1.p, n * 4));
    cudaStream_t st = nullptr;
    SCUDA(cudaMemcpy(drow.p, m->coo_row_id, n * 4, cudaMemcpyHostToDevice));
    SCUDA(cudaMemcpy(dcol.p, m->coo_col_id, n * 4, cudaMemcpyHostToDevice));
    SCUDA(cudaMemcpy(dval.p, m->coo_data, n * 4, cudaMemcpyHostToDevice));
    const unsigned g = (unsigned)((n + 255) / 256);
    pack_keys_kernel<<<g, 256, 0, st>>>(static_cast<int*>(drow.p), static_cast<int*>(dcol.p), n, cb,
                                        static_cast<uint64_t*>(k0.p), static_cast<unsigned*>(v0.p));
    SCUDA(cudaGetLastError());
    uint64_t* kres = nullptr;
    unsigned* vres = nullptr;
    int rc = device_radix_sort_pairs(static_cast<uint64_t*>(k0.p), static_cast<uint64_t*>(k1.p),
                                     static_cast<unsigned*>(v0.p), static_cast<unsigned*>(v1.p), n, rb + cb, st, &kres,
                                     &vres);
    if (rc) return rc;
    unpack_kernel<<<g, 256, 0, st>>>(kres, vres, static_cast<float*>(dval.p), n, cb, static_cast<int*>(drow.p),
                                     static_cast<int*>(dcol.p), static_cast<float*>(dval2.p));
    SCUDA(cudaGetLastError());
    SCUDA(cudaMemcpy(m->coo_row_id, drow.p, n * 4, cudaMemcpyDeviceToHost));
    SCUDA(cudaMemcpy(m->coo_col_id, dcol.p, n * 4, cudaMemcpyDeviceToHost));
    SCUDA(cudaMemcpy(m->coo_data, dval2.p, n * 4, cudaMemcpyDeviceToHost));
    return CSP_OK;
}

}  // namespace csp

extern "C" int csp_sort_coo_device(coo_matrix_if* mat)
{
    using namespace csp;
    clear_error();
    int rc = check_coo(mat);
    if (rc) return rc;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return set_error(CSP_ENODEV, "csp_sort_coo_device needs a CUDA device");
    return device_sort_coo(mat);
}
