// The Cocktail analyzer's counting passes on the device (CSP_ANALYZE_ON_DEVICE).
//
// The reference partitioner (analyze.cpp) spends most of its time on two integer
// counts over every nonzero: the nonzeros per diagonal offset (count_dia_nnz,
// clSpMV_NV/src/analyze.cpp:804) and, for each of the eight b4 block shapes and every
// block row, the number of distinct blocks and the nonzeros they hold, all blocks and
// those above a fill threshold (count_blocks, :1582).  Both are exact integer counts,
// so computing them here leaves every decision, and the partition, byte for byte what
// the host computes.
//
//   count_dia:    a histogram of col - row + threshold with warp-aggregated integer
//                 atomics (the lanes of a warp that hit one bin add once);
//   count_blocks: one thread per (shape, block row) merging the block row's BH rows,
//                 each sorted by column, block column by block column (col / bw), so
//                 every block is counted once without sorting or hashing.
#include <cuda_runtime.h>
#include <climits>
#include <vector>

#include "csp/clspmv.h"
#include "internal.h"
#include "engine.h"

namespace csp {
namespace {

__global__ void __launch_bounds__(256) dia_count_kernel(const int* __restrict__ row, const int* __restrict__ col, int nnz,
                                                        int threshold, int nbins, int* __restrict__ count)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i - threadIdx.x < nnz;
         i += (long long)gridDim.x * blockDim.x) {
        const bool in = i < nnz;
        const int o = in ? __ldg(col + i) - __ldg(row + i) + threshold : -1;
        const bool ok = in && o >= 0 && o < nbins;
        const unsigned act = __ballot_sync(0xffffffffu, ok);
        if (!ok) continue;
        const unsigned same = __match_any_sync(act, o);
        if ((threadIdx.x & 31) == __ffs(same) - 1) atomicAdd(count + o, __popc(same));
    }
}

// Block row br of a BH x bw shape: {partial blocks, partial nnz, blocks, nnz}.
template <int BH>
__global__ void __launch_bounds__(256) block_count_kernel(const int* __restrict__ rp, const int* __restrict__ col, int h,
                                                          int bw, int thr, int nbr, int4* __restrict__ out)
{
    const int br = blockIdx.x * blockDim.x + threadIdx.x;
    if (br >= nbr) return;
    int p[BH], e[BH], head[BH];
#pragma unroll
    for (int q = 0; q < BH; q++) {
        const int r = br * BH + q;
        p[q] = r < h ? __ldg(rp + r) : 0;
        e[q] = r < h ? __ldg(rp + r + 1) : 0;
        head[q] = p[q] < e[q] ? __ldg(col + p[q]) / bw : INT_MAX;
    }
    int pb = 0, pn = 0, fb = 0, fn = 0;
    while (true) {
        int bc = INT_MAX;
#pragma unroll
        for (int q = 0; q < BH; q++) bc = min(bc, head[q]);
        if (bc == INT_MAX) break;
        int cnt = 0;
#pragma unroll
        for (int q = 0; q < BH; q++) {
            while (head[q] == bc) {
                cnt++;
                p[q]++;
                head[q] = p[q] < e[q] ? __ldg(col + p[q]) / bw : INT_MAX;
            }
        }
        fb++;
        fn += cnt;
        if (cnt > thr) {
            pb++;
            pn += cnt;
        }
    }
    out[br] = make_int4(pb, pn, fb, fn);
}

struct DevBuf {
    void* p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
};

#define ACUDA(call)                                                 \
    do {                                                            \
        cudaError_t _e = (call);                                    \
        if (_e != cudaSuccess) return cuda_error(_e, #call);        \
    } while (0)

}  // namespace

int device_count_dia(const int* row, const int* col, int nnz, int threshold, std::vector<int>& count)
{
    const int nbins = 2 * threshold + 1;
    count.assign((size_t)nbins, 0);
    if (nnz == 0) return CSP_OK;
    DevBuf dr, dc, dn;
    ACUDA(cudaMalloc(&dr.p, (size_t)nnz * 4));
    ACUDA(cudaMalloc(&dc.p, (size_t)nnz * 4));
    ACUDA(cudaMalloc(&dn.p, (size_t)nbins * 4));
    ACUDA(cudaMemcpy(dr.p, row, (size_t)nnz * 4, cudaMemcpyHostToDevice));
    ACUDA(cudaMemcpy(dc.p, col, (size_t)nnz * 4, cudaMemcpyHostToDevice));
    ACUDA(cudaMemset(dn.p, 0, (size_t)nbins * 4));
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long want = ((long long)nnz + 255) / 256;
    const int grid = (int)std::min<long long>(want, (long long)sms * 8);
    dia_count_kernel<<<grid, 256>>>(static_cast<int*>(dr.p), static_cast<int*>(dc.p), nnz, threshold, nbins,
                                    static_cast<int*>(dn.p));
    ACUDA(cudaGetLastError());
    ACUDA(cudaMemcpy(count.data(), dn.p, (size_t)nbins * 4, cudaMemcpyDeviceToHost));
    return CSP_OK;
}

int device_count_blocks(const int* rp, const int* col, int h, int nnz, const int* bh, const int* bw, const int* threshold,
                        int nshapes, std::vector<std::vector<BlockCounts>>& out)
{
    static_assert(sizeof(BlockCounts) == sizeof(int4), "BlockCounts is the kernel's int4 {partial blocks, partial nnz, blocks, nnz}");
    out.assign((size_t)nshapes, std::vector<BlockCounts>());
    DevBuf drp, dcol, dout;
    ACUDA(cudaMalloc(&drp.p, ((size_t)h + 1) * 4));
    ACUDA(cudaMalloc(&dcol.p, std::max<size_t>((size_t)nnz * 4, 4)));
    ACUDA(cudaMemcpy(drp.p, rp, ((size_t)h + 1) * 4, cudaMemcpyHostToDevice));
    if (nnz) ACUDA(cudaMemcpy(dcol.p, col, (size_t)nnz * 4, cudaMemcpyHostToDevice));
    ACUDA(cudaMalloc(&dout.p, std::max<size_t>((size_t)h * sizeof(int4), sizeof(int4))));
    for (int s = 0; s < nshapes; s++) {
        const int nbr = h / bh[s] + (h % bh[s] != 0);
        out[s].resize((size_t)nbr);
        if (nbr == 0) continue;
        const unsigned g = (unsigned)((nbr + 255) / 256);
        const int* r = static_cast<const int*>(drp.p);
        const int* c = static_cast<const int*>(dcol.p);
        int4* o = static_cast<int4*>(dout.p);
        switch (bh[s]) {
        case 1: block_count_kernel<1><<<g, 256>>>(r, c, h, bw[s], threshold[s], nbr, o); break;
        case 2: block_count_kernel<2><<<g, 256>>>(r, c, h, bw[s], threshold[s], nbr, o); break;
        case 4: block_count_kernel<4><<<g, 256>>>(r, c, h, bw[s], threshold[s], nbr, o); break;
        case 8: block_count_kernel<8><<<g, 256>>>(r, c, h, bw[s], threshold[s], nbr, o); break;
        default: return set_error(CSP_EINVAL, "device block count: block height %d", bh[s]);
        }
        ACUDA(cudaGetLastError());
        ACUDA(cudaMemcpy(out[s].data(), o, (size_t)nbr * sizeof(int4), cudaMemcpyDeviceToHost));
    }
    return CSP_OK;
}

}  // namespace csp
