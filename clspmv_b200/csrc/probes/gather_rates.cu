// Random-gather rate probe (a standalone measurement program, not part of the library).
//
// Measures random 4-byte reads per second from the places an SpMV kernel can read x
// from: a global array of kGtPer * kGtCluster floats (1.5 MB, L2-resident after the
// first pass) through the load/store path (LDG) and through the texture path (a linear
// texture object over the same array), both paths interleaved, a 64 KB global array
// that stays in L1 (again through each path), one CTA's shared memory (kGtPer floats)
// and the shared memory of the 8 CTAs of a thread-block cluster (distributed shared
// memory).  Prints one JSON line.
//
//   clspmv_b200/bin/gather_rates
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <stdio.h>
#include <algorithm>
#include <functional>

namespace {

// Random 4-byte gathers with in-register hashed indices (no index stream), from three
// places: a global array kGtPer * kGtCluster floats long (L2-resident after the first
// pass), this CTA's shared memory (kGtPer floats), and the shared memory of the 8 CTAs
// of a thread-block cluster (distributed shared memory, kGtPer floats each).
constexpr int kGtPer = 49152;
constexpr int kGtCluster = 8;
constexpr int kGtThreads = 512;
constexpr int kGtIters = 256;
constexpr int kGtSmall = 16384;   // 64 KB: stays in each SM's L1 after the first touches

__device__ __forceinline__ unsigned gt_hash(unsigned a)
{
    a ^= a >> 16;
    a *= 0x7feb352dU;
    a ^= a >> 15;
    a *= 0x846ca68bU;
    a ^= a >> 16;
    return a;
}

__global__ void __launch_bounds__(kGtThreads, 1) gt_global(const float* __restrict__ src, float* __restrict__ out)
{
    unsigned h = gt_hash(blockIdx.x * kGtThreads + threadIdx.x);
    float acc = 0.0f;
#pragma unroll 8
    for (int it = 0; it < kGtIters; it++) {
        h = gt_hash(h + it);
        acc += __ldg(src + h % (kGtPer * kGtCluster));
    }
    out[blockIdx.x * kGtThreads + threadIdx.x] = acc;
}

template <int N>
__global__ void __launch_bounds__(kGtThreads, 1) gt_ldg(const float* __restrict__ src, float* __restrict__ out)
{
    unsigned h = gt_hash(blockIdx.x * kGtThreads + threadIdx.x);
    float acc = 0.0f;
#pragma unroll 8
    for (int it = 0; it < kGtIters; it++) {
        h = gt_hash(h + it);
        acc += __ldg(src + h % N);
    }
    out[blockIdx.x * kGtThreads + threadIdx.x] = acc;
}

template <int N>
__global__ void __launch_bounds__(kGtThreads, 1) gt_tex(cudaTextureObject_t tex, float* __restrict__ out)
{
    unsigned h = gt_hash(blockIdx.x * kGtThreads + threadIdx.x);
    float acc = 0.0f;
#pragma unroll 8
    for (int it = 0; it < kGtIters; it++) {
        h = gt_hash(h + it);
        acc += tex1Dfetch<float>(tex, (int)(h % N));
    }
    out[blockIdx.x * kGtThreads + threadIdx.x] = acc;
}

// half of the gathers through each path, interleaved
__global__ void __launch_bounds__(kGtThreads, 1) gt_mixed(const float* __restrict__ src, cudaTextureObject_t tex,
                                                          float* __restrict__ out)
{
    unsigned h = gt_hash(blockIdx.x * kGtThreads + threadIdx.x);
    float acc = 0.0f;
#pragma unroll 4
    for (int it = 0; it < kGtIters; it += 2) {
        h = gt_hash(h + it);
        acc += __ldg(src + h % (kGtPer * kGtCluster));
        h = gt_hash(h + it + 1);
        acc += tex1Dfetch<float>(tex, (int)(h % (kGtPer * kGtCluster)));
    }
    out[blockIdx.x * kGtThreads + threadIdx.x] = acc;
}

__global__ void __launch_bounds__(kGtThreads, 1) gt_shared(const float* __restrict__ src, float* __restrict__ out)
{
    extern __shared__ float gs[];
    for (int i = threadIdx.x; i < kGtPer; i += kGtThreads) gs[i] = src[i];
    __syncthreads();
    unsigned h = gt_hash(blockIdx.x * kGtThreads + threadIdx.x);
    float acc = 0.0f;
#pragma unroll 8
    for (int it = 0; it < kGtIters; it++) {
        h = gt_hash(h + it);
        acc += gs[h % kGtPer];
    }
    out[blockIdx.x * kGtThreads + threadIdx.x] = acc;
}

__global__ void __cluster_dims__(kGtCluster, 1, 1) __launch_bounds__(kGtThreads, 1)
    gt_cluster(const float* __restrict__ src, float* __restrict__ out)
{
    namespace cg = cooperative_groups;
    extern __shared__ float gs[];
    cg::cluster_group cl = cg::this_cluster();
    const unsigned rank = cl.block_rank();
    for (int i = threadIdx.x; i < kGtPer; i += kGtThreads) gs[i] = src[rank * kGtPer + i];
    cl.sync();
    unsigned h = gt_hash(blockIdx.x * kGtThreads + threadIdx.x);
    float acc = 0.0f;
#pragma unroll 8
    for (int it = 0; it < kGtIters; it++) {
        h = gt_hash(h + it);
        const unsigned idx = h % (kGtPer * kGtCluster);
        acc += cl.map_shared_rank(gs, idx / kGtPer)[idx % kGtPer];
    }
    cl.sync();   // no CTA leaves while the others may still read its shared memory
    out[blockIdx.x * kGtThreads + threadIdx.x] = acc;
}

float time_ms(cudaStream_t st, int reps, const std::function<void()>& f)
{
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    f();
    cudaEventRecord(e0, st);
    for (int i = 0; i < reps; i++) f();
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return ms / reps;
}

}  // namespace

int main()
{
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        fprintf(stderr, "gather_rates: no CUDA device\n");
        return 1;
    }
    const int grid = std::max(kGtCluster, sms / kGtCluster * kGtCluster);
    float *src = nullptr, *out = nullptr;
    if (cudaMalloc(&src, sizeof(float) * kGtPer * kGtCluster) != cudaSuccess ||
        cudaMalloc(&out, sizeof(float) * grid * kGtThreads) != cudaSuccess) {
        fprintf(stderr, "gather_rates: device allocation failed\n");
        return 1;
    }
    cudaStream_t st;
    cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    const size_t smem = sizeof(float) * kGtPer;
    cudaMemsetAsync(src, 0, sizeof(float) * kGtPer * kGtCluster, st);
    cudaFuncSetAttribute(gt_shared, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(gt_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const double n = (double)grid * kGtThreads * kGtIters;
    cudaResourceDesc rd = {};
    rd.resType = cudaResourceTypeLinear;
    rd.res.linear.devPtr = src;
    rd.res.linear.desc = cudaCreateChannelDesc<float>();
    rd.res.linear.sizeInBytes = sizeof(float) * kGtPer * kGtCluster;
    cudaTextureDesc td = {};
    td.readMode = cudaReadModeElementType;
    cudaTextureObject_t tex = 0;
    if (cudaCreateTextureObject(&tex, &rd, &td, nullptr) != cudaSuccess) {
        fprintf(stderr, "gather_rates: texture object creation failed\n");
        return 1;
    }
    const double l2 = n / (time_ms(st, 5, [&] { gt_global<<<grid, kGtThreads, 0, st>>>(src, out); }) * 1e-3);
    const double tx = n / (time_ms(st, 5, [&] { gt_tex<kGtPer * kGtCluster><<<grid, kGtThreads, 0, st>>>(tex, out); }) * 1e-3);
    const double mx = n / (time_ms(st, 5, [&] { gt_mixed<<<grid, kGtThreads, 0, st>>>(src, tex, out); }) * 1e-3);
    const double l1 = n / (time_ms(st, 5, [&] { gt_ldg<kGtSmall><<<grid, kGtThreads, 0, st>>>(src, out); }) * 1e-3);
    const double t1 = n / (time_ms(st, 5, [&] { gt_tex<kGtSmall><<<grid, kGtThreads, 0, st>>>(tex, out); }) * 1e-3);
    const double sh = n / (time_ms(st, 5, [&] { gt_shared<<<grid, kGtThreads, smem, st>>>(src, out); }) * 1e-3);
    cudaError_t e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) {
        fprintf(stderr, "gather_rates: %s\n", cudaGetErrorString(e));
        return 1;
    }
    double cl = n / (time_ms(st, 5, [&] { gt_cluster<<<grid, kGtThreads, smem, st>>>(src, out); }) * 1e-3);
    e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) cl = -1.0;   // no thread-block clusters on this device
    printf("{\"array_bytes\": %.0f, \"l2_per_s\": %.4e, \"tex_l2_per_s\": %.4e, \"ldg_tex_mixed_l2_per_s\": %.4e, "
           "\"small_array_bytes\": %.0f, \"l1_per_s\": %.4e, \"tex_l1_per_s\": %.4e, \"shared_per_s\": %.4e, "
           "\"cluster_per_s\": %.4e}\n",
           (double)sizeof(float) * kGtPer * kGtCluster, l2, tx, mx, (double)sizeof(float) * kGtSmall, l1, t1, sh, cl);
    cudaDestroyTextureObject(tex);
    cudaStreamDestroy(st);
    cudaFree(src);
    cudaFree(out);
    return 0;
}
