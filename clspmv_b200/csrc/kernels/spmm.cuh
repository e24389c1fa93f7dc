// Multiple right-hand sides: Y += A * X with X (n x k) and Y (m x k) row-major, so
// the k values of one column index are contiguous and every gather is a coalesced
// row segment.  A lane group of G = min(k, 32) lanes serves one (block) row, lane l
// owning right-hand sides l, l + G, ...; the group's entries are staged in shared
// memory by coalesced loads and read back as broadcasts.
#pragma once

#include "common.cuh"

namespace csp {
namespace dev {

constexpr int kSpmmThreads = 256;

// CSR: one group per row.
template <class V, int G>
__global__ void __launch_bounds__(kSpmmThreads) csr_spmm_kernel(const int* __restrict__ rp, const int* __restrict__ col,
                                                                const V* __restrict__ val, const float* __restrict__ x,
                                                                float* __restrict__ y, int m, int k)
{
    __shared__ int s_col[kSpmmThreads];
    __shared__ float s_val[kSpmmThreads];
    const int lane = threadIdx.x % G;
    const int gbase = threadIdx.x - lane;   // this group's slice of the staging arrays
    // groups of one warp run different trip counts: each synchronises only its own lanes
    const unsigned gmask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << ((threadIdx.x & 31) - lane));
    const int row = (int)(((long long)blockIdx.x * kSpmmThreads + threadIdx.x) / G);
    const bool valid = row < m;
    const int s = valid ? __ldg(rp + row) : 0, e = valid ? __ldg(rp + row + 1) : 0;
    for (int c0 = 0; c0 < k; c0 += G) {
        const int c = c0 + lane;
        float acc = 0.0f;
        for (int j0 = s; j0 < e; j0 += G) {
            const int n = min(G, e - j0);
            __syncwarp(gmask);
            if (lane < n) {
                s_col[gbase + lane] = __ldg(col + j0 + lane);
                s_val[gbase + lane] = Val<V>::ld(val + j0 + lane);
            }
            __syncwarp(gmask);
            if (c < k)
                for (int t = 0; t < n; t++) acc += s_val[gbase + t] * __ldg(x + (size_t)s_col[gbase + t] * k + c);
        }
        if (valid && c < k) y[(size_t)row * k + c] += acc;
    }
}

// Generic BCSR (block-element-major data[e * aligned + block]): one group per block row.
// The staged block values take kSpmmThreads * BH * BW floats of shared memory, so
// blocks are limited to 36 elements (6 x 6).
template <class V, int BH, int BW, int G>
__global__ void __launch_bounds__(kSpmmThreads) bcsr_spmm_kernel(const int* __restrict__ rp, const int* __restrict__ col,
                                                                 const V* __restrict__ data, const float* __restrict__ x,
                                                                 float* __restrict__ y, int nbr, int aligned, int m, int n,
                                                                 int k)
{
    constexpr int BS = BH * BW;
    __shared__ float s_val[kSpmmThreads * BS];
    __shared__ int s_col[kSpmmThreads];
    const int lane = threadIdx.x % G;
    const int gbase = threadIdx.x - lane;
    const unsigned gmask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << ((threadIdx.x & 31) - lane));
    const int br = (int)(((long long)blockIdx.x * kSpmmThreads + threadIdx.x) / G);
    const bool valid = br < nbr;
    const int s = valid ? __ldg(rp + br) : 0, e = valid ? __ldg(rp + br + 1) : 0;
    for (int c0 = 0; c0 < k; c0 += G) {
        const int c = c0 + lane;
        float acc[BH];
#pragma unroll
        for (int h = 0; h < BH; h++) acc[h] = 0.0f;
        for (int j0 = s; j0 < e; j0 += G) {
            const int nb = min(G, e - j0);
            __syncwarp(gmask);
            if (lane < nb) {
                s_col[gbase + lane] = __ldg(col + j0 + lane);
#pragma unroll
                for (int q = 0; q < BS; q++) s_val[(gbase + lane) * BS + q] = Val<V>::ld(data + (size_t)q * aligned + j0 + lane);
            }
            __syncwarp(gmask);
            if (c < k) {
                for (int t = 0; t < nb; t++) {
                    const int bc = s_col[gbase + t];
                    const float* bv = s_val + (gbase + t) * BS;
                    float xv[BW];
#pragma unroll
                    for (int w = 0; w < BW; w++) xv[w] = (bc + w < n) ? __ldg(x + (size_t)(bc + w) * k + c) : 0.0f;
#pragma unroll
                    for (int h = 0; h < BH; h++)
#pragma unroll
                        for (int w = 0; w < BW; w++) acc[h] += bv[h * BW + w] * xv[w];
                }
            }
        }
        if (valid && c < k) {
#pragma unroll
            for (int h = 0; h < BH; h++) {
                const int r = br * BH + h;
                if (r < m) y[(size_t)r * k + c] += acc[h];
            }
        }
    }
}

// Generic BCSR with k a multiple of 4: register-blocked.  A block row is served by
// L = CW * S lanes: CW lanes each own 4 consecutive right-hand sides (128-bit loads of
// X and Y rows) and S sub-groups split the block row's blocks, summed by shuffles at
// the end.  Block values are staged element-major -> shared memory by coalesced loads
// (one block per lane of the group) and read back as broadcasts.  Columns beyond
// 4 * CW are handled in further passes.
template <class V, int BH, int BW, int CW, int S>
__global__ void __launch_bounds__(kSpmmThreads) bcsr_spmm4_kernel(const int* __restrict__ rp, const int* __restrict__ col,
                                                                  const V* __restrict__ data, const float* __restrict__ x,
                                                                  float* __restrict__ y, int nbr, int aligned, int m, int n,
                                                                  int k)
{
    constexpr int BS = BH * BW;
    constexpr int L = CW * S;
    __shared__ float s_val[kSpmmThreads * BS];
    __shared__ int s_col[kSpmmThreads];
    const int lane = threadIdx.x % L;
    const int cw = lane % CW, sub = lane / CW;
    const int gbase = threadIdx.x - lane;
    const unsigned gmask = (L == 32) ? 0xffffffffu : (((1u << L) - 1u) << ((threadIdx.x & 31) - lane));
    const int br = (int)(((long long)blockIdx.x * kSpmmThreads + threadIdx.x) / L);
    const bool valid = br < nbr;
    const int s = valid ? __ldg(rp + br) : 0, e = valid ? __ldg(rp + br + 1) : 0;
    for (int c0 = 0; c0 < k; c0 += 4 * CW) {
        const int c = c0 + 4 * cw;
        const bool active = c < k;
        float4 acc[BH];
#pragma unroll
        for (int h = 0; h < BH; h++) acc[h] = make_float4(0.f, 0.f, 0.f, 0.f);
        // the Y rows this lane updates, requested before the block loads and X gathers
        float4 yo[BH];
#pragma unroll
        for (int h = 0; h < BH; h++) {
            const int r = br * BH + h;
            yo[h] = (valid && active && sub == 0 && r < m) ? *reinterpret_cast<const float4*>(y + (size_t)r * k + c)
                                                            : make_float4(0.f, 0.f, 0.f, 0.f);
        }
        for (int j0 = s; j0 < e; j0 += L) {
            const int nb = min(L, e - j0);
            __syncwarp(gmask);
            if (lane < nb) {
                s_col[gbase + lane] = __ldg(col + j0 + lane);
#pragma unroll
                for (int q = 0; q < BS; q++) s_val[(gbase + lane) * BS + q] = Val<V>::ld(data + (size_t)q * aligned + j0 + lane);
            }
            __syncwarp(gmask);
            if (active) {
                // U blocks of this sub-group at a time: their X rows are requested together.
                // With 8 float4 lanes (k >= 32), U = 2 keeps the kernel at 58 registers,
                // 4 CTAs per SM; U = 4 took 80 and ran 17 % slower on 3x3 blocks at k = 32
                constexpr int U = (BW <= 3 && CW < 8) ? 4 : 2;
                for (int t0 = sub; t0 < nb; t0 += S * U) {
                    float4 xv[U][BW];
#pragma unroll
                    for (int u = 0; u < U; u++) {
                        const int t = t0 + u * S;
                        const int bc = t < nb ? s_col[gbase + t] : 0;
#pragma unroll
                        for (int w = 0; w < BW; w++)
                            xv[u][w] = (t < nb && bc + w < n)
                                           ? __ldg(reinterpret_cast<const float4*>(x + (size_t)(bc + w) * k + c))
                                           : make_float4(0.f, 0.f, 0.f, 0.f);
                    }
#pragma unroll
                    for (int u = 0; u < U; u++) {
                        const int t = t0 + u * S;
                        if (t >= nb) break;
                        const float* bv = s_val + (gbase + t) * BS;
#pragma unroll
                        for (int h = 0; h < BH; h++)
#pragma unroll
                            for (int w = 0; w < BW; w++) {
                                const float a = bv[h * BW + w];
                                acc[h].x += a * xv[u][w].x;
                                acc[h].y += a * xv[u][w].y;
                                acc[h].z += a * xv[u][w].z;
                                acc[h].w += a * xv[u][w].w;
                            }
                    }
                }
            }
        }
        // sum the S sub-groups (lanes cw, cw + CW, ...)
#pragma unroll
        for (int h = 0; h < BH; h++) {
#pragma unroll
            for (int o = CW; o < L; o <<= 1) {
                acc[h].x += __shfl_xor_sync(gmask, acc[h].x, o, L);
                acc[h].y += __shfl_xor_sync(gmask, acc[h].y, o, L);
                acc[h].z += __shfl_xor_sync(gmask, acc[h].z, o, L);
                acc[h].w += __shfl_xor_sync(gmask, acc[h].w, o, L);
            }
        }
        if (valid && active && sub == 0) {
#pragma unroll
            for (int h = 0; h < BH; h++) {
                const int r = br * BH + h;
                if (r < m) {
                    float4 o = yo[h];
                    o.x += acc[h].x;
                    o.y += acc[h].y;
                    o.z += acc[h].z;
                    o.w += acc[h].w;
                    *reinterpret_cast<float4*>(y + (size_t)r * k + c) = o;
                }
            }
        }
    }
}

}  // namespace dev
}  // namespace csp
