// Multiple right-hand sides: Y += A * X with X (n x k) and Y (m x k) row-major, so
// the k values of one column index are contiguous and every gather is a coalesced
// row segment.  A lane group of G = min(k, 32) lanes serves one (block) row, lane l
// owning right-hand sides l, l + G, ...; the group's entries are staged in shared
// memory by coalesced loads and read back as broadcasts.
#pragma once

#include <type_traits>

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

namespace csp {
namespace dev {

// ---------------------------------------------------------------------------
// Generic BCSR SpMM on tensor cores: k a multiple of 32, blocks of BH <= 8 rows and
// BW <= 4 columns (mma.sync.m16n8k8, TF32 operands, FP32 accumulation).
//
// One warp per block row.  For each panel of 32 right-hand sides the block row's
// BH x 32 output is two 16 x 8 MMA tiles D[m][n]: M = 16 right-hand sides, N = the
// block row's rows (BH of 8), K = the columns of two blocks per step, each block's BW
// columns padded to 4.  Lane (g, t) = (lane / 4, lane % 4) feeds
//   A (16 x 8, X^T):  X[col(t)][rhs(g)], X[col(t)][rhs(g + 8)], and the same at t + 4,
//   B (8 x 8, A^T):   A[row g][col t] of the step's first and second block,
// and the right-hand sides are numbered so that tile tau's rows g and g + 8 are
// right-hand sides 4g + 2tau and 4g + 2tau + 1: one 128-bit load of X[col][4g .. 4g + 3]
// gives a lane both tiles' A entries of one column, and lane t's outputs (rows 2t and
// 2t + 1) are two 128-bit Y rows segments.  Padding columns (t >= BW) and rows
// (g >= BH) contribute zeros; they cost no loads.
//
// FP32 accuracy from TF32 operands: every operand v is split into vh = tf32(v) (round
// to nearest) and the exact remainder vl = v - vh, and a * x is taken as
// ah*xh + (ah*xl + al*xh) -- three MMAs, the two small terms in their own accumulator
// so they do not perturb the large one's rounding (the dropped al*xl is below 2^-22 of
// |a x|).  BF16 values are exact in TF32 (al = 0): two MMAs.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void mma_tf32(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                         uint32_t b1)
{
    asm volatile("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
                 "{%0, %1, %2, %3};"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// High and low TF32 parts of v: hi = v rounded to nearest (ties away from zero) at
// TF32's 10 fraction bits -- half a TF32 ulp (bit 12) added to the magnitude bits, the
// 13 low bits cleared -- and the exact remainder lo = v - hi, passed as raw FP32 bits
// (the MMA reads its top 19).  Finite |v| below 2^128 (1 - 2^-11) only.
__device__ __forceinline__ void tf32_split(float v, uint32_t& hi, uint32_t& lo)
{
    hi = (__float_as_uint(v) + 0x1000u) & 0xffffe000u;
    lo = __float_as_uint(v - __uint_as_float(hi));
}

constexpr int kMmaThreads = 256;   // 8 warps, one block row each

template <class V, int BH, int BW, int KS>
__global__ void __launch_bounds__(kMmaThreads) bcsr_spmm_mma_kernel(const int* __restrict__ rp, const int* __restrict__ col,
                                                                    const V* __restrict__ data, const float* __restrict__ x,
                                                                    float* __restrict__ y, int nbr, int aligned, int m,
                                                                    int n, int k)
{
    static_assert(BH >= 1 && BH <= 8 && BW >= 1 && BW <= 4, "block shape");
    constexpr bool kExactA = !std::is_same<V, float>::value;   // BF16 values: exact in TF32
    const int lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    const int br = (int)(((long long)blockIdx.x * kMmaThreads + threadIdx.x) >> 5);
    if (br >= nbr) return;   // the whole warp leaves together
    const int s = __ldg(rp + br), e = __ldg(rp + br + 1);
    const bool xlane = t < BW;                // lanes whose column is a real one
    const bool alane = xlane && g < BH;       // lanes holding a matrix value
    const V* __restrict__ plane = data + (size_t)(alane ? g * BW + t : 0) * aligned;
    // lane t's output rows 2t and 2t + 1
    const int r0 = br * BH + 2 * t, r1 = r0 + 1;
    const bool w0 = 2 * t < BH && r0 < m, w1 = 2 * t + 1 < BH && r1 < m;
    for (int c0 = 0; c0 < k; c0 += 32) {
        const int cx = c0 + 4 * g;
        // the Y rows this lane updates, requested before the block loads and X gathers
        float4 y0 = w0 ? *reinterpret_cast<const float4*>(y + (size_t)r0 * k + cx) : make_float4(0.f, 0.f, 0.f, 0.f);
        float4 y1 = w1 ? *reinterpret_cast<const float4*>(y + (size_t)r1 * k + cx) : make_float4(0.f, 0.f, 0.f, 0.f);
        float big[2][4], small[2][4];
#pragma unroll
        for (int u = 0; u < 2; u++)
#pragma unroll
            for (int q = 0; q < 4; q++) big[u][q] = small[u][q] = 0.0f;
        for (int j0 = s; j0 < e; j0 += 2 * KS) {
            // every load of KS steps (2 KS blocks) first
            float4 xv[KS][2];
            float av[KS][2];
#pragma unroll
            for (int u = 0; u < KS; u++)
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int j = j0 + 2 * u + h;
                    const bool vj = j < e;
                    const int bc = vj ? __ldg(col + j) : 0;
                    xv[u][h] = (vj && xlane && bc + t < n)
                                   ? __ldg(reinterpret_cast<const float4*>(x + (size_t)(bc + t) * k + cx))
                                   : make_float4(0.f, 0.f, 0.f, 0.f);
                    av[u][h] = (vj && alane) ? Val<V>::ld(plane + j) : 0.0f;
                }
#pragma unroll
            for (int u = 0; u < KS; u++) {
                if (j0 + 2 * u >= e) break;
                uint32_t xh[2][4], xl[2][4];
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    tf32_split(xv[u][h].x, xh[h][0], xl[h][0]);
                    tf32_split(xv[u][h].y, xh[h][1], xl[h][1]);
                    tf32_split(xv[u][h].z, xh[h][2], xl[h][2]);
                    tf32_split(xv[u][h].w, xh[h][3], xl[h][3]);
                }
                uint32_t ah0, ah1, al0 = 0, al1 = 0;
                if (kExactA) {
                    ah0 = __float_as_uint(av[u][0]);
                    ah1 = __float_as_uint(av[u][1]);
                } else {
                    tf32_split(av[u][0], ah0, al0);
                    tf32_split(av[u][1], ah1, al1);
                }
                // tile 0: right-hand sides 4g, 4g + 1 (x, y components); tile 1: 4g + 2, 4g + 3 (z, w)
#pragma unroll
                for (int tau = 0; tau < 2; tau++) {
                    const int p = 2 * tau, q = 2 * tau + 1;
                    mma_tf32(small[tau], xl[0][p], xl[0][q], xl[1][p], xl[1][q], ah0, ah1);
                    if (!kExactA) mma_tf32(small[tau], xh[0][p], xh[0][q], xh[1][p], xh[1][q], al0, al1);
                    mma_tf32(big[tau], xh[0][p], xh[0][q], xh[1][p], xh[1][q], ah0, ah1);
                }
            }
        }
        // D[m][n] fragments: d[0] = (g, 2t), d[1] = (g, 2t + 1), d[2] = (g + 8, 2t), d[3] = (g + 8, 2t + 1)
        float d[2][4];
#pragma unroll
        for (int u = 0; u < 2; u++)
#pragma unroll
            for (int q = 0; q < 4; q++) d[u][q] = big[u][q] + small[u][q];
        if (w0) {
            y0.x += d[0][0];
            y0.y += d[0][2];
            y0.z += d[1][0];
            y0.w += d[1][2];
            *reinterpret_cast<float4*>(y + (size_t)r0 * k + cx) = y0;
        }
        if (w1) {
            y1.x += d[0][1];
            y1.y += d[0][3];
            y1.z += d[1][1];
            y1.w += d[1][3];
            *reinterpret_cast<float4*>(y + (size_t)r1 * k + cx) = y1;
        }
    }
}

}  // namespace dev
}  // namespace csp
