// COO -> DIA, BDIA and generic BCSR layout builds on the device
// (clSpMV_NV/include/matrix_storage.h:937 coo2dia, :1185 coo2bdia, :1595 coo2bcsr).
// They fill the same host structs as csp_coo2dia / csp_coo2bdia / csp_coo2bcsr (BDIA:
// the device DIA, then the host's banding of its offsets), byte for byte whenever no two entries
// share a (row, col) position, with the grouping, counting and scattering done by
// kernels:
//
//   DIA:  a stable radix sort of the entries' diagonal offsets groups them by diagonal
//         in ascending offset order, the first entry of each group being the diagonal's
//         first entry in input order; a scan of the key changes numbers the diagonals;
//         the entries then go to data[diagonal * length + row].  The padding rule
//         (reject once the diagonals already found cover 2 * nnz slots) and the row
//         check are decided from those first entries, so the same error comes back, at
//         the same entry, as from the host build.
//   BCSR: a stable radix sort of (block row, block column) keys groups the entries by
//         block in the reference's order (block rows, then ascending block column); a
//         scan of the key changes numbers the blocks; per-block-row counts and a scan
//         give the row pointers; the entries go to data[element * aligned + block].
//
// Duplicate (row, col) entries: the last one in input order is kept.  (The host DIA
// build does the same; the host BCSR build keeps the last one in the order its
// std::sort leaves them in, which is not specified, so for duplicates the host build
// remains the byte-exact one.)
#include <cuda_runtime.h>
#include <limits.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <algorithm>
#include <vector>

#include "csp/clspmv.h"
#include "internal.h"
#include "engine.h"
#include "device_sort.h"

namespace csp {
namespace {

constexpr int kLT = 256;
constexpr int kAbsent = 0x7f7f7f7f;   // memset(0x7f) pattern: "no such entry"

struct DMem {
    void* p = nullptr;
    ~DMem() { if (p) cudaFree(p); }
    template <class T> T* as() const { return static_cast<T*>(p); }
};

#define LCUDA(call)                                                 \
    do {                                                            \
        cudaError_t _e = (call);                                    \
        if (_e != cudaSuccess) return cuda_error(_e, #call);        \
    } while (0)

inline unsigned grid_of(long long n) { return (unsigned)((n + kLT - 1) / kLT); }

int bits_for(long long v)
{
    int b = 0;
    while (v > 0) { b++; v >>= 1; }
    return std::max(b, 1);
}

// ---- DIA ----

__global__ void __launch_bounds__(kLT) dia_keys_kernel(const int* __restrict__ row, const int* __restrict__ col, int nnz,
                                                       int h, int len, uint64_t* __restrict__ keys,
                                                       unsigned* __restrict__ idx, int* __restrict__ badrow)
{
    const long long i = (long long)blockIdx.x * kLT + threadIdx.x;
    if (i >= nnz) return;
    const int r = row[i];
    if (r >= len) atomicMin(badrow, (int)i);
    keys[i] = (uint64_t)((long long)col[i] - r + h - 1);
    idx[i] = (unsigned)i;
}

// start[] holds the exclusive scan of the key changes: the group of sorted position p
__global__ void __launch_bounds__(kLT) dia_groups_kernel(const uint64_t* __restrict__ keys, const unsigned* __restrict__ idx,
                                                         const unsigned* __restrict__ start, long long n, int h,
                                                         int* __restrict__ offs, int* __restrict__ firsts,
                                                         unsigned* __restrict__ eslot)
{
    const long long p = (long long)blockIdx.x * kLT + threadIdx.x;
    if (p >= n) return;
    const bool head = p == 0 || keys[p] != keys[p - 1];
    const unsigned g = start[p] - (head ? 0u : 1u);
    eslot[idx[p]] = g;
    if (head) {
        offs[g] = (int)((long long)keys[p] - (h - 1));
        firsts[g] = (int)idx[p];   // stable sort: the group's first entry in input order
    }
}

__global__ void __launch_bounds__(kLT) dia_winner_kernel(const int* __restrict__ row, int nnz, int len,
                                                         const unsigned* __restrict__ eslot, int* __restrict__ winner)
{
    const long long i = (long long)blockIdx.x * kLT + threadIdx.x;
    if (i >= nnz) return;
    atomicMax(winner + (size_t)eslot[i] * len + row[i], (int)i);
}

__global__ void __launch_bounds__(kLT) dia_place_kernel(const int* __restrict__ row, const float* __restrict__ val, int nnz,
                                                        int len, const unsigned* __restrict__ eslot,
                                                        const int* __restrict__ winner, float* __restrict__ data)
{
    const long long i = (long long)blockIdx.x * kLT + threadIdx.x;
    if (i >= nnz) return;
    const size_t q = (size_t)eslot[i] * len + row[i];
    if (winner[q] == (int)i) data[q] = val[i];
}

// a position whose key differs from the one before starts a group
__global__ void __launch_bounds__(kLT) key_change_kernel(const uint64_t* __restrict__ keys, long long n,
                                                         unsigned* __restrict__ flag)
{
    const long long p = (long long)blockIdx.x * kLT + threadIdx.x;
    if (p < n) flag[p] = (p == 0 || keys[p] != keys[p - 1]) ? 1u : 0u;
}

// ---- BCSR ----

__global__ void __launch_bounds__(kLT) block_keys_kernel(const int* __restrict__ row, const int* __restrict__ col, int nnz,
                                                         int bw, int bh, int cb, uint64_t* __restrict__ keys,
                                                         unsigned* __restrict__ idx)
{
    const long long i = (long long)blockIdx.x * kLT + threadIdx.x;
    if (i >= nnz) return;
    keys[i] = ((uint64_t)(unsigned)(row[i] / bh) << cb) | (unsigned)(col[i] / bw);
    idx[i] = (unsigned)i;
}

// flag[] has been scanned in place (exclusive): a key change at p starts block flag[p]
__global__ void __launch_bounds__(kLT) block_list_kernel(const uint64_t* __restrict__ keys, const unsigned* __restrict__ start,
                                                         long long n, int cb, int bw, int* __restrict__ colid,
                                                         unsigned* __restrict__ rowcnt)
{
    const long long p = (long long)blockIdx.x * kLT + threadIdx.x;
    if (p >= n) return;
    const bool head = p == 0 || keys[p] != keys[p - 1];
    if (!head) return;
    const uint64_t k = keys[p];
    colid[start[p]] = (int)(k & ((1ull << cb) - 1ull)) * bw;
    atomicAdd(rowcnt + (k >> cb), 1u);
}

__global__ void __launch_bounds__(kLT) block_winner_kernel(const uint64_t* __restrict__ keys, const unsigned* __restrict__ idx,
                                                           const unsigned* __restrict__ start, long long n,
                                                           const int* __restrict__ row, const int* __restrict__ col, int bw,
                                                           int bh, int al, int* __restrict__ winner)
{
    const long long p = (long long)blockIdx.x * kLT + threadIdx.x;
    if (p >= n) return;
    const bool head = p == 0 || keys[p] != keys[p - 1];
    const unsigned blk = start[p] - (head ? 0u : 1u);
    const int e = (int)idx[p], r = row[e], c = col[e];
    const int inner = (r % bh) * bw + c % bw;
    atomicMax(winner + (size_t)inner * al + blk, e);
}

__global__ void __launch_bounds__(kLT) block_place_kernel(const uint64_t* __restrict__ keys, const unsigned* __restrict__ idx,
                                                          const unsigned* __restrict__ start, long long n,
                                                          const int* __restrict__ row, const int* __restrict__ col,
                                                          const float* __restrict__ val, int bw, int bh, int al,
                                                          const int* __restrict__ winner, float* __restrict__ data)
{
    const long long p = (long long)blockIdx.x * kLT + threadIdx.x;
    if (p >= n) return;
    const bool head = p == 0 || keys[p] != keys[p - 1];
    const unsigned blk = start[p] - (head ? 0u : 1u);
    const int e = (int)idx[p], r = row[e], c = col[e];
    const size_t q = (size_t)((r % bh) * bw + c % bw) * al + blk;
    if (winner[q] == e) data[q] = val[e];
}

template <class T>
T* host_alloc(size_t n, bool zero = false)
{
    if (n == 0) n = 1;
    return static_cast<T*>(zero ? calloc(n, sizeof(T)) : malloc(n * sizeof(T)));
}

int upload_coo(const coo_matrix_if* s, DMem& row, DMem& col, DMem& val)
{
    const size_t n = (size_t)s->matinfo.nnz;
    LCUDA(cudaMalloc(&row.p, n * 4));
    LCUDA(cudaMalloc(&col.p, n * 4));
    LCUDA(cudaMalloc(&val.p, n * 4));
    LCUDA(cudaMemcpy(row.p, s->coo_row_id, n * 4, cudaMemcpyHostToDevice));
    LCUDA(cudaMemcpy(col.p, s->coo_col_id, n * 4, cudaMemcpyHostToDevice));
    LCUDA(cudaMemcpy(val.p, s->coo_data, n * 4, cudaMemcpyHostToDevice));
    return CSP_OK;
}

int need_device(const char* what)
{
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return set_error(CSP_ENODEV, "%s needs a CUDA device", what);
    return CSP_OK;
}

int coo2dia_device(coo_matrix_if* s, dia_matrix_iif* d, int alignment)
{
    d->matinfo = s->matinfo;
    const int h = s->matinfo.height, w = s->matinfo.width, nnz = s->matinfo.nnz;
    d->dia_length = std::min(w, h);
    const int len = csp_aligned_length(d->dia_length, alignment);
    if (nnz == 0) {
        d->dia_num = 0;
        d->dia_length_aligned = len;
        d->dia_offsets = host_alloc<int>(0);
        d->dia_data = host_alloc<float>(0);
        if (!d->dia_offsets || !d->dia_data) return set_error(CSP_ENOMEM, "coo2dia");
        return CSP_OK;
    }
    if (nnz >= kAbsent) return set_error(CSP_EUNSUP, "coo2dia on the device: too many entries");
    const long long n = nnz;
    DMem row, col, val, k0, k1, v0, v1, start, bad, eslot;
    int rc = upload_coo(s, row, col, val);
    if (rc) return rc;
    LCUDA(cudaMalloc(&k0.p, n * 8));
    LCUDA(cudaMalloc(&k1.p, n * 8));
    LCUDA(cudaMalloc(&v0.p, n * 4));
    LCUDA(cudaMalloc(&v1.p, n * 4));
    LCUDA(cudaMalloc(&start.p, n * 4));
    LCUDA(cudaMalloc(&eslot.p, n * 4));
    LCUDA(cudaMalloc(&bad.p, 4));
    LCUDA(cudaMemset(bad.p, 0x7f, 4));
    cudaStream_t st = nullptr;
    dia_keys_kernel<<<grid_of(n), kLT, 0, st>>>(row.as<int>(), col.as<int>(), nnz, h, len, k0.as<uint64_t>(),
                                                 v0.as<unsigned>(), bad.as<int>());
    LCUDA(cudaGetLastError());
    uint64_t* keys = nullptr;
    unsigned* idx = nullptr;
    if ((rc = device_radix_sort_pairs(k0.as<uint64_t>(), k1.as<uint64_t>(), v0.as<unsigned>(), v1.as<unsigned>(), n,
                                      bits_for((long long)h + w - 2), st, &keys, &idx)))
        return rc;
    key_change_kernel<<<grid_of(n), kLT, 0, st>>>(keys, n, start.as<unsigned>());
    LCUDA(cudaGetLastError());
    unsigned last_flag = 0, last_start = 0;
    LCUDA(cudaMemcpy(&last_flag, start.as<unsigned>() + n - 1, 4, cudaMemcpyDeviceToHost));
    if ((rc = device_exclusive_scan(start.as<unsigned>(), (size_t)n, st))) return rc;
    LCUDA(cudaMemcpy(&last_start, start.as<unsigned>() + n - 1, 4, cudaMemcpyDeviceToHost));
    const int D = (int)(last_start + last_flag);
    DMem doffs, dfirsts;
    LCUDA(cudaMalloc(&doffs.p, (size_t)D * 4));
    LCUDA(cudaMalloc(&dfirsts.p, (size_t)D * 4));
    dia_groups_kernel<<<grid_of(n), kLT, 0, st>>>(keys, idx, start.as<unsigned>(), n, h, doffs.as<int>(), dfirsts.as<int>(),
                                                   eslot.as<unsigned>());
    LCUDA(cudaGetLastError());
    std::vector<int> offs((size_t)D), firsts((size_t)D);
    int badrow = kAbsent;
    LCUDA(cudaMemcpy(offs.data(), doffs.p, (size_t)D * 4, cudaMemcpyDeviceToHost));
    LCUDA(cudaMemcpy(firsts.data(), dfirsts.p, (size_t)D * 4, cudaMemcpyDeviceToHost));
    LCUDA(cudaMemcpy(&badrow, bad.p, 4, cudaMemcpyDeviceToHost));
    // The host build rejects when it meets a new diagonal while the K it already holds
    // cover 2 * nnz slots (K * len >= 2 * nnz), i.e. at the first entry of the
    // (K + 1)-th diagonal in input order; a row beyond the length fails at its entry.
    long long K = D;   // diagonals allowed before the rejection
    if (len > 0) K = (2LL * nnz + len - 1) / len;
    else K = 0;
    long long reject_at = LLONG_MAX;
    if ((long long)D > K) {
        std::nth_element(firsts.begin(), firsts.begin() + K, firsts.end());
        reject_at = firsts[(size_t)K];
    }
    if (badrow != kAbsent && (long long)badrow <= reject_at)
        return set_error(CSP_EFORMAT, "coo2dia: row %d beyond the diagonal length %d", s->coo_row_id[badrow], len);
    if (reject_at != LLONG_MAX) {
        d->dia_num = (int)K;
        d->dia_length_aligned = len;
        d->dia_offsets = nullptr;
        d->dia_data = nullptr;
        return set_error(CSP_EFORMAT, "coo2dia: too much padding for the DIA format");
    }
    const size_t cells = (size_t)D * len;
    DMem data, winner;
    LCUDA(cudaMalloc(&data.p, std::max<size_t>(cells, 1) * 4));
    LCUDA(cudaMalloc(&winner.p, std::max<size_t>(cells, 1) * 4));
    LCUDA(cudaMemset(data.p, 0, cells * 4));
    LCUDA(cudaMemset(winner.p, 0xff, cells * 4));
    dia_winner_kernel<<<grid_of(n), kLT, 0, st>>>(row.as<int>(), nnz, len, eslot.as<unsigned>(), winner.as<int>());
    LCUDA(cudaGetLastError());
    dia_place_kernel<<<grid_of(n), kLT, 0, st>>>(row.as<int>(), val.as<float>(), nnz, len, eslot.as<unsigned>(),
                                                  winner.as<int>(), data.as<float>());
    LCUDA(cudaGetLastError());
    d->dia_num = D;
    d->dia_length_aligned = len;
    d->dia_offsets = host_alloc<int>((size_t)D);
    d->dia_data = host_alloc<float>(cells);
    if (!d->dia_offsets || !d->dia_data) return set_error(CSP_ENOMEM, "coo2dia");
    memcpy(d->dia_offsets, offs.data(), (size_t)D * 4);   // `offs` is still in ascending order
    LCUDA(cudaMemcpy(d->dia_data, data.p, cells * 4, cudaMemcpyDeviceToHost));
    return CSP_OK;
}

int coo2bcsr_device(coo_matrix_if* s, bcsr_matrix_if* d, unsigned bw, unsigned bh, int alignment)
{
    int rc = ensure_sorted(s);
    if (rc) return rc;
    d->matinfo = s->matinfo;
    d->bcsr_bwidth = bw;
    d->bcsr_bheight = bh;
    const int h = s->matinfo.height, w = s->matinfo.width, nnz = s->matinfo.nnz;
    const int brows = h / (int)bh + (h % (int)bh != 0);
    const unsigned bs = bw * bh;
    d->bcsr_row_num = brows;
    d->bcsr_row_ptr = host_alloc<int>((size_t)brows + 1);
    if (!d->bcsr_row_ptr) return set_error(CSP_ENOMEM, "coo2bcsr");
    if (nnz == 0) {
        const int al = csp_aligned_length(0, alignment);
        memset(d->bcsr_row_ptr, 0, ((size_t)brows + 1) * 4);
        d->bcsr_aligned_size = al;
        d->bcsr_block_num = 0;
        d->bcsr_col_id = host_alloc<int>(0);
        d->bcsr_data = host_alloc<float>((size_t)al * bs, true);
        if (!d->bcsr_col_id || !d->bcsr_data) return set_error(CSP_ENOMEM, "coo2bcsr");
        return CSP_OK;
    }
    const int cb = bits_for(((long long)std::max(w, 1) - 1) / bw);
    const int rb = bits_for((long long)brows - 1);
    DMem row, col, val, k0, k1, v0, v1, start, cnt;
    if ((rc = upload_coo(s, row, col, val))) return rc;
    const long long n = nnz;
    LCUDA(cudaMalloc(&k0.p, n * 8));
    LCUDA(cudaMalloc(&k1.p, n * 8));
    LCUDA(cudaMalloc(&v0.p, n * 4));
    LCUDA(cudaMalloc(&v1.p, n * 4));
    LCUDA(cudaMalloc(&start.p, n * 4));
    LCUDA(cudaMalloc(&cnt.p, ((size_t)brows + 1) * 4));
    cudaStream_t st = nullptr;
    block_keys_kernel<<<grid_of(n), kLT, 0, st>>>(row.as<int>(), col.as<int>(), nnz, (int)bw, (int)bh, cb, k0.as<uint64_t>(),
                                                   v0.as<unsigned>());
    LCUDA(cudaGetLastError());
    uint64_t* keys = nullptr;
    unsigned* idx = nullptr;
    if ((rc = device_radix_sort_pairs(k0.as<uint64_t>(), k1.as<uint64_t>(), v0.as<unsigned>(), v1.as<unsigned>(), n, rb + cb,
                                      st, &keys, &idx)))
        return rc;
    key_change_kernel<<<grid_of(n), kLT, 0, st>>>(keys, n, start.as<unsigned>());
    LCUDA(cudaGetLastError());
    unsigned last_flag = 0, last_start = 0;
    LCUDA(cudaMemcpy(&last_flag, start.as<unsigned>() + n - 1, 4, cudaMemcpyDeviceToHost));
    if ((rc = device_exclusive_scan(start.as<unsigned>(), (size_t)n, st))) return rc;
    LCUDA(cudaMemcpy(&last_start, start.as<unsigned>() + n - 1, 4, cudaMemcpyDeviceToHost));
    const int nb = (int)(last_start + last_flag);
    const int al = csp_aligned_length(nb, alignment);
    DMem colid, data, winner;
    LCUDA(cudaMalloc(&colid.p, (size_t)nb * 4));
    LCUDA(cudaMemset(cnt.p, 0, ((size_t)brows + 1) * 4));
    block_list_kernel<<<grid_of(n), kLT, 0, st>>>(keys, start.as<unsigned>(), n, cb, (int)bw, colid.as<int>(),
                                                   cnt.as<unsigned>());
    LCUDA(cudaGetLastError());
    if ((rc = device_exclusive_scan(cnt.as<unsigned>(), (size_t)brows + 1, st))) return rc;
    const size_t cells = (size_t)al * bs;
    LCUDA(cudaMalloc(&data.p, std::max<size_t>(cells, 1) * 4));
    LCUDA(cudaMalloc(&winner.p, std::max<size_t>(cells, 1) * 4));
    LCUDA(cudaMemset(data.p, 0, cells * 4));
    LCUDA(cudaMemset(winner.p, 0xff, cells * 4));
    block_winner_kernel<<<grid_of(n), kLT, 0, st>>>(keys, idx, start.as<unsigned>(), n, row.as<int>(), col.as<int>(), (int)bw,
                                                     (int)bh, al, winner.as<int>());
    LCUDA(cudaGetLastError());
    block_place_kernel<<<grid_of(n), kLT, 0, st>>>(keys, idx, start.as<unsigned>(), n, row.as<int>(), col.as<int>(),
                                                    val.as<float>(), (int)bw, (int)bh, al, winner.as<int>(), data.as<float>());
    LCUDA(cudaGetLastError());
    d->bcsr_aligned_size = al;
    d->bcsr_block_num = nb;
    d->bcsr_col_id = host_alloc<int>((size_t)nb);
    d->bcsr_data = host_alloc<float>(cells);
    if (!d->bcsr_col_id || !d->bcsr_data) return set_error(CSP_ENOMEM, "coo2bcsr");
    LCUDA(cudaMemcpy(d->bcsr_row_ptr, cnt.p, ((size_t)brows + 1) * 4, cudaMemcpyDeviceToHost));
    LCUDA(cudaMemcpy(d->bcsr_col_id, colid.p, (size_t)nb * 4, cudaMemcpyDeviceToHost));
    LCUDA(cudaMemcpy(d->bcsr_data, data.p, cells * 4, cudaMemcpyDeviceToHost));
    return CSP_OK;
}

}  // namespace
}  // namespace csp

extern "C" int csp_coo2dia_device(coo_matrix_if* s, dia_matrix_iif* d, int alignment)
{
    using namespace csp;
    clear_error();
    int rc = check_coo(s);
    if (rc || !d) return rc ? rc : set_error(CSP_EINVAL, "null DIA");
    if ((rc = need_device("csp_coo2dia_device"))) return rc;
    return coo2dia_device(s, d, alignment);
}

extern "C" int csp_coo2bdia_device(coo_matrix_if* s, bdia_matrix_iif* d, int alignment)
{
    using namespace csp;
    clear_error();
    if (!d) return set_error(CSP_EINVAL, "null BDIA");
    dia_matrix_iif dia;
    csp_init_dia_matrix(&dia);
    int rc = check_coo(s);
    if (!rc) rc = need_device("csp_coo2bdia_device");
    if (!rc) rc = coo2dia_device(s, &dia, alignment);
    d->matinfo = s ? s->matinfo : d->matinfo;
    if (rc) return rc;
    return bdia_from_dia(&dia, d);
}

extern "C" int csp_coo2bcsr_device(coo_matrix_if* s, bcsr_matrix_if* d, unsigned bw, unsigned bh, int alignment)
{
    using namespace csp;
    clear_error();
    int rc = check_coo(s);
    if (rc || !d) return rc ? rc : set_error(CSP_EINVAL, "null BCSR");
    if (bw == 0 || bh == 0) return set_error(CSP_EINVAL, "coo2bcsr: zero block size");
    if ((rc = need_device("csp_coo2bcsr_device"))) return rc;
    return coo2bcsr_device(s, d, bw, bh, alignment);
}
