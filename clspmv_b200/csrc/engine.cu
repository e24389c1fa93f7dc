// Device engine of the Cocktail SpMV: uploads every sub-matrix of a cocktail,
// selects one kernel per sub-matrix and launches them into one accumulated
// result, the role of clSpMV_NV/src/spmv_cocktail.cpp (init_mat_kernels :1593,
// do_spmv :1091, the cpy_* functions :1462-1591, free_mat_kernels :1616).
//
// Launch order per SpMV is the reference's (do_spmv :1091-1135): BDIA, DIA,
// SBELL, BELL, BCSR, SELL, ELL, CSR, COO (segment pass + fix-up pass).  Every
// kernel reads x and read-modify-writes y on one stream, so the parts compose
// without synchronisation; with CSP_FLAG_GRAPH the whole sequence is one CUDA
// graph replayed per SpMV.
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "csp/clspmv.h"
#include "internal.h"
#include "engine.h"
#include "kernels/flat.cuh"
#include "kernels/diag.cuh"
#include "kernels/block.cuh"
#include "kernels/spmm.cuh"
#include "kernels/xpanel.cuh"

namespace csp {

static thread_local std::string g_last_error;

int set_error(int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

void clear_error() { g_last_error.clear(); }

int cuda_error(cudaError_t e, const char* what)
{
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
        return set_error(CSP_ENODEV, "%s: %s", what, cudaGetErrorString(e));
    if (e == cudaErrorMemoryAllocation) return set_error(CSP_ENOMEM, "%s: %s", what, cudaGetErrorString(e));
    return set_error(CSP_ECUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define CSP_CUDA(call)                                              \
    do {                                                            \
        cudaError_t _e = (call);                                    \
        if (_e != cudaSuccess) return cuda_error(_e, #call);        \
    } while (0)

// --------------------------------------------------------------------------
// device memory
// --------------------------------------------------------------------------
int Engine::alloc(void** p, size_t bytes)
{
    *p = nullptr;
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) return cuda_error(e, "cudaMalloc");
    allocations.push_back(*p);
    device_bytes += bytes;
    return CSP_OK;
}

// Copies n host ints to a new device array of at least `cap` entries (zero tail).
int Engine::upload_int(int** d, const int* h, size_t n, size_t cap)
{
    cap = std::max(cap, n);
    int rc = alloc(reinterpret_cast<void**>(d), cap * sizeof(int));
    if (rc) return rc;
    if (cap > n) CSP_CUDA(cudaMemset(*d + n, 0, (cap - n) * sizeof(int)));
    if (n) CSP_CUDA(cudaMemcpy(*d, h, n * sizeof(int), cudaMemcpyHostToDevice));
    return CSP_OK;
}

// Matrix values in the handle's storage type (FP32, or BF16 with CSP_FLAG_BF16).
int Engine::upload_val(void** d, const float* h, size_t n, size_t cap)
{
    cap = std::max(cap, n);
    const size_t es = bf16 ? 2 : 4;
    int rc = alloc(d, cap * es);
    if (rc) return rc;
    if (cap > n) CSP_CUDA(cudaMemset(static_cast<char*>(*d) + n * es, 0, (cap - n) * es));
    if (!n) return CSP_OK;
    if (!bf16) {
        CSP_CUDA(cudaMemcpy(*d, h, n * 4, cudaMemcpyHostToDevice));
    } else {
        std::vector<uint16_t> t(n);
        for (size_t i = 0; i < n; i++) t[i] = to_bf16(h[i]);
        CSP_CUDA(cudaMemcpy(*d, t.data(), n * 2, cudaMemcpyHostToDevice));
    }
    return CSP_OK;
}

Engine::~Engine()
{
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    for (auto& kv : iter_graphs) if (kv.second) cudaGraphExecDestroy(kv.second);
    if (l2_window && own_stream) {
        // drop the window and return the persisting lines to normal use
        cudaStreamAttrValue attr = {};
        attr.accessPolicyWindow.num_bytes = 0;
        cudaStreamSetAttribute(own_stream, cudaStreamAttributeAccessPolicyWindow, &attr);
        cudaCtxResetPersistingL2Cache();
    }
    for (void* p : allocations) cudaFree(p);
    if (own_stream) cudaStreamDestroy(own_stream);
}

static inline int pad_to(int v, int a) { return (v + a - 1) / a * a; }

// Every column id a kernel will dereference must lie in [0, hi): a struct filled by
// hand with a stray index is refused here instead of faulting on the device.
static int check_ids(const int* ids, size_t n, long long hi, const char* what)
{
    for (size_t i = 0; i < n; i++)
        if (ids[i] < 0 || ids[i] >= hi) return set_error(CSP_EINVAL, "%s: index %d at %zu outside [0, %lld)", what, ids[i], i, hi);
    return CSP_OK;
}

static int check_row_ptr(const int* rp, int rows, const char* what)
{
    if (rp[0] != 0) return set_error(CSP_EINVAL, "%s: row pointer does not start at 0", what);
    for (int i = 0; i < rows; i++)
        if (rp[i + 1] < rp[i]) return set_error(CSP_EINVAL, "%s: row pointer decreases at %d", what, i);
    return CSP_OK;
}
static inline unsigned grid_for(long long threads, int block) { return (unsigned)((threads + block - 1) / block); }

// CSR adaptive work blocks: chunks of rows longer than kAdaptNnz first, then runs of
// whole rows (at most kAdaptThreads rows, at most kAdaptNnz entries each).
void make_adaptive_blocks(const int* rp, int m, std::vector<int4>& blocks, std::vector<int4>& longs, int& nslots)
{
    std::vector<int4> runs;
    blocks.clear();
    longs.clear();
    nslots = 0;
    int r = 0;
    while (r < m) {
        const int len = rp[r + 1] - rp[r];
        if (len > dev::kAdaptNnz) {
            const int lid = (int)longs.size();
            const int nch = (len + dev::kAdaptNnz - 1) / dev::kAdaptNnz;
            longs.push_back(make_int4(r, nslots, nch, 0));
            for (int k = 0; k < nch; k++)
                blocks.push_back(make_int4(k, -(lid + 1), rp[r] + k * dev::kAdaptNnz,
                                           std::min(rp[r] + (k + 1) * dev::kAdaptNnz, rp[r + 1])));
            nslots += nch;
            r++;
            continue;
        }
        const int start = r;
        long long acc = 0;
        while (r < m && r - start < dev::kAdaptThreads) {
            const int l = rp[r + 1] - rp[r];
            if (l > dev::kAdaptNnz || acc + l > dev::kAdaptNnz) break;
            acc += l;
            r++;
        }
        runs.push_back(make_int4(start, r - start, rp[start], rp[r]));
    }
    blocks.insert(blocks.end(), runs.begin(), runs.end());
}

// --------------------------------------------------------------------------
// Per-format setup.  Each validates the struct, uploads it and fixes the launch.
// --------------------------------------------------------------------------
int Engine::add_csr(const csr_matrix_if& c, int method)
{
    const int m = c.matinfo.height;
    if (m < 0 || !c.csr_row_ptr) return set_error(CSP_EINVAL, "CSR part: bad row pointer");
    const int nnz = c.csr_row_ptr[m];
    if (nnz < 0 || (nnz > 0 && (!c.csr_col_id || !c.csr_data))) return set_error(CSP_EINVAL, "CSR part: bad arrays");
    if (m > height) return set_error(CSP_EINVAL, "CSR part taller than the cocktail");
    int rc;
    if ((rc = check_row_ptr(c.csr_row_ptr, m, "CSR part")) || (rc = check_ids(c.csr_col_id, nnz, width, "CSR part")))
        return rc;
    if (method == CSP_METH_XPANEL) {
        if (nrhs > 1) return set_error(CSP_EUNSUP, "x-panel CSR part with several right-hand sides");
        std::vector<int> rows((size_t)nnz);
        for (int r = 0; r < m; r++)
            for (int j = c.csr_row_ptr[r]; j < c.csr_row_ptr[r + 1]; j++) rows[j] = r;
        return add_xpanel(rows.data(), c.csr_col_id, c.csr_data, nnz, true);
    }
    Part p;
    p.kind = PART_CSR;
    p.method = method;
    p.m = m;
    p.nnz = nnz;
    if (method == 6) {
        // float4 scalar kernel on the row-padded CSR (util.cpp:31 pad_csr with 4)
        csr_matrix_if padded;
        csp_init_csr_matrix(&padded);
        rc = csp_pad_csr(&c, &padded, 4);
        if (rc) { csp_free_csr_matrix(&padded); return rc; }
        const int pn = padded.matinfo.nnz;
        if ((rc = upload_int(&p.i0, padded.csr_row_ptr, (size_t)m + 1, (size_t)m + 1)) ||
            (rc = upload_int(&p.i1, padded.csr_col_id, pn, (size_t)pad_to(pn, 4) + 4)) ||
            (rc = upload_val(&p.v, padded.csr_data, pn, (size_t)pad_to(pn, 4) + 4))) {
            csp_free_csr_matrix(&padded);
            return rc;
        }
        csp_free_csr_matrix(&padded);
    } else {
        if ((rc = upload_int(&p.i0, c.csr_row_ptr, (size_t)m + 1, (size_t)m + 1)) ||
            (rc = upload_int(&p.i1, c.csr_col_id, nnz, (size_t)pad_to(nnz, 4) + 4)) ||
            (rc = upload_val(&p.v, c.csr_data, nnz, (size_t)pad_to(nnz, 4) + 4)))
            return rc;
    }
    if (method == 2) {
        std::vector<int4> blocks, longs;
        int nslots = 0;
        make_adaptive_blocks(c.csr_row_ptr, m, blocks, longs, nslots);
        p.nblocks = (int)blocks.size();
        if ((rc = alloc(reinterpret_cast<void**>(&p.blocks), std::max<size_t>(blocks.size(), 1) * sizeof(int4))) ||
            (rc = alloc(reinterpret_cast<void**>(&p.long_rows), std::max<size_t>(longs.size(), 1) * sizeof(int4))) ||
            (rc = alloc(reinterpret_cast<void**>(&p.scratch_val), std::max(nslots, 1) * sizeof(float))) ||
            (rc = alloc(reinterpret_cast<void**>(&p.scratch_row), std::max<size_t>(longs.size(), 1) * sizeof(int))))
            return rc;
        if (!blocks.empty()) CSP_CUDA(cudaMemcpy(p.blocks, blocks.data(), blocks.size() * sizeof(int4), cudaMemcpyHostToDevice));
        if (!longs.empty()) CSP_CUDA(cudaMemcpy(p.long_rows, longs.data(), longs.size() * sizeof(int4), cudaMemcpyHostToDevice));
        CSP_CUDA(cudaMemset(p.scratch_row, 0, std::max<size_t>(longs.size(), 1) * sizeof(int)));   // arrival counters
    }
    if (method == 3) {
        const double mean = m ? (double)nnz / m : 0.0;
        int g = 2;
        while (g < 32 && g * 2 <= mean) g *= 2;  // ~ one 4-wide vector per lane per row
        p.group = g;
    }
    parts.push_back(p);
    return CSP_OK;
}

int Engine::add_coo(const coo_matrix_if& c, int method)
{
    const int nnz = c.matinfo.nnz;
    if (nnz < 0 || (nnz > 0 && (!c.coo_row_id || !c.coo_col_id || !c.coo_data)))
        return set_error(CSP_EINVAL, "COO part: bad arrays");
    if (nnz == 0) return CSP_OK;
    for (int i = 0; i + 1 < nnz; i++)
        if (c.coo_row_id[i] > c.coo_row_id[i + 1]) return set_error(CSP_EINVAL, "COO part: rows not sorted");
    for (int i = 0; i < nnz; i++)
        if (c.coo_row_id[i] < 0 || c.coo_row_id[i] >= height || c.coo_col_id[i] < 0 || c.coo_col_id[i] >= width)
            return set_error(CSP_EINVAL, "COO part: entry %d out of range", i);
    if (method == CSP_METH_XPANEL) return add_xpanel(c.coo_row_id, c.coo_col_id, c.coo_data, nnz, false);
    Part p;
    p.kind = PART_COO;
    p.method = 0;
    p.nnz = nnz;
    // pad to whole 128-entry tiles with (last row, last col, 0.0)
    const int npad = pad_to(nnz, 128);
    std::vector<int> r(c.coo_row_id, c.coo_row_id + nnz), cl(c.coo_col_id, c.coo_col_id + nnz);
    std::vector<float> v(c.coo_data, c.coo_data + nnz);
    r.resize(npad, c.coo_row_id[nnz - 1]);
    cl.resize(npad, c.coo_col_id[nnz - 1]);
    v.resize(npad, 0.0f);
    p.npad = npad;
    p.nwarps = (npad + dev::kCooChunk - 1) / dev::kCooChunk;
    int rc;
    if ((rc = upload_int(&p.i0, r.data(), npad, npad)) || (rc = upload_int(&p.i1, cl.data(), npad, npad)) ||
        (rc = upload_val(&p.v, v.data(), npad, npad)))
        return rc;
    // rows that cross a chunk boundary ("spans", see coo_segment_kernel)
    std::vector<int> span_head((size_t)p.nwarps, -1);
    std::vector<int4> spans;
    for (int w = 1; w < p.nwarps; w++) {
        const int b = w * dev::kCooChunk;
        if (r[b - 1] != r[b]) continue;
        if (!spans.empty() && spans.back().x == r[b] && spans.back().y + spans.back().z == w) spans.back().z++;
        else spans.push_back(make_int4(r[b], w - 1, 2, 0));
        span_head[w] = (int)spans.size() - 1;
    }
    const size_t ns = std::max<size_t>(spans.size(), 1);
    if ((rc = upload_int(&p.span_head, span_head.data(), span_head.size(), span_head.size())) ||
        (rc = alloc(reinterpret_cast<void**>(&p.spans), ns * sizeof(int4))) ||
        (rc = alloc(reinterpret_cast<void**>(&p.scratch_row), ns * sizeof(int))) ||
        (rc = alloc(reinterpret_cast<void**>(&p.scratch_val), (size_t)2 * p.nwarps * sizeof(float))))
        return rc;
    if (!spans.empty()) CSP_CUDA(cudaMemcpy(p.spans, spans.data(), spans.size() * sizeof(int4), cudaMemcpyHostToDevice));
    CSP_CUDA(cudaMemset(p.scratch_row, 0, ns * sizeof(int)));   // arrival counters
    parts.push_back(p);
    return CSP_OK;
}

// x-panel layout (kernels/xpanel.cuh) of nnz entries sorted by row, indices already
// validated.  Entries are regrouped by column panel (stable, so rows stay sorted inside
// a panel), each panel padded to whole tiles; runs of one row inside a tile get slots
// numbered row by row, in panel order inside a row.
int Engine::add_xpanel(const int* rows, const int* cols, const float* vals, int nnz, bool from_csr)
{
    using dev::kXpTile;
    if (nnz == 0) return CSP_OK;
    Part p;
    p.kind = PART_XPANEL;
    p.method = CSP_METH_XPANEL;
    p.nnz = nnz;
    p.from_csr = from_csr;
    // the widest panel that fits beside the tile rings in one CTA's shared memory
    int dev_id = 0, optin = 0, sms = 0;
    CSP_CUDA(cudaGetDevice(&dev_id));
    CSP_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev_id));
    CSP_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev_id));
    const size_t ring = bf16 ? dev::xpanel_ring_bytes<__nv_bfloat16>() : dev::xpanel_ring_bytes<float>();
    const long long room = ((long long)optin - (long long)ring) / 4 / 64 * 64;
    if (room < 64) return set_error(CSP_EUNSUP, "x-panel part: %d bytes of shared memory per block are too few", optin);
    p.panel_w = (int)std::min<long long>({room, dev::kXpPanelMax, pad_to(std::max(width, 1), 4)});
    const int P = (width + p.panel_w - 1) / p.panel_w;
    p.npanels = P;
    // stable counting sort by panel
    std::vector<long long> cnt((size_t)P + 1, 0);
    for (int i = 0; i < nnz; i++) cnt[(size_t)cols[i] / p.panel_w + 1]++;
    std::vector<int> tile0((size_t)P + 1, 0);
    for (int q = 0; q < P; q++) {
        const long long t = tile0[q] + (cnt[q + 1] + kXpTile - 1) / kXpTile;
        if (t >= INT32_MAX / kXpTile) return set_error(CSP_EUNSUP, "x-panel part: too many entries");
        tile0[q + 1] = (int)t;
    }
    for (int q = 0; q < P; q++) cnt[q + 1] += cnt[q];
    std::vector<int> order((size_t)nnz);
    {
        std::vector<long long> next(cnt.begin(), cnt.end() - 1);
        for (int i = 0; i < nnz; i++) order[(size_t)next[(size_t)cols[i] / p.panel_w]++] = i;
    }
    const int T = tile0[P];
    const size_t slots_len = (size_t)T * kXpTile;
    // a run starts at every tile start and every row change
    auto starts_run = [&](long long j, long long b) {
        return (j - b) % kXpTile == 0 || rows[order[(size_t)j - 1]] != rows[order[(size_t)j]];
    };
    std::vector<int> nruns((size_t)height, 0);
    for (int q = 0; q < P; q++)
        for (long long j = cnt[q]; j < cnt[q + 1]; j++)
            if (starts_run(j, cnt[q])) nruns[rows[order[(size_t)j]]]++;
    // rows of one run add it to y from the main kernel (one writer, no slot); the
    // others are listed with their slot ranges for the merge
    std::vector<int> run_ptr, run_rows;
    std::vector<long long> first((size_t)height, -1);
    run_ptr.push_back(0);
    long long total = 0;
    for (int r = 0; r < height; r++) {
        if (nruns[r] < 2) continue;
        first[r] = total;
        total += nruns[r];
        run_rows.push_back(r);
        run_ptr.push_back((int)total);
    }
    if (total >= INT32_MAX) return set_error(CSP_EUNSUP, "x-panel part: too many runs");
    // per-entry slots (or -(row + 1) for a one-run row), panel-local columns and values
    // in tile order
    std::vector<int> slot(slots_len, 0);
    std::vector<unsigned short> lcol(slots_len, 0);
    std::vector<float> val(slots_len, 0.0f);
    for (int q = 0; q < P; q++) {
        const long long b = cnt[q], e = cnt[q + 1];
        const size_t o = (size_t)tile0[q] * kXpTile;
        int cur = 0;
        for (long long j = b; j < e; j++) {
            const int i = order[(size_t)j];
            if (starts_run(j, b)) cur = nruns[rows[i]] == 1 ? -(rows[i] + 1) : (int)(first[rows[i]]++);
            slot[o + (size_t)(j - b)] = cur;
            lcol[o + (size_t)(j - b)] = (unsigned short)(cols[i] - q * p.panel_w);
            val[o + (size_t)(j - b)] = vals[i];
        }
        // pad entries extend the panel's last run (0 * x[panel start])
        for (long long j = e - b; j % kXpTile != 0; j++) slot[o + (size_t)j] = cur;
    }
    p.ntiles = T;
    p.nrun_rows = (int)run_rows.size();
    const bool all_rows = p.nrun_rows == height;
    // listed rows with many slots, merged by a lane group each
    std::vector<int> long_list;
    for (int i = 0; i < p.nrun_rows; i++)
        if (run_ptr[i + 1] - run_ptr[i] > dev::kXpShortRuns) long_list.push_back(i);
    p.nlong = (int)long_list.size();

    int rc;
    if ((rc = upload_int(&p.i0, slot.data(), slots_len, slots_len)) ||
        (rc = upload_val(&p.v, val.data(), slots_len, slots_len)) ||
        (rc = alloc(reinterpret_cast<void**>(&p.lcol), slots_len * sizeof(unsigned short))) ||
        (rc = upload_int(&p.tile0, tile0.data(), tile0.size(), tile0.size())) ||
        (rc = upload_int(&p.run_ptr, run_ptr.data(), run_ptr.size(), run_ptr.size())) ||
        (rc = alloc(reinterpret_cast<void**>(&p.partial), std::max<size_t>((size_t)total, 1) * sizeof(float))))
        return rc;
    CSP_CUDA(cudaMemcpy(p.lcol, lcol.data(), slots_len * sizeof(unsigned short), cudaMemcpyHostToDevice));
    if (!all_rows && (rc = upload_int(&p.run_rows, run_rows.data(), run_rows.size(), run_rows.size()))) return rc;
    if ((rc = upload_int(&p.long_list, long_list.data(), long_list.size(), std::max<size_t>(long_list.size(), 1)))) return rc;
    // grid: as many CTAs as fit on the device at once, but no more than the tiles need:
    // each CTA's entries should outweigh the x panel it copies
    p.smem = (size_t)p.panel_w * sizeof(float) + ring;
    auto kern = bf16 ? reinterpret_cast<const void*>(&dev::xpanel_kernel<__nv_bfloat16>)
                     : reinterpret_cast<const void*>(&dev::xpanel_kernel<float>);
    CSP_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p.smem));
    int per_sm = 0;
    CSP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, dev::kXpThreads, p.smem));
    const long long resident = (long long)sms * std::max(per_sm, 1);
    const long long by_work = std::max<long long>(1, (long long)slots_len * 10 / (long long)(p.panel_w * 4));
    p.ncta = (int)std::max<long long>(1, std::min({resident, by_work, (long long)T}));
    parts.push_back(p);
    return CSP_OK;
}

int Engine::add_ell(const ell_matrix_if& e, int method)
{
    const int m = e.matinfo.height;
    if (e.ell_num < 0 || e.ell_height_aligned < m || (e.ell_num > 0 && (!e.ell_col_id || !e.ell_data)))
        return set_error(CSP_EINVAL, "ELL part: bad fields");
    Part p;
    p.kind = PART_ELL;
    p.method = (method == 1 && e.ell_height_aligned % 4 == 0) ? 1 : 0;
    p.m = m;
    p.k = e.ell_num;
    p.stride = e.ell_height_aligned;
    const size_t n = (size_t)e.ell_num * e.ell_height_aligned;
    int rc;
    if (m > height) return set_error(CSP_EINVAL, "ELL part taller than the cocktail");
    if ((rc = check_ids(e.ell_col_id, n, width, "ELL part"))) return rc;   // the 4-row kernel reads alignment rows too
    if ((rc = upload_int(&p.i1, e.ell_col_id, n, n)) || (rc = upload_val(&p.v, e.ell_data, n, n))) return rc;
    parts.push_back(p);
    return CSP_OK;
}

int Engine::add_sell(const sell_matrix_if& s, int method)
{
    const int m = s.matinfo.height;
    const int H = (int)s.sell_slice_height;
    if (H <= 0 || s.sell_slice_num * (long long)H < m || !s.sell_slice_ptr) return set_error(CSP_EINVAL, "SELL part: bad fields");
    const int total = s.sell_slice_ptr[s.sell_slice_num];
    if (total > 0 && (!s.sell_col_id || !s.sell_data)) return set_error(CSP_EINVAL, "SELL part: bad arrays");
    Part p;
    p.kind = PART_SELL;
    p.method = (method != 2 && H % 4 == 0) ? 1 : 0;  // 1: four rows per thread
    p.m = m;
    p.stride = H;
    int rc;
    if (m > height) return set_error(CSP_EINVAL, "SELL part taller than the cocktail");
    for (int i = 0; i < s.sell_slice_num; i++)
        if (s.sell_slice_ptr[i + 1] < s.sell_slice_ptr[i] || (s.sell_slice_ptr[i + 1] - s.sell_slice_ptr[i]) % H != 0 ||
            s.sell_slice_ptr[0] != 0)
            return set_error(CSP_EINVAL, "SELL part: slice pointer %d inconsistent with slice height %d", i, H);
    if ((rc = check_ids(s.sell_col_id, (size_t)total, width, "SELL part"))) return rc;
    if ((rc = upload_int(&p.i0, s.sell_slice_ptr, (size_t)s.sell_slice_num + 1, (size_t)s.sell_slice_num + 1)) ||
        (rc = upload_int(&p.i1, s.sell_col_id, total, total)) || (rc = upload_val(&p.v, s.sell_data, total, total)))
        return rc;
    parts.push_back(p);
    return CSP_OK;
}

int Engine::add_dia(const dia_matrix_iif& d, int method)
{
    const int len = d.dia_length_aligned;
    if (d.dia_num < 0 || len < 0 || (d.dia_num > 0 && (!d.dia_offsets || !d.dia_data)))
        return set_error(CSP_EINVAL, "DIA part: bad fields");
    if (d.dia_num > 12000) return set_error(CSP_EUNSUP, "DIA part: %d diagonals (at most 12000)", d.dia_num);
    Part p;
    p.kind = PART_DIA;
    p.m = std::min(std::min(d.matinfo.height, height), len);
    p.k = d.dia_num;
    p.stride = len;
    p.method = ((method == 1 || method == 3) && len % 4 == 0) ? 1 : 0;
    const size_t n = (size_t)d.dia_num * len;
    int rc;
    if ((rc = upload_int(&p.i0, d.dia_offsets, d.dia_num, d.dia_num)) || (rc = upload_val(&p.v, d.dia_data, n, n))) return rc;
    parts.push_back(p);
    return CSP_OK;
}

int Engine::add_bdia(const bdia_matrix_iif& b, int method)
{
    const int len = b.bdia_length_aligned;
    if (b.bdia_band_num < 0 || len < 0 || (b.bdia_band_num > 0 && (!b.bdia_offsets || !b.bdia_bptr || !b.bdia_data)))
        return set_error(CSP_EINVAL, "BDIA part: bad fields");
    Part p;
    p.kind = PART_BDIA;
    p.m = std::min(std::min(b.matinfo.height, height), len);
    p.k = b.bdia_band_num;
    p.stride = len;
    const int ndia = b.bdia_band_num ? b.bdia_bptr[b.bdia_band_num] : 0;
    int maxw = 1;
    for (int i = 0; i < b.bdia_band_num; i++) maxw = std::max(maxw, b.bdia_bptr[i + 1] - b.bdia_bptr[i]);
    p.maxw = maxw;
    // reference numbering (spmv_cocktail.cpp:339-358): 0 nlvec, 1 staged, 2 staged (g4),
    // 3 v4_nlvec, 4 v4 staged
    p.method = ((method == 0 || method == 3) && len % 4 == 0) ? 0 : 1;
    if (maxw > 8000) p.method = 0;   // staged window would not fit in shared memory
    if (p.method == 0 && len % 4 != 0) return set_error(CSP_EUNSUP, "BDIA part: band wider than 8000 with unaligned length");
    for (int i = 0; i < b.bdia_band_num; i++)
        if (b.bdia_bptr[i + 1] < b.bdia_bptr[i] || b.bdia_bptr[0] != 0) return set_error(CSP_EINVAL, "BDIA part: bad band pointer");
    const size_t n = (size_t)ndia * len;
    int rc;
    if ((rc = upload_int(&p.i0, b.bdia_offsets, b.bdia_band_num, b.bdia_band_num)) ||
        (rc = upload_int(&p.i1, b.bdia_bptr, (size_t)b.bdia_band_num + 1, (size_t)b.bdia_band_num + 1)) ||
        (rc = upload_val(&p.v, b.bdia_data, n, n)))
        return rc;
    parts.push_back(p);
    return CSP_OK;
}

static bool b4_shape_ok(unsigned bw, unsigned bh)
{
    return (bw == 4 || bw == 8) && (bh == 1 || bh == 2 || bh == 4 || bh == 8);
}

int Engine::add_bell(const b4ell_matrix_if& b, int method)
{
    if (!b4_shape_ok(b.b4ell_bwidth, b.b4ell_bheight)) return set_error(CSP_EUNSUP, "BELL part: block %ux%u", b.b4ell_bheight, b.b4ell_bwidth);
    if (b.b4ell_float4_aligned % 4 != 0 || b.b4ell_float4_aligned < 4 * b.b4ell_row_num || b.b4ell_height_aligned < b.b4ell_row_num)
        return set_error(CSP_EINVAL, "BELL part: bad alignment");
    Part p;
    p.kind = PART_BELL;
    p.method = method;
    p.bw = (int)b.b4ell_bwidth;
    p.bh = (int)b.b4ell_bheight;
    p.m = b.matinfo.height;
    p.nbr = b.b4ell_row_num;
    p.k = b.b4ell_block_num;
    p.stride = b.b4ell_height_aligned;
    p.f4 = b.b4ell_float4_aligned;
    const size_t nc = (size_t)b.b4ell_height_aligned * b.b4ell_block_num;
    const size_t nd = (size_t)b.b4ell_float4_aligned * b.b4ell_bheight * (b.b4ell_bwidth / 4) * b.b4ell_block_num;
    int rc;
    for (int k = 0; k < b.b4ell_block_num; k++)
        if ((rc = check_ids(b.b4ell_col_id + (size_t)k * b.b4ell_height_aligned, (size_t)b.b4ell_row_num,
                            (x_len - (long long)b.b4ell_bwidth) / 4 + 1, "BELL part")))
            return rc;
    if ((rc = upload_int(&p.i1, b.b4ell_col_id, nc, nc)) || (rc = upload_val(&p.v, b.b4ell_data, nd, nd))) return rc;
    parts.push_back(p);
    return CSP_OK;
}

int Engine::add_sbell(const sbell_matrix_if& s, int method)
{
    if (!b4_shape_ok(s.sbell_bwidth, s.sbell_bheight)) return set_error(CSP_EUNSUP, "SBELL part: block %ux%u", s.sbell_bheight, s.sbell_bwidth);
    if (s.sbell_slice_height == 0 || !s.sbell_slice_ptr || s.sbell_slice_num * (long long)s.sbell_slice_height < s.sbell_row_num)
        return set_error(CSP_EINVAL, "SBELL part: bad fields");
    Part p;
    p.kind = PART_SBELL;
    p.method = method;
    p.bw = (int)s.sbell_bwidth;
    p.bh = (int)s.sbell_bheight;
    p.m = s.matinfo.height;
    p.nbr = s.sbell_row_num;
    p.stride = (int)s.sbell_slice_height;
    const int total = s.sbell_slice_ptr[s.sbell_slice_num];
    const size_t nd = (size_t)total * s.sbell_bwidth * s.sbell_bheight;
    int rc;
    for (int i = 0; i < s.sbell_slice_num; i++)
        if (s.sbell_slice_ptr[0] != 0 || s.sbell_slice_ptr[i + 1] < s.sbell_slice_ptr[i] ||
            (s.sbell_slice_ptr[i + 1] - s.sbell_slice_ptr[i]) % (int)s.sbell_slice_height != 0)
            return set_error(CSP_EINVAL, "SBELL part: bad slice pointer");
    if ((rc = check_ids(s.sbell_col_id, (size_t)total, (x_len - (long long)s.sbell_bwidth) / 4 + 1, "SBELL part"))) return rc;
    if ((rc = upload_int(&p.i0, s.sbell_slice_ptr, (size_t)s.sbell_slice_num + 1, (size_t)s.sbell_slice_num + 1)) ||
        (rc = upload_int(&p.i1, s.sbell_col_id, total, total)) || (rc = upload_val(&p.v, s.sbell_data, nd, nd)))
        return rc;
    parts.push_back(p);
    return CSP_OK;
}

int Engine::add_bcsr(const b4csr_matrix_if& b, int method)
{
    if (!b4_shape_ok(b.b4csr_bwidth, b.b4csr_bheight)) return set_error(CSP_EUNSUP, "BCSR part: block %ux%u", b.b4csr_bheight, b.b4csr_bwidth);
    if (b.b4csr_aligned_size % 4 != 0 || b.b4csr_aligned_size < 4 * b.b4csr_block_num || !b.b4csr_row_ptr)
        return set_error(CSP_EINVAL, "BCSR part: bad alignment");
    Part p;
    p.kind = PART_BCSR;
    p.method = method;
    p.bw = (int)b.b4csr_bwidth;
    p.bh = (int)b.b4csr_bheight;
    p.m = b.matinfo.height;
    p.nbr = b.b4csr_row_num;
    p.stride = b.b4csr_aligned_size;
    const size_t nd = (size_t)b.b4csr_aligned_size * b.b4csr_bheight * (b.b4csr_bwidth / 4);
    int rc;
    if ((rc = check_row_ptr(b.b4csr_row_ptr, b.b4csr_row_num, "BCSR part"))) return rc;
    if (b.b4csr_row_ptr[b.b4csr_row_num] > b.b4csr_block_num) return set_error(CSP_EINVAL, "BCSR part: row pointer past the blocks");
    if ((rc = check_ids(b.b4csr_col_id, (size_t)b.b4csr_block_num, (x_len - (long long)b.b4csr_bwidth) / 4 + 1, "BCSR part"))) return rc;
    if ((rc = upload_int(&p.i0, b.b4csr_row_ptr, (size_t)b.b4csr_row_num + 1, (size_t)b.b4csr_row_num + 1)) ||
        (rc = upload_int(&p.i1, b.b4csr_col_id, b.b4csr_block_num, b.b4csr_block_num)) ||
        (rc = upload_val(&p.v, b.b4csr_data, nd, nd)))
        return rc;
    parts.push_back(p);
    return CSP_OK;
}

int Engine::add_generic_bcsr(const bcsr_matrix_if& b, int method)
{
    const unsigned bw = b.bcsr_bwidth, bh = b.bcsr_bheight;
    if (!((bh == 3 && bw == 3) || (bh == 2 && bw == 2) || (bh == 4 && bw == 4) || (bh == 1 && bw == 1) || (bh == 6 && bw == 6) ||
          (bh == 8 && bw == 8)))
        return set_error(CSP_EUNSUP, "generic BCSR: block %ux%u not compiled", bh, bw);
    if (!b.bcsr_row_ptr || b.bcsr_aligned_size < b.bcsr_block_num) return set_error(CSP_EINVAL, "generic BCSR: bad fields");
    Part p;
    p.kind = PART_GBCSR;
    p.method = method;
    p.bw = (int)bw;
    p.bh = (int)bh;
    p.m = b.matinfo.height;
    p.nbr = b.bcsr_row_num;
    p.stride = b.bcsr_aligned_size;
    size_t nd = (size_t)b.bcsr_aligned_size * bw * bh;
    int rc;
    if ((rc = check_row_ptr(b.bcsr_row_ptr, b.bcsr_row_num, "generic BCSR"))) return rc;
    if (b.bcsr_row_ptr[b.bcsr_row_num] > b.bcsr_block_num) return set_error(CSP_EINVAL, "generic BCSR: row pointer past the blocks");
    if ((rc = check_ids(b.bcsr_col_id, (size_t)b.bcsr_block_num, width, "generic BCSR"))) return rc;
    if ((rc = upload_int(&p.i0, b.bcsr_row_ptr, (size_t)b.bcsr_row_num + 1, (size_t)b.bcsr_row_num + 1))) return rc;
    // one right-hand side, blocks of at most 16 elements: work items of whole block rows
    // for the adaptive kernel (kernels/block.cuh bcsr_adaptive_kernel), unless a block
    // row is too long for one CTA
    std::vector<int4> work;
    bool fits = nrhs == 1 && bw * bh <= 16;
    if (fits) {
        const int* rp = b.bcsr_row_ptr;
        int r0 = 0;
        for (int r = 0; r < p.nbr && fits; r++) {
            if (rp[r + 1] - rp[r] > dev::kGbBlocks - 3) fits = false;
            else if (r - r0 == dev::kGbRows || rp[r + 1] - rp[r0] > dev::kGbBlocks - 3) {
                work.push_back(make_int4(r0, r - r0, rp[r0], rp[r]));
                r0 = r;
            }
        }
        if (fits && p.nbr > r0) work.push_back(make_int4(r0, p.nbr - r0, rp[r0], rp[p.nbr]));
        fits = fits && !work.empty();
    }
    const int nblk = b.bcsr_block_num;
    if (!fits) {
        if ((rc = upload_int(&p.i1, b.bcsr_col_id, nblk, (size_t)pad_to(nblk, 4) + 4)) ||
            (rc = upload_val(&p.v, b.bcsr_data, nd, nd)))
            return rc;
    } else {
        // each item at a multiple of 4, its blocks in column order (stable) dealt to the
        // lanes of its 128-block chunks (kernels/block.cuh); tgt = row-order position - s,
        // 0xffff on empty slots
        std::vector<int> perm((size_t)nblk);
        for (int k = 0; k < nblk; k++) perm[k] = k;
        size_t total = 0;
        for (const int4& w : work) total += (size_t)pad_to(w.w - w.z, 4);
        std::vector<int> col(total + 4, 0), src(total, -1);
        std::vector<unsigned short> tgt(col.size(), 0xffff);
        size_t ds = 0;
        for (int4& w : work) {
            const int s = w.z, cnt = w.w - w.z;
            std::stable_sort(perm.begin() + s, perm.begin() + w.w,
                             [&](int a, int c) { return b.bcsr_col_id[a] < b.bcsr_col_id[c]; });
            const int nfull = cnt / 128, tail_lanes = pad_to(cnt - 128 * nfull, 4) / 4;
            for (int rk = 0; rk < cnt; rk++) {
                const int base = rk / 128 * 128, T = rk / 128 < nfull ? 32 : tail_lanes, r = rk - base;
                const size_t slot = ds + (size_t)(base + 4 * (r % T) + r / T);
                src[slot] = perm[s + rk];
                col[slot] = b.bcsr_col_id[perm[s + rk]];
                tgt[slot] = (unsigned short)(perm[s + rk] - s);
            }
            w.y |= cnt << 16;
            w.w = (int)ds;
            ds += (size_t)pad_to(cnt, 4);
        }
        p.stride = (int)total;
        nd = total * bw * bh;
        std::vector<float> data(nd);
        const size_t al = (size_t)b.bcsr_aligned_size;
        for (size_t e = 0; e < (size_t)bw * bh; e++)
            for (size_t k = 0; k < total; k++) data[e * total + k] = src[k] < 0 ? 0.0f : b.bcsr_data[e * al + src[k]];
        if ((rc = upload_int(&p.i1, col.data(), col.size(), col.size())) ||
            (rc = upload_val(&p.v, data.data(), nd, nd)) ||
            (rc = alloc(reinterpret_cast<void**>(&p.lcol), tgt.size() * sizeof(unsigned short))) ||
            (rc = alloc(reinterpret_cast<void**>(&p.blocks), work.size() * sizeof(int4))))
            return rc;
        CSP_CUDA(cudaMemcpy(p.lcol, tgt.data(), tgt.size() * sizeof(unsigned short), cudaMemcpyHostToDevice));
        CSP_CUDA(cudaMemcpy(p.blocks, work.data(), work.size() * sizeof(int4), cudaMemcpyHostToDevice));
        p.nblocks = (int)work.size();
    }
    parts.push_back(p);
    return CSP_OK;
}

// --------------------------------------------------------------------------
// Launches
// --------------------------------------------------------------------------
template <class V>
static void launch_spmm(const Part& p, const float* x, float* y, int n, int k, bool tensor, cudaStream_t st)
{
    using namespace dev;
    const V* v = static_cast<const V*>(p.v);
    if (tensor && p.kind == PART_GBCSR && k % 32 == 0 && p.bh <= 8 && p.bw <= 4) {
        // tensor cores: one warp per block row, two blocks per MMA step
        if (p.nbr == 0) return;
        const unsigned g = grid_for((long long)p.nbr * 32, kMmaThreads);
#define CSP_MMA(BH, BW) \
    bcsr_spmm_mma_kernel<V, BH, BW, 2><<<g, kMmaThreads, 0, st>>>(p.i0, p.i1, v, x, y, p.nbr, p.stride, p.m, n, k)
        switch (p.bh * 10 + p.bw) {
        case 11: CSP_MMA(1, 1); break; case 22: CSP_MMA(2, 2); break; case 33: CSP_MMA(3, 3); break;
        case 44: CSP_MMA(4, 4); break;
        default: break;
        }
#undef CSP_MMA
        if (p.bh * 10 + p.bw == 11 || p.bh * 10 + p.bw == 22 || p.bh * 10 + p.bw == 33 || p.bh * 10 + p.bw == 44) return;
    }
    const int G = k >= 32 ? 32 : (k > 16 ? 32 : (k > 8 ? 16 : (k > 4 ? 8 : (k > 2 ? 4 : 2))));
    if (p.kind == PART_CSR) {
        if (p.m == 0) return;
        const unsigned g = grid_for((long long)p.m * G, kSpmmThreads);
        switch (G) {
        case 2: csr_spmm_kernel<V, 2><<<g, kSpmmThreads, 0, st>>>(p.i0, p.i1, v, x, y, p.m, k); break;
        case 4: csr_spmm_kernel<V, 4><<<g, kSpmmThreads, 0, st>>>(p.i0, p.i1, v, x, y, p.m, k); break;
        case 8: csr_spmm_kernel<V, 8><<<g, kSpmmThreads, 0, st>>>(p.i0, p.i1, v, x, y, p.m, k); break;
        case 16: csr_spmm_kernel<V, 16><<<g, kSpmmThreads, 0, st>>>(p.i0, p.i1, v, x, y, p.m, k); break;
        default: csr_spmm_kernel<V, 32><<<g, kSpmmThreads, 0, st>>>(p.i0, p.i1, v, x, y, p.m, k); break;
        }
    } else if (p.kind == PART_GBCSR && k % 4 == 0) {
        // register-blocked: CW lanes x 4 right-hand sides, 4 sub-groups over the blocks
        if (p.nbr == 0) return;
        const int CW = k >= 32 ? 8 : (k >= 16 ? 4 : (k >= 8 ? 2 : 1));
        const unsigned g = grid_for((long long)p.nbr * CW * 4, kSpmmThreads);
#define CSP_GB4(BH, BW)                                                                                                          \
    do {                                                                                                                         \
        switch (CW) {                                                                                                            \
        case 1: bcsr_spmm4_kernel<V, BH, BW, 1, 4><<<g, kSpmmThreads, 0, st>>>(p.i0, p.i1, v, x, y, p.nbr, p.stride, p.m, n, k); break; \
        case 2: bcsr_spmm4_kernel<V, BH, BW, 2, 4><<<g, kSpmmThreads, 0, st>>>(p.i0, p.i1, v, x, y, p.nbr, p.stride, p.m, n, k); break; \
        case 4: bcsr_spmm4_kernel<V, BH, BW, 4, 4><<<g, kSpmmThreads, 0, st>>>(p.i0, p.i1, v, x, y, p.nbr, p.stride, p.m, n, k); break; \
        default: bcsr_spmm4_kernel<V, BH, BW, 8, 4><<<g, kSpmmThreads, 0, st>>>(p.i0, p.i1, v, x, y, p.nbr, p.stride, p.m, n, k); break; \
        }                                                                                                                        \
    } while (0)
        switch (p.bh * 10 + p.bw) {
        case 11: CSP_GB4(1, 1); break; case 22: CSP_GB4(2, 2); break; case 33: CSP_GB4(3, 3); break;
        case 44: CSP_GB4(4, 4); break; case 66: CSP_GB4(6, 6); break;
        }
#undef CSP_GB4
    } else if (p.kind == PART_GBCSR) {
        if (p.nbr == 0) return;
        const unsigned g = grid_for((long long)p.nbr * G, kSpmmThreads);
#define CSP_GBM(BH, BW)                                                                                                          \
    do {                                                                                                                         \
        switch (G) {                                                                                                             \
        case 2: bcsr_spmm_kernel<V, BH, BW, 2><<<g, kSpmmThreads, 0, st>>>(p.i0, p.i1, v, x, y, p.nbr, p.stride, p.m, n, k); break;   \
        case 4: bcsr_spmm_kernel<V, BH, BW, 4><<<g, kSpmmThreads, 0, st>>>(p.i0, p.i1, v, x, y, p.nbr, p.stride, p.m, n, k); break;   \
        case 8: bcsr_spmm_kernel<V, BH, BW, 8><<<g, kSpmmThreads, 0, st>>>(p.i0, p.i1, v, x, y, p.nbr, p.stride, p.m, n, k); break;   \
        case 16: bcsr_spmm_kernel<V, BH, BW, 16><<<g, kSpmmThreads, 0, st>>>(p.i0, p.i1, v, x, y, p.nbr, p.stride, p.m, n, k); break; \
        default: bcsr_spmm_kernel<V, BH, BW, 32><<<g, kSpmmThreads, 0, st>>>(p.i0, p.i1, v, x, y, p.nbr, p.stride, p.m, n, k); break; \
        }                                                                                                                        \
    } while (0)
        switch (p.bh * 10 + p.bw) {
        case 11: CSP_GBM(1, 1); break; case 22: CSP_GBM(2, 2); break; case 33: CSP_GBM(3, 3); break;
        case 44: CSP_GBM(4, 4); break; case 66: CSP_GBM(6, 6); break;
        }
#undef CSP_GBM
    }
}

template <class V>
static void launch_part(const Part& p, const float* x, float* y, int n, cudaStream_t st)
{
    using namespace dev;
    const V* v = static_cast<const V*>(p.v);
    switch (p.kind) {
    case PART_CSR: {
        if (p.m == 0) return;
        switch (p.method) {
        case 0: csr_vector_kernel<V, 32><<<grid_for((long long)p.m * 32, 256), 256, 0, st>>>(p.i0, p.i1, v, x, y, p.m); break;
        case 1: csr_block_row_kernel<V, 128><<<p.m, 128, 0, st>>>(p.i0, p.i1, v, x, y, p.m); break;
        case 2: csr_adaptive_kernel<V><<<p.nblocks, kAdaptThreads, 0, st>>>(p.i0, p.i1, v, x, y, p.blocks, p.long_rows,
                                                                             p.scratch_val, p.scratch_row); break;
        case 3: {
            const unsigned g = grid_for((long long)p.m * p.group, 256);
            switch (p.group) {
            case 2: csr_vector_kernel<V, 2><<<g, 256, 0, st>>>(p.i0, p.i1, v, x, y, p.m); break;
            case 4: csr_vector_kernel<V, 4><<<g, 256, 0, st>>>(p.i0, p.i1, v, x, y, p.m); break;
            case 8: csr_vector_kernel<V, 8><<<g, 256, 0, st>>>(p.i0, p.i1, v, x, y, p.m); break;
            case 16: csr_vector_kernel<V, 16><<<g, 256, 0, st>>>(p.i0, p.i1, v, x, y, p.m); break;
            default: csr_vector_kernel<V, 32><<<g, 256, 0, st>>>(p.i0, p.i1, v, x, y, p.m); break;
            }
            break;
        }
        case 4: csr_scalar_kernel<V, 1><<<grid_for(p.m, 256), 256, 0, st>>>(p.i0, p.i1, v, x, y, p.m); break;
        case 5: csr_scalar_kernel<V, 4><<<grid_for(p.m, 256), 256, 0, st>>>(p.i0, p.i1, v, x, y, p.m); break;
        case 6: csr_scalar4_kernel<V><<<grid_for(p.m, 256), 256, 0, st>>>(p.i0, p.i1, v, x, y, p.m); break;
        }
        break;
    }
    case PART_COO: {
        coo_segment_kernel<V><<<grid_for((long long)p.nwarps * 32, 256), 256, 0, st>>>(p.i0, p.i1, v, x, y, p.npad, p.nwarps,
                                                                                      p.span_head, p.spans, p.scratch_row,
                                                                                      p.scratch_val);
        break;
    }
    case PART_ELL:
        if (p.m == 0) return;
        if (p.method == 1) ell_kernel<V, 4><<<grid_for((p.m + 3) / 4, 256), 256, 0, st>>>(p.i1, v, x, y, p.m, p.k, p.stride);
        else ell_kernel<V, 1><<<grid_for(p.m, 256), 256, 0, st>>>(p.i1, v, x, y, p.m, p.k, p.stride);
        break;
    case PART_SELL:
        if (p.m == 0) return;
        if (p.method == 1) sell4_kernel<V><<<grid_for((p.m + 3) / 4, 256), 256, 0, st>>>(p.i0, p.i1, v, x, y, p.m, p.stride);
        else sell1_kernel<V><<<grid_for(p.m, 256), 256, 0, st>>>(p.i0, p.i1, v, x, y, p.m, p.stride);
        break;
    case PART_DIA: {
        if (p.m == 0) return;
        const size_t sm = (size_t)std::max(p.k, 1) * sizeof(int);
        if (p.method == 1) dia4_kernel<V><<<grid_for((p.m + 3) / 4, kDiaThreads), kDiaThreads, sm, st>>>(p.i0, v, x, y, p.m, n, p.k, p.stride);
        else dia_kernel<V, 2><<<grid_for(p.m, kDiaThreads * 2), kDiaThreads, sm, st>>>(p.i0, v, x, y, p.m, n, p.k, p.stride);
        break;
    }
    case PART_BDIA: {
        if (p.m == 0) return;
        if (p.method == 0) {
            bdia4_kernel<V><<<grid_for((p.m + 3) / 4, kDiaThreads), kDiaThreads, 0, st>>>(p.i0, p.i1, v, x, y, p.m, n, p.k, p.stride);
        } else {
            const size_t sm = (size_t)(kDiaThreads * 4 + p.maxw) * sizeof(float);
            bdia_staged_kernel<V, 4><<<grid_for(p.m, kDiaThreads * 4), kDiaThreads, sm, st>>>(p.i0, p.i1, v, x, y, p.m, n, p.k, p.stride);
        }
        break;
    }
    case PART_BELL: {
        if (p.nbr == 0) return;
        const unsigned g = grid_for(p.nbr, 256);
#define CSP_BELL(BH, BW4) bell_b4_kernel<V, BH, BW4><<<g, 256, 0, st>>>(p.i1, v, x, y, p.nbr, p.k, p.stride, p.f4, p.m)
        const int key = p.bh * 10 + p.bw / 4;
        switch (key) {
        case 11: CSP_BELL(1, 1); break; case 21: CSP_BELL(2, 1); break; case 41: CSP_BELL(4, 1); break; case 81: CSP_BELL(8, 1); break;
        case 12: CSP_BELL(1, 2); break; case 22: CSP_BELL(2, 2); break; case 42: CSP_BELL(4, 2); break; case 82: CSP_BELL(8, 2); break;
        }
#undef CSP_BELL
        break;
    }
    case PART_SBELL: {
        if (p.nbr == 0) return;
        const unsigned g = grid_for(p.nbr, 256);
#define CSP_SBELL(BH, BW4) sbell_b4_kernel<V, BH, BW4><<<g, 256, 0, st>>>(p.i0, p.i1, v, x, y, p.nbr, p.stride, p.m)
        const int key = p.bh * 10 + p.bw / 4;
        switch (key) {
        case 11: CSP_SBELL(1, 1); break; case 21: CSP_SBELL(2, 1); break; case 41: CSP_SBELL(4, 1); break; case 81: CSP_SBELL(8, 1); break;
        case 12: CSP_SBELL(1, 2); break; case 22: CSP_SBELL(2, 2); break; case 42: CSP_SBELL(4, 2); break; case 82: CSP_SBELL(8, 2); break;
        }
#undef CSP_SBELL
        break;
    }
    case PART_BCSR: {
        if (p.nbr == 0) return;
        const int G = (p.method == 1) ? 32 : 8;
        const unsigned g = grid_for((long long)p.nbr * G, 256);
#define CSP_BCSR(BH, BW4)                                                                                                   \
    do {                                                                                                                    \
        if (G == 32) bcsr_b4_kernel<V, BH, BW4, 32><<<g, 256, 0, st>>>(p.i0, p.i1, v, x, y, p.nbr, p.stride, p.m);       \
        else bcsr_b4_kernel<V, BH, BW4, 8><<<g, 256, 0, st>>>(p.i0, p.i1, v, x, y, p.nbr, p.stride, p.m);                \
    } while (0)
        const int key = p.bh * 10 + p.bw / 4;
        switch (key) {
        case 11: CSP_BCSR(1, 1); break; case 21: CSP_BCSR(2, 1); break; case 41: CSP_BCSR(4, 1); break; case 81: CSP_BCSR(8, 1); break;
        case 12: CSP_BCSR(1, 2); break; case 22: CSP_BCSR(2, 2); break; case 42: CSP_BCSR(4, 2); break; case 82: CSP_BCSR(8, 2); break;
        }
#undef CSP_BCSR
        break;
    }
    case PART_XPANEL: {
        dev::xpanel_kernel<V><<<p.ncta, kXpThreads, p.smem, st>>>(
            p.tile0, p.ntiles, p.npanels, p.i0, p.lcol, v, x, n, p.panel_w, p.partial, y);
        // at least one CTA even when every row has one run: the launch count stays fixed
        const long long mthreads = (long long)grid_for(p.nrun_rows, 256) * 256 + (long long)p.nlong * kXpMergeLanes;
        xpanel_merge_kernel<<<grid_for(std::max(mthreads, 1LL), 256), 256, 0, st>>>(p.run_ptr, p.run_rows, p.nrun_rows, p.long_list,
                                                                     p.nlong, p.partial, y);
        break;
    }
    case PART_GBCSR: {
        if (p.nbr == 0) return;
        if (p.nblocks > 0) {
#define CSP_GBA(BH, BW) bcsr_adaptive_kernel<V, BH, BW><<<p.nblocks, kGbThreads, 0, st>>>(p.i0, p.i1, v, x, y, p.blocks, p.lcol, p.stride, p.m, n)
            switch (p.bh * 10 + p.bw) {
            case 11: CSP_GBA(1, 1); break; case 22: CSP_GBA(2, 2); break; case 33: CSP_GBA(3, 3); break;
            case 44: CSP_GBA(4, 4); break;
            }
#undef CSP_GBA
            return;
        }
        const unsigned g = grid_for((long long)p.nbr * 8, 256);
#define CSP_GB(BH, BW) bcsr_generic_kernel<V, BH, BW, 8><<<g, 256, 0, st>>>(p.i0, p.i1, v, x, y, p.nbr, p.stride, p.m, n)
        switch (p.bh * 10 + p.bw) {
        case 11: CSP_GB(1, 1); break; case 22: CSP_GB(2, 2); break; case 33: CSP_GB(3, 3); break;
        case 44: CSP_GB(4, 4); break; case 66: CSP_GB(6, 6); break; case 88: CSP_GB(8, 8); break;
        }
#undef CSP_GB
        break;
    }
    }
}

int Engine::launches_per_spmv() const
{
    int n = 0;
    for (const Part& p : parts) n += p.kind == PART_XPANEL ? 2 : 1;
    return n;
}

int Engine::enqueue_parts(const std::vector<Part>& ps, const float* x, float* y, int n, cudaStream_t st)
{
    for (const Part& p : ps) {
        if (nrhs > 1) {
            if (bf16) launch_spmm<__nv_bfloat16>(p, x, y, n, nrhs, tensor_spmm, st);
            else launch_spmm<float>(p, x, y, n, nrhs, tensor_spmm, st);
        } else {
            if (bf16) launch_part<__nv_bfloat16>(p, x, y, n, st);
            else launch_part<float>(p, x, y, n, st);
        }
    }
    CSP_CUDA(cudaGetLastError());
    return CSP_OK;
}

int Engine::enqueue_once(cudaStream_t st) { return enqueue_parts(parts, d_x, d_y, width, st); }

int Engine::spmv(int ntimes)
{
    if (ntimes < 0) return set_error(CSP_EINVAL, "ntimes < 0");
    cudaStream_t st = stream;
    if (!use_graph) {
        for (int i = 0; i < ntimes; i++) {
            int rc = enqueue_once(st);
            if (rc) return rc;
        }
        return CSP_OK;
    }
    if (!graph_exec || graph_stream != st) {
        if (graph_exec) { cudaGraphExecDestroy(graph_exec); graph_exec = nullptr; }
        cudaGraph_t g;
        CSP_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        int rc = enqueue_once(st);
        cudaError_t e = cudaStreamEndCapture(st, &g);
        if (rc) { if (e == cudaSuccess) cudaGraphDestroy(g); return rc; }
        if (e != cudaSuccess) return cuda_error(e, "cudaStreamEndCapture");
        e = cudaGraphInstantiate(&graph_exec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return cuda_error(e, "cudaGraphInstantiate");
        graph_stream = st;
    }
    for (int i = 0; i < ntimes; i++) CSP_CUDA(cudaGraphLaunch(graph_exec, st));
    return CSP_OK;
}

// The reference's solver loop (eval.cpp:19 example(): do_spmv, then the result becomes
// the next vector) on the device: `iterations` times y += A x; x = y.  With
// CSP_FLAG_GRAPH, kIterChunk iterations are captured as one CUDA graph (and the
// remainder as another), so a long loop costs one graph launch per chunk.
int Engine::iterate_once(cudaStream_t st)
{
    int rc = enqueue_once(st);
    if (rc) return rc;
    CSP_CUDA(cudaMemcpyAsync(d_x, d_y, (size_t)height * sizeof(float), cudaMemcpyDeviceToDevice, st));
    return CSP_OK;
}

int Engine::iterate(int iterations)
{
    if (iterations < 0) return set_error(CSP_EINVAL, "iterations < 0");
    if (width != height) return set_error(CSP_EINVAL, "iterate needs a square matrix (%d x %d)", height, width);
    if (nrhs != 1) return set_error(CSP_EUNSUP, "iterate with several right-hand sides");
    cudaStream_t st = stream;
    if (!use_graph) {
        for (int i = 0; i < iterations; i++) {
            int rc = iterate_once(st);
            if (rc) return rc;
        }
        return CSP_OK;
    }
    auto graph_of = [&](int n, cudaGraphExec_t* out) -> int {
        cudaGraphExec_t& ge = iter_graphs[n];
        if (!ge || iter_stream != st) {
            if (ge) { cudaGraphExecDestroy(ge); ge = nullptr; }
            cudaGraph_t g;
            CSP_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            int rc = CSP_OK;
            for (int i = 0; i < n && !rc; i++) rc = iterate_once(st);
            cudaError_t e = cudaStreamEndCapture(st, &g);
            if (rc) { if (e == cudaSuccess) cudaGraphDestroy(g); return rc; }
            if (e != cudaSuccess) return cuda_error(e, "cudaStreamEndCapture");
            e = cudaGraphInstantiate(&ge, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return cuda_error(e, "cudaGraphInstantiate");
        }
        *out = ge;
        return CSP_OK;
    };
    if (iter_stream != st) {
        for (auto& kv : iter_graphs) if (kv.second) cudaGraphExecDestroy(kv.second);
        iter_graphs.clear();
    }
    int rc;
    cudaGraphExec_t ge = nullptr;
    const int full = iterations / kIterChunk, rest = iterations % kIterChunk;
    if (full) {
        if ((rc = graph_of(kIterChunk, &ge))) return rc;
        for (int i = 0; i < full; i++) CSP_CUDA(cudaGraphLaunch(ge, st));
    }
    if (rest) {
        if ((rc = graph_of(rest, &ge))) return rc;
        CSP_CUDA(cudaGraphLaunch(ge, st));
    }
    iter_stream = st;
    return CSP_OK;
}

// CSP_FLAG_L2_PERSIST: x (all right-hand sides) marked persisting in L2 for the
// handle's own stream, with as much persisting L2 reserved for this process's context
// as the device allows (up to the size of x).  The reservation and the window end with
// the context / the handle.
int Engine::set_l2_window()
{
    int dev_id = 0, max_persist = 0, max_window = 0;
    CSP_CUDA(cudaGetDevice(&dev_id));
    CSP_CUDA(cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, dev_id));
    CSP_CUDA(cudaDeviceGetAttribute(&max_window, cudaDevAttrMaxAccessPolicyWindowSize, dev_id));
    if (max_persist <= 0 || max_window <= 0) return set_error(CSP_EUNSUP, "device has no persisting L2");
    const size_t xb = (size_t)x_len * nrhs * sizeof(float);
    size_t cur = 0;
    CSP_CUDA(cudaDeviceGetLimit(&cur, cudaLimitPersistingL2CacheSize));
    const size_t want = std::min(xb, (size_t)max_persist);
    if (cur < want) CSP_CUDA(cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, want));
    cudaStreamAttrValue attr = {};
    attr.accessPolicyWindow.base_ptr = d_x;
    attr.accessPolicyWindow.num_bytes = std::min(xb, (size_t)max_window);
    attr.accessPolicyWindow.hitRatio = std::min(1.0f, (float)want / (float)attr.accessPolicyWindow.num_bytes);
    attr.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
    attr.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
    CSP_CUDA(cudaStreamSetAttribute(own_stream, cudaStreamAttributeAccessPolicyWindow, &attr));
    l2_window = true;
    return CSP_OK;
}

int Engine::init_common(int w, int h, int nz, const float* vec, const float* res, int flags, int k)
{
    width = w;
    height = h;
    nnz = nz;
    if (width < 0 || height < 0) return set_error(CSP_EINVAL, "negative matrix size");
    if (k < 1) return set_error(CSP_EINVAL, "nrhs must be >= 1");
    nrhs = k;
    bf16 = (flags & CSP_FLAG_BF16) != 0;
    use_graph = (flags & CSP_FLAG_GRAPH) != 0;
    tensor_spmm = (flags & CSP_FLAG_TENSOR_CORES) != 0;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) return set_error(CSP_ENODEV, "no CUDA device: %s", cudaGetErrorString(e));
    CSP_CUDA(cudaStreamCreateWithFlags(&own_stream, cudaStreamNonBlocking));
    stream = own_stream;
    // x: zero-padded to a multiple of 64 (block kernels read float4s up to the padded width);
    // y: padded to a multiple of 1024 like the reference (spmv_cocktail.cpp:234)
    x_len = pad_to(std::max(width, 1), 64) + 64;
    y_len = pad_to(std::max(height, 1), 1024);
    int rc;
    if ((rc = alloc(reinterpret_cast<void**>(&d_x), (size_t)x_len * nrhs * 4)) ||
        (rc = alloc(reinterpret_cast<void**>(&d_y), (size_t)y_len * nrhs * 4)))
        return rc;
    CSP_CUDA(cudaMemset(d_x, 0, (size_t)x_len * nrhs * 4));
    CSP_CUDA(cudaMemset(d_y, 0, (size_t)y_len * nrhs * 4));
    if (vec && width) CSP_CUDA(cudaMemcpy(d_x, vec, (size_t)width * nrhs * 4, cudaMemcpyHostToDevice));
    if (res && height) CSP_CUDA(cudaMemcpy(d_y, res, (size_t)height * nrhs * 4, cudaMemcpyHostToDevice));
    if ((flags & CSP_FLAG_L2_PERSIST) && (rc = set_l2_window())) return rc;
    return CSP_OK;
}

int Engine::init(const cocktail_iif* mat, const float* vec, const float* res, int flags, int k)
{
    if (!mat) return set_error(CSP_EINVAL, "null cocktail");
    int rc = init_common(mat->mat_width, mat->mat_height, mat->mat_nnz, vec, res, flags, k);
    if (rc) return rc;
    static_assert(sizeof(bcsr_matrix_if) == sizeof(b4csr_matrix_if) &&
                      offsetof(bcsr_matrix_if, bcsr_row_ptr) == offsetof(b4csr_matrix_if, b4csr_row_ptr) &&
                      offsetof(bcsr_matrix_if, bcsr_data) == offsetof(b4csr_matrix_if, b4csr_data),
                  "generic and b4 BCSR structs share one layout");
    const bool generic_bcsr = mat->ifusebcsr && mat->bcsr_meth_num == CSP_METH_GENERIC_BCSR;
    if (nrhs > 1) {
        if (mat->ifusebdia || mat->ifusedia || mat->ifusesbell || mat->ifusebell || (mat->ifusebcsr && !generic_bcsr) ||
            mat->ifusesell || mat->ifuseell || mat->ifusecoo)
            return set_error(CSP_EUNSUP, "several right-hand sides run on CSR and generic BCSR parts (and csp_init_bcsr_kernels)");
        if (generic_bcsr && mat->bcsr.b4csr_bwidth * mat->bcsr.b4csr_bheight > 36)
            return set_error(CSP_EUNSUP, "several right-hand sides need blocks of <= 36 elements");
        if (flags & CSP_FLAG_ADJOINT) return set_error(CSP_EUNSUP, "adjoint with several right-hand sides");
    }
    // parts, in the reference's launch order
    if (mat->ifusebdia && (rc = add_bdia(mat->bdia, mat->bdia_meth_num))) return rc;
    if (mat->ifusedia && (rc = add_dia(mat->dia, mat->dia_meth_num))) return rc;
    if (mat->ifusesbell && (rc = add_sbell(mat->sbell, mat->sbell_meth_num))) return rc;
    if (mat->ifusebell && (rc = add_bell(mat->bell, mat->bell_meth_num))) return rc;
    if (generic_bcsr) {
        // the member holds a generic BCSR (same fields as the b4 struct, see CSP_METH_GENERIC_BCSR)
        if ((rc = add_generic_bcsr(*reinterpret_cast<const bcsr_matrix_if*>(&mat->bcsr), 0))) return rc;
    } else if (mat->ifusebcsr && (rc = add_bcsr(mat->bcsr, mat->bcsr_meth_num))) {
        return rc;
    }
    if (mat->ifusesell && (rc = add_sell(mat->sell, mat->sell_meth_num))) return rc;
    if (mat->ifuseell && (rc = add_ell(mat->ell, mat->ell_meth_num))) return rc;
    if (mat->ifusecsr && (rc = add_csr(mat->csr, mat->csr_meth_num))) return rc;
    if (mat->ifusecoo && (rc = add_coo(mat->coo, mat->coo_meth_num))) return rc;
    if ((flags & CSP_FLAG_ADJOINT) && (rc = build_adjoint(mat))) return rc;
    CSP_CUDA(cudaDeviceSynchronize());
    return CSP_OK;
}

int Engine::init_bcsr(const bcsr_matrix_if* b, const float* vec, const float* res, int flags, int k)
{
    if (!b) return set_error(CSP_EINVAL, "null BCSR");
    if ((flags & CSP_FLAG_ADJOINT) && k > 1) return set_error(CSP_EUNSUP, "adjoint with several right-hand sides");
    if (k > 1 && b->bcsr_bwidth * b->bcsr_bheight > 36) return set_error(CSP_EUNSUP, "several right-hand sides need blocks of <= 36 elements");
    int rc = init_common(b->matinfo.width, b->matinfo.height, b->matinfo.nnz, vec, res, flags, k);
    if (rc) return rc;
    if ((rc = add_generic_bcsr(*b, 0))) return rc;
    if ((flags & CSP_FLAG_ADJOINT) && (rc = build_adjoint_gbcsr(*b))) return rc;
    CSP_CUDA(cudaDeviceSynchronize());
    return CSP_OK;
}

}  // namespace csp

// ==========================================================================
// C ABI
// ==========================================================================
using csp::Engine;
using csp::set_error;
using csp::cuda_error;


#define CSP_HANDLE_CHECK(h) \
    do { if (!(h)) return set_error(CSP_EINVAL, "null handle"); } while (0)

extern "C" {

const char* csp_error_string(int code)
{
    switch (code) {
    case CSP_OK: return "CSP_OK";
    case CSP_EINVAL: return "CSP_EINVAL";
    case CSP_ENOMEM: return "CSP_ENOMEM";
    case CSP_ECUDA: return "CSP_ECUDA";
    case CSP_EFORMAT: return "CSP_EFORMAT";
    case CSP_ENODEV: return "CSP_ENODEV";
    case CSP_EUNSUP: return "CSP_EUNSUP";
    case CSP_EIO: return "CSP_EIO";
    case CSP_ETIMEOUT: return "CSP_ETIMEOUT";
    default: return "CSP_E?";
    }
}

const char* csp_last_error(void) { return csp::g_last_error.c_str(); }
const char* csp_version(void) { return "clspmv_b200 0.1.0 (sm_100a)"; }

int csp_init_mat_kernels_ex(const cocktail_iif* mat, const float* vec, const float* res, int nrhs, int flags, csp_handle** out)
{
    if (!out) return set_error(CSP_EINVAL, "null output handle");
    *out = nullptr;
    csp_handle* h = new (std::nothrow) csp_handle();
    if (!h) return set_error(CSP_ENOMEM, "handle");
    int rc = h->eng.init(mat, vec, res, flags, nrhs);
    if (rc) { delete h; return rc; }
    *out = h;
    return CSP_OK;
}

int csp_init_mat_kernels(const cocktail_iif* mat, const float* vec, const float* res, int flags, csp_handle** out)
{
    return csp_init_mat_kernels_ex(mat, vec, res, 1, flags, out);
}

int csp_init_bcsr_kernels(const bcsr_matrix_if* b, const float* vec, const float* res, int nrhs, int flags, csp_handle** out)
{
    if (!out) return set_error(CSP_EINVAL, "null output handle");
    *out = nullptr;
    csp_handle* h = new (std::nothrow) csp_handle();
    if (!h) return set_error(CSP_ENOMEM, "handle");
    int rc = h->eng.init_bcsr(b, vec, res, flags, nrhs);
    if (rc) { delete h; return rc; }
    *out = h;
    return CSP_OK;
}

int csp_do_spmv(csp_handle* h, int ntimes) { CSP_HANDLE_CHECK(h); return h->eng.spmv(ntimes); }
int csp_iterate(csp_handle* h, int iterations) { CSP_HANDLE_CHECK(h); return h->eng.iterate(iterations); }

int csp_synchronize(csp_handle* h)
{
    CSP_HANDLE_CHECK(h);
    cudaError_t e = cudaStreamSynchronize(h->eng.stream);
    return e == cudaSuccess ? CSP_OK : cuda_error(e, "cudaStreamSynchronize");
}

static int copy_in(csp_handle* h, float* dst, int cap, const void* src, int n, cudaMemcpyKind kind)
{
    if (!src || n < 0 || n > cap) return set_error(CSP_EINVAL, "copy of %d elements into a buffer of %d", n, cap);
    cudaError_t e = cudaMemcpyAsync(dst, src, (size_t)n * 4, kind, h->eng.stream);
    if (e != cudaSuccess) return cuda_error(e, "cudaMemcpyAsync");
    // a pageable host source may be reused by the caller on return
    if (kind == cudaMemcpyHostToDevice) {
        e = cudaStreamSynchronize(h->eng.stream);
        if (e != cudaSuccess) return cuda_error(e, "cudaStreamSynchronize");
    }
    return CSP_OK;
}

int csp_cpy_vector_from_cpu(csp_handle* h, const float* vec, int n)
{
    CSP_HANDLE_CHECK(h);
    return copy_in(h, h->eng.d_x, h->eng.width * h->eng.nrhs, vec, n, cudaMemcpyHostToDevice);
}
int csp_cpy_vector_from_gpu(csp_handle* h, const float* dvec, int n)
{
    CSP_HANDLE_CHECK(h);
    return copy_in(h, h->eng.d_x, h->eng.width * h->eng.nrhs, dvec, n, cudaMemcpyDeviceToDevice);
}
int csp_cpy_result_from_cpu(csp_handle* h, const float* res, int n)
{
    CSP_HANDLE_CHECK(h);
    return copy_in(h, h->eng.d_y, h->eng.height * h->eng.nrhs, res, n, cudaMemcpyHostToDevice);
}
int csp_cpy_result_from_gpu(csp_handle* h, const float* dres, int n)
{
    CSP_HANDLE_CHECK(h);
    return copy_in(h, h->eng.d_y, h->eng.height * h->eng.nrhs, dres, n, cudaMemcpyDeviceToDevice);
}
int csp_cpy_result_to_cpu(csp_handle* h, float* res, int n)
{
    CSP_HANDLE_CHECK(h);
    if (!res || n < 0 || n > h->eng.height * h->eng.nrhs) return set_error(CSP_EINVAL, "bad result copy");
    cudaError_t e = cudaMemcpyAsync(res, h->eng.d_y, (size_t)n * 4, cudaMemcpyDeviceToHost, h->eng.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->eng.stream);
    return e == cudaSuccess ? CSP_OK : cuda_error(e, "result to cpu");
}
int csp_cpy_result_to_gpu(csp_handle* h, float* dres, int n)
{
    CSP_HANDLE_CHECK(h);
    if (!dres || n < 0 || n > h->eng.height * h->eng.nrhs) return set_error(CSP_EINVAL, "bad result copy");
    cudaError_t e = cudaMemcpyAsync(dres, h->eng.d_y, (size_t)n * 4, cudaMemcpyDeviceToDevice, h->eng.stream);
    return e == cudaSuccess ? CSP_OK : cuda_error(e, "result to gpu");
}

int csp_free_mat_kernels(csp_handle* h)
{
    if (!h) return CSP_OK;
    cudaStreamSynchronize(h->eng.stream);
    delete h;
    return CSP_OK;
}

int csp_get_vec_device_ptr(csp_handle* h, float** p) { CSP_HANDLE_CHECK(h); if (!p) return set_error(CSP_EINVAL, "null"); *p = h->eng.d_x; return CSP_OK; }
int csp_get_res_device_ptr(csp_handle* h, float** p) { CSP_HANDLE_CHECK(h); if (!p) return set_error(CSP_EINVAL, "null"); *p = h->eng.d_y; return CSP_OK; }

int csp_set_stream(csp_handle* h, void* stream)
{
    CSP_HANDLE_CHECK(h);
    h->eng.stream = stream ? static_cast<cudaStream_t>(stream) : h->eng.own_stream;
    return CSP_OK;
}
int csp_get_stream(csp_handle* h, void** stream) { CSP_HANDLE_CHECK(h); if (!stream) return set_error(CSP_EINVAL, "null"); *stream = h->eng.stream; return CSP_OK; }
int csp_launches_per_spmv(csp_handle* h, int* n) { CSP_HANDLE_CHECK(h); if (!n) return set_error(CSP_EINVAL, "null"); *n = h->eng.launches_per_spmv(); return CSP_OK; }
int csp_device_bytes(csp_handle* h, size_t* b) { CSP_HANDLE_CHECK(h); if (!b) return set_error(CSP_EINVAL, "null"); *b = h->eng.device_bytes; return CSP_OK; }

}  // extern "C"
