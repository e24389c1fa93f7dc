// Batched execution: many matrices, one persistent launch (kernels/batch.cuh).
//
// csp_batch_create builds, per matrix, the CSR of A and of A^T on the host,
// chooses a batch format (device autotuner, byte model, or the caller's), stores
// A and A^T in it in one device arena, and cuts every stored operator into work
// items of a few thousand slots.  A run is one launch of batch_kernel over the
// item list of the requested directions; with CSP_FLAG_GRAPH each direction set
// is a captured CUDA graph.  csp_batch_run_plain runs the same work as per-matrix
// plain CSR launches, the baseline the batch is measured against.
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdio.h>
#include <string.h>
#include <algorithm>
#include <climits>
#include <cmath>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "csp/clspmv.h"
#include "internal.h"
#include "engine.h"
#include "kernels/batch.cuh"

namespace csp {
namespace {

#define BCUDA(call)                                                 \
    do {                                                            \
        cudaError_t _e = (call);                                    \
        if (_e != cudaSuccess) return cuda_error(_e, #call);        \
    } while (0)

constexpr int kItemSlots = 2048;   // target stored slots per (warp) work item

inline long long pad_ll(long long v, long long a) { return (v + a - 1) / a * a; }

struct HCsr {
    int m = 0, n = 0;
    std::vector<int> rp, col;
    std::vector<float> val;
};

// CSR of a COO in any order: stable counting sort on rows, then columns sorted
// inside each row (duplicates keep their input order).
void csr_of(const coo_matrix_if* a, HCsr& c)
{
    const int m = a->matinfo.height, nnz = a->matinfo.nnz;
    c.m = m;
    c.n = a->matinfo.width;
    c.rp.assign((size_t)m + 1, 0);
    for (int i = 0; i < nnz; i++) c.rp[(size_t)a->coo_row_id[i] + 1]++;
    for (int r = 0; r < m; r++) c.rp[r + 1] += c.rp[r];
    std::vector<int> pos(c.rp.begin(), c.rp.end() - 1);
    std::vector<int> idx((size_t)nnz);
    for (int i = 0; i < nnz; i++) idx[(size_t)pos[a->coo_row_id[i]]++] = i;
    for (int r = 0; r < m; r++)
        std::stable_sort(idx.begin() + c.rp[r], idx.begin() + c.rp[r + 1],
                         [a](int p, int q) { return a->coo_col_id[p] < a->coo_col_id[q]; });
    c.col.resize((size_t)nnz);
    c.val.resize((size_t)nnz);
    for (int i = 0; i < nnz; i++) {
        c.col[i] = a->coo_col_id[idx[i]];
        c.val[i] = a->coo_data[idx[i]];
    }
}

// A^T: counting sort on the column; inside a row of A^T the entries come in
// increasing row of A, i.e. increasing column of A^T.
void transpose(const HCsr& a, HCsr& t)
{
    const int nnz = a.rp[a.m];
    t.m = a.n;
    t.n = a.m;
    t.rp.assign((size_t)t.m + 1, 0);
    for (int i = 0; i < nnz; i++) t.rp[(size_t)a.col[i] + 1]++;
    for (int r = 0; r < t.m; r++) t.rp[r + 1] += t.rp[r];
    std::vector<int> pos(t.rp.begin(), t.rp.end() - 1);
    t.col.resize((size_t)nnz);
    t.val.resize((size_t)nnz);
    for (int r = 0; r < a.m; r++)
        for (int j = a.rp[r]; j < a.rp[r + 1]; j++) {
            const int q = pos[a.col[j]]++;
            t.col[q] = r;
            t.val[q] = a.val[j];
        }
}

// ---------------------------------------------------------------------------
// features and the format choice
// ---------------------------------------------------------------------------
int ilog2i(long long v)
{
    int k = 0;
    while (v > 1) { v >>= 1; k++; }
    return k;
}

void features(const HCsr& c, int flags, csp_batch_features& f)
{
    memset(&f, 0, sizeof(f));
    const int m = c.m, n = c.n, nnz = c.rp[m];
    f.rows = m;
    f.cols = n;
    f.nnz = nnz;
    double sum2 = 0.0;
    for (int r = 0; r < m; r++) {
        const int l = c.rp[r + 1] - c.rp[r];
        f.max_row = std::max(f.max_row, l);
        sum2 += (double)l * l;
    }
    // diagonals
    std::vector<int> offs;
    bool dia_ok = true;
    for (int r = 0; r < m && dia_ok; r++)
        for (int j = c.rp[r]; j < c.rp[r + 1]; j++) {
            const int o = c.col[j] - r;
            if (std::find(offs.begin(), offs.end(), o) == offs.end()) {
                if ((int)offs.size() == dev::kBatchMaxDiag) { dia_ok = false; break; }
                offs.push_back(o);
            }
        }
    f.ndiag = dia_ok ? (int)offs.size() : -1;
    f.dia_slots = dia_ok ? (long long)offs.size() * pad_ll(m, 32) : 0;
    // sliced ELL
    const int H[2] = {32, 128};
    for (int h = 0; h < 2; h++) {
        long long slots = 0;
        for (int s0 = 0; s0 < m; s0 += H[h]) {
            int w = 0;
            for (int r = s0; r < std::min(m, s0 + H[h]); r++) w = std::max(w, c.rp[r + 1] - c.rp[r]);
            slots += (long long)w * H[h];
        }
        f.sell_slots[h] = slots;
    }
    // blocks
    for (int b = 2; b <= 4; b++) {
        long long blocks = 0;
        std::vector<int> cols;
        for (int r0 = 0; r0 < m; r0 += b) {
            cols.clear();
            for (int r = r0; r < std::min(m, r0 + b); r++)
                for (int j = c.rp[r]; j < c.rp[r + 1]; j++) cols.push_back(c.col[j] - c.col[j] % b);
            std::sort(cols.begin(), cols.end());
            blocks += std::unique(cols.begin(), cols.end()) - cols.begin();
        }
        f.bcsr_blocks[b - 2] = blocks;
    }
    // candidates: CSR always; the padded formats while they store at most 1.5x the entries
    // (sliced ELL: 2x, since its per-row lane needs no reduction and short, even rows --
    // the transposes of long-row matrices -- often come just above 1.5x)
    const double lim = 1.5 * nnz + 64, sell_lim = 2.0 * nnz + 64;
    unsigned feas = 1u << CSP_BFMT_CSR;
    if (nnz > 0) {
        if (f.sell_slots[0] <= sell_lim && f.sell_slots[0] < INT_MAX) feas |= 1u << CSP_BFMT_SELL32;
        if (f.sell_slots[1] <= sell_lim && f.sell_slots[1] < INT_MAX) feas |= 1u << CSP_BFMT_SELL128;
        if (dia_ok && (double)offs.size() * m <= lim && f.dia_slots < INT_MAX) feas |= 1u << CSP_BFMT_DIA;
        for (int b = 2; b <= 4; b++)
            if ((double)f.bcsr_blocks[b - 2] * b * b <= lim && f.bcsr_blocks[b - 2] * b * b < INT_MAX)
                feas |= 1u << (CSP_BFMT_BCSR2 + b - 2);
    }
    f.feasible = feas;
    // byte model: matrix bytes of A and A^T plus the gradient store
    const double es = (flags & CSP_FLAG_BF16) ? 2.0 : 4.0;
    double best = 0.0;
    f.model_format = CSP_BFMT_CSR;
    for (int fmt = 0; fmt < CSP_BFMT_COUNT; fmt++) {
        if (!(feas & (1u << fmt))) continue;
        double bytes = 0.0;
        switch (fmt) {
        case CSP_BFMT_CSR: bytes = 2.0 * ((es + 4.0) * nnz + 4.0 * m) + 4.0 * nnz; break;
        case CSP_BFMT_SELL32: bytes = (2.0 * (es + 4.0) + 4.0) * f.sell_slots[0]; break;
        case CSP_BFMT_SELL128: bytes = (2.0 * (es + 4.0) + 4.0) * f.sell_slots[1]; break;
        case CSP_BFMT_DIA: bytes = (2.0 * es + 4.0) * f.dia_slots; break;
        default: {
            const int b = fmt - CSP_BFMT_BCSR2 + 2;
            bytes = 2.0 * (4.0 + es * b * b) * f.bcsr_blocks[b - 2] + 4.0 * b * b * f.bcsr_blocks[b - 2];
        }
        }
        if (fmt == CSP_BFMT_CSR || bytes < best) {
            best = bytes;
            f.model_format = fmt;
        }
    }
    // signature: structure classes that share a decision
    const double mean = m ? (double)nnz / m : 0.0;
    const double var = m ? std::max(0.0, sum2 / m - mean * mean) : 0.0;
    const double cv = mean > 0 ? std::sqrt(var) / mean : 0.0;
    // the byte model's choice stands for the structure; the rest buckets size and row lengths
    const long long key[] = {f.model_format,
                             ilog2i(std::max(m, 1)) / 2,
                             ilog2i(std::max(n, 1)) / 2,
                             (long long)std::floor(std::log2(mean + 1.0) * 2.0),
                             std::min(8LL, (long long)std::floor(cv * 2.0)),
                             ilog2i(std::max(f.max_row, 1)),
                             f.ndiag < 0 ? -1 : f.ndiag / 4,
                             (flags & CSP_FLAG_BF16) ? 1 : 0};
    unsigned long long h = 1469598103934665603ULL;
    for (long long k : key)
        for (int i = 0; i < 8; i++) {
            h ^= (unsigned long long)((k >> (8 * i)) & 0xff);
            h *= 1099511628211ULL;
        }
    f.signature = h;
}

// ---------------------------------------------------------------------------
// stored operators
// ---------------------------------------------------------------------------
struct HPart {
    int kind = dev::BK_CSR, m = 0, n = 0, k = 0, stride = 0, nbr = 0;
    std::vector<int> i0, i1;
    std::vector<float> v;
    std::vector<int4> blocks, longs;
    int npartial = 0;
    long long slots = 0;            // stored slots (gradient length)
    std::vector<dev::BatchItem> ranges;   // work items (part index filled in later)
};

dev::BatchItem range_item(int v0, int v1, int4 blk = make_int4(0, 0, 0, 0))
{
    dev::BatchItem it;
    it.part = 0;
    it.v0 = v0;
    it.v1 = v1;
    it.pad = 0;
    it.blk = blk;
    return it;
}

// groups consecutive virtual blocks into items of about kItemSlots slots
void cut_items(HPart& p, int nvb, const std::vector<long long>& vb_slots)
{
    p.ranges.clear();
    int start = 0;
    long long acc = 0;
    for (int vb = 0; vb < nvb; vb++) {
        acc += vb_slots[vb];
        if (acc >= kItemSlots || vb == nvb - 1) {
            p.ranges.push_back(range_item(start, vb + 1));
            start = vb + 1;
            acc = 0;
        }
    }
}

// CSR work blocks of one warp: runs of whole rows with at most dev::kWarpNnz entries
// and dev::kWarpRows rows {first row, rows, first entry, end entry}, or the chunks of a
// row longer than kWarpNnz {chunk, -(long row + 1), first entry, end entry} with the
// long row {row, first partial slot, chunks, -}.
void make_warp_blocks(const std::vector<int>& rp, int m, std::vector<int4>& blocks, std::vector<int4>& longs, int& nslots)
{
    blocks.clear();
    longs.clear();
    nslots = 0;
    int r = 0;
    while (r < m) {
        const int len = rp[r + 1] - rp[r];
        if (len > dev::kWarpNnz) {
            const int lid = (int)longs.size();
            const int nch = (len + dev::kWarpNnz - 1) / dev::kWarpNnz;
            longs.push_back(make_int4(r, nslots, nch, 0));
            for (int k = 0; k < nch; k++)
                blocks.push_back(make_int4(k, -(lid + 1), rp[r] + k * dev::kWarpNnz,
                                           std::min(rp[r] + (k + 1) * dev::kWarpNnz, rp[r + 1])));
            nslots += nch;
            r++;
            continue;
        }
        const int start = r;
        long long acc = 0;
        while (r < m && r - start < dev::kWarpRows) {
            const int l = rp[r + 1] - rp[r];
            if (l > dev::kWarpNnz || acc + l > dev::kWarpNnz) break;
            acc += l;
            r++;
        }
        blocks.push_back(make_int4(start, r - start, rp[start], rp[r]));
    }
}

void build_csr(const HCsr& c, HPart& p)
{
    const int nnz = c.rp[c.m];
    p.kind = dev::BK_CSR;
    p.m = c.m;
    p.n = c.n;
    p.i0 = c.rp;
    p.i1 = c.col;
    p.i1.resize((size_t)pad_ll(nnz, 4) + 4, 0);
    p.v = c.val;
    p.v.resize(p.i1.size(), 0.0f);
    make_warp_blocks(c.rp, c.m, p.blocks, p.longs, p.npartial);
    p.slots = nnz;
    p.ranges.clear();
    for (int b = 0; b < (int)p.blocks.size(); b++) p.ranges.push_back(range_item(b, b + 1, p.blocks[b]));
}

void build_sell(const HCsr& c, int H, HPart& p)
{
    const int m = c.m;
    const int S = (m + H - 1) / H;
    p.kind = dev::BK_SELL;
    p.m = m;
    p.n = c.n;
    p.stride = H;
    p.nbr = S;
    p.i0.assign((size_t)S + 1, 0);
    for (int s = 0; s < S; s++) {
        int w = 0;
        for (int r = s * H; r < std::min(m, (s + 1) * H); r++) w = std::max(w, c.rp[r + 1] - c.rp[r]);
        p.i0[s + 1] = p.i0[s] + w * H;
    }
    p.slots = p.i0[S];
    p.i1.assign((size_t)p.slots, -1);
    p.v.assign((size_t)p.slots, 0.0f);
    for (int r = 0; r < m; r++) {
        const int s = r / H, lr = r % H;
        for (int j = c.rp[r]; j < c.rp[r + 1]; j++) {
            const size_t q = (size_t)p.i0[s] + (size_t)(j - c.rp[r]) * H + lr;
            p.i1[q] = c.col[j];
            p.v[q] = c.val[j];
        }
    }
    // virtual blocks of 32 rows (a lane per row), inside one slice (H is 32 or 128)
    const int nvb = (m + dev::kBatchSellRows - 1) / dev::kBatchSellRows;
    std::vector<long long> vs((size_t)nvb);
    for (int vb = 0; vb < nvb; vb++) {
        const int s = vb * dev::kBatchSellRows / H;
        vs[vb] = (long long)(p.i0[s + 1] - p.i0[s]) / H * dev::kBatchSellRows;
    }
    cut_items(p, nvb, vs);
}

void build_dia(const HCsr& c, HPart& p)
{
    const int m = c.m;
    std::vector<int> offs;
    for (int r = 0; r < m; r++)
        for (int j = c.rp[r]; j < c.rp[r + 1]; j++) offs.push_back(c.col[j] - r);
    std::sort(offs.begin(), offs.end());
    offs.erase(std::unique(offs.begin(), offs.end()), offs.end());
    p.kind = dev::BK_DIA;
    p.m = m;
    p.n = c.n;
    p.k = (int)offs.size();
    p.stride = (int)pad_ll(m, 32);
    p.i0 = offs;
    p.slots = (long long)p.k * p.stride;
    p.v.assign((size_t)p.slots, 0.0f);
    for (int r = 0; r < m; r++)
        for (int j = c.rp[r]; j < c.rp[r + 1]; j++) {
            const int d = (int)(std::lower_bound(offs.begin(), offs.end(), c.col[j] - r) - offs.begin());
            p.v[(size_t)d * p.stride + r] += c.val[j];   // duplicates share a slot
        }
    const int rows_per_vb = dev::kBatchDiaRows;
    const int nvb = (m + rows_per_vb - 1) / rows_per_vb;
    cut_items(p, nvb, std::vector<long long>((size_t)nvb, (long long)rows_per_vb * std::max(p.k, 1)));
}

void build_bcsr(const HCsr& c, int B, HPart& p)
{
    const int m = c.m;
    const int nbr = (m + B - 1) / B;
    p.kind = dev::BK_BCSR2 + (B - 2);
    p.m = m;
    p.n = c.n;
    p.nbr = nbr;
    p.i0.assign((size_t)nbr + 1, 0);
    p.i1.clear();
    std::vector<int> cols;
    for (int br = 0; br < nbr; br++) {
        cols.clear();
        for (int r = br * B; r < std::min(m, br * B + B); r++)
            for (int j = c.rp[r]; j < c.rp[r + 1]; j++) cols.push_back(c.col[j] - c.col[j] % B);
        std::sort(cols.begin(), cols.end());
        cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
        p.i1.insert(p.i1.end(), cols.begin(), cols.end());
        p.i0[br + 1] = (int)p.i1.size();
    }
    const int nb = p.i0[nbr];
    const int al = (int)pad_ll(std::max(nb, 1), 4);
    p.stride = al;
    p.slots = (long long)B * B * al;
    p.v.assign((size_t)p.slots, 0.0f);
    for (int r = 0; r < m; r++) {
        const int br = r / B;
        const int* b0 = p.i1.data() + p.i0[br];
        const int* b1 = p.i1.data() + p.i0[br + 1];
        for (int j = c.rp[r]; j < c.rp[r + 1]; j++) {
            const int cc = c.col[j];
            const int blk = (int)(std::lower_bound(b0, b1, cc - cc % B) - p.i1.data());
            const int q = (r % B) * B + cc % B;
            p.v[(size_t)q * al + blk] += c.val[j];
        }
    }
    const int brpv = dev::kBatchBcsrRows;   // block rows per virtual block
    const int nvb = (nbr + brpv - 1) / brpv;
    std::vector<long long> vs((size_t)nvb);
    for (int vb = 0; vb < nvb; vb++)
        vs[vb] = (long long)B * B * (p.i0[std::min(nbr, (vb + 1) * brpv)] - p.i0[vb * brpv]);
    cut_items(p, nvb, vs);
}

void build_part(int fmt, const HCsr& c, HPart& p)
{
    switch (fmt) {
    case CSP_BFMT_SELL32: build_sell(c, 32, p); break;
    case CSP_BFMT_SELL128: build_sell(c, 128, p); break;
    case CSP_BFMT_DIA: build_dia(c, p); break;
    case CSP_BFMT_BCSR2: build_bcsr(c, 2, p); break;
    case CSP_BFMT_BCSR3: build_bcsr(c, 3, p); break;
    case CSP_BFMT_BCSR4: build_bcsr(c, 4, p); break;
    default: build_csr(c, p); break;
    }
}

// ---------------------------------------------------------------------------
// device arena: one allocation, 256-byte aligned sub-ranges
// ---------------------------------------------------------------------------
struct Arena {
    char* base = nullptr;
    size_t size = 0, used = 0;
    std::vector<std::pair<size_t, std::vector<char>>> staged;   // (offset, bytes) uploads

    size_t take(size_t bytes)
    {
        const size_t o = used;
        used += (bytes + 255) / 256 * 256;
        return o;
    }
    template <class T> size_t stage(const std::vector<T>& h, size_t min_count = 0)
    {
        const size_t n = std::max(h.size(), min_count);
        const size_t o = take(std::max<size_t>(n * sizeof(T), 16));
        if (!h.empty()) {
            std::vector<char> b(h.size() * sizeof(T));
            memcpy(b.data(), h.data(), b.size());
            staged.emplace_back(o, std::move(b));
        }
        return o;
    }
    int commit()
    {
        size = std::max<size_t>(used, 256);
        BCUDA(cudaMalloc(reinterpret_cast<void**>(&base), size));
        BCUDA(cudaMemset(base, 0, size));
        for (auto& s : staged) BCUDA(cudaMemcpy(base + s.first, s.second.data(), s.second.size(), cudaMemcpyHostToDevice));
        staged.clear();
        staged.shrink_to_fit();
        return CSP_OK;
    }
    void release()
    {
        if (base) cudaFree(base);
        base = nullptr;
        size = used = 0;
        staged.clear();
    }
};

// values in the storage type
std::vector<uint16_t> bf16_of(const std::vector<float>& v)
{
    std::vector<uint16_t> t(v.size());
    for (size_t i = 0; i < v.size(); i++) t[i] = to_bf16(v[i]);
    return t;
}

// Offsets of one stored operator inside the arena (resolved to pointers after commit).
struct PartOffs {
    size_t i0 = 0, i1 = 0, v = 0, longs = 0, partial = 0, arrivals = 0;
};

PartOffs stage_part(Arena& a, const HPart& p, bool bf16)
{
    PartOffs o;
    o.i0 = a.stage(p.i0);
    o.i1 = a.stage(p.i1);
    o.v = bf16 ? a.stage(bf16_of(p.v)) : a.stage(p.v);
    o.longs = a.stage(p.longs);
    o.partial = a.take(std::max<size_t>((size_t)p.npartial * 4, 16));
    o.arrivals = a.take(std::max<size_t>(p.longs.size() * 4, 16));
    return o;
}

dev::BatchPart make_desc(const HPart& p, const PartOffs& o, char* base)
{
    dev::BatchPart d;
    memset(&d, 0, sizeof(d));
    d.kind = p.kind;
    d.m = p.m;
    d.n = p.n;
    d.k = p.k;
    d.stride = p.stride;
    d.nbr = p.nbr;
    d.i0 = reinterpret_cast<const int*>(base + o.i0);
    d.i1 = reinterpret_cast<const int*>(base + o.i1);
    d.v = base + o.v;
    d.long_rows = reinterpret_cast<const int4*>(base + o.longs);
    d.partial = reinterpret_cast<float*>(base + o.partial);
    d.arrivals = reinterpret_cast<int*>(base + o.arrivals);
    return d;
}

int occupancy_grid(bool bf16, int nitems)
{
    int dev_id = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev_id);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev_id);
    if (bf16)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dev::batch_kernel<__nv_bfloat16>, dev::kBatchThreads, 0);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dev::batch_kernel<float>, dev::kBatchThreads, 0);
    const int g = std::max(1, sms) * std::max(1, per_sm);
    return std::max(1, std::min(g, (nitems + dev::kBatchWarps - 1) / dev::kBatchWarps));
}

// One launch over `nitems` items: the item counter zeroed on the stream, then the kernel.
int launch_batch(bool bf16, const dev::BatchPart* parts, const dev::BatchItem* items, int nitems, int* counter,
                 unsigned long long* cycles, int grid, cudaStream_t st)
{
    if (nitems <= 0) return CSP_OK;
    BCUDA(cudaMemsetAsync(counter, 0, sizeof(int), st));
    if (bf16)
        dev::batch_kernel<__nv_bfloat16><<<grid, dev::kBatchThreads, 0, st>>>(parts, items, nitems, counter, cycles);
    else
        dev::batch_kernel<float><<<grid, dev::kBatchThreads, 0, st>>>(parts, items, nitems, counter, cycles);
    BCUDA(cudaGetLastError());
    return CSP_OK;
}

// process-wide decision cache: signature -> format
std::mutex g_cache_mu;
std::map<unsigned long long, int> g_cache;

void cache_read(const char* path)
{
    if (!path) return;
    FILE* f = fopen(path, "r");
    if (!f) return;
    char line[256];
    std::lock_guard<std::mutex> lk(g_cache_mu);
    while (fgets(line, sizeof(line), f)) {
        unsigned long long k = 0;
        int fmt = -1;
        if (sscanf(line, "%llx batch %d", &k, &fmt) == 2 && fmt >= 0 && fmt < CSP_BFMT_COUNT) g_cache[k] = fmt;
    }
    fclose(f);
}

void cache_write(const char* path, unsigned long long k, int fmt, double cost)
{
    {
        std::lock_guard<std::mutex> lk(g_cache_mu);
        g_cache[k] = fmt;
    }
    if (!path) return;
    FILE* f = fopen(path, "a");
    if (!f) return;
    fprintf(f, "%016llx batch %d %.4f\n", k, fmt, cost);
    fclose(f);
}

bool cache_get(unsigned long long k, int& fmt)
{
    std::lock_guard<std::mutex> lk(g_cache_mu);
    auto it = g_cache.find(k);
    if (it == g_cache.end()) return false;
    fmt = it->second;
    return true;
}

}  // namespace
}  // namespace csp

using namespace csp;

// ---------------------------------------------------------------------------
// the batch object
// ---------------------------------------------------------------------------
struct csp_batch {
    int n = 0;
    int flags = 0;
    bool bf16 = false, adjoint = false, use_graph = false;
    std::vector<int> fmt, fmt_t;   // formats of A and of A^T
    std::vector<long long> xoff, yoff, goff;
    Arena arena;
    float *x = nullptr, *y = nullptr, *ybar = nullptr, *xbar = nullptr, *abar = nullptr, *yscratch = nullptr;
    int* counter = nullptr;   // the persistent kernel's item counter
    std::vector<dev::BatchPart> hparts;      // [fwd(n) | fwd+grad(n) | grad only(n) | adj(n)]
    dev::BatchPart* dparts = nullptr;
    dev::BatchItem* ditems[4] = {nullptr, nullptr, nullptr, nullptr};   // by `what`
    int nitems[4] = {0, 0, 0, 0};
    int grid[4] = {1, 1, 1, 1};
    std::vector<std::vector<dev::BatchItem>> ranges_fwd, ranges_adj;   // per matrix
    std::vector<int> plain_g;                                 // csp_batch_run_plain lanes per row (A, A^T)
    cudaStream_t own_stream = nullptr, stream = nullptr;
    cudaGraphExec_t graph[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaStream_t graph_stream[4] = {nullptr, nullptr, nullptr, nullptr};

    ~csp_batch()
    {
        for (auto& g : graph)
            if (g) cudaGraphExecDestroy(g);
        arena.release();
        if (own_stream) cudaStreamDestroy(own_stream);
    }
};

namespace {

// Builds the item list of one direction set from per-part ranges.
std::vector<dev::BatchItem> items_for(const csp_batch* b, int what)
{
    std::vector<dev::BatchItem> it;
    const int n = b->n;
    auto add = [&](const std::vector<dev::BatchItem>& rs, int part) {
        for (dev::BatchItem r : rs) {
            r.part = part;
            it.push_back(r);
        }
    };
    for (int i = 0; i < n; i++) {
        if (what & CSP_BATCH_FWD) add(b->ranges_fwd[i], (what & CSP_BATCH_ADJ) ? n + i : i);
        else if (what & CSP_BATCH_ADJ) add(b->ranges_fwd[i], 2 * n + i);
        if (what & CSP_BATCH_ADJ) add(b->ranges_adj[i], 3 * n + i);
    }
    return it;
}

// Device timing of candidate formats for one side of the batch -- the stored matrices
// A (forward, with the value-gradient store when `grad`) or their transposes A^T
// (adjoint) -- for every signature class without a cached decision: each round stores
// up to 4 representative operators of every class in that round's candidate format and
// runs them in the persistent kernel a few times with per-part cycle counters; a class
// takes the format with the fewest cycles per stored entry.  `salt` separates the two
// sides' classes in the decision cache.
int tune_classes(const std::vector<HCsr>& M, const std::vector<csp_batch_features>& F, bool grad,
                 unsigned long long salt, int flags, const char* cache_path, std::vector<int>& choice)
{
    const bool bf16 = (flags & CSP_FLAG_BF16) != 0;
    const int n = (int)M.size();
    std::map<unsigned long long, std::vector<int>> classes;
    for (int i = 0; i < n; i++) {
        int f = -1;
        const unsigned long long sig = F[i].signature ^ salt;
        if (cache_get(sig, f)) choice[i] = (F[i].feasible & (1u << f)) ? f : F[i].model_format;
        else classes[sig].push_back(i);
    }
    if (classes.empty()) return CSP_OK;
    struct Cls { unsigned long long sig; std::vector<int> reps; unsigned feas; double cost[CSP_BFMT_COUNT]; };
    std::vector<Cls> cls;
    for (auto& kv : classes) {
        Cls c;
        c.sig = kv.first;
        std::vector<int> m = kv.second;
        std::sort(m.begin(), m.end(), [&](int p, int q) { return F[p].nnz > F[q].nnz; });
        m.resize(std::min<size_t>(m.size(), 4));
        c.reps = m;
        c.feas = F[m[0]].feasible;
        for (int r : m) c.feas &= F[r].feasible;
        for (double& x : c.cost) x = -1.0;
        cls.push_back(c);
    }
    cudaStream_t st;
    BCUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    int rc = CSP_OK;
    for (int fmt = 0; fmt < CSP_BFMT_COUNT && rc == CSP_OK; fmt++) {
        Arena ar;
        std::vector<HPart> hp;
        std::vector<PartOffs> po;
        std::vector<int> owner;   // class of each timed operator
        std::vector<size_t> vx, vy, vg;
        for (int c = 0; c < (int)cls.size(); c++) {
            if (!(cls[c].feas & (1u << fmt))) continue;
            for (int r : cls[c].reps) {
                hp.emplace_back();
                build_part(fmt, M[r], hp.back());
                owner.push_back(c);
            }
        }
        if (hp.empty()) continue;
        for (const HPart& p : hp) {
            po.push_back(stage_part(ar, p, bf16));
            vx.push_back(ar.take((size_t)p.n * 4 + 16));
            vy.push_back(ar.take((size_t)p.m * 4 + 16));
            vg.push_back(ar.take((size_t)p.slots * 4 + 16));
        }
        const size_t o_parts = ar.take(hp.size() * sizeof(dev::BatchPart));
        std::vector<dev::BatchItem> items;
        for (int q = 0; q < (int)hp.size(); q++)
            for (dev::BatchItem r : hp[q].ranges) {
                r.part = q;
                items.push_back(r);
            }
        const size_t o_items = ar.stage(items);
        const size_t o_cyc = ar.take(hp.size() * 8);
        const size_t o_ctr = ar.take(sizeof(int));
        if ((rc = ar.commit())) break;
        std::vector<dev::BatchPart> d;
        for (int q = 0; q < (int)hp.size(); q++) {
            dev::BatchPart bp = make_desc(hp[q], po[q], ar.base);
            bp.x = reinterpret_cast<float*>(ar.base + vx[q]);
            bp.y = reinterpret_cast<float*>(ar.base + vy[q]);
            bp.ybar = bp.y;   // any readable vector of the right length
            bp.abar = reinterpret_cast<float*>(ar.base + vg[q]);
            bp.grad = grad ? 1 : 0;
            d.push_back(bp);
        }
        cudaError_t e = cudaMemcpy(ar.base + o_parts, d.data(), d.size() * sizeof(dev::BatchPart), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) { rc = cuda_error(e, "batch tuning upload"); ar.release(); break; }
        const int grid = occupancy_grid(bf16, (int)items.size());
        auto* parts = reinterpret_cast<const dev::BatchPart*>(ar.base + o_parts);
        auto* ditems = reinterpret_cast<const dev::BatchItem*>(ar.base + o_items);
        auto* cyc = reinterpret_cast<unsigned long long*>(ar.base + o_cyc);
        auto* ctr = reinterpret_cast<int*>(ar.base + o_ctr);
        rc = launch_batch(bf16, parts, ditems, (int)items.size(), ctr, nullptr, grid, st);
        if (!rc) {
            e = cudaMemsetAsync(cyc, 0, hp.size() * 8, st);
            if (e != cudaSuccess) rc = cuda_error(e, "batch tuning");
        }
        const int reps = 3;
        for (int k = 0; k < reps && !rc; k++) rc = launch_batch(bf16, parts, ditems, (int)items.size(), ctr, cyc, grid, st);
        std::vector<unsigned long long> hc(hp.size());
        if (!rc) {
            e = cudaMemcpyAsync(hc.data(), cyc, hp.size() * 8, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) rc = cuda_error(e, "batch tuning timing");
        }
        ar.release();
        if (rc) break;
        std::vector<double> sum(cls.size(), 0.0);
        for (int q = 0; q < (int)hp.size(); q++) sum[owner[q]] += (double)hc[q] / reps;
        for (int c = 0; c < (int)cls.size(); c++) {
            if (!(cls[c].feas & (1u << fmt))) continue;
            long long nnz = 0;
            for (int r : cls[c].reps) nnz += F[r].nnz;
            cls[c].cost[fmt] = sum[c] / (double)std::max(1LL, nnz);
        }
    }
    cudaStreamDestroy(st);
    if (rc) return rc;
    for (Cls& c : cls) {
        int best = CSP_BFMT_CSR;
        for (int f = 0; f < CSP_BFMT_COUNT; f++)
            if (c.cost[f] >= 0.0 && (c.cost[best] < 0.0 || c.cost[f] < c.cost[best])) best = f;
        cache_write(cache_path, c.sig, best, c.cost[best]);
        for (int i : classes[c.sig]) choice[i] = (F[i].feasible & (1u << best)) ? best : F[i].model_format;
    }
    return CSP_OK;
}

float* vec_of(csp_batch* b, int which)
{
    switch (which) {
    case CSP_BV_X: return b->x;
    case CSP_BV_Y: return b->y;
    case CSP_BV_YBAR: return b->ybar;
    case CSP_BV_XBAR: return b->xbar;
    case CSP_BV_ABAR: return b->abar;
    }
    return nullptr;
}

size_t vec_len(const csp_batch* b, int which)
{
    switch (which) {
    case CSP_BV_X:
    case CSP_BV_XBAR: return (size_t)b->xoff[b->n];
    case CSP_BV_Y:
    case CSP_BV_YBAR: return (size_t)b->yoff[b->n];
    case CSP_BV_ABAR: return (size_t)b->goff[b->n];
    }
    return 0;
}

}  // namespace

extern "C" {

int csp_batch_features_of(const coo_matrix_if* mat, int flags, csp_batch_features* out)
{
    clear_error();
    if (!out) return set_error(CSP_EINVAL, "null output");
    int rc = check_coo(mat);
    if (rc) return rc;
    HCsr c;
    csr_of(mat, c);
    features(c, flags, *out);
    return CSP_OK;
}

int csp_batch_create(const coo_matrix_if* const* mats, int n, const csp_batch_opts* opts, csp_batch** out)
{
    clear_error();
    if (!out) return set_error(CSP_EINVAL, "null output");
    *out = nullptr;
    if (!mats || n <= 0) return set_error(CSP_EINVAL, "empty batch");
    csp_batch_opts o = {0, CSP_BFMT_AUTO, CSP_BATCH_TUNE_MODEL, nullptr};
    if (opts) o = *opts;
    if (o.format < CSP_BFMT_AUTO || o.format >= CSP_BFMT_COUNT) return set_error(CSP_EINVAL, "unknown batch format %d", o.format);
    if (o.tune != CSP_BATCH_TUNE_MODEL && o.tune != CSP_BATCH_TUNE_DEVICE) return set_error(CSP_EINVAL, "unknown tune mode %d", o.tune);
    int rc;
    for (int i = 0; i < n; i++)
        if ((rc = check_coo(mats[i]))) return set_error(rc, "batch matrix %d: %s", i, csp_last_error());
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return set_error(CSP_ENODEV, "no CUDA device");

    std::unique_ptr<csp_batch> b(new csp_batch);
    b->n = n;
    b->flags = o.flags;
    b->bf16 = (o.flags & CSP_FLAG_BF16) != 0;
    b->adjoint = (o.flags & CSP_FLAG_ADJOINT) != 0;
    b->use_graph = (o.flags & CSP_FLAG_GRAPH) != 0;
    std::vector<HCsr> A((size_t)n), AT;
    std::vector<csp_batch_features> F((size_t)n);
    for (int i = 0; i < n; i++) {
        csr_of(mats[i], A[i]);
        features(A[i], o.flags, F[i]);
    }
    const bool need_t = b->adjoint;
    std::vector<csp_batch_features> FT;
    if (need_t) {
        AT.resize((size_t)n);
        FT.resize((size_t)n);
        for (int i = 0; i < n; i++) {
            transpose(A[i], AT[i]);
            features(AT[i], o.flags, FT[i]);
        }
    }
    b->fmt.assign((size_t)n, CSP_BFMT_CSR);
    b->fmt_t.assign((size_t)n, CSP_BFMT_CSR);
    b->plain_g.assign((size_t)2 * n, 1);
    for (int i = 0; i < n; i++) {
        const double nz = F[i].nnz;
        const double mean[2] = {F[i].rows ? nz / F[i].rows : 0.0, F[i].cols ? nz / F[i].cols : 0.0};
        for (int t = 0; t < 2; t++) {
            int g = 1;
            while (g < 32 && g * 2 <= mean[t]) g *= 2;
            b->plain_g[2 * i + t] = g;
        }
    }
    // A and A^T choose their formats independently (A^T of a matrix with long rows has
    // short, even ones); a forced format applies to both
    if (o.format != CSP_BFMT_AUTO) {
        for (int i = 0; i < n; i++) {
            if (!(F[i].feasible & (1u << o.format)))
                return set_error(CSP_EFORMAT, "batch matrix %d: format %d not feasible", i, o.format);
            b->fmt[i] = b->fmt_t[i] = o.format;
        }
    } else if (o.tune == CSP_BATCH_TUNE_MODEL) {
        for (int i = 0; i < n; i++) {
            b->fmt[i] = F[i].model_format;
            if (need_t) b->fmt_t[i] = FT[i].model_format;
        }
    } else {
        cache_read(o.cache_path);
        if ((rc = tune_classes(A, F, b->adjoint, 0ULL, o.flags, o.cache_path, b->fmt))) return rc;
        if (need_t && (rc = tune_classes(AT, FT, false, 0x9e3779b97f4a7c15ULL, o.flags, o.cache_path, b->fmt_t)))
            return rc;
    }

    BCUDA(cudaStreamCreateWithFlags(&b->own_stream, cudaStreamNonBlocking));
    b->stream = b->own_stream;

    // stored operators
    std::vector<HPart> fw((size_t)n), bw;
    std::vector<PartOffs> fo((size_t)n), bo;
    if (b->adjoint) { bw.resize((size_t)n); bo.resize((size_t)n); }
    b->xoff.assign((size_t)n + 1, 0);
    b->yoff.assign((size_t)n + 1, 0);
    b->goff.assign((size_t)n + 1, 0);
    b->ranges_fwd.resize((size_t)n);
    b->ranges_adj.resize((size_t)n);
    Arena& ar = b->arena;
    for (int i = 0; i < n; i++) {
        build_part(b->fmt[i], A[i], fw[i]);
        fo[i] = stage_part(ar, fw[i], b->bf16);
        b->ranges_fwd[i] = fw[i].ranges;
        b->xoff[i + 1] = b->xoff[i] + A[i].n;
        b->yoff[i + 1] = b->yoff[i] + A[i].m;
        b->goff[i + 1] = b->goff[i] + (b->adjoint ? pad_ll(fw[i].slots, 64) : 0);
        if (b->adjoint) {
            build_part(b->fmt_t[i], AT[i], bw[i]);
            bo[i] = stage_part(ar, bw[i], b->bf16);
            b->ranges_adj[i] = bw[i].ranges;
            bw[i].i0.clear(); bw[i].i0.shrink_to_fit();
            bw[i].i1.clear(); bw[i].i1.shrink_to_fit();
            bw[i].v.clear(); bw[i].v.shrink_to_fit();
        }
        fw[i].i0.clear(); fw[i].i0.shrink_to_fit();
        fw[i].i1.clear(); fw[i].i1.shrink_to_fit();
        fw[i].v.clear(); fw[i].v.shrink_to_fit();
        A[i].rp.clear(); A[i].rp.shrink_to_fit();
        A[i].col.clear(); A[i].col.shrink_to_fit();
        A[i].val.clear(); A[i].val.shrink_to_fit();
        if (need_t) { AT[i].rp.clear(); AT[i].rp.shrink_to_fit(); AT[i].col.clear(); AT[i].col.shrink_to_fit(); AT[i].val.clear(); AT[i].val.shrink_to_fit(); }
    }
    const size_t nx = (size_t)b->xoff[n], ny = (size_t)b->yoff[n], ng = (size_t)b->goff[n];
    const size_t o_x = ar.take(nx * 4 + 16), o_y = ar.take(ny * 4 + 16);
    size_t o_yb = 0, o_xb = 0, o_g = 0, o_ys = 0;
    if (b->adjoint) {
        o_yb = ar.take(ny * 4 + 16);
        o_xb = ar.take(nx * 4 + 16);
        o_g = ar.take(ng * 4 + 16);
        o_ys = ar.take(ny * 4 + 16);
    }
    const size_t o_parts = ar.take((size_t)4 * n * sizeof(dev::BatchPart));
    const size_t o_ctr = ar.take(sizeof(int));
    const int whats[3] = {CSP_BATCH_FWD, CSP_BATCH_ADJ, CSP_BATCH_FWD | CSP_BATCH_ADJ};
    size_t o_items[4] = {0, 0, 0, 0};
    for (int w : whats) {
        if ((w & CSP_BATCH_ADJ) && !b->adjoint) continue;
        std::vector<dev::BatchItem> it = items_for(b.get(), w);
        b->nitems[w] = (int)it.size();
        o_items[w] = ar.stage(it);
    }
    if ((rc = ar.commit())) return rc;
    char* base = ar.base;
    b->x = reinterpret_cast<float*>(base + o_x);
    b->y = reinterpret_cast<float*>(base + o_y);
    b->counter = reinterpret_cast<int*>(base + o_ctr);
    if (b->adjoint) {
        b->ybar = reinterpret_cast<float*>(base + o_yb);
        b->xbar = reinterpret_cast<float*>(base + o_xb);
        b->abar = reinterpret_cast<float*>(base + o_g);
        b->yscratch = reinterpret_cast<float*>(base + o_ys);
    }
    b->hparts.resize((size_t)4 * n);
    for (int i = 0; i < n; i++) {
        dev::BatchPart d = make_desc(fw[i], fo[i], base);
        d.x = b->x + b->xoff[i];
        d.y = b->y + b->yoff[i];
        b->hparts[i] = d;
        if (b->adjoint) {
            d.grad = 1;
            d.ybar = b->ybar + b->yoff[i];
            d.abar = b->abar + b->goff[i];
            b->hparts[n + i] = d;
            d.y = b->yscratch + b->yoff[i];
            b->hparts[2 * n + i] = d;
            dev::BatchPart t = make_desc(bw[i], bo[i], base);
            t.x = b->ybar + b->yoff[i];
            t.y = b->xbar + b->xoff[i];
            b->hparts[3 * n + i] = t;
        }
    }
    b->dparts = reinterpret_cast<dev::BatchPart*>(base + o_parts);
    BCUDA(cudaMemcpy(b->dparts, b->hparts.data(), b->hparts.size() * sizeof(dev::BatchPart), cudaMemcpyHostToDevice));
    for (int w : whats) {
        b->ditems[w] = reinterpret_cast<dev::BatchItem*>(base + o_items[w]);
        b->grid[w] = occupancy_grid(b->bf16, std::max(1, b->nitems[w]));
    }
    *out = b.release();
    return CSP_OK;
}

int csp_batch_free(csp_batch* b)
{
    delete b;
    return CSP_OK;
}

int csp_batch_layout(const csp_batch* b, long long* x_off, long long* y_off, long long* abar_off)
{
    if (!b) return set_error(CSP_EINVAL, "null batch");
    if (x_off) memcpy(x_off, b->xoff.data(), b->xoff.size() * sizeof(long long));
    if (y_off) memcpy(y_off, b->yoff.data(), b->yoff.size() * sizeof(long long));
    if (abar_off) memcpy(abar_off, b->goff.data(), b->goff.size() * sizeof(long long));
    return CSP_OK;
}

int csp_batch_formats(const csp_batch* b, int* formats)
{
    if (!b || !formats) return set_error(CSP_EINVAL, "null argument");
    memcpy(formats, b->fmt.data(), b->fmt.size() * sizeof(int));
    return CSP_OK;
}

int csp_batch_formats_adjoint(const csp_batch* b, int* formats)
{
    if (!b || !formats) return set_error(CSP_EINVAL, "null argument");
    if (!b->adjoint) return set_error(CSP_EUNSUP, "batch built without CSP_FLAG_ADJOINT");
    memcpy(formats, b->fmt_t.data(), b->fmt_t.size() * sizeof(int));
    return CSP_OK;
}

int csp_batch_device_ptrs(const csp_batch* b, float** x, float** y, float** ybar, float** xbar, float** abar)
{
    if (!b) return set_error(CSP_EINVAL, "null batch");
    if (x) *x = b->x;
    if (y) *y = b->y;
    if (ybar) *ybar = b->ybar;
    if (xbar) *xbar = b->xbar;
    if (abar) *abar = b->abar;
    return CSP_OK;
}

int csp_batch_copy(csp_batch* b, int which, const float* src, float* dst)
{
    if (!b) return set_error(CSP_EINVAL, "null batch");
    if ((src == nullptr) == (dst == nullptr)) return set_error(CSP_EINVAL, "exactly one of src, dst");
    float* d = vec_of(b, which);
    if (!d) return set_error(CSP_EINVAL, "vector %d not present", which);
    const size_t bytes = vec_len(b, which) * 4;
    if (!bytes) return CSP_OK;
    if (src) {
        BCUDA(cudaMemcpyAsync(d, src, bytes, cudaMemcpyHostToDevice, b->stream));
    } else {
        BCUDA(cudaMemcpyAsync(dst, d, bytes, cudaMemcpyDeviceToHost, b->stream));
        BCUDA(cudaStreamSynchronize(b->stream));
    }
    return CSP_OK;
}

int csp_batch_set_stream(csp_batch* b, void* stream)
{
    if (!b) return set_error(CSP_EINVAL, "null batch");
    b->stream = stream ? static_cast<cudaStream_t>(stream) : b->own_stream;
    return CSP_OK;
}

void* csp_batch_get_stream(const csp_batch* b) { return b ? b->stream : nullptr; }

int csp_batch_run(csp_batch* b, int what, int ntimes)
{
    clear_error();
    if (!b) return set_error(CSP_EINVAL, "null batch");
    if (what < 1 || what > 3) return set_error(CSP_EINVAL, "what must be CSP_BATCH_FWD and/or CSP_BATCH_ADJ");
    if ((what & CSP_BATCH_ADJ) && !b->adjoint) return set_error(CSP_EUNSUP, "batch built without CSP_FLAG_ADJOINT");
    if (ntimes < 0) return set_error(CSP_EINVAL, "ntimes < 0");
    cudaStream_t st = b->stream;
    if (!b->use_graph) {
        for (int k = 0; k < ntimes; k++) {
            int rc = launch_batch(b->bf16, b->dparts, b->ditems[what], b->nitems[what], b->counter, nullptr, b->grid[what], st);
            if (rc) return rc;
        }
        return CSP_OK;
    }
    if (!b->graph[what] || b->graph_stream[what] != st) {
        if (b->graph[what]) { cudaGraphExecDestroy(b->graph[what]); b->graph[what] = nullptr; }
        cudaGraph_t g;
        BCUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        int rc = launch_batch(b->bf16, b->dparts, b->ditems[what], b->nitems[what], b->counter, nullptr, b->grid[what], st);
        cudaError_t e = cudaStreamEndCapture(st, &g);
        if (rc) { if (e == cudaSuccess) cudaGraphDestroy(g); return rc; }
        if (e != cudaSuccess) return cuda_error(e, "cudaStreamEndCapture");
        e = cudaGraphInstantiate(&b->graph[what], g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return cuda_error(e, "cudaGraphInstantiate");
        b->graph_stream[what] = st;
    }
    for (int k = 0; k < ntimes; k++) BCUDA(cudaGraphLaunch(b->graph[what], st));
    return CSP_OK;
}

int csp_batch_run_plain(csp_batch* b, int what, int ntimes, int lanes)
{
    clear_error();
    if (!b) return set_error(CSP_EINVAL, "null batch");
    if (what < 1 || what > 3) return set_error(CSP_EINVAL, "what must be CSP_BATCH_FWD and/or CSP_BATCH_ADJ");
    if ((what & CSP_BATCH_ADJ) && !b->adjoint) return set_error(CSP_EUNSUP, "batch built without CSP_FLAG_ADJOINT");
    for (int f : b->fmt)
        if (f != CSP_BFMT_CSR) return set_error(CSP_EUNSUP, "plain runs need every matrix in CSR");
    if (b->adjoint)
        for (int f : b->fmt_t)
            if (f != CSP_BFMT_CSR) return set_error(CSP_EUNSUP, "plain runs need every transpose in CSR");
    if (lanes != 0 && (lanes < 1 || lanes > 32 || (lanes & (lanes - 1))))
        return set_error(CSP_EINVAL, "lanes must be 0 or a power of two up to 32");
    cudaStream_t st = b->stream;
    const int n = b->n;
    // CSR-vector SpMV with the lanes per row picked from the mean row length
    auto vec = [&](const dev::BatchPart& p, int g, const float* x, float* y) {
        const int m = p.m;
        if (m == 0) return;
        const unsigned grid = (unsigned)(((long long)m * g + 255) / 256);
        const int* rp = p.i0;
        const int* col = p.i1;
#define CSP_PV(V, G) dev::csr_vector_kernel<V, G><<<grid, 256, 0, st>>>(rp, col, static_cast<const V*>(p.v), x, y, m)
#define CSP_PVG(V)                                                       \
    switch (g) {                                                         \
    case 1: CSP_PV(V, 1); break;                                         \
    case 2: CSP_PV(V, 2); break;                                         \
    case 4: CSP_PV(V, 4); break;                                         \
    case 8: CSP_PV(V, 8); break;                                         \
    case 16: CSP_PV(V, 16); break;                                       \
    default: CSP_PV(V, 32); break;                                       \
    }
        if (b->bf16) { CSP_PVG(__nv_bfloat16) } else { CSP_PVG(float) }
#undef CSP_PVG
#undef CSP_PV
    };
    for (int k = 0; k < ntimes; k++) {
        for (int i = 0; i < n; i++) {
            const dev::BatchPart& f = b->hparts[i];
            if (what & CSP_BATCH_FWD) vec(f, lanes ? lanes : b->plain_g[2 * i], f.x, f.y);
            if (what & CSP_BATCH_ADJ) {
                if (f.m) {
                    const unsigned grid = (unsigned)(((long long)f.m * 32 + 255) / 256);
                    dev::csr_grad_kernel<<<grid, 256, 0, st>>>(f.i0, f.i1, b->ybar + b->yoff[i], f.x, b->abar + b->goff[i], f.m);
                }
                const dev::BatchPart& t = b->hparts[3 * n + i];
                vec(t, lanes ? lanes : b->plain_g[2 * i + 1], t.x, t.y);
            }
        }
    }
    BCUDA(cudaGetLastError());
    return CSP_OK;
}

int csp_batch_synchronize(csp_batch* b)
{
    if (!b) return set_error(CSP_EINVAL, "null batch");
    BCUDA(cudaStreamSynchronize(b->stream));
    return CSP_OK;
}

int csp_batch_launches(const csp_batch* b, int what, int plain)
{
    if (!b || what < 1 || what > 3) return 0;
    if (!plain) return b->nitems[what] > 0 ? 1 : 0;
    int c = 0;
    for (int i = 0; i < b->n; i++) {
        if ((what & CSP_BATCH_FWD) && b->hparts[i].m) c++;
        if (what & CSP_BATCH_ADJ) c += (b->hparts[i].m ? 1 : 0) + (b->hparts[3 * b->n + i].m ? 1 : 0);
    }
    return c;
}

size_t csp_batch_device_bytes(const csp_batch* b) { return b ? b->arena.size : 0; }

int csp_batch_pattern(const csp_batch* b, int i, int* rows, int* cols)
{
    clear_error();
    if (!b || !rows || !cols) return set_error(CSP_EINVAL, "null argument");
    if (i < 0 || i >= b->n) return set_error(CSP_EINVAL, "matrix %d outside the batch", i);
    const dev::BatchPart& p = b->hparts[i];
    const long long slots = b->goff[i + 1] - b->goff[i];
    for (long long s = 0; s < slots; s++) rows[s] = cols[s] = -1;
    if (!b->adjoint) return CSP_OK;
    // the structure arrays are read back from the device
    auto rd = [&](const int* d, size_t count, std::vector<int>& h) -> int {
        h.resize(count);
        if (count) BCUDA(cudaMemcpy(h.data(), d, count * 4, cudaMemcpyDeviceToHost));
        return CSP_OK;
    };
    std::vector<int> i0, i1;
    int rc;
    switch (p.kind) {
    case dev::BK_CSR: {
        if ((rc = rd(p.i0, (size_t)p.m + 1, i0))) return rc;
        if ((rc = rd(p.i1, (size_t)i0[p.m], i1))) return rc;
        for (int r = 0; r < p.m; r++)
            for (int j = i0[r]; j < i0[r + 1]; j++) { rows[j] = r; cols[j] = i1[j]; }
        break;
    }
    case dev::BK_SELL: {
        const int H = p.stride;
        if ((rc = rd(p.i0, (size_t)p.nbr + 1, i0))) return rc;
        if ((rc = rd(p.i1, (size_t)i0[p.nbr], i1))) return rc;
        for (int s = 0; s < p.nbr; s++) {
            const int w = (i0[s + 1] - i0[s]) / H;
            for (int k = 0; k < w; k++)
                for (int lr = 0; lr < H; lr++) {
                    const int q = i0[s] + k * H + lr, r = s * H + lr;
                    if (r < p.m && i1[q] >= 0) { rows[q] = r; cols[q] = i1[q]; }
                }
        }
        break;
    }
    case dev::BK_DIA: {
        if ((rc = rd(p.i0, (size_t)p.k, i0))) return rc;
        for (int d = 0; d < p.k; d++)
            for (int r = 0; r < p.m; r++) {
                const int c = r + i0[d];
                if (c >= 0 && c < p.n) { rows[(size_t)d * p.stride + r] = r; cols[(size_t)d * p.stride + r] = c; }
            }
        break;
    }
    default: {
        const int B = p.kind - dev::BK_BCSR2 + 2;
        if ((rc = rd(p.i0, (size_t)p.nbr + 1, i0))) return rc;
        if ((rc = rd(p.i1, (size_t)i0[p.nbr], i1))) return rc;
        for (int br = 0; br < p.nbr; br++)
            for (int j = i0[br]; j < i0[br + 1]; j++)
                for (int h = 0; h < B; h++)
                    for (int w = 0; w < B; w++) {
                        const int r = br * B + h, c = i1[j] + w;
                        if (r < p.m && c < p.n) {
                            const size_t q = (size_t)(h * B + w) * p.stride + j;
                            rows[q] = r;
                            cols[q] = c;
                        }
                    }
        break;
    }
    }
    return CSP_OK;
}

}  // extern "C"
