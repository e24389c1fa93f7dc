// On-device autotuner for the Cocktail partition (CSP_ANALYZE_AUTOTUNE).
//
// The reference chooses formats from GFLOPS tables measured once on a 2012 GPU
// (clSpMV_NV/src/analyze.cpp, benchmark/*.ben).  Here the candidates are built for
// the actual matrix and timed on the actual device: every format whose padding stays
// within bounds, each kernel variant, SELL slice heights 32 and 128, the eight b4
// block shapes where sampled block fill is high enough, and two splits (ELL of the
// common row length + adaptive CSR for the overflow; SELL with per-slice quantile
// widths + adaptive CSR).  Each candidate runs a few SpMVs with L2 flushed before
// each, the fastest median wins, and the choice is recorded under a 64-bit hash of
// the sparsity pattern (and flags) so the next call on that pattern only rebuilds it.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <algorithm>
#include <map>
#include <string>
#include <vector>

#include "csp/clspmv.h"
#include "internal.h"
#include "engine.h"

namespace csp {

static thread_local std::string g_choice;

namespace {

struct Coo {
    const coo_matrix_if* m;
    std::vector<int> rp;     // row pointer
    int maxlen = 0;
};

uint64_t pattern_hash(const coo_matrix_if* m, int flags)
{
    uint64_t h = 1469598103934665603ULL;
    auto mix = [&h](uint64_t v) {
        for (int i = 0; i < 8; i++) { h ^= (v >> (8 * i)) & 0xff; h *= 1099511628211ULL; }
    };
    mix((uint64_t)m->matinfo.height);
    mix((uint64_t)m->matinfo.width);
    mix((uint64_t)m->matinfo.nnz);
    mix((uint64_t)flags);
    for (int i = 0; i < m->matinfo.nnz; i++) mix(((uint64_t)(uint32_t)m->coo_row_id[i] << 32) | (uint32_t)m->coo_col_id[i]);
    return h;
}

void info_of(const coo_matrix_if* m, cocktail_iif* c)
{
    c->mat_width = m->matinfo.width;
    c->mat_height = m->matinfo.height;
    c->mat_nnz = m->matinfo.nnz;
}

// ELL holding the first k entries of every row; the rest as CSR (adaptive kernel).
int build_ell_split(const Coo& a, int k, int csr_meth, cocktail_iif* c)
{
    const coo_matrix_if* m = a.m;
    const int h = m->matinfo.height;
    const int hal = csp_aligned_length(h, 32);
    ell_matrix_if& e = c->ell;
    e.matinfo.width = m->matinfo.width;
    e.matinfo.height = h;
    e.ell_num = k;
    e.ell_height_aligned = hal;
    e.ell_col_id = static_cast<int*>(calloc((size_t)hal * k + 1, sizeof(int)));
    e.ell_data = static_cast<float*>(calloc((size_t)hal * k + 1, sizeof(float)));
    std::vector<int> rrp((size_t)h + 1, 0), rcol;
    std::vector<float> rval;
    int ell_nnz = 0;
    for (int r = 0; r < h; r++) {
        int last = 0, j = 0;
        for (int q = a.rp[r]; q < a.rp[r + 1]; q++, j++) {
            if (j < k) {
                e.ell_col_id[r + (size_t)j * hal] = last = m->coo_col_id[q];
                e.ell_data[r + (size_t)j * hal] = m->coo_data[q];
                ell_nnz++;
            } else {
                rcol.push_back(m->coo_col_id[q]);
                rval.push_back(m->coo_data[q]);
            }
        }
        for (; j < k; j++) e.ell_col_id[r + (size_t)j * hal] = last;
        rrp[r + 1] = (int)rcol.size();
    }
    e.matinfo.nnz = ell_nnz;
    c->ifuseell = true;
    c->ell_meth_num = 1;
    if (!rcol.empty()) {
        csr_matrix_if& s = c->csr;
        s.matinfo.width = m->matinfo.width;
        s.matinfo.height = h;
        s.matinfo.nnz = (int)rcol.size();
        s.csr_row_ptr = static_cast<int*>(malloc(rrp.size() * sizeof(int)));
        s.csr_col_id = static_cast<int*>(malloc(rcol.size() * sizeof(int)));
        s.csr_data = static_cast<float*>(malloc(rval.size() * sizeof(float)));
        memcpy(s.csr_row_ptr, rrp.data(), rrp.size() * sizeof(int));
        memcpy(s.csr_col_id, rcol.data(), rcol.size() * sizeof(int));
        memcpy(s.csr_data, rval.data(), rval.size() * sizeof(float));
        c->ifusecsr = true;
        c->csr_meth_num = csr_meth;
    }
    return CSP_OK;
}

// SELL (slices of sh rows) whose slice width is the q-quantile row length of the
// slice; longer rows overflow to CSR (adaptive kernel).
int build_sell_split(const Coo& a, int sh, double q, int csr_meth, cocktail_iif* c)
{
    const coo_matrix_if* m = a.m;
    const int h = m->matinfo.height;
    const int ns = h / sh + (h % sh != 0);
    std::vector<int> width(ns), sp((size_t)ns + 1, 0), lens;
    for (int s = 0; s < ns; s++) {
        lens.clear();
        for (int r = s * sh; r < std::min((s + 1) * sh, h); r++) lens.push_back(a.rp[r + 1] - a.rp[r]);
        std::sort(lens.begin(), lens.end());
        width[s] = lens[std::min((size_t)(q * lens.size()), lens.size() - 1)];
        sp[s + 1] = sp[s] + width[s] * sh;
    }
    sell_matrix_if& e = c->sell;
    e.matinfo.width = m->matinfo.width;
    e.matinfo.height = h;
    e.sell_slice_height = (unsigned)sh;
    e.sell_slice_num = ns;
    e.sell_slice_ptr = static_cast<int*>(malloc(sp.size() * sizeof(int)));
    memcpy(e.sell_slice_ptr, sp.data(), sp.size() * sizeof(int));
    e.sell_col_id = static_cast<int*>(calloc((size_t)sp[ns] + 1, sizeof(int)));
    e.sell_data = static_cast<float*>(calloc((size_t)sp[ns] + 1, sizeof(float)));
    std::vector<int> rrp((size_t)h + 1, 0), rcol;
    std::vector<float> rval;
    int sell_nnz = 0;
    for (int s = 0; s < ns; s++) {
        int* col = e.sell_col_id + sp[s];
        float* val = e.sell_data + sp[s];
        for (int lr = 0; lr < sh; lr++) {
            const int r = s * sh + lr;
            int last = 0, j = 0;
            if (r < h) {
                for (int x = a.rp[r]; x < a.rp[r + 1]; x++, j++) {
                    if (j < width[s]) {
                        col[j * sh + lr] = last = m->coo_col_id[x];
                        val[j * sh + lr] = m->coo_data[x];
                        sell_nnz++;
                    } else {
                        rcol.push_back(m->coo_col_id[x]);
                        rval.push_back(m->coo_data[x]);
                    }
                }
                rrp[r + 1] = (int)rcol.size();
            }
            for (; j < width[s]; j++) col[j * sh + lr] = last;
        }
    }
    e.matinfo.nnz = sell_nnz;
    c->ifusesell = true;
    c->sell_meth_num = 0;
    if (!rcol.empty()) {
        csr_matrix_if& s = c->csr;
        s.matinfo.width = m->matinfo.width;
        s.matinfo.height = h;
        s.matinfo.nnz = (int)rcol.size();
        s.csr_row_ptr = static_cast<int*>(malloc(rrp.size() * sizeof(int)));
        s.csr_col_id = static_cast<int*>(malloc(rcol.size() * sizeof(int)));
        s.csr_data = static_cast<float*>(malloc(rval.size() * sizeof(float)));
        memcpy(s.csr_row_ptr, rrp.data(), rrp.size() * sizeof(int));
        memcpy(s.csr_col_id, rcol.data(), rcol.size() * sizeof(int));
        memcpy(s.csr_data, rval.data(), rval.size() * sizeof(float));
        c->ifusecsr = true;
        c->csr_meth_num = csr_meth;
    }
    return CSP_OK;
}

// Rows of at most t entries as a COO part (a segmented reduction gathering x from L2:
// few entries, no partial sums to merge), longer rows whole as a CSR part with kernel
// csr_meth (the x-panel one for random columns: its partial sums and merge then cover
// only the long rows).
int build_coo_split(const Coo& a, int t, int csr_meth, cocktail_iif* c)
{
    const coo_matrix_if* m = a.m;
    const int h = m->matinfo.height;
    std::vector<int> srow, scol, rrp((size_t)h + 1, 0), rcol;
    std::vector<float> sval, rval;
    for (int r = 0; r < h; r++) {
        const bool shortrow = a.rp[r + 1] - a.rp[r] <= t;
        for (int q = a.rp[r]; q < a.rp[r + 1]; q++) {
            if (shortrow) {
                srow.push_back(r);
                scol.push_back(m->coo_col_id[q]);
                sval.push_back(m->coo_data[q]);
            } else {
                rcol.push_back(m->coo_col_id[q]);
                rval.push_back(m->coo_data[q]);
            }
        }
        rrp[r + 1] = (int)rcol.size();
    }
    if (srow.empty() || rcol.empty()) return set_error(CSP_EFORMAT, "coo split: one side is empty");
    coo_matrix_if& o = c->coo;
    o.matinfo.width = m->matinfo.width;
    o.matinfo.height = h;
    o.matinfo.nnz = (int)srow.size();
    o.coo_row_id = static_cast<int*>(malloc(srow.size() * sizeof(int)));
    o.coo_col_id = static_cast<int*>(malloc(scol.size() * sizeof(int)));
    o.coo_data = static_cast<float*>(malloc(sval.size() * sizeof(float)));
    memcpy(o.coo_row_id, srow.data(), srow.size() * sizeof(int));
    memcpy(o.coo_col_id, scol.data(), scol.size() * sizeof(int));
    memcpy(o.coo_data, sval.data(), sval.size() * sizeof(float));
    c->ifusecoo = true;
    csr_matrix_if& e = c->csr;
    e.matinfo.width = m->matinfo.width;
    e.matinfo.height = h;
    e.matinfo.nnz = (int)rcol.size();
    e.csr_row_ptr = static_cast<int*>(malloc(rrp.size() * sizeof(int)));
    e.csr_col_id = static_cast<int*>(malloc(rcol.size() * sizeof(int)));
    e.csr_data = static_cast<float*>(malloc(rval.size() * sizeof(float)));
    memcpy(e.csr_row_ptr, rrp.data(), rrp.size() * sizeof(int));
    memcpy(e.csr_col_id, rcol.data(), rcol.size() * sizeof(int));
    memcpy(e.csr_data, rval.data(), rval.size() * sizeof(float));
    c->ifusecsr = true;
    c->csr_meth_num = csr_meth;
    return CSP_OK;
}

// Builds the candidate named `name` into c (fresh, zeroed).  Names: csr<m>, coo,
// ell, sell<sh>, dia<m>, bdia<m>, bcsr<bh>x<bw>m<m>, bell<bh>x<bw>, sbell<bh>x<bw>,
// ell<k>+csr<m>, sellq<sh>+csr<m> (m = the overflow CSR part's kernel), coo<t>+csr<m>
// (rows of at most t entries as COO, the others as CSR), gbcsr<bh>x<bw>
// (generic BCSR in the cocktail's bcsr member, CSP_METH_GENERIC_BCSR).  csr16 is the
// x-panel kernel (CSP_METH_XPANEL).
int build(const Coo& a, const std::string& name, cocktail_iif* c)
{
    coo_matrix_if* m = const_cast<coo_matrix_if*>(a.m);
    csp_init_cocktail(c);
    info_of(m, c);
    int x = 0, y = 0, z = 0;
    if (sscanf(name.c_str(), "ell%d+csr%d", &x, &y) == 2) return build_ell_split(a, x, y, c);
    if (sscanf(name.c_str(), "sellq%d+csr%d", &x, &y) == 2) return build_sell_split(a, x, 0.75, y, c);
    if (sscanf(name.c_str(), "coo%d+csr%d", &x, &y) == 2) return build_coo_split(a, x, y, c);
    if (sscanf(name.c_str(), "gbcsr%dx%d", &x, &y) == 2) {
        c->ifusebcsr = true;
        c->bcsr_meth_num = CSP_METH_GENERIC_BCSR;
        // built on the device unless duplicate entries make the host build's choice
        // among them the byte-exact one
        auto* gb = reinterpret_cast<bcsr_matrix_if*>(&c->bcsr);
        int rc = ensure_sorted(m);
        if (rc) return rc;
        return coo_has_duplicates(m) ? csp_coo2bcsr(m, gb, (unsigned)y, (unsigned)x, 32)
                                     : csp_coo2bcsr_device(m, gb, (unsigned)y, (unsigned)x, 32);
    }
    if (sscanf(name.c_str(), "bcsr%dx%dm%d", &x, &y, &z) == 3) {
        c->ifusebcsr = true;
        c->bcsr_meth_num = z;
        return csp_coo2b4csr(m, &c->bcsr, (unsigned)y, (unsigned)x, 32);
    }
    if (sscanf(name.c_str(), "sbell%dx%d", &x, &y) == 2) {
        c->ifusesbell = true;
        return csp_coo2sbell(m, &c->sbell, (unsigned)y, (unsigned)x, 32);
    }
    if (sscanf(name.c_str(), "bell%dx%d", &x, &y) == 2) {
        c->ifusebell = true;
        return csp_coo2b4ell(m, &c->bell, (unsigned)y, (unsigned)x, 32, 0);
    }
    if (sscanf(name.c_str(), "bdia%d", &x) == 1) {
        c->ifusebdia = true;
        c->bdia_meth_num = x;
        return csp_coo2bdia_device(m, &c->bdia, 32);
    }
    if (sscanf(name.c_str(), "dia%d", &x) == 1) {
        c->ifusedia = true;
        c->dia_meth_num = x;
        return csp_coo2dia_device(m, &c->dia, 32);
    }
    if (sscanf(name.c_str(), "sell%d", &x) == 1) {
        c->ifusesell = true;
        c->sell_meth_num = 0;
        return csp_coo2sell(m, &c->sell, (unsigned)x);
    }
    if (name == "ell") {
        c->ifuseell = true;
        c->ell_meth_num = 1;
        return csp_coo2ell(m, &c->ell, 32, 0);
    }
    if (sscanf(name.c_str(), "csr%d", &x) == 1) {
        c->ifusecsr = true;
        c->csr_meth_num = x;
        return csp_coo2csr(m, &c->csr);
    }
    if (name == "coo") {
        c->ifusecoo = true;
        coo_matrix_if& o = c->coo;
        const int n = m->matinfo.nnz;
        o.matinfo = m->matinfo;
        o.coo_row_id = static_cast<int*>(malloc((size_t)std::max(n, 1) * sizeof(int)));
        o.coo_col_id = static_cast<int*>(malloc((size_t)std::max(n, 1) * sizeof(int)));
        o.coo_data = static_cast<float*>(malloc((size_t)std::max(n, 1) * sizeof(float)));
        memcpy(o.coo_row_id, m->coo_row_id, (size_t)n * sizeof(int));
        memcpy(o.coo_col_id, m->coo_col_id, (size_t)n * sizeof(int));
        memcpy(o.coo_data, m->coo_data, (size_t)n * sizeof(float));
        return CSP_OK;
    }
    return set_error(CSP_EINVAL, "autotune: unknown candidate %s", name.c_str());
}

// Sampled fill of bh x bw blocks (nonzeros / stored block slots) over up to 2048
// evenly spaced block rows.
double sampled_fill(const Coo& a, int bh, int bw)
{
    const coo_matrix_if* m = a.m;
    const int h = m->matinfo.height;
    const int nbr = h / bh + (h % bh != 0);
    const int step = std::max(1, nbr / 2048);
    long long nz = 0, blocks = 0;
    std::vector<int> cols;
    for (int br = 0; br < nbr; br += step) {
        cols.clear();
        for (int r = br * bh; r < std::min(br * bh + bh, h); r++)
            for (int q = a.rp[r]; q < a.rp[r + 1]; q++) cols.push_back(m->coo_col_id[q] / bw);
        nz += (long long)cols.size();
        std::sort(cols.begin(), cols.end());
        blocks += std::unique(cols.begin(), cols.end()) - cols.begin();
    }
    return blocks ? (double)nz / ((double)blocks * bh * bw) : 0.0;
}

std::vector<std::string> candidates(const Coo& a)
{
    const coo_matrix_if* m = a.m;
    const int h = m->matinfo.height, w = m->matinfo.width;
    const long long nnz = m->matinfo.nnz;
    const double mean = h ? (double)nnz / h : 0.0;
    // generic BCSR block shapes (any alignment of the block grid the b4 formats need)
    std::vector<std::string> blocks;
    double best_fill = 0.0;
    for (int b : {2, 3, 4, 6, 8}) {
        const double fill = sampled_fill(a, b, b);
        if (fill < 0.5) continue;
        best_fill = std::max(best_fill, fill);
        blocks.push_back("gbcsr" + std::to_string(b) + "x" + std::to_string(b));
    }
    // a matrix made of dense blocks: the block layouts and plain CSR (the baseline) only;
    // flat formats would store every block entry with its own column id
    if (best_fill >= 0.95) {
        blocks.insert(blocks.begin(), "csr2");
        return blocks;
    }
    std::vector<std::string> c = {"csr2", "coo", "csr16"};
    c.insert(c.end(), blocks.begin(), blocks.end());
    if (mean >= 12.0) c.push_back("csr0");
    if (a.maxlen <= 64 && mean >= 2.0) c.push_back("csr3");
    // ELL / SELL when the padding stays below 1.5x / 2x of the nonzeros
    if ((long long)a.maxlen * csp_aligned_length(h, 32) <= nnz * 3 / 2) c.push_back("ell");
    for (int sh : {32, 128}) {
        long long slots = 0;
        for (int s = 0; s * sh < h; s++) {
            int mx = 0;
            for (int r = s * sh; r < std::min((s + 1) * sh, h); r++) mx = std::max(mx, a.rp[r + 1] - a.rp[r]);
            slots += (long long)mx * sh;
        }
        if (slots <= 2 * nnz) c.push_back("sell" + std::to_string(sh));
    }
    // splits for irregular rows: ELL of the length covering 90 % of rows
    {
        std::vector<int> lens((size_t)h);
        for (int r = 0; r < h; r++) lens[r] = a.rp[r + 1] - a.rp[r];
        std::sort(lens.begin(), lens.end());
        const int k = lens.empty() ? 0 : lens[(size_t)(0.9 * (lens.size() - 1))];
        for (const char* tail : {"+csr2", "+csr16"}) {
            if (k > 0 && k < a.maxlen) c.push_back("ell" + std::to_string(k) + tail);
            if (a.maxlen > 2 * mean + 1) c.push_back(std::string("sellq32") + tail);
        }
        // short rows through COO, long rows whole through the x-panel kernel
        if (a.maxlen > 64)
            for (int t : {4, 8, 16})
                if (t < a.maxlen) c.push_back("coo" + std::to_string(t) + "+csr16");
    }
    if (h == w && nnz > 0) {
        // DIA only if the padded storage stays within the reference's 2x rule: a failed
        // conversion drops the DIA and BDIA candidates (see autotune_partition)
        c.push_back("dia0");
        c.push_back("dia1");
        c.push_back("bdia0");
        c.push_back("bdia1");
    }
    static const int bhs[4] = {1, 2, 4, 8};
    for (int bw : {4, 8})
        for (int bh : bhs) {
            if (bh * bw < 4) continue;
            const double fill = sampled_fill(a, bh, bw);
            if (fill < 0.5) continue;
            const std::string s = std::to_string(bh) + "x" + std::to_string(bw);
            c.push_back("bcsr" + s + "m0");
            c.push_back("bcsr" + s + "m1");
            c.push_back("sbell" + s);
            c.push_back("bell" + s);
        }
    return c;
}

// Median of `reps` SpMVs, each after an L2-clearing write of `flush`.
int time_candidate(const cocktail_iif* c, int flags, void* flush, size_t flush_bytes, int reps, double* ms)
{
    csp_handle* h = nullptr;
    int rc = csp_init_mat_kernels(c, nullptr, nullptr, flags, &h);
    if (rc) return rc;
    cudaStream_t st = nullptr;
    csp_get_stream(h, reinterpret_cast<void**>(&st));
    std::vector<float> t;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    rc = csp_do_spmv(h, 2);
    for (int i = 0; i < reps && !rc; i++) {
        cudaMemsetAsync(flush, i & 1, flush_bytes, st);
        cudaEventRecord(e0, st);
        rc = csp_do_spmv(h, 1);
        cudaEventRecord(e1, st);
        if (cudaEventSynchronize(e1) != cudaSuccess) { rc = set_error(CSP_ECUDA, "autotune timing"); break; }
        float x = 0.0f;
        cudaEventElapsedTime(&x, e0, e1);
        t.push_back(x);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    csp_free_mat_kernels(h);
    if (rc) return rc;
    std::sort(t.begin(), t.end());
    *ms = t[t.size() / 2];
    return CSP_OK;
}

// Candidates that differ only in the kernel method share one conversion: the key of
// that conversion ("" for candidates converted on their own), and the method applied to
// a shared copy.
std::string conversion_key(const std::string& name)
{
    int x = 0, y = 0, z = 0;
    if (name.find('+') != std::string::npos) return "";
    if (sscanf(name.c_str(), "bcsr%dx%dm%d", &x, &y, &z) == 3) return "bcsr" + std::to_string(x) + "x" + std::to_string(y);
    if (sscanf(name.c_str(), "bdia%d", &x) == 1) return "bdia";
    if (sscanf(name.c_str(), "dia%d", &x) == 1) return "dia";
    return "";
}

void set_method(const std::string& name, cocktail_iif* c)
{
    int x = 0, y = 0, z = 0;
    if (sscanf(name.c_str(), "bcsr%dx%dm%d", &x, &y, &z) == 3) c->bcsr_meth_num = z;
    else if (sscanf(name.c_str(), "bdia%d", &x) == 1) c->bdia_meth_num = x;
    else if (sscanf(name.c_str(), "dia%d", &x) == 1) c->dia_meth_num = x;
}

bool cache_lookup(const char* path, uint64_t key, std::string& name)
{
    if (!path) return false;
    FILE* f = fopen(path, "r");
    if (!f) return false;
    char line[512];
    bool hit = false;
    while (fgets(line, sizeof(line), f)) {
        unsigned long long k = 0;
        char nm[256];
        if (sscanf(line, "%llx %255s", &k, nm) == 2 && k == key) { name = nm; hit = true; }
    }
    fclose(f);
    return hit;
}

void cache_store(const char* path, uint64_t key, const std::string& name, double ms)
{
    if (!path) return;
    FILE* f = fopen(path, "a");
    if (!f) return;
    fprintf(f, "%016llx %s %.6f\n", (unsigned long long)key, name.c_str(), ms);
    fclose(f);
}

}  // namespace

int autotune_partition(coo_matrix_if* coo, cocktail_iif* out, const csp_analyze_opts* opts)
{
    g_choice.clear();
    int rc = ensure_sorted(coo);
    if (rc) return rc;
    Coo a;
    a.m = coo;
    const int h = coo->matinfo.height;
    a.rp.assign((size_t)h + 1, 0);
    for (int i = 0; i < coo->matinfo.nnz; i++) a.rp[(size_t)coo->coo_row_id[i] + 1]++;
    for (int r = 0; r < h; r++) {
        a.rp[r + 1] += a.rp[r];
        a.maxlen = std::max(a.maxlen, a.rp[r + 1] - a.rp[r]);
    }
    const int flags = opts->flags & CSP_FLAG_BF16;
    const uint64_t key = pattern_hash(coo, flags);
    std::string best;
    if (cache_lookup(opts->cache_path, key, best)) {
        rc = build(a, best, out);
        if (rc == CSP_OK) { g_choice = best; return CSP_OK; }
        csp_free_cocktail(out);
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return set_error(CSP_ENODEV, "autotune needs a CUDA device");
    const size_t flush_bytes = 192u << 20;   // larger than L2 (126 MB)
    void* flush = nullptr;
    if (cudaMalloc(&flush, flush_bytes) != cudaSuccess) return set_error(CSP_ENOMEM, "autotune flush buffer");
    double best_ms = 1e30;
    // conversions shared by several candidates, owned here until the end; `best_conv` is
    // the key of the one the best candidate shares ("" if it owns its arrays)
    std::map<std::string, cocktail_iif> conv;
    std::map<std::string, bool> conv_failed;
    std::string best_conv;
    for (const std::string& name : candidates(a)) {
        const std::string key = conversion_key(name);
        cocktail_iif c;
        if (key.empty()) {
            if (build(a, name, &c) != CSP_OK) { csp_free_cocktail(&c); clear_error(); continue; }
        } else {
            if (conv_failed[key]) continue;
            auto it = conv.find(key);
            if (it == conv.end()) {
                cocktail_iif cc;
                if (build(a, name, &cc) != CSP_OK) {
                    csp_free_cocktail(&cc);
                    clear_error();
                    conv_failed[key] = true;
                    continue;
                }
                it = conv.emplace(key, cc).first;
            }
            c = it->second;   // shallow: the arrays stay owned by conv
            set_method(name, &c);
        }
        double ms = 0.0;
        const int trc = time_candidate(&c, flags, flush, flush_bytes, 5, &ms);
        if (opts->verbose) printf("autotune %-16s %s %.3f us\n", name.c_str(), trc ? "failed" : "", ms * 1e3);
        if (trc == CSP_OK && ms < best_ms) {
            if (!best.empty() && best_conv.empty()) csp_free_cocktail(out);
            *out = c;
            best = name;
            best_ms = ms;
            best_conv = key;
        } else {
            if (key.empty()) csp_free_cocktail(&c);
            clear_error();
        }
    }
    for (auto& kv : conv)
        if (kv.first != best_conv) csp_free_cocktail(&kv.second);
    cudaFree(flush);
    if (best.empty()) return set_error(CSP_EFORMAT, "autotune: no candidate partition ran");
    g_choice = best;
    cache_store(opts->cache_path, key, best, best_ms);
    return CSP_OK;
}

}  // namespace csp

extern "C" const char* csp_autotune_choice(void) { return csp::g_choice.c_str(); }
