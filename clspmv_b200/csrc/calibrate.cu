// Calibration tables for the reference analyzer, measured on this device
// (csp_benchmark_tables).  The reference ships tables measured once on a 2012 GPU
// (clSpMV_NV/benchmark/*.ben), written by its bench_* programs
// (clSpMV_NV/src/bench_{dia,bdia,ell,sell,csr,coo,bcsr,bell,sbell,overhead}.cpp and the
// `benchmarking` script).  This file writes the same ten tables with the same record
// layout -- the structure parameters of a synthetic matrix, then one GFLOPS figure per
// kernel method, GFLOPS = 2 * nnz / time of one SpMV -- for this library's kernels on
// the current GPU, so csp_analyze_matrix in CSP_ANALYZE_REFERENCE mode can make its
// decisions from B200 numbers.
//
// The synthetic families are the reference's: a banded matrix of all-ones values whose
// rows hold `width` consecutive columns centred on the diagonal (shifted inwards at the
// edges), in each format's own storage; diagonal formats get `width` centred diagonals;
// block formats get `blocknum` consecutive block columns per block row.  One method
// column is measured per kernel variant the engine selects from that format's
// *_meth_num (SELL: slice height 32, then 128).  The CSR and COO tables carry one
// work-group count (the SM count): this library's kernels size their own grids.
// Times are CUDA-event times of back-to-back SpMVs after three warm-up ones, like the
// reference's timing loops (which do not clear caches either).
#include <cuda_runtime.h>
#include <errno.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <string>
#include <vector>

#include "csp/clspmv.h"
#include "internal.h"
#include "engine.h"

namespace csp {
namespace {

__global__ void calib_null_kernel(int* sink)
{
    // never true for the grids used here; keeps the launch from being optimised away
    if (sink && blockIdx.x == 0x7fffffff) sink[threadIdx.x] = 0;
}

struct Grid {
    std::vector<int> dims_large;   // 1024 .. 2M (DIA, BDIA, ELL, SELL, COO, BELL, SBELL)
    std::vector<int> dims_small;   // 1024 .. 256K (CSR, BCSR)
    std::vector<int> dia_widths;   // 1, 3, ..., 15, 19, ..., 63
    std::vector<int> ell_widths;   // 1, 2, 4, ..., 128
    std::vector<int> csr_widths;   // 2, 8, 32, ..., 2048
    std::vector<int> bcsr_blocks;  // 2, 4, ..., 512
    std::vector<int> bell_blocks;  // 1, 3, ..., 15, 19, ..., 31
    int ntimes;
};

std::vector<int> thin(const std::vector<int>& v, size_t step)
{
    std::vector<int> o;
    for (size_t i = 0; i < v.size(); i += step) o.push_back(v[i]);
    if (!v.empty() && o.back() != v.back()) o.push_back(v.back());
    return o;
}

Grid make_grid(int level)
{
    Grid g;
    for (int s = 1024; s <= 2 * 1024 * 1024; s *= 2) g.dims_large.push_back(s);
    for (int s = 1024; s <= 262144; s *= 2) g.dims_small.push_back(s);
    for (int w = 1; w < 64;) { g.dia_widths.push_back(w); w += (w < 14) ? 2 : 4; }
    for (int k = 1; k <= 128; k *= 2) g.ell_widths.push_back(k);
    for (int k = 2; k <= 2048; k *= 4) g.csr_widths.push_back(k);
    for (int b = 2; b <= 512; b *= 2) g.bcsr_blocks.push_back(b);
    for (int b = 1; b < 32;) { g.bell_blocks.push_back(b); b += (b < 14) ? 2 : 4; }
    g.ntimes = 100;
    if (level == 1) {   // every third size, every other width
        g.dims_large = thin(g.dims_large, 3);
        g.dims_small = thin(g.dims_small, 3);
        g.dia_widths = thin(g.dia_widths, 2);
        g.ell_widths = thin(g.ell_widths, 2);
        g.bcsr_blocks = thin(g.bcsr_blocks, 2);
        g.bell_blocks = thin(g.bell_blocks, 2);
        g.ntimes = 30;
    } else if (level == 0) {   // two sizes, two widths: a format check
        g.dims_large = {4096, 65536};
        g.dims_small = {4096, 65536};
        g.dia_widths = {3, 9};
        g.ell_widths = {2, 8};
        g.csr_widths = {2, 32};
        g.bcsr_blocks = {2, 8};
        g.bell_blocks = {1, 5};
        g.ntimes = 5;
    }
    return g;
}

// Milliseconds of one SpMV of `mat` (only one format used), averaged over ntimes
// back-to-back SpMVs after three warm-up ones.
int time_cocktail(const cocktail_iif& mat, int ntimes, double* ms)
{
    csp_handle* h = nullptr;
    int rc = csp_init_mat_kernels(&mat, nullptr, nullptr, 0, &h);
    if (rc) return rc;
    void* sv = nullptr;
    csp_get_stream(h, &sv);
    cudaStream_t st = static_cast<cudaStream_t>(sv);
    cudaEvent_t a = nullptr, b = nullptr;
    cudaError_t e = cudaEventCreate(&a);
    if (e == cudaSuccess) e = cudaEventCreate(&b);
    if (e == cudaSuccess && (rc = csp_do_spmv(h, 3)) == CSP_OK) {
        e = cudaEventRecord(a, st);
        if (e == cudaSuccess && (rc = csp_do_spmv(h, ntimes)) == CSP_OK) {
            e = cudaEventRecord(b, st);
            if (e == cudaSuccess) e = cudaEventSynchronize(b);
            float t = 0.0f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&t, a, b);
            *ms = (double)t / ntimes;
        }
    }
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    csp_free_mat_kernels(h);
    if (rc) return rc;
    return e == cudaSuccess ? CSP_OK : cuda_error(e, "calibration timing");
}

// Columns of a banded row: `width` consecutive columns centred on `row`, shifted inwards
// at the edges (the reference's synthetic matrices, e.g. bench_csr.cpp:232).
inline int band_start(int row, int width, int limit)
{
    int start = row - width / 2;
    if (start < 0) start = 0;
    if (start + width > limit) start = limit - width;
    return start;
}

struct Out {
    FILE* f = nullptr;
    ~Out() { if (f) fclose(f); }
};

int open_table(const std::string& dir, const char* name, Out& o)
{
    const std::string p = dir + "/" + name;
    o.f = fopen(p.c_str(), "w");
    if (!o.f) return set_error(CSP_EIO, "cannot write %s", p.c_str());
    return CSP_OK;
}

inline double gflops(double nnz, double ms) { return ms > 0.0 ? 2.0 * nnz / (ms * 1e-3) / 1e9 : 0.0; }

int table_dia(const std::string& dir, const Grid& g, bool banded)
{
    Out o;
    int rc = open_table(dir, banded ? "bdia.ben" : "dia.ben", o);
    if (rc) return rc;
    const int nmeth = banded ? 5 : 4;
    for (int size : g.dims_large)
        for (int width : g.dia_widths) {
            double nnz = size;
            for (int i = 2; i < width; i += 2) nnz += 2.0 * (size - i / 2);
            std::vector<int> off(width);
            std::vector<float> data((size_t)width * size, 1.0f);
            for (int i = 0; i < width; i++) off[i] = -(width / 2) + i;
            int bptr[2] = {0, width};
            int boff[1] = {-(width / 2)};
            fprintf(o.f, "%d %d", size, width);
            for (int m = 0; m < nmeth; m++) {
                cocktail_iif c;
                csp_init_cocktail(&c);
                c.mat_width = c.mat_height = size;
                c.mat_nnz = (int)nnz;
                if (banded) {
                    c.ifusebdia = true;
                    c.bdia_meth_num = m;
                    bdia_matrix_iif& b = c.bdia;
                    b.matinfo = {size, size, (int)nnz};
                    b.bdia_band_num = 1;
                    b.bdia_length = b.bdia_length_aligned = size;
                    b.bdia_offsets = boff;
                    b.bdia_bptr = bptr;
                    b.bdia_data = data.data();
                } else {
                    c.ifusedia = true;
                    c.dia_meth_num = m;
                    dia_matrix_iif& d = c.dia;
                    d.matinfo = {size, size, (int)nnz};
                    d.dia_num = width;
                    d.dia_length = d.dia_length_aligned = size;
                    d.dia_offsets = off.data();
                    d.dia_data = data.data();
                }
                double ms = 0.0;
                if ((rc = time_cocktail(c, g.ntimes, &ms))) return rc;
                fprintf(o.f, " %f", gflops(nnz, ms));
            }
            fprintf(o.f, "\n");
        }
    return CSP_OK;
}

int table_ell(const std::string& dir, const Grid& g, bool sliced)
{
    Out o;
    int rc = open_table(dir, sliced ? "sell.ben" : "ell.ben", o);
    if (rc) return rc;
    for (int size : g.dims_large)
        for (int k : g.ell_widths) {
            if ((long long)size * k > 104857600) break;
            const size_t nnz = (size_t)size * k;
            fprintf(o.f, "%d %d", size, k);
            for (int m = 0; m < 2; m++) {
                cocktail_iif c;
                csp_init_cocktail(&c);
                c.mat_width = c.mat_height = size;
                c.mat_nnz = (int)nnz;
                std::vector<int> col(nnz);
                std::vector<float> val(nnz, 1.0f);
                std::vector<int> sp;
                if (!sliced) {
                    for (int r = 0; r < size; r++) {
                        const int s0 = band_start(r, k, size);
                        for (int j = 0; j < k; j++) col[(size_t)j * size + r] = s0 + j;
                    }
                    c.ifuseell = true;
                    c.ell_meth_num = m;
                    c.ell.matinfo = {size, size, (int)nnz};
                    c.ell.ell_num = k;
                    c.ell.ell_height_aligned = size;
                    c.ell.ell_col_id = col.data();
                    c.ell.ell_data = val.data();
                } else {
                    const int sh = m == 0 ? 32 : 128;   // method 0: WARPSIZE slices, 1: SELL_GROUP_SIZE
                    const int ns = size / sh;
                    sp.resize((size_t)ns + 1);
                    for (int s = 0; s <= ns; s++) sp[s] = s * sh * k;
                    for (int s = 0; s < ns; s++)
                        for (int hh = 0; hh < sh; hh++) {
                            const int r = s * sh + hh;
                            const int s0 = band_start(r, k, size);
                            for (int j = 0; j < k; j++) col[(size_t)s * sh * k + (size_t)j * sh + hh] = s0 + j;
                        }
                    c.ifusesell = true;
                    c.sell_meth_num = m;
                    c.sell.matinfo = {size, size, (int)nnz};
                    c.sell.sell_slice_height = (unsigned)sh;
                    c.sell.sell_slice_num = ns;
                    c.sell.sell_slice_ptr = sp.data();
                    c.sell.sell_col_id = col.data();
                    c.sell.sell_data = val.data();
                }
                double ms = 0.0;
                if ((rc = time_cocktail(c, g.ntimes, &ms))) return rc;
                fprintf(o.f, " %f", gflops((double)nnz, ms));
            }
            fprintf(o.f, "\n");
        }
    return CSP_OK;
}

int table_rows(const std::string& dir, const Grid& g, bool coo, int groups)
{
    Out o;
    int rc = open_table(dir, coo ? "coo.ben" : "csr.ben", o);
    if (rc) return rc;
    const std::vector<int>& dims = coo ? g.dims_large : g.dims_small;
    const std::vector<int>& widths = coo ? g.ell_widths : g.csr_widths;
    const long long cap = coo ? 69905067LL : 104857600LL;
    const int nmeth = coo ? 1 : 2;
    for (int size : dims)
        for (int k : widths) {
            if ((long long)size * k > cap || k > size) break;
            const size_t nnz = (size_t)size * k;
            std::vector<int> rows(coo ? nnz : 0), col(nnz), rp(coo ? 0 : (size_t)size + 1);
            std::vector<float> val(nnz, 1.0f);
            for (int r = 0; r < size; r++) {
                const int s0 = band_start(r, k, size);
                for (int j = 0; j < k; j++) {
                    col[(size_t)r * k + j] = s0 + j;
                    if (coo) rows[(size_t)r * k + j] = r;
                }
            }
            if (!coo)
                for (int r = 0; r <= size; r++) rp[r] = r * k;
            fprintf(o.f, "%d %d %d", size, k, groups);
            for (int m = 0; m < nmeth; m++) {
                cocktail_iif c;
                csp_init_cocktail(&c);
                c.mat_width = c.mat_height = size;
                c.mat_nnz = (int)nnz;
                if (coo) {
                    c.ifusecoo = true;
                    c.coo_meth_num = m;
                    c.coo.matinfo = {size, size, (int)nnz};
                    c.coo.coo_row_id = rows.data();
                    c.coo.coo_col_id = col.data();
                    c.coo.coo_data = val.data();
                } else {
                    c.ifusecsr = true;
                    c.csr_meth_num = m;
                    c.csr.matinfo = {size, size, (int)nnz};
                    c.csr.csr_row_ptr = rp.data();
                    c.csr.csr_col_id = col.data();
                    c.csr.csr_data = val.data();
                }
                double ms = 0.0;
                if ((rc = time_cocktail(c, g.ntimes, &ms))) return rc;
                fprintf(o.f, " %f", gflops((double)nnz, ms));
            }
            fprintf(o.f, "\n");
        }
    return CSP_OK;
}

// BCSR (b4 layout, one method), BELL (b4 layout, two methods), SBELL (slices of 32 block
// rows, one method); block shapes in the analyzer's order: bw 4 then 8, bh 1, 2, 4, 8.
enum BlockKind { BK_BCSR, BK_BELL, BK_SBELL };

int table_block(const std::string& dir, const Grid& g, BlockKind kind)
{
    Out o;
    int rc = open_table(dir, kind == BK_BCSR ? "bcsr.ben" : (kind == BK_BELL ? "bell.ben" : "sbell.ben"), o);
    if (rc) return rc;
    const int nmeth = kind == BK_BELL ? 2 : 1;
    const std::vector<int>& dims = kind == BK_BCSR ? g.dims_small : g.dims_large;
    const std::vector<int>& blocks = kind == BK_BCSR ? g.bcsr_blocks : g.bell_blocks;
    for (int bw = 4; bw <= 8; bw += 4)
        for (int bh = 1; bh <= 8; bh *= 2)
            for (int size : dims)
                for (int bn : blocks) {
                    if ((long long)size * bn * bw > 209715200LL) break;
                    if (kind == BK_BCSR && bn * bw >= size) break;
                    const int nbr = size / bh, ncols = size / bw;
                    if (bn > ncols) break;
                    const size_t nblk = (size_t)nbr * bn;
                    const size_t nnz = nblk * bw * bh;
                    std::vector<float> data(nnz, 1.0f);
                    std::vector<int> col(nblk), rp, sp;
                    if (kind == BK_BCSR) {
                        rp.resize((size_t)nbr + 1);
                        for (int i = 0; i <= nbr; i++) rp[i] = i * bn;
                        for (int i = 0; i < nbr; i++) {
                            const int s0 = band_start(i, bn, ncols);
                            for (int j = 0; j < bn; j++) col[(size_t)i * bn + j] = s0 + j;
                        }
                    } else if (kind == BK_BELL) {
                        for (int i = 0; i < nbr; i++) {
                            const int s0 = band_start(i, bn, ncols);
                            for (int j = 0; j < bn; j++) col[(size_t)j * nbr + i] = s0 + j;
                        }
                    } else {
                        const int sh = 32, ns = nbr / sh;
                        sp.resize((size_t)ns + 1);
                        for (int s = 0; s <= ns; s++) sp[s] = s * sh * bn;
                        for (int s = 0; s < ns; s++)
                            for (int hh = 0; hh < sh; hh++) {
                                const int s0 = band_start(s * sh + hh, bn, ncols);
                                for (int j = 0; j < bn; j++) col[(size_t)s * sh * bn + (size_t)j * sh + hh] = s0 + j;
                            }
                    }
                    fprintf(o.f, "%d %d %d %d", bh, bw, size, bn);
                    for (int m = 0; m < nmeth; m++) {
                        cocktail_iif c;
                        csp_init_cocktail(&c);
                        c.mat_width = c.mat_height = size;
                        c.mat_nnz = (int)nnz;
                        if (kind == BK_BCSR) {
                            c.ifusebcsr = true;
                            c.bcsr_meth_num = m;
                            b4csr_matrix_if& b = c.bcsr;
                            b.matinfo = {size, size, (int)nnz};
                            b.b4csr_bwidth = (unsigned)bw;
                            b.b4csr_bheight = (unsigned)bh;
                            b.b4csr_row_num = nbr;
                            b.b4csr_aligned_size = (int)(4 * nblk);
                            b.b4csr_block_num = (int)nblk;
                            b.b4csr_row_ptr = rp.data();
                            b.b4csr_col_id = col.data();
                            b.b4csr_data = data.data();
                        } else if (kind == BK_BELL) {
                            c.ifusebell = true;
                            c.bell_meth_num = m;
                            b4ell_matrix_if& b = c.bell;
                            b.matinfo = {size, size, (int)nnz};
                            b.b4ell_bwidth = (unsigned)bw;
                            b.b4ell_bheight = (unsigned)bh;
                            b.b4ell_row_num = nbr;
                            b.b4ell_block_num = bn;
                            b.b4ell_height_aligned = nbr;
                            b.b4ell_float4_aligned = 4 * nbr;
                            b.b4ell_col_id = col.data();
                            b.b4ell_data = data.data();
                        } else {
                            c.ifusesbell = true;
                            c.sbell_meth_num = m;
                            sbell_matrix_if& b = c.sbell;
                            b.matinfo = {size, size, (int)nnz};
                            b.sbell_bwidth = (unsigned)bw;
                            b.sbell_bheight = (unsigned)bh;
                            b.sbell_slice_height = 32;
                            b.sbell_slice_num = nbr / 32;
                            b.sbell_row_num = nbr;
                            b.sbell_slice_ptr = sp.data();
                            b.sbell_col_id = col.data();
                            b.sbell_data = data.data();
                        }
                        double ms = 0.0;
                        if ((rc = time_cocktail(c, g.ntimes, &ms))) return rc;
                        fprintf(o.f, " %f", gflops((double)nnz, ms));
                    }
                    fprintf(o.f, "\n");
                }
    return CSP_OK;
}

// Launch overhead in microseconds per launch of an empty kernel, back to back
// (bench_overhead.cpp: work groups from the SM count doubling to 131,702, work-group
// sizes 64, 128, 256).
int table_overhead(const std::string& dir, int sms, int ntimes)
{
    Out o;
    int rc = open_table(dir, "overhead.ben", o);
    if (rc) return rc;
    cudaStream_t st = nullptr;
    cudaEvent_t a = nullptr, b = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&a);
    if (e == cudaSuccess) e = cudaEventCreate(&b);
    for (int groups = sms; groups <= 131702 && e == cudaSuccess; groups *= 2)
        for (int threads = 64; threads <= 256 && e == cudaSuccess; threads *= 2) {
            for (int i = 0; i < 10; i++) calib_null_kernel<<<groups, threads, 0, st>>>(nullptr);
            e = cudaEventRecord(a, st);
            for (int i = 0; i < ntimes && e == cudaSuccess; i++) calib_null_kernel<<<groups, threads, 0, st>>>(nullptr);
            if (e == cudaSuccess) e = cudaEventRecord(b, st);
            if (e == cudaSuccess) e = cudaEventSynchronize(b);
            float t = 0.0f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&t, a, b);
            if (e == cudaSuccess) e = cudaGetLastError();
            if (e == cudaSuccess) fprintf(o.f, "%d %d %f\n", groups, threads, (double)t * 1000.0 / ntimes);
        }
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    if (st) cudaStreamDestroy(st);
    return e == cudaSuccess ? CSP_OK : cuda_error(e, "overhead calibration");
}

}  // namespace
}  // namespace csp

extern "C" int csp_benchmark_tables(const char* clspmv_path, int level)
{
    using namespace csp;
    clear_error();
    if (!clspmv_path || !*clspmv_path) return set_error(CSP_EINVAL, "null output directory");
    if (level < 0 || level > 2) return set_error(CSP_EINVAL, "level must be 0, 1 or 2");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return set_error(CSP_ENODEV, "no CUDA device");
    const std::string dir = std::string(clspmv_path) + "/benchmark";
    if (mkdir(clspmv_path, 0755) != 0 && errno != EEXIST) return set_error(CSP_EIO, "cannot create %s", clspmv_path);
    if (mkdir(dir.c_str(), 0755) != 0 && errno != EEXIST) return set_error(CSP_EIO, "cannot create %s", dir.c_str());
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return set_error(CSP_ECUDA, "device query failed");
    const Grid g = make_grid(level);
    int rc;
    if ((rc = table_overhead(dir, sms, g.ntimes)) || (rc = table_dia(dir, g, false)) || (rc = table_dia(dir, g, true)) ||
        (rc = table_ell(dir, g, false)) || (rc = table_ell(dir, g, true)) || (rc = table_rows(dir, g, false, sms)) ||
        (rc = table_rows(dir, g, true, sms)) || (rc = table_block(dir, g, BK_BCSR)) || (rc = table_block(dir, g, BK_BELL)) ||
        (rc = table_block(dir, g, BK_SBELL)))
        return rc;
    return CSP_OK;
}
