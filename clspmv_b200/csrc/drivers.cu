// Evaluation and single-format drivers: csp_evaluate (spmv_cocktail.cpp:1434
// evaluate + :1137 check_and_time), csp_spmv_all and the csp_spmv_<fmt>
// drivers (clSpMV_NV/src/spmv_all.cpp:196-246 and the spmv_<fmt>.cpp files),
// and the MatrixMarket reader (fileio.cpp:10 ReadMMF).
//
// Like the reference, each check runs one SpMV on x = vec against a serial COO
// result and reports the reference's comparison numbers (util.cpp:93
// two_vec_compare), then times repeated SpMVs.  Timing uses CUDA events on the
// handle's stream after three warm-up SpMVs.  Nothing is printed.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <vector>

#include "csp/clspmv.h"
#include "internal.h"
#include "engine.h"

namespace csp {

// Bytes an SpMV must move at minimum (values + indices of each part in its own
// structure class, x once, y read and written), the numerator of every GB/s
// figure this library reports.
double algorithmic_bytes(const cocktail_iif* m, int value_bytes)
{
    double b = 4.0 * m->mat_width + 8.0 * m->mat_height;
    if (m->ifusebdia) b += (double)value_bytes * m->bdia.matinfo.nnz + 8.0 * m->bdia.bdia_band_num;
    if (m->ifusedia) b += (double)value_bytes * m->dia.matinfo.nnz + 4.0 * m->dia.dia_num;
    if (m->ifusesbell) {
        const double nb = m->sbell.matinfo.nnz;  // block counts are not kept; values as stored nonzeros
        b += (double)value_bytes * nb + 4.0 * (m->sbell.sbell_row_num + 1);
    }
    if (m->ifusebell) b += (double)value_bytes * m->bell.matinfo.nnz + 4.0 * (m->bell.b4ell_row_num + 1);
    if (m->ifusebcsr) {
        const double bs = (double)m->bcsr.b4csr_bwidth * m->bcsr.b4csr_bheight;
        b += (double)value_bytes * bs * m->bcsr.b4csr_block_num + 4.0 * m->bcsr.b4csr_block_num + 4.0 * (m->bcsr.b4csr_row_num + 1);
    }
    if (m->ifusesell) b += (value_bytes + 4.0) * m->sell.matinfo.nnz + 4.0 * (m->sell.matinfo.height + 1);
    if (m->ifuseell) b += (value_bytes + 4.0) * m->ell.matinfo.nnz + 4.0 * (m->ell.matinfo.height + 1);
    if (m->ifusecsr) b += (value_bytes + 4.0) * m->csr.matinfo.nnz + 4.0 * (m->csr.matinfo.height + 1);
    if (m->ifusecoo) b += (value_bytes + 4.0) * m->coo.matinfo.nnz + 4.0 * (m->coo.matinfo.height + 1);
    return b;
}

static void compare_vectors(const float* a, const float* b, int n, csp_report* r)
{
    double dist = 0.0, maxdiff = 0.0, maxratio = 0.0;
    for (int i = 0; i < n; i++) {
        const double t = (double)a[i] - (double)b[i];
        dist += t * t;
        const float ta = fabsf(a[i]), tb = fabsf(b[i]);
        const double diff = fabs((double)ta - (double)tb);
        const float mab = ta > tb ? ta : tb;
        const double ratio = mab > 0 ? diff / mab : 0.0;
        if (diff > maxdiff) maxdiff = diff;
        if (ratio > maxratio) maxratio = ratio;
    }
    r->l2_distance = sqrt(dist);
    r->max_diff = maxdiff;
    r->max_ratio_diff = maxratio;
}

// Serial COO product in storage order, the reference's spmv_only (util.cpp:85), used
// only to check the device result.
static void serial_coo(const coo_matrix_if* c, const float* x, float* y)
{
    for (int i = 0; i < c->matinfo.height; i++) y[i] = 0.0f;
    for (int i = 0; i < c->matinfo.nnz; i++) y[c->coo_row_id[i]] += c->coo_data[i] * x[c->coo_col_id[i]];
}

// One checked SpMV then `ntimes` timed SpMVs of a cocktail.
static int check_and_time(const cocktail_iif* mat, const float* vec, const float* res, const float* coores, int ntimes,
                          int flags, csp_report* rep)
{
    csp_handle* h = nullptr;
    int rc = csp_init_mat_kernels(mat, vec, res, flags, &h);
    if (rc) return rc;
    std::vector<float> out((size_t)mat->mat_height);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    float ms = 0.0f;
    cudaStream_t st = nullptr;
    if ((rc = csp_do_spmv(h, 1)) || (rc = csp_cpy_result_to_cpu(h, out.data(), mat->mat_height))) goto done;
    compare_vectors(coores, out.data(), mat->mat_height, rep);
    if (ntimes > 0) {
        csp_get_stream(h, reinterpret_cast<void**>(&st));
        if ((rc = csp_do_spmv(h, 3))) goto done;
        if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) { rc = set_error(CSP_ECUDA, "event"); goto done; }
        cudaEventRecord(e0, st);
        if ((rc = csp_do_spmv(h, ntimes))) goto done;
        cudaEventRecord(e1, st);
        if (cudaEventSynchronize(e1) != cudaSuccess) { rc = set_error(CSP_ECUDA, "timed SpMVs failed: %s", cudaGetErrorString(cudaGetLastError())); goto done; }
        cudaEventElapsedTime(&ms, e0, e1);
        rep->ms = ms / ntimes;
        rep->gflops = 2.0 * mat->mat_nnz / (rep->ms * 1e-3) / 1e9;
        rep->gbytes = algorithmic_bytes(mat, (flags & CSP_FLAG_BF16) ? 2 : 4) / (rep->ms * 1e-3) / 1e9;
    }
done:
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    csp_free_mat_kernels(h);
    return rc;
}

struct Variant {
    cocktail_iif mat;
    int method;
};

static void set_info(cocktail_iif* c, const coo_matrix_if* coo)
{
    c->mat_width = coo->matinfo.width;
    c->mat_height = coo->matinfo.height;
    c->mat_nnz = coo->matinfo.nnz;
}

// Runs every kernel variant of one format and keeps the fastest (spmv_all method n).
static int run_format(coo_matrix_if* coo, int method, int ntimes, csp_report* report)
{
    int rc = check_coo(coo);
    if (rc) return rc;
    if ((rc = ensure_sorted(coo))) return rc;
    const int w = coo->matinfo.width, h = coo->matinfo.height;
    std::vector<float> x((size_t)w, 1.0f), y0((size_t)h, 0.0f), ref((size_t)h);
    serial_coo(coo, x.data(), ref.data());
    memset(report, 0, sizeof(*report));
    report->ms = 1e30;
    report->method = -1;
    bool any = false;
    auto try_one = [&](cocktail_iif& c, int code) -> int {
        csp_report r;
        memset(&r, 0, sizeof(r));
        int e = check_and_time(&c, x.data(), y0.data(), ref.data(), ntimes, 0, &r);
        if (e) return e;
        if (!any || r.ms < report->ms) {
            *report = r;
            report->method = code;
            report->group_num = 0;
        }
        any = true;
        return CSP_OK;
    };
    static const unsigned bhs[4] = {1, 2, 4, 8};
    switch (method) {
    case 1:
    case 2: {
        cocktail_iif c;
        csp_init_cocktail(&c);
        set_info(&c, coo);
        if ((rc = csp_coo2csr(coo, &c.csr))) { csp_free_cocktail(&c); return rc; }
        c.ifusecsr = true;
        const int ms1[3] = {4, 5, 6}, ms2[4] = {0, 1, 2, 3};
        const int* ms = method == 1 ? ms1 : ms2;
        const int nm = method == 1 ? 3 : 4;
        for (int i = 0; i < nm && !rc; i++) { c.csr_meth_num = ms[i]; rc = try_one(c, ms[i]); }
        csp_free_cocktail(&c);
        return rc;
    }
    case 3:
    case 4: {
        cocktail_iif c;
        csp_init_cocktail(&c);
        set_info(&c, coo);
        if (method == 3) {
            if ((rc = csp_coo2bdia(coo, &c.bdia, 32))) { csp_free_cocktail(&c); return rc; }
            c.ifusebdia = true;
            for (int mth = 0; mth < 5 && !rc; mth++) { c.bdia_meth_num = mth; rc = try_one(c, mth); }
        } else {
            if ((rc = csp_coo2dia(coo, &c.dia, 32))) { csp_free_cocktail(&c); return rc; }
            c.ifusedia = true;
            for (int mth = 0; mth < 4 && !rc; mth++) { c.dia_meth_num = mth; rc = try_one(c, mth); }
        }
        csp_free_cocktail(&c);
        return rc;
    }
    case 5: {
        cocktail_iif c;
        csp_init_cocktail(&c);
        set_info(&c, coo);
        if ((rc = csp_coo2ell(coo, &c.ell, 32, 0))) { csp_free_cocktail(&c); return rc; }
        c.ifuseell = true;
        for (int mth = 0; mth < 2 && !rc; mth++) { c.ell_meth_num = mth; rc = try_one(c, mth); }
        csp_free_cocktail(&c);
        return rc;
    }
    case 6: {
        cocktail_iif c;
        csp_init_cocktail(&c);
        set_info(&c, coo);
        c.coo.matinfo = coo->matinfo;
        c.coo.coo_row_id = coo->coo_row_id;
        c.coo.coo_col_id = coo->coo_col_id;
        c.coo.coo_data = coo->coo_data;
        c.ifusecoo = true;
        rc = try_one(c, 0);
        return rc;  // arrays belong to the caller
    }
    case 7:
    case 8:
    case 10: {
        for (unsigned bw = 4; bw <= 8 && !rc; bw += 4)
            for (int bi = 0; bi < 4 && !rc; bi++) {
                const unsigned bh = bhs[bi];
                cocktail_iif c;
                csp_init_cocktail(&c);
                set_info(&c, coo);
                int code = (int)(bh * 10 + bw);
                if (method == 7) {
                    if (csp_coo2b4ell(coo, &c.bell, bw, bh, 32, 0) == CSP_OK) {
                        c.ifusebell = true;
                        rc = try_one(c, code);
                    }
                } else if (method == 8) {
                    if (csp_coo2b4csr(coo, &c.bcsr, bw, bh, 32) == CSP_OK) {
                        c.ifusebcsr = true;
                        for (int mth = 0; mth < 2 && !rc; mth++) { c.bcsr_meth_num = mth; rc = try_one(c, code * 10 + mth); }
                    }
                } else {
                    if (csp_coo2sbell(coo, &c.sbell, bw, bh, 32) == CSP_OK) {
                        c.ifusesbell = true;
                        rc = try_one(c, code);
                    }
                }
                csp_free_cocktail(&c);
            }
        if (!rc && !any) return set_error(CSP_EFORMAT, "no block shape could represent the matrix");
        return rc;
    }
    case 9: {
        const unsigned shs[2] = {32, 128};
        for (int i = 0; i < 2 && !rc; i++) {
            cocktail_iif c;
            csp_init_cocktail(&c);
            set_info(&c, coo);
            if ((rc = csp_coo2sell(coo, &c.sell, shs[i]))) { csp_free_cocktail(&c); return rc; }
            c.ifusesell = true;
            c.sell_meth_num = i;
            rc = try_one(c, i);
            csp_free_cocktail(&c);
        }
        return rc;
    }
    default:
        return set_error(CSP_EINVAL, "spmv_all: unknown method %d", method);
    }
}

}  // namespace csp

using namespace csp;

extern "C" {

int csp_evaluate(const cocktail_iif* mat, const float* vec, const float* res, const float* coores, int ntimes, csp_report* report)
{
    if (!mat || !vec || !coores || !report) return set_error(CSP_EINVAL, "csp_evaluate: null argument");
    memset(report, 0, sizeof(*report));
    return check_and_time(mat, vec, res, coores, ntimes, 0, report);
}

int csp_spmv_all(coo_matrix_if* coo, int method, int ntimes, csp_report* report)
{
    if (!report) return set_error(CSP_EINVAL, "null report");
    return run_format(coo, method, ntimes, report);
}
int csp_spmv_csr_scalar(coo_matrix_if* c, int n, csp_report* r) { return csp_spmv_all(c, 1, n, r); }
int csp_spmv_csr_vector(coo_matrix_if* c, int n, csp_report* r) { return csp_spmv_all(c, 2, n, r); }
int csp_spmv_bdia(coo_matrix_if* c, int n, csp_report* r) { return csp_spmv_all(c, 3, n, r); }
int csp_spmv_dia(coo_matrix_if* c, int n, csp_report* r) { return csp_spmv_all(c, 4, n, r); }
int csp_spmv_ell(coo_matrix_if* c, int n, csp_report* r) { return csp_spmv_all(c, 5, n, r); }
int csp_spmv_coo(coo_matrix_if* c, int n, csp_report* r) { return csp_spmv_all(c, 6, n, r); }
int csp_spmv_bell(coo_matrix_if* c, int n, csp_report* r) { return csp_spmv_all(c, 7, n, r); }
int csp_spmv_bcsr(coo_matrix_if* c, int n, csp_report* r) { return csp_spmv_all(c, 8, n, r); }
int csp_spmv_sell(coo_matrix_if* c, int n, csp_report* r) { return csp_spmv_all(c, 9, n, r); }
int csp_spmv_sbell(coo_matrix_if* c, int n, csp_report* r) { return csp_spmv_all(c, 10, n, r); }

// fileio.cpp:10 ReadMMF: header "%%MatrixMarket matrix coordinate <field> <symmetry>",
// comment lines, "rows cols nnz", then 1-based entries.  Pattern matrices get 1.0;
// symmetric ones are mirrored (diagonal once) and sorted; general ones sorted if needed.
// Unlike the reference, an "integer" field's values are read rather than misparsed.
int csp_read_mmf(const char* filename, coo_matrix_if* mat) { return csp_read_mmf_ex(filename, mat, 0); }

int csp_read_mmf_ex(const char* filename, coo_matrix_if* mat, int flags)
{
    if (!filename || !mat) return set_error(CSP_EINVAL, "null argument");
    FILE* f = fopen(filename, "r");
    if (!f) return set_error(CSP_EIO, "cannot open %s", filename);
    char tok[5][128];
    for (int i = 0; i < 5; i++)
        if (fscanf(f, "%127s", tok[i]) != 1) { fclose(f); return set_error(CSP_EIO, "bad MatrixMarket header"); }
    const bool has_value = strcmp(tok[3], "pattern") != 0;
    const bool sym = strcmp(tok[4], "symmetric") == 0;
    char line[2048];
    int h = 0, w = 0, nnz = 0;
    while (true) {
        if (!fgets(line, sizeof(line), f)) { fclose(f); return set_error(CSP_EIO, "missing size line"); }
        char* p = line;
        while (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r') p++;
        if (*p == 0 || *p == '%') continue;
        if (sscanf(p, "%d %d %d", &h, &w, &nnz) != 3) { fclose(f); return set_error(CSP_EIO, "bad size line"); }
        break;
    }
    if (h < 0 || w < 0 || nnz < 0) { fclose(f); return set_error(CSP_EIO, "negative sizes"); }
    std::vector<int> r((size_t)nnz), c((size_t)nnz);
    std::vector<float> v((size_t)nnz, 1.0f);
    int ndiag = 0;
    for (int i = 0; i < nnz; i++) {
        if (fscanf(f, "%d %d", &r[i], &c[i]) != 2) { fclose(f); return set_error(CSP_EIO, "entry %d unreadable", i); }
        r[i]--;
        c[i]--;
        if (has_value) {
            double d = 0.0;
            if (fscanf(f, "%lf", &d) != 1) { fclose(f); return set_error(CSP_EIO, "value %d unreadable", i); }
            v[i] = (float)d;
        }
        if (r[i] == c[i]) ndiag++;
    }
    fclose(f);
    const long long total = sym ? 2LL * nnz - ndiag : nnz;
    mat->matinfo.height = h;
    mat->matinfo.width = w;
    mat->matinfo.nnz = (int)total;
    mat->coo_row_id = (int*)malloc(sizeof(int) * (size_t)(total ? total : 1));
    mat->coo_col_id = (int*)malloc(sizeof(int) * (size_t)(total ? total : 1));
    mat->coo_data = (float*)malloc(sizeof(float) * (size_t)(total ? total : 1));
    if (!mat->coo_row_id || !mat->coo_col_id || !mat->coo_data) return set_error(CSP_ENOMEM, "read_mmf");
    size_t k = 0;
    for (int i = 0; i < nnz; i++) {
        mat->coo_row_id[k] = r[i]; mat->coo_col_id[k] = c[i]; mat->coo_data[k] = v[i]; k++;
        if (sym && r[i] != c[i]) { mat->coo_row_id[k] = c[i]; mat->coo_col_id[k] = r[i]; mat->coo_data[k] = v[i]; k++; }
    }
    if (flags & CSP_MMF_SORT_ON_DEVICE) return coo_is_sorted(mat) ? CSP_OK : csp_sort_coo_device(mat);
    if (sym) return csp_sort_coo(mat);
    return ensure_sorted(mat);
}

}  // extern "C"
