/*
 * ORACLE -- test infrastructure only.  Never linked into, loaded by or called from
 * the product library or its Python package; only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg use it, to check and to time against.
 *
 * A plain-C restatement of the reference's serial SpMV semantics
 * (clSpMV_NV/include/spmv_serial.h) plus an FP64 reference product and the
 * per-row error bound the parity tests apply.
 *
 * Semantics (every function): res += A * vec, the reference's accumulate form
 * (clSpMV_NV/src/eval.cpp:40-42).  FP32 functions keep the reference's
 * summation order, so they agree bit for bit with the compiled reference;
 * tests/test_oracle_pin.py checks exactly that.
 *
 * Parity pinning: the reference ships no golden vectors or fixtures
 * (its only checks are GPU-vs-serial COO, clSpMV_NV/src/util.cpp:93-172, and
 * format-vs-COO exact equality, spmv_serial.h:332-565).  This oracle is pinned
 * against the reference's own serial code compiled from its sources
 * (oracle/_ref, built by oracle/Makefile) and against committed fixtures
 * generated from it (tests/golden/).
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

/* spmv_serial.h:199 csr_spmv: per row, accumulate in FP32 from 0, then add to res. */
void orc_csr_spmv_f32(int height, const int* row_ptr, const int* col, const float* val,
                      const float* vec, float* res)
{
    for (int r = 0; r < height; r++) {
        float acc = 0.0f;
        for (int j = row_ptr[r]; j < row_ptr[r + 1]; j++)
            acc += val[j] * vec[col[j]];
        res[r] += acc;
    }
}

/* spmv_serial.h:184 coo_spmv: element by element into res, in storage order. */
void orc_coo_spmv_f32(int nnz, const int* row, const int* col, const float* val,
                      const float* vec, float* res)
{
    for (int i = 0; i < nnz; i++)
        res[row[i]] += val[i] * vec[col[i]];
}

/* spmv_serial.h:12 dia_spmv: for each padded row, sum over diagonals (bounds-checked x). */
void orc_dia_spmv_f32(int dia_num, int length_aligned, const int* offsets, const float* data,
                      const float* vec, int vec_size, float* res)
{
    for (int r = 0; r < length_aligned; r++) {
        float acc = 0.0f;
        for (int d = 0; d < dia_num; d++) {
            int c = r + offsets[d];
            float v = (c >= 0 && c < vec_size) ? vec[c] : 0.0f;
            acc += v * data[r + d * length_aligned];
        }
        res[r] += acc;
    }
}

/* spmv_serial.h:60 bdia_spmv: bands of consecutive diagonals. */
void orc_bdia_spmv_f32(int band_num, int length_aligned, const int* offsets, const int* bptr,
                       const float* data, const float* vec, int vec_size, float* res)
{
    for (int r = 0; r < length_aligned; r++) {
        float acc = 0.0f;
        for (int b = 0; b < band_num; b++) {
            int off = offsets[b];
            for (int d = bptr[b]; d < bptr[b + 1]; d++, off++) {
                int c = r + off;
                float v = (c >= 0 && c < vec_size) ? vec[c] : 0.0f;
                acc += v * data[r + d * length_aligned];
            }
        }
        res[r] += acc;
    }
}

/* spmv_serial.h:93 ell_spmv: column-major ELL, slot by slot straight into res. */
void orc_ell_spmv_f32(int height, int ell_num, int height_aligned, const int* col,
                      const float* data, const float* vec, float* res)
{
    for (int k = 0; k < ell_num; k++)
        for (int r = 0; r < height; r++)
            res[r] += data[k * height_aligned + r] * vec[col[k * height_aligned + r]];
}

/* spmv_serial.h:113 sell_spmv: per slice, slot by slot straight into res. */
void orc_sell_spmv_f32(int height, unsigned slice_height, int slice_num, const int* slice_ptr,
                       const int* col, const float* data, const float* vec, float* res)
{
    for (int s = 0; s < slice_num; s++) {
        int start = slice_ptr[s];
        int width = (slice_ptr[s + 1] - start) / (int)slice_height;
        int first = s * (int)slice_height;
        for (int k = 0; k < width; k++)
            for (int r = first; r < first + (int)slice_height && r < height; r++) {
                int idx = start + (r - first) + k * (int)slice_height;
                res[r] += data[idx] * vec[col[idx]];
            }
    }
}

/* spmv_serial.h:220 bcsr_spmv: block element k outermost, blocks inner, straight into res. */
void orc_bcsr_spmv_f32(int height, int row_num, unsigned bw, unsigned bh, int aligned,
                       const int* row_ptr, const int* col, const float* data,
                       const float* vec, int vec_size, float* res)
{
    unsigned bs = bw * bh;
    for (int i = 0; i < row_num; i++) {
        int r0 = i * (int)bh;
        for (unsigned k = 0; k < bs; k++) {
            int ic = (int)(k % bw), ir = (int)(k / bw);
            for (int j = row_ptr[i]; j < row_ptr[i + 1]; j++) {
                int c = col[j] + ic, r = r0 + ir;
                if (c < vec_size && r < height)
                    res[r] += data[j + (int)k * aligned] * vec[c];
            }
        }
    }
}

/* spmv_serial.h:252 bell_spmv (generic BELL, block-element-major per block column). */
void orc_bell_spmv_f32(int row_num, int block_num, unsigned bw, unsigned bh, int height_aligned,
                       const int* col, const float* data, const float* vec, float* res)
{
    int colsize = height_aligned * (int)(bw * bh);
    for (int i = 0; i < block_num; i++)
        for (int j = 0; j < row_num; j++)
            for (unsigned k = 0; k < bw * bh; k++) {
                float d = data[j + (int)k * height_aligned + i * colsize];
                int c = col[i * height_aligned + j] + (int)(k % bw);
                res[j * (int)bh + (int)(k / bw)] += d * vec[c];
            }
}

/* spmv_serial.h:138 sbell_spmv (b4 layout, slices of block rows). */
void orc_sbell_spmv_f32(int height, int width, unsigned bw, unsigned bh, unsigned sh, int slice_num,
                        const int* slice_ptr, const int* col, const float* data,
                        const float* vec, float* res)
{
    unsigned bs = bw * bh;
    for (int i = 0; i < slice_num; i++) {
        int start = slice_ptr[i];
        int ellnum = (slice_ptr[i + 1] - start) / (int)sh;
        for (unsigned s = 0; s < sh; s++) {
            int coloff = start + (int)s;
            int dataoff = start * (int)bs + (int)s * 4;
            for (int j = 0; j < ellnum; j++) {
                int c = col[coloff] * 4;
                for (unsigned w4 = 0; w4 < bw / 4; w4++) {
                    for (unsigned h = 0; h < bh; h++) {
                        int r = (i * (int)sh + (int)s) * (int)bh + (int)h;
                        if (r < height) {
                            for (int w = 0; w < 4; w++) {
                                if (c + w >= width) break;
                                res[r] += data[dataoff + w] * vec[c + w];
                            }
                        }
                        dataoff += (int)sh * 4;
                    }
                    c += 4;
                }
                coloff += (int)sh;
            }
        }
    }
}

/*
 * FP64 reference product on CSR: out[r] = res0[r] + sum_j a_rj * vec[c_j], evaluated in
 * double, and bound[r] = sum_j |a_rj * vec[c_j]| + res0_weight * |res0[r]|, the scale
 * of row r's rounding error.  A test accepts row r when |y_r - out[r]| <= tol * bound[r];
 * with tol = 1e-5 and res0_weight = 2^-23 / 1e-5 that is the FP32 bound
 * 1e-5 * sum_j |a_rj x_j| + 2^-23 * |res0[r]| (the final FP32 add of res0 rounds by at
 * most 2^-24 of the result).  `transpose` != 0 computes A^T * vec instead (out has
 * `width` rows): the adjoint d(vec) = A^T * res_bar.
 */
void orc_csr_spmv_f64(int height, int width, const int* row_ptr, const int* col, const float* val,
                      const float* vec, const float* res0, double res0_weight, int transpose,
                      double* out, double* bound)
{
    int n_out = transpose ? width : height;
    for (int i = 0; i < n_out; i++) {
        double r0 = res0 ? (double)res0[i] : 0.0;
        out[i] = r0;
        bound[i] = res0_weight * fabs(r0);
    }
    for (int r = 0; r < height; r++) {
        for (int j = row_ptr[r]; j < row_ptr[r + 1]; j++) {
            if (!transpose) {
                double p = (double)val[j] * (double)vec[col[j]];
                out[r] += p;
                bound[r] += fabs(p);
            } else {
                double p = (double)val[j] * (double)vec[r];
                out[col[j]] += p;
                bound[col[j]] += fabs(p);
            }
        }
    }
}

/*
 * Value gradient of y = A x on the CSR pattern: abar[j] = res_bar[row(j)] * vec[col[j]]
 * (the derivative of y_row with respect to a_row,col, weighted by res_bar).  The
 * reference has no adjoint; this is the definition, used to time a CPU counterpart of
 * the device's gradient pass.
 */
void orc_csr_value_grad_f32(int height, const int* row_ptr, const int* col, const float* res_bar,
                            const float* vec, float* abar)
{
    for (int r = 0; r < height; r++) {
        float yb = res_bar[r];
        for (int j = row_ptr[r]; j < row_ptr[r + 1]; j++) abar[j] = yb * vec[col[j]];
    }
}

/*
 * Largest per-row error relative to its bound: max_i |y_i - yhat_i| / bound_i.
 * A row whose bound is 0 must match exactly; any difference there returns +inf.
 * `worst` receives the row index (or -1).
 */
double orc_max_rel_err(int n, const float* y, const double* yhat, const double* bound, int* worst)
{
    double m = 0.0;
    int w = -1;
    for (int i = 0; i < n; i++) {
        double d = fabs((double)y[i] - yhat[i]);
        double e;
        if (bound[i] > 0.0) e = d / bound[i];
        else e = (d == 0.0) ? 0.0 : INFINITY;
        if (e != e) e = INFINITY; /* NaN in y */
        if (e > m) { m = e; w = i; }
    }
    if (worst) *worst = w;
    return m;
}

/* The reference's own comparison numbers (util.cpp:93 two_vec_compare), computed silently:
 * out[0] = L2 distance, out[1] = max | |a| - |b| |, out[2] = max relative form. */
void orc_two_vec_compare(int n, const float* a, const float* b, double* out)
{
    double dist = 0.0, maxdiff = 0.0, maxratio = 0.0;
    for (int i = 0; i < n; i++) {
        double t = (double)a[i] - (double)b[i];
        dist += t * t;
        float ta = a[i] < 0 ? -a[i] : a[i];
        float tb = b[i] < 0 ? -b[i] : b[i];
        double diff = (double)ta - (double)tb;
        if (diff < 0) diff = -diff;
        float mab = ta > tb ? ta : tb;
        double ratio = mab > 0 ? diff / mab : 0.0;
        if (diff > maxdiff) maxdiff = diff;
        if (ratio > maxratio) maxratio = ratio;
    }
    out[0] = sqrt(dist);
    out[1] = maxdiff;
    out[2] = maxratio;
}
