// Adjoint of the Cocktail SpMV (no counterpart in the reference):
//   xbar += A^T * ybar      by a precomputed transposed structure, and
//   abar[slot] = ybar[row] * x[col] over every stored slot (the gradient of
//                ybar^T (A x) with respect to the stored values).
//
// With CSP_FLAG_ADJOINT, csp_init_mat_kernels also builds A^T once: each DIA/BDIA
// part of a square matrix becomes a transposed DIA part (offsets negated, data
// shifted along the diagonal), every other part's nonzeros are gathered into one
// transposed CSR run by the adaptive CSR kernel.  The transposed product therefore
// reuses the forward kernels, is deterministic and needs no atomics; it doubles the
// matrix memory.  abar follows the forward parts in launch order, each in its own
// storage layout; csp_adjoint_pattern writes the (row, col) of every slot.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>
#include <algorithm>
#include <numeric>
#include <vector>

#include "csp/clspmv.h"
#include "internal.h"
#include "engine.h"
#include "kernels/adjoint.cuh"

namespace csp {

namespace {


// Every stored slot of a b4 block layout (matrix_storage.h:2203 SBELL, :2010 BELL,
// :1741 BCSR): f(i, row, col) with i the slot's index in the part's data array and
// row -1 where the slot lies outside the matrix (alignment rows and columns).
template <class F> void for_each_sbell_slot(const sbell_matrix_if& s, F f)
{
    const int bw = (int)s.sbell_bwidth, bh = (int)s.sbell_bheight, sh = (int)s.sbell_slice_height, bw4 = bw / 4;
    const size_t total = (size_t)s.sbell_slice_ptr[s.sbell_slice_num] * bw * bh;
    std::vector<char> seen(total, 0);
    for (int br = 0; br < s.sbell_row_num; br++) {
        const int sl = br / sh, lr = br % sh;
        const int cs = s.sbell_slice_ptr[sl];
        const int width = (s.sbell_slice_ptr[sl + 1] - cs) / sh;
        for (int k = 0; k < width; k++) {
            const int c4 = s.sbell_col_id[cs + lr + k * sh];
            for (int h = 0; h < bh; h++)
                for (int w4 = 0; w4 < bw4; w4++)
                    for (int w = 0; w < 4; w++) {
                        const size_t i = (size_t)cs * bw * bh + (size_t)k * sh * bw4 * bh * 4 + (size_t)h * sh * 4 +
                                         (size_t)w4 * sh * bh * 4 + (size_t)lr * 4 + w;
                        const int r = br * bh + h, c = (c4 + w4) * 4 + w;
                        const bool in = r < s.matinfo.height && c < s.matinfo.width;
                        f(i, in ? r : -1, in ? c : -1);
                        seen[i] = 1;
                    }
        }
    }
    for (size_t i = 0; i < total; i++)
        if (!seen[i]) f(i, -1, -1);   // slice rows past the last block row
}

template <class F> void for_each_bell_slot(const b4ell_matrix_if& b, F f)
{
    const int bw4 = (int)b.b4ell_bwidth / 4, bh = (int)b.b4ell_bheight, f4 = b.b4ell_float4_aligned;
    const size_t total = (size_t)f4 * bh * bw4 * b.b4ell_block_num;
    std::vector<char> seen(total, 0);
    for (int br = 0; br < b.b4ell_row_num; br++)
        for (int k = 0; k < b.b4ell_block_num; k++) {
            const int c4 = b.b4ell_col_id[(size_t)k * b.b4ell_height_aligned + br];
            for (int h = 0; h < bh; h++)
                for (int w4 = 0; w4 < bw4; w4++)
                    for (int w = 0; w < 4; w++) {
                        const size_t i = (size_t)k * f4 * bw4 * bh + (size_t)h * f4 + (size_t)w4 * f4 * bh + (size_t)br * 4 + w;
                        const int r = br * bh + h, c = (c4 + w4) * 4 + w;
                        const bool in = r < b.matinfo.height && c < b.matinfo.width;
                        f(i, in ? r : -1, in ? c : -1);
                        seen[i] = 1;
                    }
        }
    for (size_t i = 0; i < total; i++)
        if (!seen[i]) f(i, -1, -1);   // alignment block rows
}

template <class F> void for_each_bcsr_slot(const b4csr_matrix_if& b, F f)
{
    const int bw4 = (int)b.b4csr_bwidth / 4, bh = (int)b.b4csr_bheight, al = b.b4csr_aligned_size;
    const size_t total = (size_t)al * bh * bw4;
    std::vector<char> seen(total, 0);
    for (int br = 0; br < b.b4csr_row_num; br++)
        for (int j = b.b4csr_row_ptr[br]; j < b.b4csr_row_ptr[br + 1]; j++) {
            const int c4 = b.b4csr_col_id[j];
            for (int h = 0; h < bh; h++)
                for (int w4 = 0; w4 < bw4; w4++)
                    for (int w = 0; w < 4; w++) {
                        const size_t i = (size_t)w4 * al * bh + (size_t)h * al + (size_t)j * 4 + w;
                        const int r = br * bh + h, c = (c4 + w4) * 4 + w;
                        const bool in = r < b.matinfo.height && c < b.matinfo.width;
                        f(i, in ? r : -1, in ? c : -1);
                        seen[i] = 1;
                    }
        }
    for (size_t i = 0; i < total; i++)
        if (!seen[i]) f(i, -1, -1);   // alignment slots past the last block
}

// Nonzeros of a generic BCSR (matrix_storage.h:1595 layout: element e of block j at
// row brow(j) * bh + e / bw, column col[j] + e % bw).
void gather_generic_bcsr(const bcsr_matrix_if& b, std::vector<Entry>& out)
{
    const int bw = (int)b.bcsr_bwidth, bh = (int)b.bcsr_bheight, al = b.bcsr_aligned_size;
    for (int br = 0; br < b.bcsr_row_num; br++)
        for (int j = b.bcsr_row_ptr[br]; j < b.bcsr_row_ptr[br + 1]; j++)
            for (int q = 0; q < bh * bw; q++) {
                const int r = br * bh + q / bw, c = b.bcsr_col_id[j] + q % bw;
                const float v = b.bcsr_data[(size_t)q * al + j];
                if (r < b.matinfo.height && c < b.matinfo.width && v != 0.0f) out.push_back(Entry{r, c, v});
            }
}

const bcsr_matrix_if& generic_of(const cocktail_iif* mat)
{
    return *reinterpret_cast<const bcsr_matrix_if*>(&mat->bcsr);
}

// Nonzeros of the non-diagonal parts of `mat`, gathered from their host layouts.
void gather_entries(const cocktail_iif* mat, bool include_diag, std::vector<Entry>& out)
{
    auto add = [&out](int r, int c, float v) { if (v != 0.0f) out.push_back(Entry{r, c, v}); };
    if (include_diag && mat->ifusedia) {
        const dia_matrix_iif& d = mat->dia;
        const int rows = std::min(d.matinfo.height, d.dia_length_aligned);
        for (int k = 0; k < d.dia_num; k++)
            for (int r = 0; r < rows; r++) {
                const int c = r + d.dia_offsets[k];
                if (c >= 0 && c < d.matinfo.width) add(r, c, d.dia_data[(size_t)k * d.dia_length_aligned + r]);
            }
    }
    if (include_diag && mat->ifusebdia) {
        const bdia_matrix_iif& b = mat->bdia;
        const int rows = std::min(b.matinfo.height, b.bdia_length_aligned);
        for (int band = 0; band < b.bdia_band_num; band++)
            for (int k = b.bdia_bptr[band]; k < b.bdia_bptr[band + 1]; k++) {
                const int o = b.bdia_offsets[band] + (k - b.bdia_bptr[band]);
                for (int r = 0; r < rows; r++) {
                    const int c = r + o;
                    if (c >= 0 && c < b.matinfo.width) add(r, c, b.bdia_data[(size_t)k * b.bdia_length_aligned + r]);
                }
            }
    }
    auto add_slot = [&](size_t i, int r, int c, const float* data) { if (r >= 0) add(r, c, data[i]); };
    if (mat->ifusesbell) for_each_sbell_slot(mat->sbell, [&](size_t i, int r, int c) { add_slot(i, r, c, mat->sbell.sbell_data); });
    if (mat->ifusebell) for_each_bell_slot(mat->bell, [&](size_t i, int r, int c) { add_slot(i, r, c, mat->bell.b4ell_data); });
    if (mat->ifusebcsr && mat->bcsr_meth_num == CSP_METH_GENERIC_BCSR) gather_generic_bcsr(generic_of(mat), out);
    else if (mat->ifusebcsr) for_each_bcsr_slot(mat->bcsr, [&](size_t i, int r, int c) { add_slot(i, r, c, mat->bcsr.b4csr_data); });
    if (mat->ifusesell) {
        const sell_matrix_if& s = mat->sell;
        const int H = (int)s.sell_slice_height;
        for (int sl = 0; sl < s.sell_slice_num; sl++) {
            const int b = s.sell_slice_ptr[sl], width = (s.sell_slice_ptr[sl + 1] - b) / H;
            for (int k = 0; k < width; k++)
                for (int lr = 0; lr < H; lr++) {
                    const int r = sl * H + lr;
                    if (r < s.matinfo.height) add(r, s.sell_col_id[b + k * H + lr], s.sell_data[b + k * H + lr]);
                }
        }
    }
    if (mat->ifuseell) {
        const ell_matrix_if& e = mat->ell;
        for (int k = 0; k < e.ell_num; k++)
            for (int r = 0; r < e.matinfo.height; r++)
                add(r, e.ell_col_id[(size_t)k * e.ell_height_aligned + r], e.ell_data[(size_t)k * e.ell_height_aligned + r]);
    }
    if (mat->ifusecsr) {
        const csr_matrix_if& s = mat->csr;
        for (int r = 0; r < s.matinfo.height; r++)
            for (int j = s.csr_row_ptr[r]; j < s.csr_row_ptr[r + 1]; j++) add(r, s.csr_col_id[j], s.csr_data[j]);
    }
    if (mat->ifusecoo) {
        const coo_matrix_if& s = mat->coo;
        for (int i = 0; i < s.matinfo.nnz; i++) add(s.coo_row_id[i], s.coo_col_id[i], s.coo_data[i]);
    }
}

// Transposed DIA of a square DIA part: offset -o, data_T[c] = data[c - o].
void transpose_dia(int n, int len, const std::vector<int>& off, const float* data, int valid_rows,
                   std::vector<int>& off_t, std::vector<float>& data_t)
{
    const int nd = (int)off.size();
    off_t.resize(nd);
    data_t.assign((size_t)nd * len, 0.0f);
    for (int dt = 0; dt < nd; dt++) {
        const int d = nd - 1 - dt;
        const int o = off[d];
        off_t[dt] = -o;
        for (int c = 0; c < std::min(len, n); c++) {
            const int r = c - o;
            if (r >= 0 && r < valid_rows) data_t[(size_t)dt * len + c] = data[(size_t)d * len + r];
        }
    }
}

}  // namespace

// A value-gradient segment given by the (row, col) of each slot (row -1: padding).
int Engine::add_slot_list(Seg& s, const std::vector<int>& rows, const std::vector<int>& cols)
{
    int *d_r = nullptr, *d_c = nullptr;
    int rc;
    if ((rc = upload_int(&d_r, rows.data(), rows.size(), std::max<size_t>(rows.size(), 1))) ||
        (rc = upload_int(&d_c, cols.data(), cols.size(), std::max<size_t>(cols.size(), 1))))
        return rc;
    s.kind = SEG_LIST;
    s.a0 = d_r;
    s.a1 = d_c;
    s.count = rows.size();
    return CSP_OK;
}

// Adjoint of a generic BCSR handle (csp_init_bcsr_kernels with CSP_FLAG_ADJOINT): A^T
// as one transposed CSR part of the blocks' nonzeros, and value gradients over every
// slot of the caller's BCSR layout (data[e * aligned + block], matrix_storage.h:1595),
// element e of a block being row e / bw, column e % bw; alignment slots, and slots
// of a partial last block row or column, get row -1.
// The value-gradient segment of a generic BCSR part: every slot of the caller's layout.
int Engine::gbcsr_segment(const bcsr_matrix_if& b, Seg& s)
{
    const int bw = (int)b.bcsr_bwidth, bh = (int)b.bcsr_bheight, al = b.bcsr_aligned_size, nb = b.bcsr_block_num;
    std::vector<int> brow((size_t)std::max(nb, 1), -1);
    for (int br = 0; br < b.bcsr_row_num; br++)
        for (int j = b.bcsr_row_ptr[br]; j < b.bcsr_row_ptr[br + 1]; j++) brow[j] = br;
    int *d_brow = nullptr, *d_col = nullptr;
    int rc;
    if ((rc = upload_int(&d_brow, brow.data(), (size_t)nb, std::max<size_t>(nb, 1))) ||
        (rc = upload_int(&d_col, b.bcsr_col_id, (size_t)nb, std::max<size_t>(nb, 1))))
        return rc;
    s.kind = SEG_GBCSR;
    s.a0 = d_brow;
    s.a1 = d_col;
    s.p0 = al;
    s.p1 = nb;
    s.p2 = bh * 16 + bw;
    s.count = (size_t)al * bh * bw;
    return CSP_OK;
}

// Adjoint of a generic BCSR handle (csp_init_bcsr_kernels with CSP_FLAG_ADJOINT): A^T
// as one transposed CSR part of the blocks' nonzeros, and value gradients over every
// slot of the caller's BCSR layout (data[e * aligned + block], matrix_storage.h:1595),
// element e of a block being row e / bw, column e % bw; alignment slots, and slots
// of a partial last block row or column, get row -1.
int Engine::build_adjoint_gbcsr(const bcsr_matrix_if& b)
{
    adjoint = true;
    std::vector<Entry> e;
    gather_generic_bcsr(b, e);
    int rc = add_transposed_csr(e);
    if (rc) return rc;
    Seg s;
    s.offset = 0;
    if ((rc = gbcsr_segment(b, s))) return rc;
    segs.push_back(s);
    abar_total = s.count;
    return CSP_OK;
}

// A^T of the given entries (of A) as one CSR part of adj_parts, the adaptive kernel.
int Engine::add_transposed_csr(std::vector<Entry>& e)
{
    if (e.empty()) return CSP_OK;
    std::swap(width, height);
    std::swap(parts, adj_parts);
    std::stable_sort(e.begin(), e.end(), [](const Entry& p, const Entry& q) { return p.c != q.c ? p.c < q.c : p.r < q.r; });
    csr_matrix_if t;
    csp_init_csr_matrix(&t);
    std::vector<int> rp((size_t)height + 1, 0), col(e.size());
    std::vector<float> val(e.size());
    for (size_t i = 0; i < e.size(); i++) {
        rp[(size_t)e[i].c + 1]++;
        col[i] = e[i].r;
        val[i] = e[i].v;
    }
    for (int i = 0; i < height; i++) rp[i + 1] += rp[i];
    t.matinfo.width = width;
    t.matinfo.height = height;
    t.matinfo.nnz = (int)e.size();
    t.csr_row_ptr = rp.data();
    t.csr_col_id = col.data();
    t.csr_data = val.data();
    const int rc = add_csr(t, 2);
    std::swap(parts, adj_parts);
    std::swap(width, height);
    return rc;
}

int Engine::build_adjoint(const cocktail_iif* mat)
{
    adjoint = true;
    const bool square = width == height;
    int rc;
    // --- transposed parts (built with rows and columns swapped) ---
    std::swap(width, height);
    std::swap(parts, adj_parts);
    auto add_tdia = [&](const std::vector<int>& off, const float* data, int len, int valid_rows, int method) {
        std::vector<int> off_t;
        std::vector<float> data_t;
        transpose_dia(height, len, off, data, valid_rows, off_t, data_t);
        dia_matrix_iif t;
        csp_init_dia_matrix(&t);
        t.matinfo.width = width;
        t.matinfo.height = height;
        t.dia_num = (int)off_t.size();
        t.dia_length = height;
        t.dia_length_aligned = len;
        t.dia_offsets = off_t.data();
        t.dia_data = data_t.data();
        return add_dia(t, method);
    };
    rc = CSP_OK;
    if (square && mat->ifusebdia) {
        const bdia_matrix_iif& b = mat->bdia;
        std::vector<int> off;
        for (int band = 0; band < b.bdia_band_num; band++)
            for (int k = b.bdia_bptr[band]; k < b.bdia_bptr[band + 1]; k++) off.push_back(b.bdia_offsets[band] + (k - b.bdia_bptr[band]));
        rc = add_tdia(off, b.bdia_data, b.bdia_length_aligned, std::min(b.matinfo.height, b.bdia_length_aligned), 1);
    }
    if (!rc && square && mat->ifusedia) {
        const dia_matrix_iif& d = mat->dia;
        std::vector<int> off(d.dia_offsets, d.dia_offsets + d.dia_num);
        rc = add_tdia(off, d.dia_data, d.dia_length_aligned, std::min(d.matinfo.height, d.dia_length_aligned), 1);
    }
    std::swap(parts, adj_parts);
    std::swap(width, height);
    if (rc) return rc;
    {
        std::vector<Entry> e;
        gather_entries(mat, !square, e);
        if ((rc = add_transposed_csr(e))) return rc;
    }

    // --- value-gradient segments over the forward parts, in launch order ---
    abar_total = 0;
    for (const Part& p : parts) {
        Seg s;
        s.offset = abar_total;
        switch (p.kind) {
        case PART_DIA: {
            s.kind = SEG_DIA;
            s.a0 = p.i0;
            s.p0 = p.k;
            s.p1 = p.stride;
            s.p2 = p.m;
            s.count = (size_t)p.k * p.stride;
            break;
        }
        case PART_BDIA: {
            const bdia_matrix_iif& b = mat->bdia;
            std::vector<int> off;
            for (int band = 0; band < b.bdia_band_num; band++)
                for (int k = b.bdia_bptr[band]; k < b.bdia_bptr[band + 1]; k++) off.push_back(b.bdia_offsets[band] + (k - b.bdia_bptr[band]));
            int* d_off = nullptr;
            if ((rc = upload_int(&d_off, off.data(), off.size(), std::max<size_t>(off.size(), 1)))) return rc;
            s.kind = SEG_DIA;
            s.a0 = d_off;
            s.p0 = (int)off.size();
            s.p1 = p.stride;
            s.p2 = p.m;
            s.count = off.size() * (size_t)p.stride;
            break;
        }
        case PART_CSR: {
            const csr_matrix_if& c = mat->csr;
            std::vector<int> rows((size_t)c.matinfo.nnz);
            for (int r = 0; r < c.matinfo.height; r++)
                for (int j = c.csr_row_ptr[r]; j < c.csr_row_ptr[r + 1]; j++) rows[j] = r;
            int *d_r = nullptr, *d_c = nullptr;
            if ((rc = upload_int(&d_r, rows.data(), rows.size(), std::max<size_t>(rows.size(), 1))) ||
                (rc = upload_int(&d_c, c.csr_col_id, (size_t)c.matinfo.nnz, std::max<size_t>(c.matinfo.nnz, 1))))
                return rc;
            s.kind = SEG_LIST;
            s.a0 = d_r;
            s.a1 = d_c;
            s.p0 = c.matinfo.nnz;
            s.count = (size_t)c.matinfo.nnz;
            break;
        }
        case PART_COO:
            s.kind = SEG_LIST;
            s.a0 = p.i0;
            s.a1 = p.i1;
            s.p0 = p.nnz;
            s.count = (size_t)p.nnz;
            break;
        case PART_XPANEL: {
            // slots follow the source part's own entry order (CSR or sorted COO), not
            // the panel regrouping of the forward layout
            std::vector<int> rows;
            const int* cols;
            if (p.from_csr) {
                const csr_matrix_if& c = mat->csr;
                rows.resize((size_t)c.matinfo.nnz);
                for (int r = 0; r < c.matinfo.height; r++)
                    for (int j = c.csr_row_ptr[r]; j < c.csr_row_ptr[r + 1]; j++) rows[j] = r;
                cols = c.csr_col_id;
            } else {
                rows.assign(mat->coo.coo_row_id, mat->coo.coo_row_id + mat->coo.matinfo.nnz);
                cols = mat->coo.coo_col_id;
            }
            int *d_r = nullptr, *d_c = nullptr;
            if ((rc = upload_int(&d_r, rows.data(), rows.size(), std::max<size_t>(rows.size(), 1))) ||
                (rc = upload_int(&d_c, cols, rows.size(), std::max<size_t>(rows.size(), 1))))
                return rc;
            s.kind = SEG_LIST;
            s.a0 = d_r;
            s.a1 = d_c;
            s.p0 = (int)rows.size();
            s.count = rows.size();
            break;
        }
        case PART_ELL:
            s.kind = SEG_ELL;
            s.a0 = p.i1;
            s.p0 = p.k;
            s.p1 = p.stride;
            s.p2 = p.m;
            s.count = (size_t)p.k * p.stride;
            break;
        case PART_SELL:
            s.kind = SEG_SELL;
            s.a0 = p.i0;
            s.a1 = p.i1;
            s.p0 = p.stride;
            s.p1 = mat->sell.sell_slice_num;
            s.p2 = p.m;
            s.count = (size_t)mat->sell.sell_slice_ptr[mat->sell.sell_slice_num];
            break;
        case PART_GBCSR:
            if ((rc = gbcsr_segment(generic_of(mat), s))) return rc;
            break;
        case PART_SBELL:
        case PART_BELL:
        case PART_BCSR: {
            // block layouts: the (row, col) of every slot, row -1 for padding
            std::vector<int> rows, cols;
            auto put = [&](size_t i, int r, int c) {
                if (i >= rows.size()) { rows.resize(i + 1, -1); cols.resize(i + 1, -1); }
                rows[i] = r;
                cols[i] = c;
            };
            if (p.kind == PART_SBELL) for_each_sbell_slot(mat->sbell, put);
            else if (p.kind == PART_BELL) for_each_bell_slot(mat->bell, put);
            else for_each_bcsr_slot(mat->bcsr, put);
            if ((rc = add_slot_list(s, rows, cols))) return rc;
            break;
        }
        default:
            s.kind = SEG_NONE;
            s.count = 0;
            abar_blocks = true;
            break;
        }
        abar_total += s.count;
        segs.push_back(s);
    }
    return CSP_OK;
}

int Engine::launch_abar(const float* ybar, float* abar, int* prow, int* pcol, cudaStream_t st)
{
    using namespace dev;
    for (const Seg& s : segs) {
        if (s.count == 0) continue;
        float* a = abar ? abar + s.offset : nullptr;
        int* pr = prow ? prow + s.offset : nullptr;
        int* pc = pcol ? pcol + s.offset : nullptr;
        const unsigned g = (unsigned)((s.count + 255) / 256);
        switch (s.kind) {
        case SEG_DIA:
            if (a && s.p1 % 4 == 0 && (reinterpret_cast<uintptr_t>(a) & 15) == 0) {
                const unsigned g4 = (unsigned)((s.p1 / 4 + 255) / 256);
                abar_dia4_kernel<<<g4, 256, (size_t)s.p0 * sizeof(int), st>>>(s.a0, s.p0, s.p1, s.p2, width, ybar, d_x, a);
            } else {
                abar_dia_kernel<<<g, 256, 0, st>>>(s.a0, s.p0, s.p1, s.p2, width, ybar, d_x, a, pr, pc);
            }
            break;
        case SEG_LIST: abar_list_kernel<<<g, 256, 0, st>>>(s.a0, s.a1, s.count, ybar, d_x, a, pr, pc); break;
        case SEG_GBCSR:
            abar_gbcsr_kernel<<<g, 256, 0, st>>>(s.a0, s.a1, s.p0, s.p1, s.p2 >> 4, s.p2 & 15, height, width, ybar, d_x, a,
                                                 pr, pc);
            break;
        case SEG_ELL: abar_ell_kernel<<<g, 256, 0, st>>>(s.a0, s.p0, s.p1, s.p2, ybar, d_x, a, pr, pc); break;
        case SEG_SELL: {
            const unsigned gs = (unsigned)(((size_t)s.p1 * s.p0 + 255) / 256);
            abar_sell_kernel<<<gs, 256, 0, st>>>(s.a0, s.a1, s.p0, s.p1, s.p2, ybar, d_x, a, pr, pc);
            break;
        }
        default: break;
        }
    }
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? CSP_OK : cuda_error(e, "adjoint value gradient");
}

}  // namespace csp

using csp::set_error;

extern "C" {

int csp_spmv_adjoint(csp_handle* h, const float* d_ybar, float* d_xbar, float* d_abar)
{
    if (!h) return set_error(CSP_EINVAL, "null handle");
    csp::Engine& e = h->eng;
    if (!e.adjoint) return set_error(CSP_EINVAL, "handle was not built with CSP_FLAG_ADJOINT");
    if (!d_ybar) return set_error(CSP_EINVAL, "null ybar");
    if (d_abar && e.abar_blocks) return set_error(CSP_EUNSUP, "value gradients of this handle's parts are not provided");
    if (d_xbar) {
        int rc = e.enqueue_parts(e.adj_parts, d_ybar, d_xbar, e.height, e.stream);
        if (rc) return rc;
    }
    if (d_abar) return e.launch_abar(d_ybar, d_abar, nullptr, nullptr, e.stream);
    return CSP_OK;
}

int csp_adjoint_slots(csp_handle* h, size_t* nslots)
{
    if (!h || !nslots) return set_error(CSP_EINVAL, "null argument");
    if (!h->eng.adjoint) return set_error(CSP_EINVAL, "handle was not built with CSP_FLAG_ADJOINT");
    *nslots = h->eng.abar_total;
    return CSP_OK;
}

int csp_adjoint_pattern(csp_handle* h, int* d_rows, int* d_cols)
{
    if (!h || !d_rows || !d_cols) return set_error(CSP_EINVAL, "null argument");
    if (!h->eng.adjoint) return set_error(CSP_EINVAL, "handle was not built with CSP_FLAG_ADJOINT");
    if (h->eng.abar_blocks) return set_error(CSP_EUNSUP, "value gradients of this handle's parts are not provided");
    return h->eng.launch_abar(nullptr, nullptr, d_rows, d_cols, h->eng.stream);
}

}  // extern "C"
