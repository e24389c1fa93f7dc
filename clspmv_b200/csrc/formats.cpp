// Host-side storage-format conversions of the clSpMV formats.
//
// Every csp_coo2* function writes arrays that are byte-identical to the
// reference conversion of the same name in clSpMV_NV/include/matrix_storage.h
// (cited per function), including the padding values the reference chooses.
// The algorithms are this library's own (hash maps and single passes where
// the reference searches linearly), but the output layouts and the padding
// rules necessarily follow the reference: the device kernels and any caller
// that fills these structs by hand rely on them.
//
// Differences that only concern inputs on which the reference has undefined
// behaviour (out-of-range indices, rows beyond the DIA length, empty leading
// rows in pad_csr): this code returns CSP_EINVAL / CSP_EFORMAT instead.
// Array regions the reference leaves uninitialised (alignment padding of the
// b4ell layout) are zero here.
#include <stdlib.h>
#include <string.h>
#include <stdint.h>
#include <algorithm>
#include <unordered_map>
#include <vector>

#include "csp/clspmv.h"
#include "internal.h"

namespace csp {

// clSpMV_NV/include/constant.h:10,9
static const int kMaxLevels = 1000;
static const long long kMaxMemObj = 838860800LL;

template <class T>
static T* xmalloc(size_t n)
{
    if (n == 0) n = 1;
    return static_cast<T*>(malloc(n * sizeof(T)));
}

template <class T>
static T* xcalloc(size_t n)
{
    if (n == 0) n = 1;
    return static_cast<T*>(calloc(n, sizeof(T)));
}

int check_coo(const coo_matrix_if* m)
{
    if (!m) return set_error(CSP_EINVAL, "null COO matrix");
    const int nnz = m->matinfo.nnz, h = m->matinfo.height, w = m->matinfo.width;
    if (nnz < 0 || h < 0 || w < 0) return set_error(CSP_EINVAL, "negative COO dimension");
    if (nnz > 0 && (!m->coo_row_id || !m->coo_col_id || !m->coo_data))
        return set_error(CSP_EINVAL, "COO arrays are null");
    for (int i = 0; i < nnz; i++) {
        if (m->coo_row_id[i] < 0 || m->coo_row_id[i] >= h || m->coo_col_id[i] < 0 || m->coo_col_id[i] >= w)
            return set_error(CSP_EINVAL, "COO entry %d (%d, %d) outside %d x %d", i,
                             m->coo_row_id[i], m->coo_col_id[i], h, w);
    }
    return CSP_OK;
}

// Row pointer of a row-sorted COO (the scan the reference repeats in coo2csr :1290-1306,
// coo2sell :1414-1431, coo2bcsr :1612-1629 ...).
static void row_pointer(const coo_matrix_if* s, std::vector<int>& rp)
{
    const int h = s->matinfo.height, nnz = s->matinfo.nnz;
    rp.assign((size_t)h + 1, 0);
    for (int i = 0; i < nnz; i++) rp[(size_t)s->coo_row_id[i] + 1]++;
    for (int r = 0; r < h; r++) rp[r + 1] += rp[r];
}

// Iterative quicksort keyed on (row, col) whose partition steps equal the reference's
// (matrix_storage.h:745-815: middle element as pivot, moved to the left end first;
// at most kMaxLevels pending ranges, else failure).  Reproducing the steps keeps the
// order of duplicate (row, col) entries identical to the reference's.
bool quicksort_coo(int* row, int* col, float* val, int n)
{
    std::vector<int> lo(kMaxLevels), hi(kMaxLevels);
    int depth = 0;
    lo[0] = 0;
    hi[0] = n;
    while (depth >= 0) {
        int left = lo[depth];
        int right = hi[depth] - 1;
        if (left >= right) {
            depth--;
            continue;
        }
        const int mid = left + (right - left) / 2;
        const int prow = row[mid], pcol = col[mid];
        const float pval = val[mid];
        row[mid] = row[left]; col[mid] = col[left]; val[mid] = val[left];
        row[left] = prow; col[left] = pcol; val[left] = pval;
        if (depth == kMaxLevels - 1) return false;
        while (left < right) {
            while (left < right && (row[right] > prow || (row[right] == prow && col[right] > pcol))) right--;
            if (left < right) {
                row[left] = row[right]; col[left] = col[right]; val[left] = val[right];
                left++;
            }
            while (left < right && (row[left] < prow || (row[left] == prow && col[left] < pcol))) left++;
            if (left < right) {
                row[right] = row[left]; col[right] = col[left]; val[right] = val[left];
                right--;
            }
        }
        row[left] = prow; col[left] = pcol; val[left] = pval;
        lo[depth + 1] = left + 1;
        hi[depth + 1] = hi[depth];
        hi[depth] = left;
        depth++;
    }
    return true;
}

bool coo_is_sorted(const coo_matrix_if* m)
{
    const int nnz = m->matinfo.nnz;
    for (int i = 0; i + 1 < nnz; i++) {
        const int r0 = m->coo_row_id[i], r1 = m->coo_row_id[i + 1];
        if (r0 > r1 || (r0 == r1 && m->coo_col_id[i] > m->coo_col_id[i + 1])) return false;
    }
    return true;
}

bool coo_has_duplicates(const coo_matrix_if* m)
{
    for (int i = 0; i + 1 < m->matinfo.nnz; i++)
        if (m->coo_row_id[i] == m->coo_row_id[i + 1] && m->coo_col_id[i] == m->coo_col_id[i + 1]) return true;
    return false;
}

int ensure_sorted(coo_matrix_if* m)
{
    if (coo_is_sorted(m)) return CSP_OK;
    if (!quicksort_coo(m->coo_row_id, m->coo_col_id, m->coo_data, m->matinfo.nnz))
        return set_error(CSP_EFORMAT, "sort_coo: partition stack exhausted");
    return CSP_OK;
}

// Blocks of one block row, in the reference's order (matrix_storage.h:1631-1697): the
// entries of bheight rows sorted by (col, row), grouped into blocks whose column is
// col - col % bwidth; each block's bwidth*bheight values row-major, later duplicates win.
struct Elem { int rowid; int colid; float data; };

void build_blocks(const coo_matrix_if* s, unsigned bw, unsigned bh, BlockRows& out)
{
    std::vector<int> rp;
    row_pointer(s, rp);
    const int h = s->matinfo.height;
    const int brows = h / (int)bh + (h % (int)bh != 0);
    const unsigned bs = bw * bh;
    out.rowptr.assign((size_t)brows + 1, 0);
    out.colid.clear();
    out.data.clear();
    out.colid.reserve(s->matinfo.nnz);
    std::vector<Elem> el;
    for (int br = 0; br < brows; br++) {
        const int r0 = br * (int)bh;
        const int start = rp[r0];
        const int end = (r0 + (int)bh <= h) ? rp[r0 + bh] : rp[h];
        int nblocks = 0;
        if (end > start) {
            el.resize((size_t)(end - start));
            for (int i = start; i < end; i++)
                el[i - start] = Elem{s->coo_row_id[i], s->coo_col_id[i], s->coo_data[i]};
            // Same comparator as the reference's compareCol (matrix_storage.h:1531-1540),
            // applied with std::sort to the same sequence, so ties land identically.
            std::sort(el.begin(), el.end(), [](const Elem& a, const Elem& b) {
                if (a.colid != b.colid) return a.colid < b.colid;
                return a.rowid < b.rowid;
            });
            int cur = -1;
            size_t base = 0;
            for (const Elem& e : el) {
                const int bcol = e.colid - e.colid % (int)bw;
                if (bcol != cur || nblocks == 0) {
                    cur = bcol;
                    base = out.data.size();
                    out.data.resize(base + bs, 0.0f);
                    out.colid.push_back(bcol);
                    nblocks++;
                }
                const unsigned inner = (unsigned)(e.rowid % (int)bh) * bw + (unsigned)(e.colid - bcol);
                out.data[base + inner] = e.data;
            }
        }
        out.rowptr[br + 1] = out.rowptr[br] + nblocks;
    }
}

// b4csr layout (matrix_storage.h:1741-1897 coo2b4csr; analyze.cpp:2113 extract_bcsr_part):
// column ids /4; data [w4 * (al * bh) + h * al + blk * 4 + w], al = aligned_length(4 * #blocks).
int write_b4csr(const BlockRows& b, unsigned bw, unsigned bh, int alignment, b4csr_matrix_if* d)
{
    const long long nb = (long long)b.colid.size();
    const unsigned bs = bw * bh, bw4 = bw / 4;
    const int al = csp_aligned_length((int)nb * 4, alignment);
    d->b4csr_bwidth = bw;
    d->b4csr_bheight = bh;
    d->b4csr_row_num = (int)b.rowptr.size() - 1;
    d->b4csr_aligned_size = al;
    d->b4csr_block_num = (int)nb;
    d->b4csr_row_ptr = xmalloc<int>(b.rowptr.size());
    d->b4csr_col_id = xmalloc<int>((size_t)nb);
    d->b4csr_data = xcalloc<float>((size_t)al * bh * bw4);
    if (!d->b4csr_row_ptr || !d->b4csr_col_id || !d->b4csr_data) return set_error(CSP_ENOMEM, "b4csr layout");
    memcpy(d->b4csr_row_ptr, b.rowptr.data(), b.rowptr.size() * sizeof(int));
    const size_t rowlen = (size_t)al * bh;
    for (long long i = 0; i < nb; i++) {
        d->b4csr_col_id[i] = b.colid[i] / 4;
        for (unsigned h = 0; h < bh; h++)
            for (unsigned w4 = 0; w4 < bw4; w4++)
                for (unsigned w = 0; w < 4; w++)
                    d->b4csr_data[w4 * rowlen + (size_t)h * al + (size_t)i * 4 + w] =
                        b.data[(size_t)i * bs + h * bw + w4 * 4 + w];
    }
    return CSP_OK;
}

// b4ell layout (matrix_storage.h:2010-2200 coo2b4ell; analyze.cpp:1888 extract_bell_part):
// `ellnum` slots per block row; short rows repeat their last block column, zero data.
int write_b4ell(const BlockRows& b, unsigned bw, unsigned bh, int alignment, int ellnum, b4ell_matrix_if* d)
{
    const int nbr = (int)b.rowptr.size() - 1;
    const unsigned bs = bw * bh, bw4 = bw / 4;
    const int hal = csp_aligned_length(nbr, alignment);
    const int f4 = csp_aligned_length(4 * nbr, alignment);
    d->b4ell_bwidth = bw;
    d->b4ell_bheight = bh;
    d->b4ell_row_num = nbr;
    d->b4ell_block_num = ellnum;
    d->b4ell_height_aligned = hal;
    d->b4ell_float4_aligned = f4;
    d->b4ell_col_id = xcalloc<int>((size_t)hal * ellnum);
    d->b4ell_data = xcalloc<float>((size_t)f4 * bh * bw4 * ellnum);
    if (!d->b4ell_col_id || !d->b4ell_data) return set_error(CSP_ENOMEM, "b4ell layout");
    const size_t colsize = (size_t)f4 * bw4 * bh, w4size = (size_t)f4 * bh;
    for (int r = 0; r < nbr; r++) {
        int last = 0, k = 0;
        for (int j = b.rowptr[r]; j < b.rowptr[r + 1]; j++, k++) {
            d->b4ell_col_id[r + (size_t)k * hal] = last = b.colid[j] / 4;
            for (unsigned h = 0; h < bh; h++)
                for (unsigned w4 = 0; w4 < bw4; w4++)
                    for (unsigned w = 0; w < 4; w++)
                        d->b4ell_data[(size_t)k * colsize + (size_t)h * f4 + w4 * w4size + (size_t)r * 4 + w] =
                            b.data[(size_t)j * bs + h * bw + w4 * 4 + w];
        }
        for (; k < ellnum; k++) d->b4ell_col_id[r + (size_t)k * hal] = last;
    }
    return CSP_OK;
}

// sbell layout (matrix_storage.h:2203-2409 coo2sbell; analyze.cpp:1660 extract_sbell_part):
// slice i holds width[i] slots for each of its `sh` block rows.
int write_sbell(const BlockRows& b, unsigned bw, unsigned bh, unsigned sh, const std::vector<int>& width,
                sbell_matrix_if* d)
{
    const int nbr = (int)b.rowptr.size() - 1;
    const int H = (int)sh;
    const int nslices = (int)width.size();
    d->sbell_bwidth = bw;
    d->sbell_bheight = bh;
    d->sbell_slice_num = nslices;
    d->sbell_row_num = nbr;
    d->sbell_slice_height = sh;
    d->sbell_slice_ptr = xmalloc<int>((size_t)nslices + 1);
    if (!d->sbell_slice_ptr) return set_error(CSP_ENOMEM, "sbell layout");
    d->sbell_slice_ptr[0] = 0;
    for (int i = 0; i < nslices; i++) d->sbell_slice_ptr[i + 1] = d->sbell_slice_ptr[i] + width[i] * H;
    const long long total = d->sbell_slice_ptr[nslices];
    const unsigned bs = bw * bh, bw4 = bw / 4;
    d->sbell_col_id = xcalloc<int>((size_t)total);
    d->sbell_data = xcalloc<float>((size_t)total * bs);
    if (!d->sbell_col_id || !d->sbell_data) return set_error(CSP_ENOMEM, "sbell layout");
    const size_t colsize = (size_t)H * bw4 * bh * 4, w4size = (size_t)H * bh * 4, hsize = (size_t)H * 4;
    for (int r = 0; r < nbr; r++) {
        const int sl = r / H, lr = r % H;
        const size_t cstart = (size_t)d->sbell_slice_ptr[sl];
        const size_t dstart = cstart * bs;
        int last = 0, k = 0;
        for (int j = b.rowptr[r]; j < b.rowptr[r + 1]; j++, k++) {
            d->sbell_col_id[cstart + lr + (size_t)k * H] = last = b.colid[j] / 4;
            for (unsigned h = 0; h < bh; h++)
                for (unsigned w4 = 0; w4 < bw4; w4++)
                    for (unsigned w = 0; w < 4; w++)
                        d->sbell_data[dstart + (size_t)k * colsize + h * hsize + w4 * w4size + (size_t)lr * 4 + w] =
                            b.data[(size_t)j * bs + h * bw + w4 * 4 + w];
        }
        for (; k < width[sl]; k++) d->sbell_col_id[cstart + lr + (size_t)k * H] = last;
    }
    return CSP_OK;
}

// The banding step of coo2bdia (matrix_storage.h:1185): runs of consecutive offsets
// of a built DIA become bands; the DIA's data moves into the BDIA unchanged (same
// layout) and the DIA is freed.
int bdia_from_dia(dia_matrix_iif* dia, bdia_matrix_iif* d)
{
    std::vector<int> boff, bcnt;
    for (int k = 0; k < dia->dia_num; k++) {
        if (k > 0 && dia->dia_offsets[k] - dia->dia_offsets[k - 1] == 1) bcnt.back()++;
        else { boff.push_back(dia->dia_offsets[k]); bcnt.push_back(1); }
    }
    d->bdia_band_num = (int)boff.size();
    d->bdia_length = dia->dia_length;
    d->bdia_length_aligned = dia->dia_length_aligned;
    d->bdia_offsets = xmalloc<int>(boff.size());
    d->bdia_bptr = xmalloc<int>(boff.size() + 1);
    if (!d->bdia_offsets || !d->bdia_bptr) { csp_free_dia_matrix(dia); return set_error(CSP_ENOMEM, "coo2bdia"); }
    d->bdia_bptr[0] = 0;
    for (size_t b = 0; b < boff.size(); b++) {
        d->bdia_offsets[b] = boff[b];
        d->bdia_bptr[b + 1] = d->bdia_bptr[b] + bcnt[b];
    }
    d->bdia_data = dia->dia_data;   // identical data layout
    dia->dia_data = nullptr;
    csp_free_dia_matrix(dia);
    return CSP_OK;
}

}  // namespace csp

using namespace csp;

extern "C" {

int csp_aligned_length(int length, int alignment)
{
    if (alignment <= 0) return length;
    if (length % alignment == 0) return length;
    return length + alignment - length % alignment;
}

int csp_if_sorted_coo(const coo_matrix_if* m) { return m && coo_is_sorted(m) ? 1 : 0; }

int csp_sort_coo(coo_matrix_if* m)
{
    if (!m) return set_error(CSP_EINVAL, "null COO matrix");
    if (!quicksort_coo(m->coo_row_id, m->coo_col_id, m->coo_data, m->matinfo.nnz))
        return set_error(CSP_EFORMAT, "sort_coo: partition stack exhausted");
    return CSP_OK;
}

// matrix_storage.h:1269 coo2csr
int csp_coo2csr(coo_matrix_if* s, csr_matrix_if* d)
{
    int rc = check_coo(s);
    if (rc || !d) return rc ? rc : set_error(CSP_EINVAL, "null CSR");
    if ((rc = ensure_sorted(s))) return rc;
    const int nnz = s->matinfo.nnz;
    d->matinfo = s->matinfo;
    std::vector<int> rp;
    row_pointer(s, rp);
    d->csr_row_ptr = xmalloc<int>(rp.size());
    d->csr_col_id = xmalloc<int>(nnz);
    d->csr_data = xmalloc<float>(nnz);
    if (!d->csr_row_ptr || !d->csr_col_id || !d->csr_data) return set_error(CSP_ENOMEM, "coo2csr");
    memcpy(d->csr_row_ptr, rp.data(), rp.size() * sizeof(int));
    memcpy(d->csr_col_id, s->coo_col_id, (size_t)nnz * sizeof(int));
    memcpy(d->csr_data, s->coo_data, (size_t)nnz * sizeof(float));
    return CSP_OK;
}

// Expands CSR rows back to COO.  (The reference's csr2coo, matrix_storage.h:1239,
// does not compile when instantiated; this is the evident intent.)
int csp_csr2coo(const csr_matrix_if* s, coo_matrix_if* d)
{
    if (!s || !d) return set_error(CSP_EINVAL, "null matrix");
    const int nnz = s->matinfo.nnz;
    d->matinfo = s->matinfo;
    d->coo_row_id = xmalloc<int>(nnz);
    d->coo_col_id = xmalloc<int>(nnz);
    d->coo_data = xmalloc<float>(nnz);
    if (!d->coo_row_id || !d->coo_col_id || !d->coo_data) return set_error(CSP_ENOMEM, "csr2coo");
    memcpy(d->coo_col_id, s->csr_col_id, (size_t)nnz * sizeof(int));
    memcpy(d->coo_data, s->csr_data, (size_t)nnz * sizeof(float));
    for (int r = 0; r < s->matinfo.height; r++)
        for (int j = s->csr_row_ptr[r]; j < s->csr_row_ptr[r + 1]; j++) d->coo_row_id[j] = r;
    return CSP_OK;
}

// matrix_storage.h:1341 coo2ell.  Column-major slots of ell_height_aligned rows; a short
// row repeats its last column id with value 0 (column 0 for an empty row); alignment
// rows are (0, 0.0).
int csp_coo2ell(coo_matrix_if* s, ell_matrix_if* d, int alignment, int ellnum)
{
    int rc = check_coo(s);
    if (rc || !d) return rc ? rc : set_error(CSP_EINVAL, "null ELL");
    if ((rc = ensure_sorted(s))) return rc;
    std::vector<int> rp;
    row_pointer(s, rp);
    const int h = s->matinfo.height;
    int maxw = 0;
    for (int r = 0; r < h; r++) maxw = std::max(maxw, rp[r + 1] - rp[r]);
    if (ellnum == 0) ellnum = maxw;
    if (ellnum < maxw) return set_error(CSP_EINVAL, "coo2ell: ellnum %d below the longest row %d", ellnum, maxw);
    d->matinfo = s->matinfo;
    d->ell_num = ellnum;
    const int hal = csp_aligned_length(h, alignment);
    d->ell_height_aligned = hal;
    const size_t total = (size_t)hal * (size_t)ellnum;
    d->ell_col_id = xcalloc<int>(total);
    d->ell_data = xcalloc<float>(total);
    if (!d->ell_col_id || !d->ell_data) return set_error(CSP_ENOMEM, "coo2ell");
    for (int r = 0; r < h; r++) {
        int last = 0;
        int k = 0;
        for (int j = rp[r]; j < rp[r + 1]; j++, k++) {
            d->ell_col_id[(size_t)k * hal + r] = last = s->coo_col_id[j];
            d->ell_data[(size_t)k * hal + r] = s->coo_data[j];
        }
        for (; k < ellnum; k++) d->ell_col_id[(size_t)k * hal + r] = last;
    }
    return CSP_OK;
}

// matrix_storage.h:1310 ell2coo: nonzero values only, row by row.
int csp_ell2coo(const ell_matrix_if* s, coo_matrix_if* d)
{
    if (!s || !d) return set_error(CSP_EINVAL, "null matrix");
    const int h = s->matinfo.height, nnz = s->matinfo.nnz, hal = s->ell_height_aligned;
    d->matinfo = s->matinfo;
    d->coo_row_id = xmalloc<int>(nnz);
    d->coo_col_id = xmalloc<int>(nnz);
    d->coo_data = xmalloc<float>(nnz);
    if (!d->coo_row_id || !d->coo_col_id || !d->coo_data) return set_error(CSP_ENOMEM, "ell2coo");
    int n = 0;
    for (int r = 0; r < h; r++)
        for (int k = 0; k < s->ell_num; k++) {
            const float v = s->ell_data[(size_t)k * hal + r];
            if (v != 0.0f) {
                if (n >= nnz) return set_error(CSP_EFORMAT, "ell2coo: more nonzeros than matinfo.nnz");
                d->coo_row_id[n] = r;
                d->coo_col_id[n] = s->ell_col_id[(size_t)k * hal + r];
                d->coo_data[n] = v;
                n++;
            }
        }
    if (n != nnz) return set_error(CSP_EFORMAT, "ell2coo: %d nonzero values, matinfo.nnz %d", n, nnz);
    return CSP_OK;
}

// matrix_storage.h:1398 coo2sell.  Slice s holds sliceheight rows as width(s) column-major
// slots, width(s) = longest row in the slice.  Padding slot k of a row copies slot k-1's
// column id; slot 0 of an empty row (and of the rows past `height` in the last slice)
// copies the slice's first stored column id.  Padding values are 0.
int csp_coo2sell(coo_matrix_if* s, sell_matrix_if* d, unsigned int sh)
{
    int rc = check_coo(s);
    if (rc || !d) return rc ? rc : set_error(CSP_EINVAL, "null SELL");
    if (sh == 0) return set_error(CSP_EINVAL, "coo2sell: slice height 0");
    if ((rc = ensure_sorted(s))) return rc;
    std::vector<int> rp;
    row_pointer(s, rp);
    const int h = s->matinfo.height;
    const int H = (int)sh;
    const int nslices = h / H + (h % H != 0);
    d->matinfo = s->matinfo;
    d->sell_slice_height = sh;
    d->sell_slice_num = nslices;
    d->sell_slice_ptr = xmalloc<int>((size_t)nslices + 1);
    if (!d->sell_slice_ptr) return set_error(CSP_ENOMEM, "coo2sell");
    d->sell_slice_ptr[0] = 0;
    long long total = 0;
    std::vector<int> width((size_t)nslices);
    for (int i = 0; i < nslices; i++) {
        int w = 0;
        for (int r = i * H; r < (i + 1) * H && r < h; r++) w = std::max(w, rp[r + 1] - rp[r]);
        width[i] = w;
        total += (long long)w * H;
        if (total > INT32_MAX) return set_error(CSP_EFORMAT, "coo2sell: padded size exceeds int32");
        d->sell_slice_ptr[i + 1] = (int)total;
    }
    d->sell_col_id = xmalloc<int>((size_t)total);
    d->sell_data = xmalloc<float>((size_t)total);
    if (!d->sell_col_id || !d->sell_data) return set_error(CSP_ENOMEM, "coo2sell");
    for (int i = 0; i < nslices; i++) {
        int* col = d->sell_col_id + d->sell_slice_ptr[i];
        float* val = d->sell_data + d->sell_slice_ptr[i];
        const int w = width[i];
        if (w == 0) continue;
        const int first = i * H;
        col[0] = 0;
        for (int r = first; r < first + H; r++) {
            const int lr = r - first;
            int k = 0;
            if (r < h) {
                for (int j = rp[r]; j < rp[r + 1]; j++, k++) {
                    col[k * H + lr] = s->coo_col_id[j];
                    val[k * H + lr] = s->coo_data[j];
                }
            }
            for (; k < w; k++) {
                const int id = k * H + lr;
                col[id] = (id >= H) ? col[id - H] : col[0];
                val[id] = 0.0f;
            }
        }
    }
    return CSP_OK;
}

// matrix_storage.h:937 coo2dia.  Diagonals sorted by offset, each dia_length_aligned long
// and indexed by row; a later duplicate (row, col) overwrites an earlier one.  Fails
// (CSP_EFORMAT, dia_num/dia_length_aligned set, no arrays) as soon as a new diagonal
// would be opened while diaCount * aligned length >= 2 * nnz (:972).
int csp_coo2dia(coo_matrix_if* s, dia_matrix_iif* d, int alignment)
{
    int rc = check_coo(s);
    if (rc || !d) return rc ? rc : set_error(CSP_EINVAL, "null DIA");
    d->matinfo = s->matinfo;
    const int h = s->matinfo.height, w = s->matinfo.width, nnz = s->matinfo.nnz;
    d->dia_length = std::min(w, h);
    const int len = csp_aligned_length(d->dia_length, alignment);
    std::unordered_map<int, int> slot;
    std::vector<int> offs;
    std::vector<std::vector<float>> data;
    for (int i = 0; i < nnz; i++) {
        const int r = s->coo_row_id[i], c = s->coo_col_id[i];
        if (r >= len) return set_error(CSP_EFORMAT, "coo2dia: row %d beyond the diagonal length %d", r, len);
        const int off = c - r;
        auto it = slot.find(off);
        if (it == slot.end()) {
            if ((long long)offs.size() * len >= 2LL * nnz) {
                d->dia_num = (int)offs.size();
                d->dia_length_aligned = len;
                d->dia_offsets = nullptr;
                d->dia_data = nullptr;
                return set_error(CSP_EFORMAT, "coo2dia: too much padding for the DIA format");
            }
            it = slot.emplace(off, (int)offs.size()).first;
            offs.push_back(off);
            data.emplace_back((size_t)len, 0.0f);
        }
        data[it->second][r] = s->coo_data[i];
    }
    std::vector<int> order(offs.size());
    for (size_t i = 0; i < order.size(); i++) order[i] = (int)i;
    std::sort(order.begin(), order.end(), [&](int a, int b) { return offs[a] < offs[b]; });
    d->dia_num = (int)offs.size();
    d->dia_length_aligned = len;
    d->dia_offsets = xmalloc<int>(offs.size());
    d->dia_data = xmalloc<float>(offs.size() * (size_t)len);
    if (!d->dia_offsets || !d->dia_data) return set_error(CSP_ENOMEM, "coo2dia");
    for (size_t k = 0; k < order.size(); k++) {
        d->dia_offsets[k] = offs[order[k]];
        memcpy(d->dia_data + k * (size_t)len, data[order[k]].data(), (size_t)len * sizeof(float));
    }
    return CSP_OK;
}

// matrix_storage.h:826 dia2coo: nonzero values, row by row, diagonal by diagonal.
int csp_dia2coo(const dia_matrix_iif* s, coo_matrix_if* d)
{
    if (!s || !d) return set_error(CSP_EINVAL, "null matrix");
    const int nnz = s->matinfo.nnz, len = s->dia_length_aligned;
    d->matinfo = s->matinfo;
    d->coo_row_id = xmalloc<int>(nnz);
    d->coo_col_id = xmalloc<int>(nnz);
    d->coo_data = xmalloc<float>(nnz);
    if (!d->coo_row_id || !d->coo_col_id || !d->coo_data) return set_error(CSP_ENOMEM, "dia2coo");
    int n = 0;
    for (int r = 0; r < len; r++)
        for (int k = 0; k < s->dia_num; k++) {
            const int c = r + s->dia_offsets[k];
            if (c < 0 || c >= s->dia_length) continue;
            const float v = s->dia_data[(size_t)k * len + r];
            if (v == 0.0f) continue;
            if (n >= nnz) return set_error(CSP_EFORMAT, "dia2coo: more nonzeros than matinfo.nnz");
            d->coo_row_id[n] = r;
            d->coo_col_id[n] = c;
            d->coo_data[n] = v;
            n++;
        }
    return ensure_sorted(d);
}

// matrix_storage.h:1185 coo2bdia: coo2dia, then runs of consecutive offsets become bands.
int csp_coo2bdia(coo_matrix_if* s, bdia_matrix_iif* d, int alignment)
{
    if (!d) return set_error(CSP_EINVAL, "null BDIA");
    dia_matrix_iif dia;
    csp_init_dia_matrix(&dia);
    int rc = csp_coo2dia(s, &dia, alignment);
    d->matinfo = s ? s->matinfo : d->matinfo;
    if (rc) return rc;
    return bdia_from_dia(&dia, d);
}

// matrix_storage.h:1137 bdia2coo.
int csp_bdia2coo(const bdia_matrix_iif* s, coo_matrix_if* d)
{
    if (!s || !d) return set_error(CSP_EINVAL, "null matrix");
    const int nnz = s->matinfo.nnz, len = s->bdia_length_aligned;
    d->matinfo = s->matinfo;
    d->coo_row_id = xmalloc<int>(nnz);
    d->coo_col_id = xmalloc<int>(nnz);
    d->coo_data = xmalloc<float>(nnz);
    if (!d->coo_row_id || !d->coo_col_id || !d->coo_data) return set_error(CSP_ENOMEM, "bdia2coo");
    int n = 0;
    for (int b = 0; b < s->bdia_band_num; b++) {
        int off = s->bdia_offsets[b];
        for (int k = s->bdia_bptr[b]; k < s->bdia_bptr[b + 1]; k++, off++)
            for (int r = 0; r < len; r++) {
                const int c = r + off;
                if (c < 0 || c >= s->bdia_length) continue;
                const float v = s->bdia_data[(size_t)k * len + r];
                if (v == 0.0f) continue;
                if (n >= nnz) return set_error(CSP_EFORMAT, "bdia2coo: more nonzeros than matinfo.nnz");
                d->coo_row_id[n] = r;
                d->coo_col_id[n] = c;
                d->coo_data[n] = v;
                n++;
            }
    }
    return ensure_sorted(d);
}

// matrix_storage.h:1595 coo2bcsr.  Block-element-major data: element k of block i at
// data[k * aligned + i], aligned = aligned_length(#blocks, alignment), zero padded.
int csp_coo2bcsr(coo_matrix_if* s, bcsr_matrix_if* d, unsigned bw, unsigned bh, int alignment)
{
    int rc = check_coo(s);
    if (rc || !d) return rc ? rc : set_error(CSP_EINVAL, "null BCSR");
    if (bw == 0 || bh == 0) return set_error(CSP_EINVAL, "coo2bcsr: zero block size");
    if ((rc = ensure_sorted(s))) return rc;
    d->matinfo = s->matinfo;
    d->bcsr_bwidth = bw;
    d->bcsr_bheight = bh;
    BlockRows b;
    build_blocks(s, bw, bh, b);
    const int nb = (int)b.colid.size();
    const unsigned bs = bw * bh;
    const int al = csp_aligned_length(nb, alignment);
    d->bcsr_row_num = (int)b.rowptr.size() - 1;
    d->bcsr_aligned_size = al;
    d->bcsr_block_num = nb;
    d->bcsr_row_ptr = xmalloc<int>(b.rowptr.size());
    d->bcsr_col_id = xmalloc<int>(nb);
    d->bcsr_data = xcalloc<float>((size_t)al * bs);
    if (!d->bcsr_row_ptr || !d->bcsr_col_id || !d->bcsr_data) return set_error(CSP_ENOMEM, "coo2bcsr");
    memcpy(d->bcsr_row_ptr, b.rowptr.data(), b.rowptr.size() * sizeof(int));
    memcpy(d->bcsr_col_id, b.colid.data(), (size_t)nb * sizeof(int));
    for (int i = 0; i < nb; i++)
        for (unsigned k = 0; k < bs; k++) d->bcsr_data[(size_t)k * al + i] = b.data[(size_t)i * bs + k];
    return CSP_OK;
}

// matrix_storage.h:1546 bcsr2coo.
int csp_bcsr2coo(const bcsr_matrix_if* s, coo_matrix_if* d)
{
    if (!s || !d) return set_error(CSP_EINVAL, "null matrix");
    const int nnz = s->matinfo.nnz;
    const unsigned bw = s->bcsr_bwidth, bh = s->bcsr_bheight, bs = bw * bh;
    d->matinfo = s->matinfo;
    d->coo_row_id = xmalloc<int>(nnz);
    d->coo_col_id = xmalloc<int>(nnz);
    d->coo_data = xmalloc<float>(nnz);
    if (!d->coo_row_id || !d->coo_col_id || !d->coo_data) return set_error(CSP_ENOMEM, "bcsr2coo");
    int n = 0;
    for (int i = 0; i < s->bcsr_row_num; i++)
        for (unsigned k = 0; k < bs; k++)
            for (int j = s->bcsr_row_ptr[i]; j < s->bcsr_row_ptr[i + 1]; j++) {
                const float v = s->bcsr_data[j + (size_t)k * s->bcsr_aligned_size];
                if (v == 0.0f) continue;
                if (n >= nnz) return set_error(CSP_EFORMAT, "bcsr2coo: more nonzeros than matinfo.nnz");
                d->coo_row_id[n] = i * (int)bh + (int)(k / bw);
                d->coo_col_id[n] = s->bcsr_col_id[j] + (int)(k % bw);
                d->coo_data[n] = v;
                n++;
            }
    if (!quicksort_coo(d->coo_row_id, d->coo_col_id, d->coo_data, n))
        return set_error(CSP_EFORMAT, "bcsr2coo: sort failed");
    return CSP_OK;
}

// matrix_storage.h:1941 coo2bell (generic block ELL built from coo2bcsr).  Column ids
// [slot * height_aligned + block_row]; data [slot * (height_aligned * bs) + k *
// height_aligned + block_row]; short block rows repeat their last block column with
// zero blocks.  bell_float4_aligned is left as the caller initialised it, as in the
// reference.
int csp_coo2bell(coo_matrix_if* s, bell_matrix_if* d, unsigned bw, unsigned bh, int alignment, int ellnum)
{
    if (!d) return set_error(CSP_EINVAL, "null BELL");
    bcsr_matrix_if b;
    csp_init_bcsr_matrix(&b);
    int rc = csp_coo2bcsr(s, &b, bw, bh, alignment);
    if (rc) { csp_free_bcsr_matrix(&b); return rc; }
    d->matinfo = s->matinfo;
    d->bell_bwidth = bw;
    d->bell_bheight = bh;
    int maxw = 0;
    for (int i = 0; i < b.bcsr_row_num; i++) maxw = std::max(maxw, b.bcsr_row_ptr[i + 1] - b.bcsr_row_ptr[i]);
    if (ellnum == 0) ellnum = maxw;
    if (ellnum < maxw) { csp_free_bcsr_matrix(&b); return set_error(CSP_EINVAL, "coo2bell: ellnum below the widest block row"); }
    const unsigned bs = bw * bh;
    const int hal = csp_aligned_length(b.bcsr_row_num, alignment);
    d->bell_block_num = ellnum;
    d->bell_row_num = b.bcsr_row_num;
    d->bell_height_aligned = hal;
    const size_t slots = (size_t)hal * ellnum;
    d->bell_col_id = xcalloc<int>(slots);
    d->bell_data = xcalloc<float>(slots * bs);
    if (!d->bell_col_id || !d->bell_data) { csp_free_bcsr_matrix(&b); return set_error(CSP_ENOMEM, "coo2bell"); }
    const size_t colsize = (size_t)hal * bs;
    for (int i = 0; i < b.bcsr_row_num; i++) {
        int last = 0, k = 0;
        for (int j = b.bcsr_row_ptr[i]; j < b.bcsr_row_ptr[i + 1]; j++, k++) {
            d->bell_col_id[i + (size_t)k * hal] = last = b.bcsr_col_id[j];
            for (unsigned e = 0; e < bs; e++)
                d->bell_data[i + (size_t)e * hal + (size_t)k * colsize] = b.bcsr_data[j + (size_t)e * b.bcsr_aligned_size];
        }
        for (; k < ellnum; k++) d->bell_col_id[i + (size_t)k * hal] = last;
    }
    csp_free_bcsr_matrix(&b);
    return CSP_OK;
}

// matrix_storage.h:1901 bell2coo.
int csp_bell2coo(const bell_matrix_if* s, coo_matrix_if* d)
{
    if (!s || !d) return set_error(CSP_EINVAL, "null matrix");
    const int nnz = s->matinfo.nnz, hal = s->bell_height_aligned;
    const unsigned bw = s->bell_bwidth, bh = s->bell_bheight, bs = bw * bh;
    d->matinfo = s->matinfo;
    d->coo_row_id = xmalloc<int>(nnz);
    d->coo_col_id = xmalloc<int>(nnz);
    d->coo_data = xmalloc<float>(nnz);
    if (!d->coo_row_id || !d->coo_col_id || !d->coo_data) return set_error(CSP_ENOMEM, "bell2coo");
    const size_t colsize = (size_t)hal * bs;
    int n = 0;
    for (int i = 0; i < s->bell_block_num; i++)
        for (int j = 0; j < s->bell_row_num; j++)
            for (unsigned k = 0; k < bs; k++) {
                const float v = s->bell_data[j + (size_t)k * hal + (size_t)i * colsize];
                if (v == 0.0f) continue;
                if (n >= nnz) return set_error(CSP_EFORMAT, "bell2coo: more nonzeros than matinfo.nnz");
                d->coo_row_id[n] = j * (int)bh + (int)(k / bw);
                d->coo_col_id[n] = s->bell_col_id[(size_t)i * hal + j] + (int)(k % bw);
                d->coo_data[n] = v;
                n++;
            }
    return ensure_sorted(d);
}

// matrix_storage.h:1741 coo2b4csr: BCSR with bwidth in {4, 8}; column ids in float4
// units; data [w4 * (al * bh) + h * al + blk * 4 + w], al = aligned_length(4 * #blocks).
int csp_coo2b4csr(coo_matrix_if* s, b4csr_matrix_if* d, unsigned bw, unsigned bh, int alignment)
{
    int rc = check_coo(s);
    if (rc || !d) return rc ? rc : set_error(CSP_EINVAL, "null B4CSR");
    if (bw == 0 || bw % 4 != 0 || bh == 0) return set_error(CSP_EINVAL, "coo2b4csr: bwidth must be a multiple of 4");
    if ((rc = ensure_sorted(s))) return rc;
    d->matinfo = s->matinfo;
    d->b4csr_bwidth = bw;
    d->b4csr_bheight = bh;
    BlockRows b;
    build_blocks(s, bw, bh, b);
    const long long nb = (long long)b.colid.size();
    if (nb > kMaxMemObj / (long long)(bw * bh * sizeof(float)))
        return set_error(CSP_EFORMAT, "coo2b4csr: %lld blocks exceed the memory-object limit", nb);
    return write_b4csr(b, bw, bh, alignment, d);
}

// matrix_storage.h:2010 coo2b4ell: block ELL in the b4 layout.  Column ids (float4
// units) [slot * height_aligned + block_row]; data [slot * (f4al * bw4 * bh) + h * f4al
// + w4 * (f4al * bh) + block_row * 4 + w], f4al = aligned_length(4 * #block rows).
int csp_coo2b4ell(coo_matrix_if* s, b4ell_matrix_if* d, unsigned bw, unsigned bh, int alignment, int ellnum)
{
    int rc = check_coo(s);
    if (rc || !d) return rc ? rc : set_error(CSP_EINVAL, "null B4ELL");
    if (bw == 0 || bw % 4 != 0 || bh == 0) return set_error(CSP_EINVAL, "coo2b4ell: bwidth must be a multiple of 4");
    if ((rc = ensure_sorted(s))) return rc;
    d->matinfo = s->matinfo;
    d->b4ell_bwidth = bw;
    d->b4ell_bheight = bh;
    BlockRows b;
    build_blocks(s, bw, bh, b);
    const int nbr = (int)b.rowptr.size() - 1;
    int maxw = 0;
    for (int i = 0; i < nbr; i++) maxw = std::max(maxw, b.rowptr[i + 1] - b.rowptr[i]);
    if (ellnum == 0) ellnum = maxw;
    if (ellnum < maxw) return set_error(CSP_EINVAL, "coo2b4ell: ellnum below the widest block row");
    if ((long long)nbr * ellnum > kMaxMemObj / (long long)(bw * bh * sizeof(float)))
        return set_error(CSP_EFORMAT, "coo2b4ell: exceeds the memory-object limit");
    return write_b4ell(b, bw, bh, alignment, ellnum, d);
}

// matrix_storage.h:2203 coo2sbell: sliced b4 block ELL, slices of `sh` block rows, slice
// width = widest block row in the slice.  Column ids [slice_ptr[s] + row_in_slice + slot
// * sh]; data [slice_ptr[s] * bs + slot * (sh * bw4 * bh * 4) + h * (sh * 4) + w4 * (sh *
// bh * 4) + row_in_slice * 4 + w].  Padding repeats the last block column, zero data.
int csp_coo2sbell(coo_matrix_if* s, sbell_matrix_if* d, unsigned bw, unsigned bh, unsigned sh)
{
    int rc = check_coo(s);
    if (rc || !d) return rc ? rc : set_error(CSP_EINVAL, "null SBELL");
    if (bw == 0 || bw % 4 != 0 || bh == 0 || sh == 0) return set_error(CSP_EINVAL, "coo2sbell: bad block or slice size");
    if ((rc = ensure_sorted(s))) return rc;
    d->matinfo = s->matinfo;
    d->sbell_bwidth = bw;
    d->sbell_bheight = bh;
    BlockRows b;
    build_blocks(s, bw, bh, b);
    const int nbr = (int)b.rowptr.size() - 1;
    const int H = (int)sh;
    const int nslices = nbr / H + (nbr % H != 0);
    d->sbell_slice_num = nslices;
    d->sbell_row_num = nbr;
    d->sbell_slice_height = sh;
    std::vector<int> width((size_t)nslices);
    long long total = 0;
    for (int i = 0; i < nslices; i++) {
        int w = 0;
        for (int r = i * H; r < (i + 1) * H && r < nbr; r++) w = std::max(w, b.rowptr[r + 1] - b.rowptr[r]);
        width[i] = w;
        total += (long long)w * H;
    }
    if (total > kMaxMemObj / (long long)(bw * bh * sizeof(float)))
        return set_error(CSP_EFORMAT, "coo2sbell: exceeds the memory-object limit");
    return write_sbell(b, bw, bh, sh, width, d);
}

// util.cpp:273 rearrange_bell_4col: a generic BELL whose block width is a multiple of 4
// rewritten in place into the float4 layout of the b4 kernels.  Element (h, w) of the
// block in ELL slot i of block row j moves from
//   data[i * hal * bw * bh + h * hal * bw + w * hal + j]            (hal = bell_height_aligned)
// to
//   data[i * f4 * w4 * bh + h * f4 + (w / 4) * f4 * bh + 4 * j + w % 4]
// with f4 = bell_float4_aligned = align(4 * row_num, alignment) and w4 = bw / 4; the
// column ids become float4 ids (divided by 4).  The slots between 4 * row_num and f4
// are zero here; the reference leaves them uninitialized.
int csp_rearrange_bell_4col(bell_matrix_if* m, int alignment)
{
    if (!m || alignment <= 0) return set_error(CSP_EINVAL, "rearrange_bell_4col: bad argument");
    const int bw = (int)m->bell_bwidth, bh = (int)m->bell_bheight;
    if (bw <= 0 || bw % 4 != 0) return set_error(CSP_EINVAL, "rearrange_bell_4col: block width %d is not a multiple of 4", bw);
    const int ellnum = m->bell_block_num, rows = m->bell_row_num, hal = m->bell_height_aligned;
    const int w4 = bw / 4;
    const int f4 = csp_aligned_length(4 * rows, alignment);
    const size_t n = (size_t)f4 * bh * w4 * ellnum;
    float* nd = xcalloc<float>(std::max<size_t>(n, 1));
    if (!nd) return set_error(CSP_ENOMEM, "rearrange_bell_4col");
    const size_t col_old = (size_t)hal * bw * bh, h_old = (size_t)hal * bw;
    const size_t col_new = (size_t)f4 * w4 * bh, w4_new = (size_t)f4 * bh;
    for (int i = 0; i < ellnum; i++)
        for (int h = 0; h < bh; h++)
            for (int w = 0; w < bw; w++)
                for (int j = 0; j < rows; j++)
                    nd[i * col_new + (size_t)h * f4 + (size_t)(w / 4) * w4_new + (size_t)j * 4 + w % 4] =
                        m->bell_data[i * col_old + (size_t)h * h_old + (size_t)w * hal + j];
    free(m->bell_data);
    m->bell_data = nd;
    m->bell_float4_aligned = f4;
    for (size_t i = 0; i < (size_t)hal * ellnum; i++) m->bell_col_id[i] /= 4;
    return CSP_OK;
}

// util.cpp:31 pad_csr: every row padded to a multiple of `alignment` with the row's last
// column id and value 0.  (An empty first row reads before the array in the reference;
// here padding of an empty row is simply empty, which is what findPaddedSize(0) asks.)
int csp_pad_csr(const csr_matrix_if* s, csr_matrix_if* d, int alignment)
{
    if (!s || !d || alignment <= 0) return set_error(CSP_EINVAL, "pad_csr: bad argument");
    const int h = s->matinfo.height;
    d->matinfo.height = h;
    d->matinfo.width = s->matinfo.width;
    d->csr_row_ptr = xmalloc<int>((size_t)h + 1);
    if (!d->csr_row_ptr) return set_error(CSP_ENOMEM, "pad_csr");
    d->csr_row_ptr[0] = 0;
    long long total = 0;
    for (int r = 0; r < h; r++) {
        total += csp_aligned_length(s->csr_row_ptr[r + 1] - s->csr_row_ptr[r], alignment);
        if (total > INT32_MAX) return set_error(CSP_EFORMAT, "pad_csr: padded size exceeds int32");
        d->csr_row_ptr[r + 1] = (int)total;
    }
    d->matinfo.nnz = (int)total;
    d->csr_col_id = xmalloc<int>((size_t)total);
    d->csr_data = xmalloc<float>((size_t)total);
    if (!d->csr_col_id || !d->csr_data) return set_error(CSP_ENOMEM, "pad_csr");
    int last = 0;
    for (int r = 0; r < h; r++) {
        int o = d->csr_row_ptr[r];
        for (int j = s->csr_row_ptr[r]; j < s->csr_row_ptr[r + 1]; j++, o++) {
            d->csr_col_id[o] = last = s->csr_col_id[j];
            d->csr_data[o] = s->csr_data[j];
        }
        for (; o < d->csr_row_ptr[r + 1]; o++) {
            d->csr_col_id[o] = last;
            d->csr_data[o] = 0.0f;
        }
    }
    return CSP_OK;
}

// ---------------------------------------------------------------------------------
// init_ / free_  (matrix_storage.h:371-651; analyze.h:146-206)
// ---------------------------------------------------------------------------------
void csp_init_coo_matrix(coo_matrix_if* m) { memset(m, 0, sizeof(*m)); }
void csp_init_csr_matrix(csr_matrix_if* m) { memset(m, 0, sizeof(*m)); }
void csp_init_ell_matrix(ell_matrix_if* m) { memset(m, 0, sizeof(*m)); }
void csp_init_sell_matrix(sell_matrix_if* m) { memset(m, 0, sizeof(*m)); }
void csp_init_dia_matrix(dia_matrix_iif* m) { memset(m, 0, sizeof(*m)); }
void csp_init_bdia_matrix(bdia_matrix_iif* m) { memset(m, 0, sizeof(*m)); }
void csp_init_bcsr_matrix(bcsr_matrix_if* m) { memset(m, 0, sizeof(*m)); }
void csp_init_bell_matrix(bell_matrix_if* m) { memset(m, 0, sizeof(*m)); }
void csp_init_b4csr_matrix(b4csr_matrix_if* m) { memset(m, 0, sizeof(*m)); }
void csp_init_b4ell_matrix(b4ell_matrix_if* m) { memset(m, 0, sizeof(*m)); }
void csp_init_sbell_matrix(sbell_matrix_if* m) { memset(m, 0, sizeof(*m)); }
void csp_init_cocktail(cocktail_iif* m) { memset(m, 0, sizeof(*m)); }

#define CSP_FREE(p) do { free(p); (p) = nullptr; } while (0)
void csp_free_coo_matrix(coo_matrix_if* m) { if (!m) return; CSP_FREE(m->coo_row_id); CSP_FREE(m->coo_col_id); CSP_FREE(m->coo_data); }
void csp_free_csr_matrix(csr_matrix_if* m) { if (!m) return; CSP_FREE(m->csr_row_ptr); CSP_FREE(m->csr_col_id); CSP_FREE(m->csr_data); }
void csp_free_ell_matrix(ell_matrix_if* m) { if (!m) return; CSP_FREE(m->ell_col_id); CSP_FREE(m->ell_data); }
void csp_free_sell_matrix(sell_matrix_if* m) { if (!m) return; CSP_FREE(m->sell_slice_ptr); CSP_FREE(m->sell_col_id); CSP_FREE(m->sell_data); }
void csp_free_dia_matrix(dia_matrix_iif* m) { if (!m) return; CSP_FREE(m->dia_offsets); CSP_FREE(m->dia_data); }
void csp_free_bdia_matrix(bdia_matrix_iif* m) { if (!m) return; CSP_FREE(m->bdia_offsets); CSP_FREE(m->bdia_bptr); CSP_FREE(m->bdia_data); }
void csp_free_bcsr_matrix(bcsr_matrix_if* m) { if (!m) return; CSP_FREE(m->bcsr_row_ptr); CSP_FREE(m->bcsr_col_id); CSP_FREE(m->bcsr_data); }
void csp_free_bell_matrix(bell_matrix_if* m) { if (!m) return; CSP_FREE(m->bell_col_id); CSP_FREE(m->bell_data); }
void csp_free_b4csr_matrix(b4csr_matrix_if* m) { if (!m) return; CSP_FREE(m->b4csr_row_ptr); CSP_FREE(m->b4csr_col_id); CSP_FREE(m->b4csr_data); }
void csp_free_b4ell_matrix(b4ell_matrix_if* m) { if (!m) return; CSP_FREE(m->b4ell_col_id); CSP_FREE(m->b4ell_data); }
void csp_free_sbell_matrix(sbell_matrix_if* m) { if (!m) return; CSP_FREE(m->sbell_slice_ptr); CSP_FREE(m->sbell_col_id); CSP_FREE(m->sbell_data); }

void csp_free_cocktail(cocktail_iif* m)
{
    if (!m) return;
    m->ifusebdia = m->ifusedia = m->ifusesbell = m->ifusebell = m->ifusebcsr = false;
    m->ifusesell = m->ifuseell = m->ifusecsr = m->ifusecoo = false;
    csp_free_bdia_matrix(&m->bdia);
    csp_free_dia_matrix(&m->dia);
    csp_free_sbell_matrix(&m->sbell);
    csp_free_b4ell_matrix(&m->bell);
    csp_free_b4csr_matrix(&m->bcsr);
    csp_free_sell_matrix(&m->sell);
    csp_free_ell_matrix(&m->ell);
    csp_free_csr_matrix(&m->csr);
    csp_free_coo_matrix(&m->coo);
}

}  // extern "C"
