// The Cocktail analyzer: partitions a COO matrix into diagonal (BDIA/DIA), block
// (SBELL/BELL/BCSR) and flat (SELL/ELL/CSR/COO) sub-matrices and picks a kernel
// variant for each, the role of clSpMV_NV/src/analyze.cpp (analyze_matrix :3704).
//
// CSP_ANALYZE_REFERENCE reproduces the reference's partition bit for bit: the same
// calibration tables ($CLSPMVPATH/benchmark/*.ben, read like ReadBench :177), the
// same bilinear GFLOPS predictions (find_fourid :294, linear_inter :401), the same
// cost comparisons evaluated in the same precision and operation order, and the
// same extraction rules, including the reference's quirks (e.g. extract_partial_block
// hands a zero block threshold to the SBELL/BELL extraction, :2711).  The shared
// prediction state (maxflop_info, analyze.h:208) is mutated across the phases exactly
// as the reference mutates it, because later decisions read fields set by earlier
// ones.  The implementation is this library's own: block counting, diagonal lookup
// and remainder bookkeeping use hash maps and direct indexing instead of the
// reference's std::map and linear searches, which changes the cost on large
// matrices but not the outcome.
//
// CSP_ANALYZE_AUTOTUNE does not use the tables: it hands the matrix to the on-device
// autotuner (autotune.cu), which times candidate partitions on the GPU.  Tables
// measured on the B200 by csp_benchmark_tables (calibrate.cu) can still drive the
// reference partitioner through CSP_ANALYZE_REFERENCE and a table path.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <algorithm>
#include <functional>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#include "csp/clspmv.h"
#include "internal.h"

namespace csp {
namespace ana {

using std::pair;
using std::vector;

// clSpMV_NV/include/constant.h
constexpr int kAlign = 32;          // GPU_ALIGNMENT
constexpr int kWarp = 32;           // WARPSIZE
constexpr int kWorkGroup = 256;     // WORK_GROUP_SIZE
constexpr int kCsrVecGroup = 128;   // CSR_VEC_GROUP_SIZE
constexpr int kBellGroup = 256;     // BELL_GROUP_SIZE
constexpr int kSellGroup = 128;     // SELL_GROUP_SIZE
constexpr int kCooGroup = 256;      // COO_GROUP_SIZE
constexpr int kMaxDiaNum = 128;     // MAX_DIA_NUM
constexpr int kBdiaImp = 5, kDiaImp = 4, kSbellImp = 1, kBellImp = 2, kBcsrImp = 1;
constexpr int kSellImp = 2, kEllImp = 2, kCsrImp = 2, kCooImp = 1;
const int kBh[8] = {1, 2, 4, 8, 1, 2, 4, 8};
const int kBw[8] = {4, 4, 4, 4, 8, 8, 8, 8};

// ---------------------------------------------------------------------------
// calibration tables (analyze.h:12-103)
// ---------------------------------------------------------------------------
struct Ov { unsigned groupnum, threadnum; double us; };
struct Row2 { unsigned dim, width; double g[5]; };                 // bdia/dia/sell/ell
struct RowB { unsigned bh, bw, dim, blocknum; double g[2]; };      // sbell/bell/bcsr
struct RowG { unsigned dim, width, groupnum; double g[2]; };       // csr/coo
struct Basic { unsigned dim, width; };

struct Tables {
    vector<Ov> overhead;
    vector<Row2> bdia, dia, sell, ell;
    vector<RowB> sbell, bell, bcsr;
    vector<RowG> csr, coo;
};

// Whitespace-separated numbers of one table file; records of `ni` integers then `nd`
// doubles, read until the data runs out (the reference's fscanf loops, :16-175).
static int read_table(const std::string& dir, const char* name, int ni, int nd,
                      const std::function<void(const long*, const double*)>& push)
{
    const std::string path = dir + "/benchmark/" + name;
    FILE* f = fopen(path.c_str(), "r");
    if (!f) return set_error(CSP_EIO, "cannot open calibration table %s", path.c_str());
    long iv[4];
    double dv[5];
    while (true) {
        int got = 0;
        for (int i = 0; i < ni; i++) got += fscanf(f, "%ld", iv + i) == 1;
        if (got < ni) break;
        for (int i = 0; i < nd; i++) {
            dv[i] = 0.0;
            if (fscanf(f, "%lf", dv + i) != 1) break;
        }
        push(iv, dv);
    }
    fclose(f);
    return CSP_OK;
}

static int read_tables(const std::string& dir, Tables& t)
{
    int rc;
    if ((rc = read_table(dir, "overhead.ben", 2, 1, [&](const long* i, const double* d) {
             t.overhead.push_back(Ov{(unsigned)i[0], (unsigned)i[1], d[0]}); })))
        return rc;
    auto diag = [&](vector<Row2>& v, int nd) {
        return [&v, nd](const long* i, const double* d) {
            Row2 r{(unsigned)i[0], (unsigned)i[1], {0, 0, 0, 0, 0}};
            for (int k = 0; k < nd; k++) r.g[k] = d[k];
            v.push_back(r);
        };
    };
    auto blk = [&](vector<RowB>& v, int nd) {
        return [&v, nd](const long* i, const double* d) {
            RowB r{(unsigned)i[0], (unsigned)i[1], (unsigned)i[2], (unsigned)i[3], {0, 0}};
            for (int k = 0; k < nd; k++) r.g[k] = d[k];
            v.push_back(r);
        };
    };
    auto grp = [&](vector<RowG>& v, int nd) {
        return [&v, nd](const long* i, const double* d) {
            RowG r{(unsigned)i[0], (unsigned)i[1], (unsigned)i[2], {0, 0}};
            for (int k = 0; k < nd; k++) r.g[k] = d[k];
            v.push_back(r);
        };
    };
    if ((rc = read_table(dir, "bdia.ben", 2, kBdiaImp, diag(t.bdia, kBdiaImp))) ||
        (rc = read_table(dir, "dia.ben", 2, kDiaImp, diag(t.dia, kDiaImp))) ||
        (rc = read_table(dir, "sbell.ben", 4, kSbellImp, blk(t.sbell, kSbellImp))) ||
        (rc = read_table(dir, "bell.ben", 4, kBellImp, blk(t.bell, kBellImp))) ||
        (rc = read_table(dir, "bcsr.ben", 4, kBcsrImp, blk(t.bcsr, kBcsrImp))) ||
        (rc = read_table(dir, "sell.ben", 2, kSellImp, diag(t.sell, kSellImp))) ||
        (rc = read_table(dir, "ell.ben", 2, kEllImp, diag(t.ell, kEllImp))) ||
        (rc = read_table(dir, "csr.ben", 3, kCsrImp, grp(t.csr, kCsrImp))) ||
        (rc = read_table(dir, "coo.ben", 3, kCooImp, grp(t.coo, kCooImp))))
        return rc;
    if (t.overhead.empty() || t.bdia.empty() || t.dia.empty() || t.sbell.empty() || t.bell.empty() || t.bcsr.empty() ||
        t.sell.empty() || t.ell.empty() || t.csr.empty() || t.coo.empty())
        return set_error(CSP_EIO, "a calibration table under %s/benchmark is empty", dir.c_str());
    return CSP_OK;
}

// ---------------------------------------------------------------------------
// predictions
// ---------------------------------------------------------------------------
struct Four { int ss, sl, ls, ll; };

// The two table dimensions bracketing `dim` and, within each, the two widths bracketing
// `width` (find_fourid :294).  Comparisons against the unsigned table fields are
// unsigned, as in the reference.
static Four find_four(const vector<Basic>& b, int dim, int width)
{
    vector<int> dims, off;
    dims.push_back((int)b[0].dim);
    off.push_back(0);
    for (size_t i = 0; i < b.size(); i++)
        if ((int)b[i].dim != dims.back()) { dims.push_back((int)b[i].dim); off.push_back((int)i); }
    off.push_back((int)b.size());
    int ds = 0, dl = 0;
    const int nd = (int)dims.size();
    if (dim < dims[0]) ds = dl = 0;
    else if (dim > dims[nd - 1]) ds = dl = nd - 1;
    else {
        for (int i = 0; i < nd; i++) {
            if (dim == dims[i]) { ds = dl = i; break; }
            if (i < nd - 1 && dims[i] < dim && dims[i + 1] > dim) { ds = i; dl = i + 1; break; }
        }
    }
    auto within = [&](int d, int& lo, int& hi) {
        const unsigned w = (unsigned)width;
        lo = hi = off[d];
        if (w < b[off[d]].width) { lo = hi = off[d]; return; }
        if (w > b[off[d + 1] - 1].width) { lo = hi = off[d + 1] - 1; return; }
        for (int i = off[d]; i < off[d + 1]; i++) {
            if (w == b[i].width) { lo = hi = i; break; }
            if (i < off[d + 1] - 1 && b[i].width < w && b[i + 1].width > w) { lo = i; hi = i + 1; }
        }
    };
    Four f;
    within(ds, f.ss, f.sl);
    within(dl, f.ls, f.ll);
    return f;
}

// linear_inter :401
static inline double lin(int small, double sv, int large, double lv, int index)
{
    if (small == large) return lv;
    return sv + ((double)(index - small)) * (lv - sv) / ((double)(large - small));
}

// maxflop_info (analyze.h:208-250)
struct Info {
    int bdia_meth = 0; double bdia_max = 0;
    int dia_meth = 0; double dia_max = 0;
    int sbell_meth[8] = {}; double sbell_max[8] = {};
    int bell_meth[8] = {}; double bell_max[8] = {};
    int bcsr_meth[8] = {}; double bcsr_max[8] = {};
    int sell_meth = 0; double sell_max = 0;
    int ell_meth = 0; double ell_max = 0;
    int csr_meth = 0, csr_group = 0; double csr_max = 0;
    int coo_meth = 0, coo_group = 0; double coo_max = 0;
    double max_dia_base = 0, max_block_base = 0, max_flat_base = 0;
};

// (int)((float)a / (float)b + 0.5): a float quotient rounded in double (:1313 ...)
static inline int per_row(int nnz, int rows) { return (int)(((float)nnz) / ((float)rows) + 0.5); }

// maxflop_{bdia,dia,sell,ell} (:431-545): best method over the bilinear prediction.
static void maxflop_basic(const vector<Row2>& t, int nimp, int rownum, int npr, int& meth, double& best)
{
    vector<Basic> basic(t.size());
    for (size_t i = 0; i < t.size(); i++) basic[i] = Basic{t[i].dim, t[i].width};
    const Four x = find_four(basic, rownum, npr);
    meth = 0;
    best = 0.0f;
    for (int i = 0; i < nimp; i++) {
        const double sv = lin((int)t[x.ss].width, t[x.ss].g[i], (int)t[x.sl].width, t[x.sl].g[i], npr);
        const double lv = lin((int)t[x.ls].width, t[x.ls].g[i], (int)t[x.ll].width, t[x.ll].g[i], npr);
        const double fv = lin((int)t[x.ss].dim, sv, (int)t[x.ll].dim, lv, rownum);
        if (fv > best) { meth = i; best = fv; }
    }
}

// maxflop_{sbell,bell,bcsr} (:547-706): per block shape, over (rows, blocks per row).
static void maxflop_block(const vector<RowB>& t, int nimp, int rownum, int npr, int* meth, double* best)
{
    int off[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    int b = 1;
    for (size_t i = 0; i < t.size() && b < 8; i++)
        if ((int)t[i].bw == kBw[b] && (int)t[i].bh == kBh[b]) off[b++] = (int)i;
    off[8] = (int)t.size();
    for (b = 0; b < 8; b++) {
        const int blocknum = (int)(((double)npr) / ((double)kBw[b]) + 0.5);
        vector<Basic> basic;
        for (int i = off[b]; i < off[b + 1]; i++) basic.push_back(Basic{t[i].dim, t[i].blocknum});
        meth[b] = 0;
        best[b] = 0.0f;
        if (basic.empty()) continue;
        Four x = find_four(basic, rownum, blocknum);
        x.ss += off[b]; x.sl += off[b]; x.ls += off[b]; x.ll += off[b];
        for (int i = 0; i < nimp; i++) {
            const double sv = lin((int)t[x.ss].blocknum, t[x.ss].g[i], (int)t[x.sl].blocknum, t[x.sl].g[i], blocknum);
            const double lv = lin((int)t[x.ls].blocknum, t[x.ls].g[i], (int)t[x.ll].blocknum, t[x.ll].g[i], blocknum);
            const double fv = lin((int)t[x.ss].dim, sv, (int)t[x.ll].dim, lv, rownum);
            if (fv > best[b]) { meth[b] = i; best[b] = fv; }
        }
    }
}

// maxflop_{csr,coo} (:708-802): also the best work-group count.  The group count is
// not reset when no method beats zero, as in the reference.
static void maxflop_group(const vector<RowG>& t, int nimp, int rownum, int npr, int& meth, int& group, double& best)
{
    vector<int> off;
    unsigned pd = t[0].dim, pw = t[0].width;
    off.push_back(0);
    for (size_t i = 0; i < t.size(); i++)
        if (pd != t[i].dim || pw != t[i].width) { off.push_back((int)i); pd = t[i].dim; pw = t[i].width; }
    off.push_back((int)t.size());
    vector<Basic> basic(off.size() - 1);
    for (size_t i = 0; i + 1 < off.size(); i++) basic[i] = Basic{t[off[i]].dim, t[off[i]].width};
    const Four x = find_four(basic, rownum, npr);
    meth = 0;
    best = 0.0f;
    const int choices = off[1] - off[0];
    for (int g = 0; g < choices; g++)
        for (int i = 0; i < nimp; i++) {
            const RowG& a = t[off[x.ss] + g];
            const RowG& b = t[off[x.sl] + g];
            const RowG& c = t[off[x.ls] + g];
            const RowG& d = t[off[x.ll] + g];
            const double sv = lin((int)a.width, a.g[i], (int)b.width, b.g[i], npr);
            const double lv = lin((int)c.width, c.g[i], (int)d.width, d.g[i], npr);
            const double fv = lin((int)a.dim, sv, (int)d.dim, lv, rownum);
            if (fv > best) { meth = i; group = (int)a.groupnum; best = fv; }
        }
}

// ---------------------------------------------------------------------------
// matrices handled by the analyzer
// ---------------------------------------------------------------------------
struct Mat {
    int w = 0, h = 0;
    vector<int> r, c;
    vector<float> v;
    int nnz() const { return (int)r.size(); }
};

static void row_ptr(const Mat& m, vector<int>& rp)
{
    rp.assign((size_t)m.h + 1, 0);
    for (int x : m.r) rp[(size_t)x + 1]++;
    for (int i = 0; i < m.h; i++) rp[i + 1] += rp[i];
}

static void sort_rows(Mat& m)
{
    coo_matrix_if t;
    t.matinfo.width = m.w;
    t.matinfo.height = m.h;
    t.matinfo.nnz = m.nnz();
    t.coo_row_id = m.r.data();
    t.coo_col_id = m.c.data();
    t.coo_data = m.v.data();
    if (!coo_is_sorted(&t)) quicksort_coo(t.coo_row_id, t.coo_col_id, t.coo_data, t.matinfo.nnz);
}

template <class T>
static T* dup(const vector<T>& v)
{
    T* p = static_cast<T*>(malloc(std::max<size_t>(v.size(), 1) * sizeof(T)));
    if (p && !v.empty()) memcpy(p, v.data(), v.size() * sizeof(T));
    return p;
}

class Analyzer {
  public:
    Analyzer(const Tables& t, cocktail_iif& out, bool on_device = false) : T(t), mat(out), on_device(on_device) {}
    void run(Mat& coo);
    int device_rc = CSP_OK;   // first error of a device counting pass (CSP_ANALYZE_ON_DEVICE)

  private:
    const Tables& T;
    cocktail_iif& mat;
    bool on_device;
    Info info;

    double overhead(int groupnum, int threadnum) const;
    void update_dia(const Mat& m);
    void update_block(const Mat& m);
    void update_flat(const Mat& m);
    void flat_only(const Mat& m, Info& in) const;

    bool extract_dia(const Mat& m, Mat& rem);
    bool extract_block(const Mat& m, Mat& rem);
    void extract_flat(const Mat& m);
    void extract_coo(const Mat& m);
    void extract_csr(const Mat& m);
    void extract_csr_coo(const Mat& m);
    bool extract_sell_ell(const Mat& m, Mat& rem);
    double estimate_flat_time(const vector<int>& rownnz, int nnz) const;
    double estimate_coo_time(int nnz, const Info& in) const;
    double estimate_csr_time(const vector<int>& rownnz, const Info& in) const;
    double estimate_csr_coo_time(const vector<int>& rownnz, int nnz, Info& in) const;
    double estimate_sell_ell_time(const vector<int>& rownnz, int nnz, const Info& in, vector<int>& remain, int& nremain) const;
};

// find_overhead :413 -- launch overhead in microseconds
double Analyzer::overhead(int groupnum, int threadnum) const
{
    const vector<Ov>& o = T.overhead;
    vector<Basic> basic(o.size());
    for (size_t i = 0; i < o.size(); i++) basic[i] = Basic{o[i].groupnum, o[i].threadnum};
    const Four x = find_four(basic, groupnum, threadnum);
    const double sv = lin((int)o[x.ss].threadnum, o[x.ss].us, (int)o[x.sl].threadnum, o[x.sl].us, threadnum);
    const double lv = lin((int)o[x.ls].threadnum, o[x.ls].us, (int)o[x.ll].threadnum, o[x.ll].us, threadnum);
    return lin((int)o[x.ss].groupnum, sv, (int)o[x.ll].groupnum, lv, groupnum);
}

// update_info_dia / _block / _flat (:1311-1357)
void Analyzer::update_dia(const Mat& m)
{
    const int npr = per_row(m.nnz(), m.h);
    maxflop_basic(T.bdia, kBdiaImp, m.h, npr, info.bdia_meth, info.bdia_max);
    maxflop_basic(T.dia, kDiaImp, m.h, npr, info.dia_meth, info.dia_max);
    double b = info.bdia_max;
    if (info.dia_max > b) b = info.dia_max;
    info.max_dia_base = b;
}

void Analyzer::update_block(const Mat& m)
{
    const int npr = per_row(m.nnz(), m.h);
    maxflop_block(T.sbell, kSbellImp, m.h, npr, info.sbell_meth, info.sbell_max);
    maxflop_block(T.bell, kBellImp, m.h, npr, info.bell_meth, info.bell_max);
    maxflop_block(T.bcsr, kBcsrImp, m.h, npr, info.bcsr_meth, info.bcsr_max);
    double b = 0.0f;
    for (int i = 0; i < 8; i++) {
        if (info.sbell_max[i] > b) b = info.sbell_max[i];
        if (info.bell_max[i] > b) b = info.bell_max[i];
        if (info.bcsr_max[i] > b) b = info.bcsr_max[i];
    }
    info.max_block_base = b;
}

void Analyzer::flat_only(const Mat& m, Info& in) const
{
    const int npr = per_row(m.nnz(), m.h);
    maxflop_basic(T.sell, kSellImp, m.h, npr, in.sell_meth, in.sell_max);
    maxflop_basic(T.ell, kEllImp, m.h, npr, in.ell_meth, in.ell_max);
    maxflop_group(T.csr, kCsrImp, m.h, npr, in.csr_meth, in.csr_group, in.csr_max);
    maxflop_group(T.coo, kCooImp, m.h, npr, in.coo_meth, in.coo_group, in.coo_max);
    double b = in.sell_max;
    if (in.ell_max > b) b = in.ell_max;
    if (in.csr_max > b) b = in.csr_max;
    if (in.coo_max > b) b = in.coo_max;
    in.max_flat_base = b;
}

void Analyzer::update_flat(const Mat& m) { flat_only(m, info); }

// ---------------------------------------------------------------------------
// diagonal part (extract_dia :1365 and its helpers :804-1309)
// ---------------------------------------------------------------------------
struct BdiaVsDia { int min_width = 1000000, range_s = 0, range_l = 0; double bdia_single = 0, dia_single = 0; };

// find_min_bdia_width :828: in the table dimension nearest `dimension`, the narrowest
// band width at which BDIA beats DIA.
static BdiaVsDia min_bdia_width(const vector<Row2>& bdia, const vector<Row2>& dia, int dimension)
{
    vector<int> dims, off;
    dims.push_back((int)bdia[0].dim);
    off.push_back(0);
    for (size_t i = 0; i < bdia.size(); i++)
        if ((int)bdia[i].dim != dims.back()) { dims.push_back((int)bdia[i].dim); off.push_back((int)i); }
    off.push_back((int)bdia.size());
    const int nd = (int)dims.size();
    int ds = 0, dl = 0;
    if (dimension < dims[0]) ds = dl = 0;
    else if (dimension > dims[nd - 1]) ds = dl = nd - 1;
    else {
        for (int i = 0; i < nd; i++) {
            if (dimension == dims[i]) { ds = dl = i; break; }
            if (i < nd - 1 && dims[i] < dimension && dims[i + 1] > dimension) { ds = i; dl = i + 1; break; }
        }
    }
    int near = ds;
    if (ds != dl) {
        const int dist_s = (int)((unsigned)dimension - bdia[off[ds]].dim);
        const int dist_l = (int)(bdia[off[dl]].dim - (unsigned)dimension);
        near = (dist_s < dist_l) ? ds : dl;
    }
    BdiaVsDia r;
    r.range_s = off[near];
    r.range_l = off[near + 1];
    for (int i = off[near]; i < off[near + 1]; i++) {
        const int width = (int)bdia[i].width;
        double mb = 0.0f, md = 0.0f;
        for (int j = 0; j < kBdiaImp; j++) if (bdia[i].g[j] > mb) mb = bdia[i].g[j];
        for (int j = 0; j < kDiaImp; j++) if (dia[i].g[j] > md) md = dia[i].g[j];
        if (width == 1) { r.bdia_single = mb; r.dia_single = md; }
        if (mb > md) { r.min_width = width; return r; }
    }
    r.min_width = 1000000;
    return r;
}

// bdia_gflop / dia_gflop :898-967: best method at the band count within the range.
static void diag_gflop(const vector<Row2>& t, int nimp, int rs, int rl, int width, double& best, int& meth)
{
    int idx = 0;
    const unsigned w = (unsigned)width;
    if (w < t[rs].width) idx = rs;
    else if (w > t[rl - 1].width) idx = rl - 1;
    else {
        for (int i = rs; i < rl; i++) {
            if (w == t[i].width) { idx = i; break; }
            if (i < rl - 1 && t[i].width < w && t[i + 1].width > w) { idx = i; break; }
        }
    }
    best = 0.0f;
    meth = 0;
    for (int i = 0; i < nimp; i++)
        if (t[idx].g[i] > best) { best = t[idx].g[i]; meth = i; }
}

static void band_runs(const vector<int>& off, vector<int>& start, vector<int>& count)
{
    start.clear();
    count.clear();
    for (size_t i = 0; i < off.size(); i++) {
        if (i > 0 && off[i] - off[i - 1] == 1) count.back()++;
        else { start.push_back(off[i]); count.push_back(1); }
    }
}

bool Analyzer::extract_dia(const Mat& m, Mat& rem)
{
    if (m.nnz() == 0) return false;
    update_dia(m);
    update_flat(m);
    const double margin = 1.05;
    const double ratio = info.max_flat_base / info.max_dia_base;
    const int least = (int)(ratio * (double)m.h * margin);
    if (least > m.h) return false;
    const int threshold = m.h - least;
    vector<int> count((size_t)2 * threshold + 1, 0);
    if (on_device && !device_rc) {
        device_rc = device_count_dia(m.r.data(), m.c.data(), m.nnz(), threshold, count);
    } else {
        for (int i = 0; i < m.nnz(); i++) {
            const int o = m.c[i] - m.r[i] + threshold;
            if (o >= 0 && o < (int)count.size()) count[o]++;
        }
    }
    vector<pair<int, int>> valid;
    for (int i = 0; i < (int)count.size(); i++)
        if (count[i] > least) valid.push_back(pair<int, int>(count[i], i));
    std::sort(valid.begin(), valid.end(), std::greater<pair<int, int>>());
    double ov = overhead(m.h / kWorkGroup, kWorkGroup);
    ov /= 1000.0;
    int cur = 0, dia_num = 0;
    double best = 1000000.0f;
    for (int i = 0; i <= kMaxDiaNum && i <= (int)valid.size(); i++) {
        if (i > 0) cur += valid[i - 1].first;
        const int left = m.nnz() - cur;
        double t = ((double)i) * ((double)m.h) / 1000000.0 / info.max_dia_base + ((double)left) / 1000000.0 / info.max_flat_base;
        if (i > 0) t += ov;
        if (left > 0) t += ov;
        if (t < best) { best = t; dia_num = i; }
    }
    if (dia_num == 0) return false;
    vector<pair<int, int>> sel;   // (table index, count)
    for (int i = 0; i < dia_num; i++) sel.push_back(pair<int, int>(valid[i].second, valid[i].first));
    std::sort(sel.begin(), sel.end());
    const BdiaVsDia bv = min_bdia_width(T.bdia, T.dia, m.h);
    const int least_band = bv.min_width;
    int band_num = 0, width = 1;
    for (size_t i = 1; i < sel.size(); i++) {
        if (sel[i].first == sel[i - 1].first + 1) width++;
        else {
            if (width >= least_band) band_num += width;
            width = 1;
        }
        if (i == sel.size() - 1 && width >= least_band) band_num += width;
    }
    const int remain_dia = dia_num - band_num;
    double bdia_partial = 0.0001f, dia_partial = 0.0001f, dia_all = 0.0001f;
    int bdia_partial_meth = 0, dia_partial_meth = 0, dia_all_meth = 0;
    if (band_num > 0) diag_gflop(T.bdia, kBdiaImp, bv.range_s, bv.range_l, band_num, bdia_partial, bdia_partial_meth);
    if (remain_dia > 0) diag_gflop(T.dia, kDiaImp, bv.range_s, bv.range_l, remain_dia, dia_partial, dia_partial_meth);
    diag_gflop(T.dia, kDiaImp, bv.range_s, bv.range_l, dia_num, dia_all, dia_all_meth);
    const double h = (double)m.h;
    const double bdia_only = ((double)band_num * h) / 1000000.0 / bdia_partial +
                             ((double)remain_dia * h) / 1000000.0 / (dia_partial * bv.bdia_single / bv.dia_single) + ov;
    const double dia_only = ((double)dia_num * h) / 1000000.0 / dia_all + ov;
    const double both = ((double)band_num * h) / 1000000.0 / bdia_partial + ((double)remain_dia * h) / 1000000.0 / dia_partial + 2 * ov;

    // diagonal offsets of the selection, ascending
    vector<int> off(sel.size());
    for (size_t i = 0; i < sel.size(); i++) off[i] = sel[i].first - threshold;
    const int len = csp_aligned_length(m.h, kAlign);
    enum { NONE = -1 };
    // slot[o + threshold] = (part, index): part 0 = DIA, 1 = BDIA
    vector<int> part((size_t)2 * threshold + 1, NONE), slot((size_t)2 * threshold + 1, 0);
    vector<int> dia_off, bdia_off;
    int dia_nnz = 0, bdia_nnz = 0;
    if (bdia_only <= dia_only && bdia_only <= both) {
        mat.ifusebdia = true;
        mat.bdia_meth_num = bdia_partial_meth;
        bdia_off = off;
        for (size_t i = 0; i < sel.size(); i++) bdia_nnz += sel[i].second;
    } else if (dia_only <= bdia_only && dia_only <= both) {
        mat.ifusedia = true;
        mat.dia_meth_num = dia_all_meth;
        dia_off = off;
        for (size_t i = 0; i < sel.size(); i++) dia_nnz += sel[i].second;
    } else {
        mat.ifusebdia = mat.ifusedia = true;
        mat.bdia_meth_num = bdia_partial_meth;
        mat.dia_meth_num = dia_partial_meth;
        vector<int> bs, bc;
        band_runs(off, bs, bc);
        size_t k = 0;
        for (size_t b = 0; b < bs.size(); b++) {
            int nz = 0;
            for (int j = 0; j < bc[b]; j++) nz += sel[k + j].second;
            vector<int>& dst = (bc[b] >= least_band) ? bdia_off : dia_off;
            (bc[b] >= least_band ? bdia_nnz : dia_nnz) += nz;
            for (int j = 0; j < bc[b]; j++) dst.push_back(bs[b] + j);
            k += bc[b];
        }
    }
    for (size_t i = 0; i < dia_off.size(); i++) { part[dia_off[i] + threshold] = 0; slot[dia_off[i] + threshold] = (int)i; }
    for (size_t i = 0; i < bdia_off.size(); i++) { part[bdia_off[i] + threshold] = 1; slot[bdia_off[i] + threshold] = (int)i; }
    float* ddata = nullptr;
    float* bdata = nullptr;
    if (mat.ifusedia) {
        dia_matrix_iif& d = mat.dia;
        d.matinfo.width = m.w;
        d.matinfo.height = m.h;
        d.matinfo.nnz = dia_nnz;
        d.dia_length = m.h;
        d.dia_length_aligned = len;
        d.dia_num = (int)dia_off.size();
        d.dia_offsets = dup(dia_off);
        d.dia_data = ddata = static_cast<float*>(calloc(std::max<size_t>(dia_off.size() * (size_t)len, 1), sizeof(float)));
    }
    if (mat.ifusebdia) {
        bdia_matrix_iif& b = mat.bdia;
        vector<int> bs, bc;
        band_runs(bdia_off, bs, bc);
        b.matinfo.width = m.w;
        b.matinfo.height = m.h;
        b.matinfo.nnz = bdia_nnz;
        b.bdia_length = m.h;
        b.bdia_length_aligned = len;
        b.bdia_band_num = (int)bs.size();
        b.bdia_offsets = dup(bs);
        vector<int> bptr(bs.size() + 1, 0);
        for (size_t i = 0; i < bs.size(); i++) bptr[i + 1] = bptr[i] + bc[i];
        b.bdia_bptr = dup(bptr);
        b.bdia_data = bdata = static_cast<float*>(calloc(std::max<size_t>(bdia_off.size() * (size_t)len, 1), sizeof(float)));
    }
    rem.w = m.w;
    rem.h = m.h;
    rem.r.clear(); rem.c.clear(); rem.v.clear();
    for (int i = 0; i < m.nnz(); i++) {
        const int o = m.c[i] - m.r[i] + threshold;
        const int p = (o >= 0 && o < (int)part.size()) ? part[o] : NONE;
        if (p == 0) ddata[(size_t)slot[o] * len + m.r[i]] = m.v[i];
        else if (p == 1) bdata[(size_t)slot[o] * len + m.r[i]] = m.v[i];
        else { rem.r.push_back(m.r[i]); rem.c.push_back(m.c[i]); rem.v.push_back(m.v[i]); }
    }
    return true;
}

// ---------------------------------------------------------------------------
// block part (extract_block :2723 and helpers :1534-2721)
// ---------------------------------------------------------------------------
struct BlockInfo { int partial_blocks = 0, partial_nnz = 0, full_blocks = 0, full_nnz = 0; };

// count_blocks :1582: per block row and shape, the number of blocks and the nonzeros
// in them, all blocks and those with more than threshold[i] entries.
static void count_blocks(const Mat& m, const vector<int>& rp, const vector<int>& threshold, vector<vector<BlockInfo>>& bc)
{
    bc.assign(8, vector<BlockInfo>());
    vector<int> cols;
    for (int s = 0; s < 8; s++) {
        const int bh = kBh[s], bw = kBw[s];
        const int nbr = m.h / bh + (m.h % bh != 0);
        bc[s].assign(nbr, BlockInfo());
        for (int br = 0; br < nbr; br++) {
            const int r0 = br * bh, r1 = std::min(r0 + bh, m.h);
            cols.clear();
            for (int j = rp[r0]; j < rp[r1]; j++) cols.push_back(m.c[j] / bw);
            std::sort(cols.begin(), cols.end());
            BlockInfo& bi = bc[s][br];
            for (size_t j = 0; j < cols.size();) {
                size_t k = j;
                while (k < cols.size() && cols[k] == cols[j]) k++;
                const int cnt = (int)(k - j);
                bi.full_blocks++;
                bi.full_nnz += cnt;
                if (cnt > threshold[s]) { bi.partial_blocks++; bi.partial_nnz += cnt; }
                j = k;
            }
        }
    }
}

// The reference's block peel (extract_{sbell,bell,bcsr}_part :1660-2261): per block row,
// entries sorted by (col, row); each block is kept if accept(entries, index within the
// row) holds, else its entries go to the remainder in block order; the remainder is
// then sorted by (row, col).
template <class Accept>
static void peel_blocks(const Mat& m, const vector<int>& rp, int bw, int bh, Accept accept, BlockRows& out, Mat& rem)
{
    const int nbr = m.h / bh + (m.h % bh != 0);
    const unsigned bs = (unsigned)(bw * bh);
    out.rowptr.assign((size_t)nbr + 1, 0);
    out.colid.clear();
    out.data.clear();
    rem.w = m.w;
    rem.h = m.h;
    rem.r.clear(); rem.c.clear(); rem.v.clear();
    struct E { int rowid, colid; float data; };
    vector<E> el;
    for (int br = 0; br < nbr; br++) {
        const int r0 = br * bh;
        const int start = rp[r0], end = (r0 + bh <= m.h) ? rp[r0 + bh] : rp[m.h];
        int blocknum = 0;
        if (end > start) {
            el.resize((size_t)(end - start));
            for (int i = start; i < end; i++) el[i - start] = E{m.r[i], m.c[i], m.v[i]};
            std::sort(el.begin(), el.end(), [](const E& a, const E& b) {
                if (a.colid != b.colid) return a.colid < b.colid;
                return a.rowid < b.rowid;
            });
            size_t e = 0;
            while (e < el.size()) {
                const int bcol = el[e].colid - el[e].colid % bw;
                size_t f = e;
                while (f < el.size() && el[f].colid - el[f].colid % bw == bcol) f++;
                blocknum++;
                if (accept((int)(f - e), blocknum, br)) {
                    const size_t base = out.data.size();
                    out.data.resize(base + bs, 0.0f);
                    for (size_t k = e; k < f; k++)
                        out.data[base + (unsigned)(el[k].rowid % bh) * bw + (unsigned)(el[k].colid - bcol)] = el[k].data;
                    out.colid.push_back(bcol);
                } else {
                    for (size_t k = e; k < f; k++) { rem.r.push_back(el[k].rowid); rem.c.push_back(el[k].colid); rem.v.push_back(el[k].data); }
                    blocknum--;
                }
                e = f;
            }
        }
        out.rowptr[br + 1] = out.rowptr[br] + blocknum;
    }
    sort_rows(rem);
}

bool Analyzer::extract_block(const Mat& m, Mat& rem)
{
    if (m.nnz() == 0) return false;
    update_block(m);
    update_flat(m);
    vector<int> rp;
    row_ptr(m, rp);
    // find_thre_max_flop :1558
    vector<int> threshold(8, 0);
    vector<double> best_block(8, 0.0f);
    for (int i = 0; i < 8; i++) {
        if (info.sbell_max[i] > best_block[i]) best_block[i] = info.sbell_max[i];
        if (info.bell_max[i] > best_block[i]) best_block[i] = info.bell_max[i];
        if (info.bcsr_max[i] > best_block[i]) best_block[i] = info.bcsr_max[i];
    }
    for (int i = 0; i < 8; i++) {
        threshold[i] = (int)((double)kBh[i] * (double)kBw[i] * info.max_flat_base / best_block[i]);
        if (threshold[i] > kBh[i] * kBw[i] - 1) threshold[i] = kBh[i] * kBw[i] - 1;
    }
    vector<vector<BlockInfo>> bc;
    if (on_device && !device_rc) {
        vector<vector<BlockCounts>> dc;
        device_rc = device_count_blocks(rp.data(), m.c.data(), m.h, m.nnz(), kBh, kBw, threshold.data(), 8, dc);
        bc.assign(8, vector<BlockInfo>());
        for (int s = 0; s < 8 && !device_rc; s++) {
            bc[s].resize(dc[s].size());
            for (size_t j = 0; j < dc[s].size(); j++) {
                bc[s][j].partial_blocks = dc[s][j].partial_blocks;
                bc[s][j].partial_nnz = dc[s][j].partial_nnz;
                bc[s][j].full_blocks = dc[s][j].full_blocks;
                bc[s][j].full_nnz = dc[s][j].full_nnz;
            }
        }
    } else {
        count_blocks(m, rp, threshold, bc);
    }
    vector<double> block_over(8, 0.0f);
    for (int i = 0; i < 8; i++) {
        block_over[i] = overhead(m.h / (kBh[i] * kSellGroup), kSellGroup);
        block_over[i] /= 1000.0;
    }
    double flatover = overhead(m.h / kWorkGroup, kWorkGroup);
    flatover /= 1000.0;
    vector<BlockInfo> sum(8);
    for (int i = 0; i < 8; i++)
        for (const BlockInfo& b : bc[i]) {
            sum[i].partial_blocks += b.partial_blocks;
            sum[i].partial_nnz += b.partial_nnz;
            sum[i].full_blocks += b.full_blocks;
            sum[i].full_nnz += b.full_nnz;
        }
    double best_full = 1000000.0f, best_partial = 1000000.0f;
    int full_id = 0, partial_id = 0;
    for (int i = 0; i < 8; i++) {
        const double ft = ((double)sum[i].full_blocks) * ((double)kBh[i]) * ((double)kBw[i]) / 1000000.0 / best_block[i] + block_over[i];
        if (ft < best_full) { best_full = ft; full_id = i; }
        vector<int> rownnz((size_t)m.h, 0);
        int flatnnz = 0;
        for (int j = 0; j < (int)bc[i].size(); j++) {
            const int diff = bc[i][j].full_nnz - bc[i][j].partial_nnz;
            const int rs = j * kBh[i];
            const int re = std::min((j + 1) * kBh[i], m.h);
            const int n = re - rs;
            const int avg = diff / n;
            for (int k = rs; k < re - 1; k++) rownnz[k] = avg;
            rownnz[re - 1] = diff - avg * (n - 1);
            flatnnz += diff;
        }
        double pt = ((double)sum[i].partial_blocks) * ((double)kBh[i]) * ((double)kBw[i]) / 1000000.0 / best_block[i] + block_over[i];
        pt += estimate_flat_time(rownnz, flatnnz);
        if (pt < best_partial) { best_partial = pt; partial_id = i; }
    }
    double fullflat = ((double)m.nnz()) / 1000000.0 / info.max_flat_base + flatover;
    fullflat *= 1.02;   // favour blocks: flat must win by more than 2 %
    if (fullflat <= best_full && fullflat <= best_partial) return false;

    const bool full = best_full <= best_partial;
    const int w = full ? full_id : partial_id;
    const int bw = kBw[w], bh = kBh[w];
    const BlockInfo& s = sum[w];
    // extract_full_block :2676 / extract_partial_block :2699
    if (info.bcsr_max[w] >= info.sbell_max[w] && info.bcsr_max[w] >= info.bell_max[w]) {
        // extract_bcsr_part :2113 (full: threshold 0, every block)
        const int thr = full ? 0 : threshold[w];
        mat.ifusebcsr = true;
        mat.bcsr_meth_num = info.bcsr_meth[w];
        BlockRows b;
        peel_blocks(m, rp, bw, bh, [thr](int n, int, int) { return n > thr; }, b, rem);
        write_b4csr(b, (unsigned)bw, (unsigned)bh, kAlign, &mat.bcsr);
        mat.bcsr.matinfo.width = m.w;
        mat.bcsr.matinfo.height = m.h;
        mat.bcsr.matinfo.nnz = full ? s.full_nnz : s.partial_nnz;
        return true;
    }
    // per block row (blocks, nonzeros) of the chosen kind
    vector<pair<int, int>> cnt(bc[w].size());
    for (size_t i = 0; i < bc[w].size(); i++)
        cnt[i] = full ? pair<int, int>(bc[w][i].full_blocks, bc[w][i].full_nnz)
                      : pair<int, int>(bc[w][i].partial_blocks, bc[w][i].partial_nnz);
    const pair<int, int> tot = full ? pair<int, int>(s.full_blocks, s.full_nnz) : pair<int, int>(s.partial_blocks, s.partial_nnz);
    const int npr = per_row(tot.second, m.h);
    maxflop_block(T.sbell, kSbellImp, m.h, npr, info.sbell_meth, info.sbell_max);
    maxflop_block(T.bell, kBellImp, m.h, npr, info.bell_meth, info.bell_max);
    int maxblk = 0;
    for (const auto& c : cnt) maxblk = std::max(maxblk, c.first);
    int brownum = m.h / bh + (m.h % bh != 0);
    const int bw4 = bw / 4;
    const int newlength = csp_aligned_length(4 * brownum, kAlign);
    double bell_ov = overhead(brownum / kBellGroup, kBellGroup);
    bell_ov /= 1000.0;
    const double avgnnz = ((double)tot.second / (double)tot.first);
    const int sh = kWarp;
    const int nslices = brownum / sh + (brownum % sh != 0);
    vector<int> slice_full(nslices, 0), slice_partial(nslices, 0);
    int bell_num = 0;
    bool use_bell = false;
    vector<int>* sbell_width = &slice_full;
    if (full) {
        // extract_full_sbell_bell :2435
        const double bell_time = ((double)maxblk * (double)newlength * (double)bh * (double)bw4) / 1000000.0 / info.bell_max[w] + bell_ov;
        for (int i = 0; i < nslices; i++) {
            int mx = 0;
            for (int j = i * sh; j < (i + 1) * sh && j < (int)cnt.size(); j++) mx = std::max(mx, cnt[j].first);
            slice_full[i] = mx;
        }
        double sbell_ov = overhead(brownum / kSellGroup, kSellGroup);
        sbell_ov /= 1000.0;
        int sbell_full = 0;
        for (int x : slice_full) sbell_full += sh * x;
        const double full_time = ((double)(sbell_full * bw * bh)) / 1000000.0 / info.sbell_max[w] + sbell_ov;
        use_bell = bell_time < full_time;
        bell_num = maxblk;
    } else {
        // extract_sbell_bell :2521
        const double remain_flop = info.max_flat_base;
        double remain_ov = overhead(m.h / kWorkGroup, kWorkGroup);
        remain_ov /= 1000.0;
        vector<int> hist((size_t)maxblk + 1, 0);
        for (const auto& c : cnt) hist[c.first]++;
        int bellnnz = 0, rows_left = brownum;
        double best = 1000000.0;
        for (int i = 0; i < (int)hist.size(); i++) {
            rows_left -= hist[i];
            double t = 0.0f;
            if (i > 0) t += ((double)i * (double)newlength * (double)bh * (double)bw4) / 1000000.0 / info.bell_max[w] + bell_ov;
            if (bellnnz < m.nnz()) t += ((double)(m.nnz() - bellnnz)) / 1000000.0 / remain_flop + remain_ov;
            if (t < best) { best = t; bell_num = i; }
            bellnnz += (int)((double)rows_left * avgnnz);
        }
        int partial_nnz = 0;
        const int full_nnz = tot.second;
        for (int i = 0; i < nslices; i++) {
            vector<int> sw;
            for (int j = i * sh; j < (i + 1) * sh && j < (int)cnt.size(); j++) sw.push_back(cnt[j].first);
            std::sort(sw.begin(), sw.end());
            slice_full[i] = sw.back();
            int pn = (int)((double)sw[0] * (double)sw.size() * avgnnz);
            int curn = pn;
            slice_partial[i] = sw[0];
            for (size_t j = 1; j < sw.size(); j++) {
                pn += (int)((double)(sw[j] - sw[j - 1]) * (double)(sw.size() - j) * avgnnz);
                const double ratio = remain_flop / info.sbell_max[w];
                if (pn > (int)(((double)(sw.size() * (size_t)sw[j] * (size_t)bw * (size_t)bh)) * ratio)) {
                    slice_partial[i] = sw[j];
                    curn = pn;
                } else {
                    break;
                }
            }
            partial_nnz += curn;
        }
        double sbell_ov = overhead(brownum / kSellGroup, kSellGroup);
        sbell_ov /= 1000.0;
        int sb_full = 0, sb_partial = 0;
        for (int x : slice_full) sb_full += sh * x;
        for (int x : slice_partial) sb_partial += sh * x;
        const double full_time = ((double)(sb_full * bw * bh)) / 1000000.0 / info.sbell_max[w] + sbell_ov +
                                 ((double)(m.nnz() - full_nnz)) / 1000000.0 / remain_flop + remain_ov;
        const double partial_time = ((double)(sb_partial * bw * bh)) / 1000000.0 / info.sbell_max[w] + sbell_ov +
                                    ((double)(m.nnz() - partial_nnz)) / 1000000.0 / remain_flop + remain_ov;
        if (best < full_time && best < partial_time) use_bell = true;
        else if (partial_time < full_time) sbell_width = &slice_partial;
    }
    // the SBELL/BELL extraction keeps every block (threshold 0) up to the chosen widths
    if (use_bell) {
        if (bell_num == 0) {   // extract_bell_part :1899: nothing kept
            rem = m;
            return true;
        }
        mat.ifusebell = true;
        mat.bell_meth_num = info.bell_meth[w];
        BlockRows b;
        const int limit = bell_num;
        peel_blocks(m, rp, bw, bh, [limit](int n, int k, int) { return n > 0 && k <= limit; }, b, rem);
        write_b4ell(b, (unsigned)bw, (unsigned)bh, kAlign, bell_num, &mat.bell);
        mat.bell.matinfo.width = m.w;
        mat.bell.matinfo.height = m.h;
        mat.bell.matinfo.nnz = m.nnz() - rem.nnz();
        return true;
    }
    mat.ifusesbell = true;
    mat.sbell_meth_num = info.sbell_meth[w];
    BlockRows b;
    const vector<int>& widths = *sbell_width;
    peel_blocks(m, rp, bw, bh, [&widths, sh](int n, int k, int br) { return n > 0 && k <= widths[br / sh]; }, b, rem);
    write_sbell(b, (unsigned)bw, (unsigned)bh, (unsigned)sh, widths, &mat.sbell);
    mat.sbell.matinfo.width = m.w;
    mat.sbell.matinfo.height = m.h;
    mat.sbell.matinfo.nnz = m.nnz() - rem.nnz();
    return true;
}

// ---------------------------------------------------------------------------
// flat part (:2836-3701)
// ---------------------------------------------------------------------------
double Analyzer::estimate_coo_time(int nnz, const Info& in) const
{
    if (nnz == 0) return 0.0f;
    double ov = overhead(in.coo_group, kCooGroup);
    ov /= 1000.0;
    return ((double)nnz) / 1000000.0 / in.coo_max + ov;
}

// Work of the busiest CSR work group under the chosen kernel (estimate_csr_time :2880,
// the same distribution as extract_csr_coo :3003-3041).
static int csr_busiest(const vector<int>& rownnz, int meth, int groups)
{
    vector<int> per(groups, 0);
    const int n = (int)rownnz.size();
    if (meth == 0) {
        const int height = kCsrVecGroup / kWarp;
        const int warps = groups * height;
        int iters = n / warps;
        if (n % warps != 0) iters++;
        for (int i = 0; i < iters; i++)
            for (int g = 0; g < groups; g++)
                for (int j = 0; j < height; j++) {
                    const long long id = (long long)i * warps + g * height + j;
                    if (id >= n) break;
                    per[g] += rownnz[id];
                }
    } else if (meth == 1) {
        for (int i = 0; (long long)i * groups < n; i++)
            for (int g = 0; g < groups; g++) {
                const long long id = (long long)i * groups + g;
                if (id >= n) break;
                per[g] += rownnz[id];
            }
    }
    int mx = 0;
    for (int g = 0; g < groups; g++) mx = std::max(mx, per[g]);
    return mx;
}

double Analyzer::estimate_csr_time(const vector<int>& rownnz, const Info& in) const
{
    const int newnnz = csr_busiest(rownnz, in.csr_meth, in.csr_group) * in.csr_group;
    double ov = overhead(in.csr_group, kCsrVecGroup);
    ov /= 1000.0;
    return ((double)newnnz) / 1000000.0 / in.csr_max + ov;
}

double Analyzer::estimate_csr_coo_time(const vector<int>& rownnz, int nnz, Info& in) const
{
    if (nnz == 0) return 0.0f;
    const int npr = per_row(nnz, (int)rownnz.size());
    maxflop_group(T.csr, kCsrImp, (int)rownnz.size(), npr, in.csr_meth, in.csr_group, in.csr_max);
    maxflop_group(T.coo, kCooImp, (int)rownnz.size(), npr, in.coo_meth, in.coo_group, in.coo_max);
    if (in.coo_max >= in.csr_max) return estimate_coo_time(nnz, in);
    const double ct = estimate_coo_time(nnz, in);
    const double rt = estimate_csr_time(rownnz, in);
    return ct < rt ? ct : rt;
}

// Shared by extract_sell_ell :3441 and estimate_sell_ell_time :3238: the best ELL width
// (over the row-length histogram) and the full/partial SELL slice widths.
struct FlatPlan {
    double ell_time = 0, sell_full_time = 0, sell_partial_time = 0;
    int ell_num = 0, ell_nnz = 0, slice_height = 0, partial_nnz = 0, full_nnz = 0;
    vector<int> slice_full, slice_partial;
};

static int slice_height_of(int sell_meth) { return sell_meth == 0 ? kWarp : (sell_meth == 1 ? kSellGroup : 0); }

static FlatPlan plan_sell_ell(const vector<int>& rownnz, int nnz, const Info& in,
                              const std::function<double(int, int)>& ovf)
{
    FlatPlan p;
    double remain_flop;
    int remain_group, remain_thread;
    if (in.csr_max > in.coo_max) { remain_flop = in.csr_max; remain_group = in.csr_group; remain_thread = kCsrVecGroup; }
    else { remain_flop = in.coo_max; remain_group = in.coo_group; remain_thread = kCooGroup; }
    double remain_ov = ovf(remain_group, remain_thread);
    remain_ov /= 1000.0;
    const int n = (int)rownnz.size();
    int maxr = 0;
    for (int x : rownnz) maxr = std::max(maxr, x);
    vector<int> hist((size_t)maxr + 1, 0);
    for (int x : rownnz) hist[x]++;
    int rownum = n, ellnnz = 0;
    double best = 1000000.0;
    double ell_ov = 0.0f;
    if (in.ell_meth == 0) ell_ov = ovf(n / kWorkGroup, kWorkGroup);
    else if (in.ell_meth == 1) ell_ov = ovf(n / (4 * kWorkGroup), kWorkGroup);
    ell_ov /= 1000.0;
    const int newlength = csp_aligned_length(n, kAlign);
    for (int i = 0; i < (int)hist.size(); i++) {
        rownum -= hist[i];
        double t = 0.0f;
        if (i > 0) t += ((double)i * (double)newlength) / 1000000.0 / in.ell_max + ell_ov;
        if (ellnnz < nnz) t += ((double)(nnz - ellnnz)) / 1000000.0 / remain_flop + remain_ov;
        if (t < best) { best = t; p.ell_num = i; p.ell_nnz = ellnnz; }
        ellnnz += rownum;
    }
    p.ell_time = best;
    const int sh = slice_height_of(in.sell_meth);
    p.slice_height = sh;
    const int nslices = n / sh + (n % sh != 0);
    p.slice_full.assign(nslices, 0);
    p.slice_partial.assign(nslices, 0);
    p.full_nnz = nnz;
    for (int i = 0; i < nslices; i++) {
        vector<int> sw;
        for (int j = i * sh; j < (i + 1) * sh && j < n; j++) sw.push_back(rownnz[j]);
        std::sort(sw.begin(), sw.end());
        p.slice_full[i] = sw.back();
        int pn = (int)((size_t)sw[0] * sw.size());
        int curn = pn;
        p.slice_partial[i] = sw[0];
        for (size_t j = 1; j < sw.size(); j++) {
            pn = (int)((size_t)pn + (size_t)(sw[j] - sw[j - 1]) * (sw.size() - j));
            const double ratio = remain_flop / in.sell_max;
            if (pn > (int)(((double)(sw.size() * (size_t)sw[j])) * ratio)) {
                p.slice_partial[i] = sw[j];
                curn = pn;
            } else {
                break;
            }
        }
        p.partial_nnz += curn;
    }
    double sell_ov = ovf(nslices, kSellGroup);
    sell_ov /= 1000.0;
    int sell_full = 0, sell_partial = 0;
    for (int x : p.slice_full) sell_full += sh * x;
    for (int x : p.slice_partial) sell_partial += sh * x;
    p.sell_full_time = ((double)sell_full) / 1000000.0 / in.sell_max + sell_ov;
    p.sell_partial_time = ((double)sell_partial) / 1000000.0 / in.sell_max + sell_ov +
                          ((double)(nnz - p.partial_nnz)) / 1000000.0 / remain_flop + remain_ov;
    return p;
}

double Analyzer::estimate_sell_ell_time(const vector<int>& rownnz, int nnz, const Info& in, vector<int>& remain, int& nremain) const
{
    nremain = 0;
    std::fill(remain.begin(), remain.end(), 0);
    if (nnz == 0) return 0.0f;
    const FlatPlan p = plan_sell_ell(rownnz, nnz, in, [this](int g, int t) { return overhead(g, t); });
    if (p.ell_time < p.sell_full_time && p.ell_time < p.sell_partial_time) {
        for (size_t i = 0; i < rownnz.size(); i++)
            if (rownnz[i] > p.ell_num) { remain[i] = rownnz[i] - p.ell_num; nremain += remain[i]; }
        return p.ell_time;
    }
    if (p.sell_partial_time < p.sell_full_time) {
        for (size_t i = 0; i < rownnz.size(); i++) {
            const int wdt = p.slice_partial[i / p.slice_height];
            if (rownnz[i] > wdt) { remain[i] = rownnz[i] - wdt; nremain += remain[i]; }
        }
        return p.sell_partial_time;
    }
    return p.sell_full_time;
}

// estimate_flat_time :3619 (a fresh prediction state, as in the reference)
double Analyzer::estimate_flat_time(const vector<int>& rownnz, int nnz) const
{
    if (nnz == 0) return 0.0f;
    Info in;
    Mat shape;
    const int npr = per_row(nnz, (int)rownnz.size());
    maxflop_basic(T.sell, kSellImp, (int)rownnz.size(), npr, in.sell_meth, in.sell_max);
    maxflop_basic(T.ell, kEllImp, (int)rownnz.size(), npr, in.ell_meth, in.ell_max);
    maxflop_group(T.csr, kCsrImp, (int)rownnz.size(), npr, in.csr_meth, in.csr_group, in.csr_max);
    maxflop_group(T.coo, kCooImp, (int)rownnz.size(), npr, in.coo_meth, in.coo_group, in.coo_max);
    double b = in.sell_max;
    if (in.ell_max > b) b = in.ell_max;
    if (in.csr_max > b) b = in.csr_max;
    if (in.coo_max > b) b = in.coo_max;
    in.max_flat_base = b;
    if (in.max_flat_base == in.coo_max) return estimate_coo_time(nnz, in);
    if (in.max_flat_base == in.csr_max) return estimate_csr_time(rownnz, in);
    vector<int> remain(rownnz.size(), 0);
    int nremain = 0;
    const double et = estimate_sell_ell_time(rownnz, nnz, in, remain, nremain);
    const double ct = estimate_csr_coo_time(remain, nremain, in);
    return et + ct;
}

// extract_coo :2846
void Analyzer::extract_coo(const Mat& m)
{
    if (m.nnz() == 0) return;
    maxflop_group(T.coo, kCooImp, m.h, per_row(m.nnz(), m.h), info.coo_meth, info.coo_group, info.coo_max);
    mat.ifusecoo = true;
    mat.coo_meth_num = info.coo_meth;
    mat.coo_group_num = info.coo_group;
    mat.coo.matinfo.height = m.h;
    mat.coo.matinfo.width = m.w;
    mat.coo.matinfo.nnz = m.nnz();
    mat.coo.coo_row_id = dup(m.r);
    mat.coo.coo_col_id = dup(m.c);
    mat.coo.coo_data = dup(m.v);
}

// extract_csr :2955
void Analyzer::extract_csr(const Mat& m)
{
    if (m.nnz() == 0) return;
    maxflop_group(T.csr, kCsrImp, m.h, per_row(m.nnz(), m.h), info.csr_meth, info.csr_group, info.csr_max);
    mat.ifusecsr = true;
    mat.csr_meth_num = info.csr_meth;
    mat.csr_group_num = info.csr_group;
    Mat s = m;
    sort_rows(s);
    vector<int> rp;
    row_ptr(s, rp);
    mat.csr.matinfo.width = m.w;
    mat.csr.matinfo.height = m.h;
    mat.csr.matinfo.nnz = m.nnz();
    mat.csr.csr_row_ptr = dup(rp);
    mat.csr.csr_col_id = dup(s.c);
    mat.csr.csr_data = dup(s.v);
}

// extract_csr_coo :2970: COO unless CSR's load-imbalance-adjusted time is lower.
void Analyzer::extract_csr_coo(const Mat& m)
{
    if (m.nnz() == 0) return;
    const int npr = per_row(m.nnz(), m.h);
    maxflop_group(T.csr, kCsrImp, m.h, npr, info.csr_meth, info.csr_group, info.csr_max);
    maxflop_group(T.coo, kCooImp, m.h, npr, info.coo_meth, info.coo_group, info.coo_max);
    if (info.coo_max >= info.csr_max) { extract_coo(m); return; }
    vector<int> cnt((size_t)m.h, 0);
    for (int x : m.r) cnt[x]++;
    double coo_ov = overhead(info.coo_group, kCooGroup);
    coo_ov /= 1000.0;
    const double coo_time = ((double)m.nnz()) / 1000000.0 / info.coo_max + coo_ov;
    const int newnnz = csr_busiest(cnt, info.csr_meth, info.csr_group) * info.csr_group;
    double csr_ov = overhead(info.csr_group, kCsrVecGroup);
    csr_ov /= 1000.0;
    const double csr_time = ((double)newnnz) / 1000000.0 / info.csr_max + csr_ov;
    if (coo_time <= csr_time) extract_coo(m);
    else extract_csr(m);
}

// extract_sell_ell :3441 (+ extract_ell :3175, extract_sell :3078).  Returns false when
// nothing was extracted (the caller then sends the whole matrix to CSR/COO).
bool Analyzer::extract_sell_ell(const Mat& m, Mat& rem)
{
    if (m.nnz() == 0) return false;
    vector<int> cnt((size_t)m.h, 0);
    for (int x : m.r) cnt[x]++;
    const FlatPlan p = plan_sell_ell(cnt, m.nnz(), info, [this](int g, int t) { return overhead(g, t); });
    vector<int> rp((size_t)m.h + 1, 0);
    for (int i = 0; i < m.h; i++) rp[i + 1] = rp[i] + cnt[i];
    rem.w = m.w;
    rem.h = m.h;
    rem.r.clear(); rem.c.clear(); rem.v.clear();
    if (p.ell_time < p.sell_full_time && p.ell_time < p.sell_partial_time) {
        const int ellnum = p.ell_num;
        if (ellnum == 0) return false;
        maxflop_basic(T.ell, kEllImp, m.h, ellnum, info.ell_meth, info.ell_max);
        mat.ifuseell = true;
        mat.ell_meth_num = info.ell_meth;
        ell_matrix_if& e = mat.ell;
        const int hal = csp_aligned_length(m.h, kAlign);
        e.matinfo.width = m.w;
        e.matinfo.height = m.h;
        e.matinfo.nnz = p.ell_nnz;
        e.ell_num = ellnum;
        e.ell_height_aligned = hal;
        e.ell_col_id = static_cast<int*>(calloc((size_t)hal * ellnum, sizeof(int)));
        e.ell_data = static_cast<float*>(calloc((size_t)hal * ellnum, sizeof(float)));
        for (int i = 0; i < m.h; i++) {
            int last = 0, k = 0;
            for (int j = rp[i]; j < rp[i + 1]; j++, k++) {
                if (k < ellnum) {
                    e.ell_col_id[i + (size_t)k * hal] = last = m.c[j];
                    e.ell_data[i + (size_t)k * hal] = m.v[j];
                } else {
                    rem.r.push_back(i); rem.c.push_back(m.c[j]); rem.v.push_back(m.v[j]);
                }
            }
            for (; k < ellnum; k++) e.ell_col_id[i + (size_t)k * hal] = last;
        }
        return true;
    }
    const bool partial = p.sell_partial_time < p.sell_full_time;
    const vector<int>& widths = partial ? p.slice_partial : p.slice_full;
    const int slice_nnz = partial ? p.partial_nnz : p.full_nnz;
    if (slice_nnz == 0) return false;
    const int sh = p.slice_height;
    mat.ifusesell = true;
    mat.sell_meth_num = info.sell_meth;
    sell_matrix_if& s = mat.sell;
    const int ns = (int)widths.size();
    s.matinfo.width = m.w;
    s.matinfo.height = m.h;
    s.matinfo.nnz = slice_nnz;
    s.sell_slice_height = (unsigned)sh;
    s.sell_slice_num = ns;
    vector<int> sp((size_t)ns + 1, 0);
    for (int i = 0; i < ns; i++) sp[i + 1] = sp[i] + widths[i] * sh;
    s.sell_slice_ptr = dup(sp);
    s.sell_col_id = static_cast<int*>(calloc(std::max(sp[ns], 1), sizeof(int)));
    s.sell_data = static_cast<float*>(calloc(std::max(sp[ns], 1), sizeof(float)));
    for (int i = 0; i < ns; i++) {
        int* col = s.sell_col_id + sp[i];
        float* val = s.sell_data + sp[i];
        const int first = i * sh;
        for (int j = first; j < first + sh; j++) {
            const int lr = j - first;
            int k = 0;
            if (j < m.h) {
                for (int q = rp[j]; q < rp[j + 1]; q++, k++) {
                    if (k < widths[i]) {
                        col[k * sh + lr] = m.c[q];
                        val[k * sh + lr] = m.v[q];
                    } else {
                        rem.r.push_back(j); rem.c.push_back(m.c[q]); rem.v.push_back(m.v[q]);
                    }
                }
            }
            for (; k < widths[i]; k++) {
                const int id = k * sh + lr;
                col[id] = (id >= sh) ? col[id - sh] : col[0];
            }
        }
    }
    return true;
}

// extract_flat :3665
void Analyzer::extract_flat(const Mat& m)
{
    if (m.nnz() == 0) return;
    update_flat(m);
    if (info.max_flat_base == info.coo_max) { extract_coo(m); return; }
    if (info.max_flat_base == info.csr_max) { extract_csr_coo(m); return; }
    Mat rem;
    if (extract_sell_ell(m, rem)) extract_csr_coo(rem);
    else extract_csr_coo(m);
}

// analyze_matrix :3704: the order of the diagonal, block and flat peels follows the
// predicted base GFLOPS of each category; DIA only for square matrices.
void Analyzer::run(Mat& coo)
{
    mat.mat_width = coo.w;
    mat.mat_height = coo.h;
    mat.mat_nnz = coo.nnz();
    update_dia(coo);
    update_block(coo);
    update_flat(coo);
    const double dia = info.max_dia_base, block = info.max_block_base, flat = info.max_flat_base;
    const bool square = coo.w == coo.h;
    Mat r1, r2;
    auto dia_then_block = [&](const Mat& m) {
        if (extract_dia(m, r1)) {
            if (extract_block(r1, r2)) extract_flat(r2);
            else extract_flat(r1);
        } else {
            if (extract_block(m, r2)) extract_flat(r2);
            else extract_flat(m);
        }
    };
    auto block_then_dia = [&](const Mat& m) {
        if (extract_block(m, r1)) {
            if (extract_dia(r1, r2)) extract_flat(r2);
            else extract_flat(r1);
        } else {
            if (extract_dia(m, r2)) extract_flat(r2);
            else extract_flat(m);
        }
    };
    auto block_only = [&](const Mat& m) {
        if (extract_block(m, r1)) extract_flat(r1);
        else extract_flat(m);
    };
    if (dia > flat) {
        if (block > flat) {
            if (dia > block) {
                if (square) dia_then_block(coo);
                else block_only(coo);
            } else {
                if (square) block_then_dia(coo);
                else block_only(coo);
            }
        } else {
            if (square) {
                if (extract_dia(coo, r1)) extract_flat(r1);
                else extract_flat(coo);
            } else {
                extract_flat(coo);
            }
        }
    } else {
        if (block > flat) block_only(coo);
        else extract_flat(coo);
    }
}

}  // namespace ana
}  // namespace csp

extern "C" int csp_analyze_matrix(coo_matrix_if* coo, cocktail_iif* mat, const csp_analyze_opts* opts)
{
    using namespace csp;
    if (!mat) return set_error(CSP_EINVAL, "null cocktail");
    int rc = check_coo(coo);
    if (rc) return rc;
    if (coo->matinfo.height == 0 || coo->matinfo.nnz == 0) {
        csp_init_cocktail(mat);
        mat->mat_width = coo->matinfo.width;
        mat->mat_height = coo->matinfo.height;
        mat->mat_nnz = coo->matinfo.nnz;
        return CSP_OK;
    }
    if (opts && opts->mode == CSP_ANALYZE_AUTOTUNE) {
        csp_init_cocktail(mat);
        return autotune_partition(coo, mat, opts);
    }
    if (opts && opts->mode != CSP_ANALYZE_REFERENCE) return set_error(CSP_EINVAL, "unknown analyze mode %d", opts->mode);
    const char* path = (opts && opts->bench_path) ? opts->bench_path : getenv("CLSPMVPATH");
    if (!path) return set_error(CSP_EINVAL, "no calibration tables: set CLSPMVPATH or csp_analyze_opts.bench_path");
    ana::Tables t;
    if ((rc = ana::read_tables(path, t))) return rc;
    if ((rc = ensure_sorted(coo))) return rc;   // the reference analyzer expects ReadMMF's sorted input
    csp_init_cocktail(mat);
    ana::Mat m;
    m.w = coo->matinfo.width;
    m.h = coo->matinfo.height;
    m.r.assign(coo->coo_row_id, coo->coo_row_id + coo->matinfo.nnz);
    m.c.assign(coo->coo_col_id, coo->coo_col_id + coo->matinfo.nnz);
    m.v.assign(coo->coo_data, coo->coo_data + coo->matinfo.nnz);
    const bool on_device = opts && (opts->flags & CSP_ANALYZE_ON_DEVICE);
    if (on_device) {
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
            return set_error(CSP_ENODEV, "CSP_ANALYZE_ON_DEVICE needs a CUDA device");
    }
    ana::Analyzer a(t, *mat, on_device);
    a.run(m);
    if (a.device_rc) {
        csp_free_cocktail(mat);
        return a.device_rc;
    }
    return CSP_OK;
}
