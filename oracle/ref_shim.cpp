// Test infrastructure only: this file is never linked into the product library.
//
// C-linkage entry points into the reference clSpMV host code, compiled from the
// reference sources where they lie (see oracle/Makefile).  The tests call these
// through ctypes to pin the oracle and to check the product's conversions and
// partitioning byte for byte.  Every argument struct is the reference template
// itself; the product's C structs (include/csp/clspmv.h) share its layout.
//
// Wrapped reference functions (clSpMV_NV/...):
//   include/matrix_storage.h : sort_coo :745, if_sorted_coo :732, coo2csr :1269,
//       coo2ell :1341, coo2sell :1398, coo2dia :937, coo2bdia :1185,
//       coo2bcsr :1595, coo2bell :1941, coo2b4csr :1741, coo2b4ell :2010,
//       coo2sbell :2203, dia2coo :826, bdia2coo :1137,
//       ell2coo :1310, bcsr2coo :1546, bell2coo :1901
//   include/spmv_serial.h    : {dia,bdia,ell,sell,sbell,coo,csr,bcsr,bell}_spmv :12-279
//   src/util.cpp             : pad_csr :31, rearrange_bell_4col :273
//   src/analyze.cpp          : analyze_matrix :3704
//   src/fileio.cpp           : ReadMMF :10
// csr2coo (matrix_storage.h:1239) is not wrapped: instantiating it fails to compile
// (it passes a csr_matrix to if_sorted_coo/sort_coo, :1241-1244).
#include <stdio.h>
#include <unistd.h>
#include <fcntl.h>
#include "matrix_storage.h"
#include "spmv_serial.h"
#include "analyze.h"
#include "util.h"
#include "fileio.h"

typedef coo_matrix<int, float> COO;
typedef csr_matrix<int, float> CSR;

extern "C" {

int ref_if_sorted_coo(COO* m) { return if_sorted_coo<int, float>(m) ? 1 : 0; }
int ref_sort_coo(COO* m) { return sort_coo<int, float>(m) ? 1 : 0; }
void ref_coo2csr(COO* s, CSR* d) { coo2csr<int, float>(s, d); }
void ref_coo2ell(COO* s, ell_matrix<int, float>* d, int alignment, int ellnum) { coo2ell<int, float>(s, d, alignment, ellnum); }
void ref_ell2coo(ell_matrix<int, float>* s, COO* d) { ell2coo<int, float>(s, d); }
void ref_coo2sell(COO* s, sell_matrix<int, float>* d, unsigned int sh) { coo2sell<int, float>(s, d, sh); }
int ref_coo2dia(COO* s, dia_matrix<int, int, float>* d, int alignment) { return coo2dia<int, int, float>(s, d, alignment) ? 1 : 0; }
void ref_dia2coo(dia_matrix<int, int, float>* s, COO* d) { dia2coo<int, int, float>(s, d); }
int ref_coo2bdia(COO* s, bdia_matrix<int, int, float>* d, int alignment) { return coo2bdia<int, int, float>(s, d, alignment) ? 1 : 0; }
void ref_bdia2coo(bdia_matrix<int, int, float>* s, COO* d) { bdia2coo<int, int, float>(s, d); }
void ref_coo2bcsr(COO* s, bcsr_matrix<int, float>* d, unsigned int bw, unsigned int bh, int alignment) { coo2bcsr<int, float>(s, d, bw, bh, alignment); }
void ref_bcsr2coo(bcsr_matrix<int, float>* s, COO* d) { bcsr2coo<int, float>(s, d); }
void ref_coo2bell(COO* s, bell_matrix<int, float>* d, unsigned int bw, unsigned int bh, int alignment, int ellnum) { coo2bell<int, float>(s, d, bw, bh, alignment, ellnum); }
void ref_bell2coo(bell_matrix<int, float>* s, COO* d) { bell2coo<int, float>(s, d); }
int ref_coo2b4csr(COO* s, b4csr_matrix<int, float>* d, unsigned int bw, unsigned int bh, int alignment) { return coo2b4csr<int, float>(s, d, bw, bh, alignment) ? 1 : 0; }
int ref_coo2b4ell(COO* s, b4ell_matrix<int, float>* d, unsigned int bw, unsigned int bh, int alignment, int ellnum) { return coo2b4ell<int, float>(s, d, bw, bh, alignment, ellnum) ? 1 : 0; }
int ref_coo2sbell(COO* s, sbell_matrix<int, float>* d, unsigned int bw, unsigned int bh, unsigned int sh) { return coo2sbell<int, float>(s, d, bw, bh, sh) ? 1 : 0; }
void ref_pad_csr(CSR* s, CSR* d, int alignment) { pad_csr(s, d, alignment); }
void ref_rearrange_bell_4col(bell_matrix<int, float>* m, int alignment) { rearrange_bell_4col(m, alignment); }

void ref_dia_spmv(dia_matrix<int, int, float>* m, float* v, float* r, int n) { dia_spmv<int, int, float>(m, v, r, n); }
void ref_bdia_spmv(bdia_matrix<int, int, float>* m, float* v, float* r, int n) { bdia_spmv<int, int, float>(m, v, r, n); }
void ref_ell_spmv(ell_matrix<int, float>* m, float* v, float* r, int n) { ell_spmv<int, float>(m, v, r, n); }
void ref_sell_spmv(sell_matrix<int, float>* m, float* v, float* r, int n) { sell_spmv<int, float>(m, v, r, n); }
void ref_sbell_spmv(sbell_matrix<int, float>* m, float* v, float* r, int n) { sbell_spmv<int, float>(m, v, r, n); }
void ref_coo_spmv(COO* m, float* v, float* r, int n) { coo_spmv<int, float>(m, v, r, n); }
void ref_csr_spmv(CSR* m, float* v, float* r, int n) { csr_spmv<int, float>(m, v, r, n); }
void ref_bcsr_spmv(bcsr_matrix<int, float>* m, float* v, float* r, int n) { bcsr_spmv<int, float>(m, v, r, n); }
void ref_bell_spmv(bell_matrix<int, float>* m, float* v, float* r, int n) { bell_spmv<int, float>(m, v, r, n); }

// The reference analyzer prints progress to stdout; `quiet` sends it to /dev/null.
void ref_analyze_matrix(COO* coo, cocktail<int, int, float>* mat, int quiet)
{
    int saved = -1;
    if (quiet) {
        fflush(stdout);
        saved = dup(1);
        int devnull = open("/dev/null", O_WRONLY);
        dup2(devnull, 1);
        close(devnull);
    }
    init_cocktail<int, int, float>(*mat);
    analyze_matrix(*coo, *mat);
    if (quiet) {
        fflush(stdout);
        dup2(saved, 1);
        close(saved);
    }
}

void ref_free_cocktail(cocktail<int, int, float>* mat) { free_cocktail<int, int, float>(*mat); }
void ref_read_mmf(char* filename, COO* mat) { ReadMMF(filename, mat); }

// Frees any array the reference malloc()ed (the tests hand back every pointer).
void ref_free(void* p) { free(p); }

}  // extern "C"
