// spmv_cocktail: the Cocktail evaluation command of clSpMV (clSpMV_NV/src/eval.cpp:93),
// on this library:  spmv_cocktail matrix.mtx
// Reads the matrix, sets x = 1 and y = 0, computes the serial COO product as the
// reference result (eval.cpp:79 spmv_only), partitions the matrix -- with the clSpMV
// calibration tables when $CLSPMVPATH is set (the reference's own decisions), else with
// the on-device autotuner -- then checks and times the Cocktail SpMV (csp_evaluate).
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <vector>

#include "csp/clspmv.h"

int main(int argc, char** argv)
{
    if (argc < 2) {
        printf("\nUsage: spmv_cocktail input_matrix.mtx");
        printf("\nThe matrix needs to be in the matrix market format\n");
        return 0;
    }
    coo_matrix_if coo;
    csp_init_coo_matrix(&coo);
    int rc = csp_read_mmf(argv[1], &coo);
    if (rc) { fprintf(stderr, "%s: %s\n", csp_error_string(rc), csp_last_error()); return 1; }
    const int h = coo.matinfo.height, w = coo.matinfo.width;
    printf("MatInfo: Width %d Height %d NNZ %d\n", w, h, coo.matinfo.nnz);
    std::vector<float> vec((size_t)w, 1.0f), res((size_t)h, 0.0f), coores((size_t)h, 0.0f);
    for (int i = 0; i < coo.matinfo.nnz; i++) coores[coo.coo_row_id[i]] += coo.coo_data[i] * vec[coo.coo_col_id[i]];
    cocktail_iif mat;
    csp_init_cocktail(&mat);
    csp_analyze_opts opts;
    memset(&opts, 0, sizeof(opts));
    opts.mode = getenv("CLSPMVPATH") ? CSP_ANALYZE_REFERENCE : CSP_ANALYZE_AUTOTUNE;
    rc = csp_analyze_matrix(&coo, &mat, &opts);
    if (rc) { fprintf(stderr, "%s: %s\n", csp_error_string(rc), csp_last_error()); csp_free_coo_matrix(&coo); return 1; }
    printf("Partition (%s):", opts.mode == CSP_ANALYZE_REFERENCE ? "reference tables" : "autotuned");
    if (mat.ifusebdia) printf(" bdia[%d] nnz %d", mat.bdia_meth_num, mat.bdia.matinfo.nnz);
    if (mat.ifusedia) printf(" dia[%d] nnz %d", mat.dia_meth_num, mat.dia.matinfo.nnz);
    if (mat.ifusesbell) printf(" sbell %ux%u nnz %d", mat.sbell.sbell_bheight, mat.sbell.sbell_bwidth, mat.sbell.matinfo.nnz);
    if (mat.ifusebell) printf(" bell %ux%u nnz %d", mat.bell.b4ell_bheight, mat.bell.b4ell_bwidth, mat.bell.matinfo.nnz);
    if (mat.ifusebcsr) printf(" bcsr %ux%u nnz %d", mat.bcsr.b4csr_bheight, mat.bcsr.b4csr_bwidth, mat.bcsr.matinfo.nnz);
    if (mat.ifusesell) printf(" sell[%d] nnz %d", mat.sell_meth_num, mat.sell.matinfo.nnz);
    if (mat.ifuseell) printf(" ell[%d] nnz %d", mat.ell_meth_num, mat.ell.matinfo.nnz);
    if (mat.ifusecsr) printf(" csr[%d] nnz %d", mat.csr_meth_num, mat.csr.matinfo.nnz);
    if (mat.ifusecoo) printf(" coo nnz %d", mat.coo.matinfo.nnz);
    printf("\n");
    csp_report r;
    rc = csp_evaluate(&mat, vec.data(), res.data(), coores.data(), 1000, &r);
    if (rc) { fprintf(stderr, "%s: %s\n", csp_error_string(rc), csp_last_error()); return 1; }
    printf("Correctness Check: Distance %e max diff %e max diff ratio %e vec size %d\n", r.l2_distance, r.max_diff,
           r.max_ratio_diff, h);
    printf("Cocktail time %lf ms GFLOPS %lf (%.1f GB/s)\n", r.ms, r.gflops, r.gbytes);
    csp_free_cocktail(&mat);
    csp_free_coo_matrix(&coo);
    return 0;
}
