// spmv_all: the single-format benchmark command of clSpMV (clSpMV_NV/src/spmv_all.cpp:158),
// on this library.  Usage and method numbers are the reference's:
//   spmv_all matrix.mtx method [ntimes]
//   0 bandwidth/launch overhead, 1 csr scalar, 2 csr vector, 3 bdia, 4 dia, 5 ell,
//   6 coo, 7 bell, 8 bcsr, 9 sell, 10 sbell
#include <stdio.h>
#include <stdlib.h>

#include "csp/clspmv.h"

static const char* kNames[11] = {"bandwidth", "csr scalar", "csr vector", "bdia", "dia", "ell",
                                 "coo", "bell", "bcsr", "sell", "sbell"};

int main(int argc, char** argv)
{
    if (argc < 2) {
        printf("\nUsage: spmv_all input_matrix.mtx method execution_times");
        printf("\nThe matrix needs to be in the matrix market format");
        printf("\nMethod 0: memory bandwidth and kernel launch overhead only");
        printf("\nMethods 1-10: csr scalar, csr vector, bdia, dia, ell, coo, bell, bcsr, sell, sbell\n");
        return 0;
    }
    const int choice = argc > 2 ? atoi(argv[2]) : 1;
    const int ntimes = argc > 3 ? atoi(argv[3]) : 20;
    if (choice < 0 || choice > 10) {
        fprintf(stderr, "unknown method %d\n", choice);
        return 2;
    }
    if (choice == 0) {
        csp_bandwidth_report b;
        int rc = csp_bandwidth_test((size_t)256 << 20, 1 << 20, &b);
        if (rc) { fprintf(stderr, "%s: %s\n", csp_error_string(rc), csp_last_error()); return 1; }
        printf("launch overhead %.2f us  copy %.1f GB/s  random gather %.1f GB/s (%.2f G elements/s)\n",
               b.launch_us, b.copy_gbs, b.gather_gbs, b.gather_per_s / 1e9);
        return 0;
    }
    coo_matrix_if coo;
    csp_init_coo_matrix(&coo);
    int rc = csp_read_mmf(argv[1], &coo);
    if (rc) { fprintf(stderr, "%s: %s\n", csp_error_string(rc), csp_last_error()); return 1; }
    printf("MatInfo: Width %d Height %d NNZ %d\n", coo.matinfo.width, coo.matinfo.height, coo.matinfo.nnz);
    csp_report r;
    rc = csp_spmv_all(&coo, choice, ntimes, &r);
    if (rc) { fprintf(stderr, "%s: %s\n", csp_error_string(rc), csp_last_error()); csp_free_coo_matrix(&coo); return 1; }
    printf("%s: best variant %d  %.4f ms  %.2f GFLOPS  %.1f GB/s\n", kNames[choice], r.method, r.ms, r.gflops, r.gbytes);
    printf("Correctness Check: Distance %e max diff %e max diff ratio %e vec size %d\n", r.l2_distance, r.max_diff,
           r.max_ratio_diff, coo.matinfo.height);
    csp_free_coo_matrix(&coo);
    return 0;
}
