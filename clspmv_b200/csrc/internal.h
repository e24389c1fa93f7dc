// Internal helpers shared by the host translation units of libclspmv_b200.
#pragma once

#include <stdarg.h>
#include <vector>
#include "csp/clspmv.h"

namespace csp {

// Records a detail message for csp_last_error() on the calling thread and returns `code`.
int set_error(int code, const char* fmt, ...);
void clear_error();

int check_coo(const coo_matrix_if* m);

// Blocks of a matrix in the reference's construction order (matrix_storage.h:1631-1697):
// per block row, entries sorted by (col, row), one block per distinct col - col % bw.
struct BlockRows {
    std::vector<int> rowptr;   // per block row
    std::vector<int> colid;    // block column (original column units)
    std::vector<float> data;   // bw*bh values per block, row-major
};
void build_blocks(const coo_matrix_if* s, unsigned bw, unsigned bh, BlockRows& out);
int write_b4csr(const BlockRows& b, unsigned bw, unsigned bh, int alignment, b4csr_matrix_if* d);
int write_b4ell(const BlockRows& b, unsigned bw, unsigned bh, int alignment, int ellnum, b4ell_matrix_if* d);
int write_sbell(const BlockRows& b, unsigned bw, unsigned bh, unsigned sh, const std::vector<int>& width,
                sbell_matrix_if* d);
bool quicksort_coo(int* row, int* col, float* val, int n);
bool coo_is_sorted(const coo_matrix_if* m);
int autotune_partition(coo_matrix_if* coo, cocktail_iif* out, const csp_analyze_opts* opts);

// The analyzer's counting passes on the current device (analyze_device.cu).
struct BlockCounts { int partial_blocks, partial_nnz, full_blocks, full_nnz; };
int device_count_dia(const int* row, const int* col, int nnz, int threshold, std::vector<int>& count);
int device_count_blocks(const int* rp, const int* col, int h, int nnz, const int* bh, const int* bw, const int* threshold,
                        int nshapes, std::vector<std::vector<BlockCounts>>& out);
int ensure_sorted(coo_matrix_if* m);
// The banding step of coo2bdia on a built DIA (consumed: its data moves into d).
int bdia_from_dia(dia_matrix_iif* dia, bdia_matrix_iif* d);
// true when a row-sorted COO holds two entries at one (row, col) position
bool coo_has_duplicates(const coo_matrix_if* m);

}  // namespace csp
