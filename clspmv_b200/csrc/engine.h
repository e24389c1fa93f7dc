// Device engine state shared by the engine, driver and adjoint translation units.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>
#include <string.h>
#include <map>
#include <vector>

#include "csp/clspmv.h"

namespace csp {

enum PartKind { PART_BDIA, PART_DIA, PART_SBELL, PART_BELL, PART_BCSR, PART_SELL, PART_ELL, PART_CSR, PART_COO, PART_GBCSR,
                PART_XPANEL };

// One uploaded sub-matrix and its launch parameters.
struct Part {
    PartKind kind = PART_CSR;
    int method = 0;
    int* i0 = nullptr;   // row_ptr / slice_ptr / offsets / COO rows
    int* i1 = nullptr;   // col ids / band pointers / COO cols
    int4* blocks = nullptr;     // CSR adaptive work blocks
    int4* long_rows = nullptr;  // CSR adaptive long rows {row, first slot, chunks, -}
    void* v = nullptr;   // values (FP32 or BF16)
    int* scratch_row = nullptr;   // COO span / CSR adaptive long-row arrival counters
    float* scratch_val = nullptr; // COO chunk shares of spans; CSR adaptive long-row partials
    int* span_head = nullptr;     // COO: span continued by each chunk's first row, or -1
    int4* spans = nullptr;        // COO: rows crossing chunk boundaries {row, first chunk, chunks, -}
    int m = 0;        // rows (or block rows' parent height)
    int nnz = 0;
    int k = 0;        // ELL width / #diagonals / #bands / BELL slots
    int stride = 0;   // ELL/DIA aligned height, SELL/SBELL slice height, BELL height_aligned, BCSR aligned size
    int f4 = 0;       // BELL float4_aligned
    int bw = 0, bh = 0, nbr = 0;
    int maxw = 0;     // BDIA widest band
    int group = 0;    // CSR sub-warp lanes per row
    int nblocks = 0;  // CSR adaptive row blocks
    int npad = 0, nwarps = 0;  // COO
    // x-panel layout (kernels/xpanel.cuh): i0 = run slot per entry, v = values
    unsigned short* lcol = nullptr;   // column inside the entry's panel
    int* tile0 = nullptr;             // first tile of each panel (npanels + 1)
    int* run_ptr = nullptr;           // slots of each listed row (nrun_rows + 1)
    int* run_rows = nullptr;          // listed rows: rows with entries, or null when all have some
    int* long_list = nullptr;         // listed rows with more than kXpShortRuns slots (nlong)
    float* partial = nullptr;         // one sum per run
    int ntiles = 0, npanels = 0, panel_w = 0, nrun_rows = 0, ncta = 0, nlong = 0;
    size_t smem = 0;                  // dynamic shared memory of the x-panel kernel
    bool from_csr = false;            // adjoint: value-gradient order follows the CSR part
};

// One matrix entry (row, column, value), as the adjoint builders gather them.
struct Entry { int r, c; float v; };

enum SegKind { SEG_NONE, SEG_DIA, SEG_LIST, SEG_ELL, SEG_SELL, SEG_GBCSR };

// One forward part's share of the value-gradient array (adjoint).
struct Seg {
    SegKind kind = SEG_NONE;
    size_t offset = 0, count = 0;
    const int* a0 = nullptr;
    const int* a1 = nullptr;
    int p0 = 0, p1 = 0, p2 = 0;
};

struct Engine {
    int width = 0, height = 0, nnz = 0;
    int nrhs = 1;            // right-hand sides: x is width x nrhs, y height x nrhs, row-major
    bool bf16 = false;
    bool use_graph = false;
    bool tensor_spmm = false;   // CSP_FLAG_TENSOR_CORES
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    float* d_x = nullptr;
    float* d_y = nullptr;
    int x_len = 0, y_len = 0;
    std::vector<Part> parts;
    std::vector<void*> allocations;
    size_t device_bytes = 0;
    cudaGraphExec_t graph_exec = nullptr;
    cudaStream_t graph_stream = nullptr;
    std::map<int, cudaGraphExec_t> iter_graphs;   // csp_iterate: graphs of n iterations
    cudaStream_t iter_stream = nullptr;
    bool l2_window = false;                         // CSP_FLAG_L2_PERSIST applied to own_stream
    static constexpr int kIterChunk = 32;
    // adjoint (CSP_FLAG_ADJOINT)
    bool adjoint = false;
    bool abar_blocks = false;          // a part without value gradients (none of the built formats)
    std::vector<Part> adj_parts;       // parts of A^T: xbar += A^T ybar
    std::vector<Seg> segs;
    size_t abar_total = 0;

    ~Engine();
    int init(const cocktail_iif* mat, const float* vec, const float* res, int flags, int k = 1);
    int init_common(int w, int h, int nz, const float* vec, const float* res, int flags, int k);
    int init_bcsr(const bcsr_matrix_if* b, const float* vec, const float* res, int flags, int k);
    int spmv(int ntimes);
    int iterate(int iterations);
    int iterate_once(cudaStream_t st);
    int set_l2_window();
    int enqueue_once(cudaStream_t st);
    int enqueue_parts(const std::vector<Part>& ps, const float* x, float* y, int n, cudaStream_t st);
    int build_adjoint(const cocktail_iif* mat);
    int build_adjoint_gbcsr(const bcsr_matrix_if& b);
    int gbcsr_segment(const bcsr_matrix_if& b, Seg& s);
    int add_transposed_csr(std::vector<Entry>& e);
    int add_slot_list(Seg& s, const std::vector<int>& rows, const std::vector<int>& cols);
    int launch_abar(const float* ybar, float* abar, int* prow, int* pcol, cudaStream_t st);
    int launches_per_spmv() const;

    int alloc(void** p, size_t bytes);
    int upload_int(int** d, const int* h, size_t n, size_t cap);
    int upload_val(void** d, const float* h, size_t n, size_t cap);

    int add_csr(const csr_matrix_if& c, int method);
    int add_coo(const coo_matrix_if& c, int method);
    int add_xpanel(const int* rows, const int* cols, const float* vals, int nnz, bool from_csr);
    int add_ell(const ell_matrix_if& e, int method);
    int add_sell(const sell_matrix_if& s, int method);
    int add_dia(const dia_matrix_iif& d, int method);
    int add_bdia(const bdia_matrix_iif& b, int method);
    int add_bell(const b4ell_matrix_if& b, int method);
    int add_sbell(const sbell_matrix_if& s, int method);
    int add_bcsr(const b4csr_matrix_if& b, int method);
    int add_generic_bcsr(const bcsr_matrix_if& b, int method);
};

int cuda_error(cudaError_t e, const char* what);

// CSR adaptive work blocks (see csr_adaptive_kernel) of rows [0, m) of row pointer rp;
// nslots = long-row chunk partial slots.
void make_adaptive_blocks(const int* rp, int m, std::vector<int4>& blocks, std::vector<int4>& longs, int& nslots);

// Round-to-nearest-even FP32 -> BF16 (NaN kept quiet).
inline uint16_t to_bf16(float f)
{
    uint32_t u;
    memcpy(&u, &f, 4);
    if ((u & 0x7fffffffu) > 0x7f800000u) return (uint16_t)((u >> 16) | 0x40);
    u += 0x7fffu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}

}  // namespace csp

// The opaque handle of the C ABI.
struct csp_handle {
    csp::Engine eng;
};
