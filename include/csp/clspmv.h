/*
 * clspmv_b200 -- C ABI of the B200 (sm_100a) Cocktail SpMV library.
 *
 * The library computes res += A * vec in FP32 (int32 indices) for a sparse
 * matrix A stored in one or more of the nine clSpMV storage formats, exactly
 * like clSpMV (clSpMV_NV/src/eval.cpp:40-42: the result buffer is accumulated,
 * never overwritten).
 *
 * Struct layout.  Every matrix struct below has the same field names, field
 * order and field types as the reference template instantiated at
 * <int, float> (or <int, int, float>) in clSpMV_NV/include/matrix_storage.h,
 * and `cocktail_iif` matches `cocktail<int, int, float>`
 * (clSpMV_NV/include/analyze.h:105-144).  Code that fills the reference
 * structs can pass them here unchanged.
 *
 * Conventions that differ from the reference:
 *   - every function returns CSP_OK (0) or a CSP_E* code and never exits or
 *     aborts (the reference calls exit(1) through CHECKERROR,
 *     clSpMV_NV/include/oclcommon.h:11, or assert);
 *   - OpenCL contexts/queues/cl_mem are replaced by an opaque csp_handle that
 *     owns the device buffers and one CUDA stream;
 *   - one handle per host thread; handles are not internally synchronised;
 *   - csp_do_spmv is asynchronous on the handle's stream; the *_to_cpu copies
 *     synchronise.
 *
 * Host arrays written by the conversion functions are malloc()ed by the
 * library and released by the matching csp_free_* function, like the
 * reference's init_/free_ pairs (matrix_storage.h:373-640).
 */
#ifndef CSP_CLSPMV_H
#define CSP_CLSPMV_H

#include <stddef.h>
#include <stdbool.h>

#ifdef __cplusplus
extern "C" {
#endif
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* ------------------------------------------------------------------------ */
/* Status codes                                                              */
/* ------------------------------------------------------------------------ */
#define CSP_OK        0
#define CSP_EINVAL    1  /* invalid argument or inconsistent struct field        */
#define CSP_ENOMEM    2  /* host or device allocation failed                     */
#define CSP_ECUDA     3  /* a CUDA runtime call failed                           */
#define CSP_EFORMAT   4  /* matrix not representable in the requested format    */
#define CSP_ENODEV    5  /* no CUDA device is visible                            */
#define CSP_EUNSUP    6  /* combination of options not supported                 */
#define CSP_EIO       7  /* file could not be read or parsed                     */
#define CSP_ETIMEOUT  8  /* a bounded device-side wait gave up                   */

/* Human-readable name of a status code. */
const char* csp_error_string(int code);
/* Detail message of the last error raised on the calling thread ("" if none). */
const char* csp_last_error(void);
/* Library version string. */
const char* csp_version(void);

/* ------------------------------------------------------------------------ */
/* Storage formats (layout-compatible with clSpMV_NV/include/matrix_storage.h) */
/* ------------------------------------------------------------------------ */
typedef struct matrixInfo_i { int width; int height; int nnz; } matrixInfo_i;  /* :15-25 */

typedef struct dia_matrix_iif {                          /* matrix_storage.h:27-47 */
    matrixInfo_i matinfo;
    int dia_num;
    int dia_length;
    int dia_length_aligned;
    int* dia_offsets;
    float* dia_data;
} dia_matrix_iif;

typedef struct bdia_matrix_iif {                         /* matrix_storage.h:71-94 */
    matrixInfo_i matinfo;
    int bdia_band_num;
    int bdia_length;
    int bdia_length_aligned;
    int* bdia_offsets;
    int* bdia_bptr;
    float* bdia_data;
} bdia_matrix_iif;

typedef struct ell_matrix_if {                           /* matrix_storage.h:96-111 */
    matrixInfo_i matinfo;
    int ell_num;
    int ell_height_aligned;
    int* ell_col_id;
    float* ell_data;
} ell_matrix_if;

typedef struct sell_matrix_if {                          /* matrix_storage.h:114-137 */
    matrixInfo_i matinfo;
    unsigned int sell_slice_height;
    int sell_slice_num;
    int* sell_slice_ptr;
    int* sell_col_id;
    float* sell_data;
} sell_matrix_if;

typedef struct coo_matrix_if {                           /* matrix_storage.h:141-152 */
    matrixInfo_i matinfo;
    int* coo_row_id;
    int* coo_col_id;
    float* coo_data;
} coo_matrix_if;

typedef struct csr_matrix_if {                           /* matrix_storage.h:155-166 */
    matrixInfo_i matinfo;
    int* csr_row_ptr;
    int* csr_col_id;
    float* csr_data;
} csr_matrix_if;

typedef struct bcsr_matrix_if {                          /* matrix_storage.h:169-199 */
    matrixInfo_i matinfo;
    unsigned int bcsr_bwidth;
    unsigned int bcsr_bheight;
    int bcsr_row_num;
    int bcsr_aligned_size;
    int bcsr_block_num;
    int* bcsr_row_ptr;
    int* bcsr_col_id;
    float* bcsr_data;
} bcsr_matrix_if;

typedef struct bell_matrix_if {                          /* matrix_storage.h:215-236 */
    matrixInfo_i matinfo;
    unsigned int bell_bwidth;
    unsigned int bell_bheight;
    int bell_row_num;
    int bell_block_num;
    int bell_height_aligned;
    int bell_float4_aligned;
    int* bell_col_id;
    float* bell_data;
} bell_matrix_if;

typedef struct b4csr_matrix_if {                         /* matrix_storage.h:266-287 */
    matrixInfo_i matinfo;
    unsigned int b4csr_bwidth;
    unsigned int b4csr_bheight;
    int b4csr_row_num;
    int b4csr_aligned_size;
    int b4csr_block_num;
    int* b4csr_row_ptr;
    int* b4csr_col_id;
    float* b4csr_data;
} b4csr_matrix_if;

typedef struct b4ell_matrix_if {                         /* matrix_storage.h:311-332 */
    matrixInfo_i matinfo;
    unsigned int b4ell_bwidth;
    unsigned int b4ell_bheight;
    int b4ell_row_num;
    int b4ell_block_num;
    int b4ell_height_aligned;
    int b4ell_float4_aligned;
    int* b4ell_col_id;
    float* b4ell_data;
} b4ell_matrix_if;

typedef struct sbell_matrix_if {                         /* matrix_storage.h:344-365 */
    matrixInfo_i matinfo;
    unsigned int sbell_bwidth;
    unsigned int sbell_bheight;
    unsigned int sbell_slice_height;
    int sbell_slice_num;
    int sbell_row_num;
    int* sbell_slice_ptr;
    int* sbell_col_id;
    float* sbell_data;
} sbell_matrix_if;

/* The Cocktail container: one optional sub-matrix per format plus the kernel
 * variant ("method") chosen for each.  Layout of cocktail<int,int,float>,
 * clSpMV_NV/include/analyze.h:105-144. */
typedef struct cocktail_iif {
    bool ifusebdia;
    bool ifusedia;
    bool ifusesbell;
    bool ifusebell;
    bool ifusebcsr;
    bool ifusesell;
    bool ifuseell;
    bool ifusecsr;
    bool ifusecoo;

    int bdia_meth_num;
    int dia_meth_num;
    int sbell_meth_num;
    int bell_meth_num;
    int bcsr_meth_num;
    int sell_meth_num;
    int ell_meth_num;
    int csr_meth_num;
    int coo_meth_num;

    int csr_group_num;
    int coo_group_num;

    int mat_width;
    int mat_height;
    int mat_nnz;

    bdia_matrix_iif bdia;
    dia_matrix_iif dia;
    sbell_matrix_if sbell;
    b4ell_matrix_if bell;
    b4csr_matrix_if bcsr;
    sell_matrix_if sell;
    ell_matrix_if ell;
    csr_matrix_if csr;
    coo_matrix_if coo;
} cocktail_iif;

/* ------------------------------------------------------------------------ */
/* init_ / free_ (matrix_storage.h:373-640; analyze.h:146-206)               */
/* free_* releases the arrays only; the info fields stay, as in the reference. */
/* ------------------------------------------------------------------------ */
void csp_init_coo_matrix(coo_matrix_if* m);
void csp_init_csr_matrix(csr_matrix_if* m);
void csp_init_ell_matrix(ell_matrix_if* m);
void csp_init_sell_matrix(sell_matrix_if* m);
void csp_init_dia_matrix(dia_matrix_iif* m);
void csp_init_bdia_matrix(bdia_matrix_iif* m);
void csp_init_bcsr_matrix(bcsr_matrix_if* m);
void csp_init_bell_matrix(bell_matrix_if* m);
void csp_init_b4csr_matrix(b4csr_matrix_if* m);
void csp_init_b4ell_matrix(b4ell_matrix_if* m);
void csp_init_sbell_matrix(sbell_matrix_if* m);
void csp_init_cocktail(cocktail_iif* m);

void csp_free_coo_matrix(coo_matrix_if* m);
void csp_free_csr_matrix(csr_matrix_if* m);
void csp_free_ell_matrix(ell_matrix_if* m);
void csp_free_sell_matrix(sell_matrix_if* m);
void csp_free_dia_matrix(dia_matrix_iif* m);
void csp_free_bdia_matrix(bdia_matrix_iif* m);
void csp_free_bcsr_matrix(bcsr_matrix_if* m);
void csp_free_bell_matrix(bell_matrix_if* m);
void csp_free_b4csr_matrix(b4csr_matrix_if* m);
void csp_free_b4ell_matrix(b4ell_matrix_if* m);
void csp_free_sbell_matrix(sbell_matrix_if* m);
void csp_free_cocktail(cocktail_iif* m);

/* ------------------------------------------------------------------------ */
/* Host-side conversions.  Output arrays are byte-identical to the reference */
/* functions named beside each declaration, including padding values.        */
/* Functions that the reference lets sort the input in place do the same.    */
/* ------------------------------------------------------------------------ */
int csp_aligned_length(int length, int alignment);                  /* matrix_storage.h:818 */
int csp_if_sorted_coo(const coo_matrix_if* m);                       /* matrix_storage.h:732 */
int csp_sort_coo(coo_matrix_if* m);                                  /* matrix_storage.h:745; CSP_EFORMAT on stack overflow */
int csp_coo2csr(coo_matrix_if* src, csr_matrix_if* dst);             /* matrix_storage.h:1269 */
int csp_csr2coo(const csr_matrix_if* src, coo_matrix_if* dst);       /* matrix_storage.h:1239 */
int csp_coo2ell(coo_matrix_if* src, ell_matrix_if* dst, int alignment, int ellnum);   /* :1341 */
int csp_ell2coo(const ell_matrix_if* src, coo_matrix_if* dst);       /* matrix_storage.h:1310 */
int csp_coo2sell(coo_matrix_if* src, sell_matrix_if* dst, unsigned int sliceheight); /* :1398 */
int csp_coo2dia(coo_matrix_if* src, dia_matrix_iif* dst, int alignment);             /* :937; CSP_EFORMAT when too padded */
int csp_dia2coo(const dia_matrix_iif* src, coo_matrix_if* dst);      /* matrix_storage.h:826 */
int csp_coo2bdia(coo_matrix_if* src, bdia_matrix_iif* dst, int alignment);           /* :1185 */
int csp_bdia2coo(const bdia_matrix_iif* src, coo_matrix_if* dst);    /* matrix_storage.h:1137 */
int csp_coo2bcsr(coo_matrix_if* src, bcsr_matrix_if* dst, unsigned int bwidth, unsigned int bheight, int alignment); /* :1595 */
int csp_bcsr2coo(const bcsr_matrix_if* src, coo_matrix_if* dst);     /* matrix_storage.h:1546 */
int csp_coo2bell(coo_matrix_if* src, bell_matrix_if* dst, unsigned int bwidth, unsigned int bheight, int alignment, int ellnum); /* :1941 */
int csp_bell2coo(const bell_matrix_if* src, coo_matrix_if* dst);     /* matrix_storage.h:1901 */
/* util.cpp:273 rearrange_bell_4col: a generic BELL with bwidth % 4 == 0 rewritten in place
 * into the b4 float4 layout (bell_float4_aligned = align(4 * row_num, alignment), column
 * ids divided by 4).  Alignment slots are zero (the reference leaves them unset). */
int csp_rearrange_bell_4col(bell_matrix_if* mat, int alignment);
int csp_coo2b4csr(coo_matrix_if* src, b4csr_matrix_if* dst, unsigned int bwidth, unsigned int bheight, int alignment); /* :1741; CSP_EFORMAT above MAX_MEM_OBJ */
int csp_coo2b4ell(coo_matrix_if* src, b4ell_matrix_if* dst, unsigned int bwidth, unsigned int bheight, int alignment, int ellnum); /* :2010 */
int csp_coo2sbell(coo_matrix_if* src, sbell_matrix_if* dst, unsigned int bwidth, unsigned int bheight, unsigned int sliceheight); /* :2203 */
int csp_pad_csr(const csr_matrix_if* src, csr_matrix_if* dst, int alignment);        /* util.cpp:31 */

/* ------------------------------------------------------------------------ */
/* Cocktail analyzer (analyze.h:257 analyze_matrix)                          */
/* ------------------------------------------------------------------------ */
#define CSP_ANALYZE_REFERENCE 0  /* reference decisions from clSpMV .ben tables      */
#define CSP_ANALYZE_AUTOTUNE  1  /* B200 decisions: measured on the device, cached   */

typedef struct csp_analyze_opts {
    int mode;                /* CSP_ANALYZE_REFERENCE or CSP_ANALYZE_AUTOTUNE            */
    const char* bench_path;  /* REFERENCE: directory holding benchmark/ *.ben; NULL = $CLSPMVPATH */
    int verbose;             /* AUTOTUNE: 1 = print each candidate's measured time        */
    const char* cache_path;  /* AUTOTUNE: file caching decisions per sparsity signature  */
    int flags;               /* AUTOTUNE: engine flags the partition is tuned for (CSP_FLAG_BF16);
                                REFERENCE: CSP_ANALYZE_ON_DEVICE                              */
} csp_analyze_opts;
/* REFERENCE mode: the analyzer's integer counting passes -- nonzeros per diagonal
 * (analyze.cpp:804 count_dia_nnz) and blocks per block row for the eight b4 shapes
 * (:1582 count_blocks) -- run on the current CUDA device; the partition is the same,
 * byte for byte.  CSP_ENODEV without a device.  No counterpart in the reference. */
#define CSP_ANALYZE_ON_DEVICE 0x100

/* Partition `coo` into the per-format sub-matrices of `mat`.  `coo` may be
 * sorted in place (as the reference does).  opts may be NULL (REFERENCE mode,
 * $CLSPMVPATH).
 * REFERENCE: the reference partition, bit for bit, from the clSpMV tables.
 * AUTOTUNE: needs a CUDA device; builds candidate partitions (each format and
 * kernel variant, slice heights 32/128, the eight b4 block shapes, ELL + CSR
 * splits), times each on the device with L2 flushed between SpMVs, keeps the
 * fastest, and records the choice under a hash of the sparsity pattern in
 * cache_path (if given) so the next call on the same pattern skips timing. */
int csp_analyze_matrix(coo_matrix_if* coo, cocktail_iif* mat, const csp_analyze_opts* opts);
/* Measure this library's kernels on the current GPU and write the analyzer's
 * calibration tables (clspmv_path/benchmark/{overhead,dia,bdia,ell,sell,csr,coo,bcsr,
 * bell,sbell}.ben) in the layout the reference's bench_* programs write
 * (clSpMV_NV/src/bench_*.cpp, the `benchmarking` script): the same synthetic banded
 * matrices, one GFLOPS column per kernel method.  CSP_ANALYZE_REFERENCE with
 * bench_path = clspmv_path then partitions from B200 measurements.  level 2: the
 * reference's full grids (minutes); 1: every third size and every other width;
 * 0: two sizes and two widths per table (seconds; a format check).  Synchronous. */
int csp_benchmark_tables(const char* clspmv_path, int level);

/* Name of the partition the last AUTOTUNE call on this thread chose ("" if none),
 * e.g. "csr2", "ell1+csr2", "bcsr4x4m0". */
const char* csp_autotune_choice(void);

/* ------------------------------------------------------------------------ */
/* Device engine (spmv_cocktail.h:111-175)                                   */
/* ------------------------------------------------------------------------ */
typedef struct csp_handle csp_handle;

#define CSP_FLAG_USE_TEX   0x1  /* accepted for API compatibility; x is always read through the read-only path */
#define CSP_FLAG_BF16      0x2  /* store matrix values as BF16, accumulate in FP32                             */
#define CSP_FLAG_GRAPH     0x4  /* replay do_spmv as one captured CUDA graph                                   */
#define CSP_FLAG_ADJOINT   0x8  /* also build the transposed structures for csp_spmv_adjoint                  */
#define CSP_FLAG_L2_PERSIST 0x10 /* keep x resident in L2: an access-policy window (persisting hits) over x on
                                    the handle's own stream, with persisting L2 reserved for this process's
                                    context up to x's size; not applied to a stream given by csp_set_stream.
                                    No counterpart in the reference. */
#define CSP_FLAG_TENSOR_CORES 0x20 /* generic BCSR SpMM (csp_init_bcsr_kernels, nrhs a multiple of 32, blocks of
                                    at most 8 rows x 4 columns) on the tensor cores: mma.sync m16n8k8 with TF32
                                    operands split in high and low parts for FP32 accuracy.  No counterpart
                                    in the reference. */

/* Kernel choice for a CSR or COO sub-matrix (csr_meth_num / coo_meth_num; no
 * counterpart in the reference): x staged in shared memory by column panels of at
 * most 32,768 columns.  The sub-matrix's nonzeros are regrouped by panel; each CTA
 * copies its panels of x into shared memory and reduces 128-entry tiles to one
 * partial sum per run of one row, and a second kernel adds every row's partials to
 * res in panel order (deterministic, two launches per SpMV).  Meant for matrices
 * whose column indices have no locality (random graphs), where gathering x from
 * global memory is bound by L2 request throughput.  One right-hand side only. */
#define CSP_METH_XPANEL    16

/* bcsr_meth_num value marking the cocktail's `bcsr` member as a generic BCSR
 * (matrix_storage.h:1595 coo2bcsr layout: column ids of the block's first column,
 * data[e * aligned + block]) of one of the block shapes csp_init_bcsr_kernels takes,
 * instead of the b4 layout.  bcsr_matrix_if and b4csr_matrix_if have the same fields
 * in the same order, so the generic matrix is stored in the member as is and
 * csp_free_cocktail frees it.  The autotuner (CSP_ANALYZE_AUTOTUNE) uses it for block
 * shapes the b4 formats cannot hold, such as 3x3.  Such a part also takes several
 * right-hand sides.  No counterpart in the reference. */
#define CSP_METH_GENERIC_BCSR 32

/* Upload every used sub-matrix of `mat`, x = vec (length mat_width) and
 * res (length mat_height; may be NULL for zeros), and select one kernel per
 * sub-matrix from its *_meth_num.  (spmv_cocktail.cpp:1593 init_mat_kernels) */
int csp_init_mat_kernels(const cocktail_iif* mat, const float* vec, const float* res, int flags, csp_handle** out);
/* Several right-hand sides (SpMM, no counterpart in the reference):
 * res (mat_height x nrhs) += A * vec (mat_width x nrhs), both row-major, so the
 * copy functions take nrhs times as many floats.  nrhs > 1 runs on CSR parts only;
 * other formats return CSP_EUNSUP (use csp_init_bcsr_kernels for block matrices). */
int csp_init_mat_kernels_ex(const cocktail_iif* mat, const float* vec, const float* res, int nrhs, int flags,
                            csp_handle** out);
/* A handle over one generic BCSR matrix (matrix_storage.h:169 layout, any block
 * shape 1x1, 2x2, 3x3, 4x4, 6x6 or 8x8; nrhs > 1 up to 6x6), e.g. the 3x3-block FEM
 * case the b4 formats cannot hold.  Same do_spmv / copy calls. */
int csp_init_bcsr_kernels(const bcsr_matrix_if* mat, const float* vec, const float* res, int nrhs, int flags,
                          csp_handle** out);
/* Enqueue ntimes SpMVs res += A*vec on the handle's stream.  (:1091 do_spmv) */
int csp_do_spmv(csp_handle* h, int ntimes);
/* The solver loop of the reference's example() (eval.cpp:19-50: do_spmv, then
 * cpy_vector_from_gpu(gpumat.res)) on the device: `iterations` times res += A*vec
 * followed by vec = res.  Square matrices, one right-hand side.  With CSP_FLAG_GRAPH
 * every 32 iterations are one CUDA graph launch.  Asynchronous on the handle's stream. */
int csp_iterate(csp_handle* h, int iterations);
/* Block until every launch on the handle's stream has finished. */
int csp_synchronize(csp_handle* h);
int csp_cpy_vector_from_cpu(csp_handle* h, const float* vec, int vec_size);     /* :1462 */
int csp_cpy_vector_from_gpu(csp_handle* h, const float* dvec, int vec_size);    /* :1513, dvec = device pointer */
int csp_cpy_result_from_cpu(csp_handle* h, const float* res, int res_size);     /* :1562 */
int csp_cpy_result_from_gpu(csp_handle* h, const float* dres, int res_size);    /* :1571 */
int csp_cpy_result_to_cpu(csp_handle* h, float* res, int res_size);             /* :1578, synchronises */
int csp_cpy_result_to_gpu(csp_handle* h, float* dres, int res_size);            /* :1585 */
int csp_free_mat_kernels(csp_handle* h);                                        /* :1616 */

/* Device pointers of the handle's x and res buffers (like gpumat.vec / gpumat.res). */
int csp_get_vec_device_ptr(csp_handle* h, float** dvec);
int csp_get_res_device_ptr(csp_handle* h, float** dres);
/* Launch on a caller-owned cudaStream_t (passed as void*); NULL = the handle's own stream. */
int csp_set_stream(csp_handle* h, void* stream);
int csp_get_stream(csp_handle* h, void** stream);
/* Number of kernel launches one csp_do_spmv(h, 1) enqueues. */
int csp_launches_per_spmv(csp_handle* h, int* launches);
/* Bytes of device memory the handle owns. */
int csp_device_bytes(csp_handle* h, size_t* bytes);

/* Correctness and timing of one engine against the serial COO result
 * (spmv_cocktail.cpp:1434 evaluate / :1137 check_and_time).  Prints nothing;
 * fills the report. */
typedef struct csp_report {
    int    method;          /* best kernel variant (format-specific numbering)    */
    double gflops;          /* 2*nnz / best time                                  */
    double gbytes;          /* algorithmic bytes / best time, GB/s                */
    double ms;              /* best time per SpMV, milliseconds                   */
    double l2_distance;     /* || y_gpu - y_coo ||_2   (util.cpp:93 two_vec_compare) */
    double max_diff;        /* max | |y_gpu| - |y_coo| |                          */
    double max_ratio_diff;  /* max of the relative form of the same               */
    int    group_num;       /* CSR/COO: work-group count used                    */
} csp_report;
int csp_evaluate(const cocktail_iif* mat, const float* vec, const float* res, const float* coores, int ntimes, csp_report* report);

/* ------------------------------------------------------------------------ */
/* spmv_all single-format drivers (NV/include/spmv_*.h:7; spmv_all.cpp:196)   */
/* method: 1 csr_scalar, 2 csr_vector, 3 bdia, 4 dia, 5 ell, 6 coo, 7 bell,   */
/* 8 bcsr, 9 sell, 10 sbell (spmv_all.cpp:164-175).  Each converts `coo`, runs */
/* every kernel variant                                                        */
/* of that format (one checked launch, 3 warm-ups, ntimes timed) and reports   */
/* the best, without printing.                                                 */
/* ------------------------------------------------------------------------ */
int csp_spmv_all(coo_matrix_if* coo, int method, int ntimes, csp_report* report);
int csp_spmv_csr_scalar(coo_matrix_if* coo, int ntimes, csp_report* report);
int csp_spmv_csr_vector(coo_matrix_if* coo, int ntimes, csp_report* report);
int csp_spmv_bdia(coo_matrix_if* coo, int ntimes, csp_report* report);
int csp_spmv_dia(coo_matrix_if* coo, int ntimes, csp_report* report);
int csp_spmv_ell(coo_matrix_if* coo, int ntimes, csp_report* report);
int csp_spmv_sell(coo_matrix_if* coo, int ntimes, csp_report* report);
int csp_spmv_coo(coo_matrix_if* coo, int ntimes, csp_report* report);
int csp_spmv_bell(coo_matrix_if* coo, int ntimes, csp_report* report);
int csp_spmv_bcsr(coo_matrix_if* coo, int ntimes, csp_report* report);
int csp_spmv_sbell(coo_matrix_if* coo, int ntimes, csp_report* report);

/* ------------------------------------------------------------------------ */
/* Adjoint (no counterpart in the reference).  Needs a handle built with      */
/* CSP_FLAG_ADJOINT, which also stores A^T (a transposed DIA per diagonal      */
/* part of a square matrix, one transposed CSR for every other part):         */
/*   d_xbar += A^T * d_ybar            (deterministic, no atomics), and        */
/*   d_abar[s] = d_ybar[row(s)] * x[col(s)] for every stored slot s of the     */
/*   forward parts, in launch order, each part in its own storage layout      */
/*   (DIA/BDIA: diagonal-major slots; CSR/COO: entry order; ELL/SELL: their     */
/*   slot order; BCSR/BELL/SBELL: their b4 data order) -- the gradient of      */
/*   ybar^T (A x) with respect to the stored values.  A handle of              */
/*   csp_init_bcsr_kernels (one right-hand side) takes CSP_FLAG_ADJOINT too:   */
/*   its slots are the caller's generic BCSR data order, data[e * aligned + j] */
/*   (element e of block j at row e / bw, column e % bw).  x is the handle's   */
/*   current vector.  All pointers are device pointers; d_xbar or d_abar may   */
/*   be NULL to skip that output.                                              */
/* ------------------------------------------------------------------------ */
int csp_spmv_adjoint(csp_handle* h, const float* d_ybar, float* d_xbar, float* d_abar);
/* Number of stored slots, the length of d_abar. */
int csp_adjoint_slots(csp_handle* h, size_t* nslots);
/* Row and column of every slot (row -1 for slots outside the matrix: alignment
 * rows and blocks, out-of-range diagonal positions, the parts of a last block row
 * or column past the matrix), into device arrays of nslots ints. */
int csp_adjoint_pattern(csp_handle* h, int* d_rows, int* d_cols);

/* ------------------------------------------------------------------------ */
/* Batched execution (no counterpart in the reference).  Many matrices of     */
/* uneven size run in ONE persistent kernel over a (matrix, row-slice) work   */
/* list: forward y_i += A_i x_i, adjoint xbar_i += A_i^T ybar_i and value      */
/* gradients abar_i[s] = ybar_i[row(s)] * x_i[col(s)] over every stored slot.  */
/* Each matrix is stored in the batch format chosen for it (format, slice     */
/* height, block size): by the device autotuner, which times the candidates   */
/* inside the persistent kernel and caches the decision per sparsity          */
/* signature, by a byte-count model, or forced by the caller.  The batch takes */
/* COO matrices (sorted copies are made when needed), not cocktails: it picks  */
/* its own formats.  Vectors are concatenated in matrix order: x and xbar of   */
/* length sum(width_i), y and ybar of sum(height_i), abar of the slots of all  */
/* matrices; csp_batch_layout gives the offsets.  Results are deterministic.   */
/* ------------------------------------------------------------------------ */
typedef struct csp_batch csp_batch;

#define CSP_BFMT_AUTO    (-1)
#define CSP_BFMT_CSR      0  /* CSR in work blocks of <= 2040 entries, long rows chunked */
#define CSP_BFMT_SELL32   1  /* sliced ELL, slice height 32                              */
#define CSP_BFMT_SELL128  2  /* sliced ELL, slice height 128                             */
#define CSP_BFMT_DIA      3  /* diagonals (at most 64)                                   */
#define CSP_BFMT_BCSR2    4  /* 2x2 blocks                                               */
#define CSP_BFMT_BCSR3    5  /* 3x3 blocks                                               */
#define CSP_BFMT_BCSR4    6  /* 4x4 blocks                                               */
#define CSP_BFMT_COUNT    7

#define CSP_BATCH_TUNE_MODEL  0  /* fewest stored bytes among the feasible formats   */
#define CSP_BATCH_TUNE_DEVICE 1  /* time the feasible formats in the persistent kernel */

#define CSP_BATCH_FWD 1          /* y += A x                                        */
#define CSP_BATCH_ADJ 2          /* xbar += A^T ybar and abar = ybar (x) x on A's slots */

#define CSP_BV_X    0
#define CSP_BV_Y    1
#define CSP_BV_YBAR 2
#define CSP_BV_XBAR 3
#define CSP_BV_ABAR 4

typedef struct csp_batch_opts {
    int flags;               /* CSP_FLAG_BF16, CSP_FLAG_GRAPH, CSP_FLAG_ADJOINT (A^T and abar) */
    int format;              /* CSP_BFMT_AUTO, or one format for every matrix (must be feasible) */
    int tune;                /* CSP_BATCH_TUNE_MODEL or CSP_BATCH_TUNE_DEVICE (format AUTO)     */
    const char* cache_path;  /* signature -> format decisions, appended; NULL: process cache only */
} csp_batch_opts;

/* Host-side structure of one matrix, as the format choice sees it. */
typedef struct csp_batch_features {
    int rows, cols, nnz, max_row;
    int ndiag;                      /* distinct diagonals, -1 if more than 64 */
    long long dia_slots;            /* ndiag * align(rows, 32)                */
    long long sell_slots[2];        /* slice heights 32 and 128               */
    long long bcsr_blocks[3];       /* block sizes 2, 3, 4                    */
    unsigned int feasible;          /* bit f: format f is a candidate         */
    int model_format;               /* the byte model's choice                */
    unsigned long long signature;   /* sparsity signature (decision cache key) */
} csp_batch_features;

int csp_batch_features_of(const coo_matrix_if* mat, int flags, csp_batch_features* out);
int csp_batch_create(const coo_matrix_if* const* mats, int n, const csp_batch_opts* opts, csp_batch** out);
int csp_batch_free(csp_batch* b);
/* n + 1 prefix offsets each (floats); any pointer may be NULL. */
int csp_batch_layout(const csp_batch* b, long long* x_off, long long* y_off, long long* abar_off);
int csp_batch_formats(const csp_batch* b, int* formats);
/* Formats of the stored transposes A_i^T (CSP_FLAG_ADJOINT batches): chosen on their own,
 * since the transpose of a matrix with long rows has short, even rows. */
int csp_batch_formats_adjoint(const csp_batch* b, int* formats);
int csp_batch_device_ptrs(const csp_batch* b, float** x, float** y, float** ybar, float** xbar, float** abar);
/* Whole-vector copies on the batch stream: host `src` -> device, or device -> host
 * `dst` (then synchronised).  Exactly one of src, dst is non-NULL. */
int csp_batch_copy(csp_batch* b, int which, const float* src, float* dst);
int csp_batch_set_stream(csp_batch* b, void* stream);   /* NULL: the batch's own stream */
void* csp_batch_get_stream(const csp_batch* b);
/* One persistent launch per repetition (a CUDA graph replay with CSP_FLAG_GRAPH). */
int csp_batch_run(csp_batch* b, int what, int ntimes);
/* The same work as per-matrix plain CSR launches (a CSR-vector SpMV per matrix
 * and direction, one gradient kernel per matrix); needs every format CSR.  `lanes`
 * per row: 1, 2, 4, 8, 16 or 32, or 0 for the power of two nearest below each
 * matrix's mean row length. */
int csp_batch_run_plain(csp_batch* b, int what, int ntimes, int lanes);
int csp_batch_synchronize(csp_batch* b);
/* Kernel launches one run (or one plain run) makes. */
int csp_batch_launches(const csp_batch* b, int what, int plain);
size_t csp_batch_device_bytes(const csp_batch* b);
/* Row and column of every slot of matrix i (host arrays of abar_off[i+1]-abar_off[i]
 * ints; row -1 for padding slots). */
int csp_batch_pattern(const csp_batch* b, int i, int* rows, int* cols);

/* ------------------------------------------------------------------------ */
/* SpMV without device allocation.  No counterpart in the reference.          */
/*                                                                            */
/* For callers that cannot allocate device memory -- code running under a     */
/* framework allocator that already owns the device, real-time loops where    */
/* cudaMalloc/cudaFree (which may synchronize the device) are forbidden,      */
/* embedders that pass only buffers they own.  Computes y += A*x for a COO    */
/* matrix held by the caller in device memory (16-byte aligned arrays), on    */
/* `stream` (NULL = legacy default stream), allocating nothing: its scratch   */
/* is a fixed 1 MiB array inside this library's device image, held by every   */
/* GPU that loads the library until the process exits, which limits nnz to   */
/* CSP_NOALLOC_MAX_NNZ (larger matrices: CSP_EINVAL).                         */
/* Preconditions, not checked on the device (checking would need a pass and a */
/* synchronization): rows sorted in nondecreasing order -- unsorted input     */
/* gives an undefined result, though no access leaves the caller's arrays --  */
/* and x and y distinct, non-overlapping arrays (d_x == d_y: CSP_EINVAL).     */
/* The first call on each device looks the array's address up for that       */
/* device and keeps it, so make it before capturing the call into a CUDA      */
/* graph; a cudaDeviceReset after that first call is not supported.  All     */
/* calls on a device share the array: calls that overlap on the GPU (other   */
/* streams, other host threads) race and must be serialized by the caller.    */
/* Nothing in the array needs clearing between calls: each call writes every  */
/* slot it reads.  Out-of-range row or column ids are skipped, not            */
/* dereferenced.                                                              */
/* ------------------------------------------------------------------------ */
#define CSP_NOALLOC_MAX_NNZ       33554432   /* 2^25 entries                          */
#define CSP_NOALLOC_SCRATCH_BYTES 1048576    /* 2 (row, partial) pairs per 512 entries */
int csp_coo_spmv_noalloc(int height, int width, int nnz, const int* d_row, const int* d_col, const float* d_val,
                         const float* d_x, float* d_y, void* stream);

/* ------------------------------------------------------------------------ */
/* spmv_all method 0 (spmv_all.cpp:196, mem_bandwidth.cpp): device memory      */
/* bandwidth and kernel launch overhead.  `bytes` per buffer (>= 1 MiB);      */
/* the gather reads 4-byte values at random indices in [0, gather_range).      */
/* ------------------------------------------------------------------------ */
typedef struct csp_bandwidth_report {
    double launch_us;     /* empty-kernel launch-to-launch time, microseconds      */
    double copy_gbs;      /* float4 device copy, read + written bytes per second   */
    double gather_gbs;    /* random gather: index and value bytes per second        */
    double gather_per_s;  /* random gather: elements per second                      */
} csp_bandwidth_report;
int csp_bandwidth_test(size_t bytes, int gather_range, csp_bandwidth_report* rep);


/* ------------------------------------------------------------------------ */
/* MatrixMarket input (fileio.cpp:10 ReadMMF): 0-based, pattern -> 1.0,       */
/* symmetric mirrored, sorted.                                               */
/* ------------------------------------------------------------------------ */
int csp_read_mmf(const char* filename, coo_matrix_if* mat);
/* csp_read_mmf with options.  CSP_MMF_SORT_ON_DEVICE: the entries are sorted by
 * (row, col) on the current CUDA device (csp_sort_coo_device) instead of the host.
 * No counterpart in the reference. */
#define CSP_MMF_SORT_ON_DEVICE 0x1
int csp_read_mmf_ex(const char* filename, coo_matrix_if* mat, int flags);
/* A host COO sorted in place by (row, col) on the current CUDA device: a stable radix
 * sort, so entries with equal (row, col) keep their input order (the reference's
 * quicksort, matrix_storage.h:745, may order such duplicates differently; without
 * duplicates the two agree byte for byte).  CSP_ENODEV without a device.  No
 * counterpart in the reference. */
int csp_sort_coo_device(coo_matrix_if* mat);

/* ------------------------------------------------------------------------ */
/* Layout builds on the current CUDA device: the same structs, filled byte for */
/* byte as by csp_coo2dia / csp_coo2bdia / csp_coo2bcsr (matrix_storage.h:937  */
/* coo2dia, :1185 coo2bdia, :1595 coo2bcsr) when no two entries share a        */
/* (row, col) position; with such                                              */
/* duplicates the last one in input order is kept.  The same errors, at the    */
/* same entry, as the host builds; CSP_ENODEV without a device.                */
/* ------------------------------------------------------------------------ */
int csp_coo2dia_device(coo_matrix_if* src, dia_matrix_iif* dst, int alignment);
int csp_coo2bdia_device(coo_matrix_if* src, bdia_matrix_iif* dst, int alignment);     /* :1185 */
int csp_coo2bcsr_device(coo_matrix_if* src, bcsr_matrix_if* dst, unsigned int bwidth, unsigned int bheight,
                        int alignment);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#ifdef __cplusplus
}
#endif
#endif /* CSP_CLSPMV_H */
