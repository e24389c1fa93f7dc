"""ctypes mirror of include/csp/clspmv.h, the C ABI of libclspmv_b200.so.

The struct classes carry the reference's names and fields
(clSpMV_NV/include/matrix_storage.h:15-365, analyze.h:105-144), so Python code reads
like the reference's C++.  Arrays inside a struct are raw pointers; the helpers below
convert between them and numpy arrays.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libclspmv_b200.so")

IP = C.POINTER(C.c_int)
FP = C.POINTER(C.c_float)

CSP_OK, CSP_EINVAL, CSP_ENOMEM, CSP_ECUDA, CSP_EFORMAT, CSP_ENODEV, CSP_EUNSUP, CSP_EIO, CSP_ETIMEOUT = range(9)
CSP_FLAG_USE_TEX, CSP_FLAG_BF16, CSP_FLAG_GRAPH, CSP_FLAG_ADJOINT, CSP_FLAG_L2_PERSIST = 0x1, 0x2, 0x4, 0x8, 0x10
CSP_FLAG_TENSOR_CORES = 0x20
CSP_METH_XPANEL = 16
CSP_METH_GENERIC_BCSR = 32
CSP_ANALYZE_ON_DEVICE = 0x100
CSP_MMF_SORT_ON_DEVICE = 0x1
CSP_ANALYZE_REFERENCE, CSP_ANALYZE_AUTOTUNE = 0, 1
CSP_NOALLOC_MAX_NNZ = 33554432
CSP_BFMT_AUTO = -1
(CSP_BFMT_CSR, CSP_BFMT_SELL32, CSP_BFMT_SELL128, CSP_BFMT_DIA, CSP_BFMT_BCSR2, CSP_BFMT_BCSR3,
 CSP_BFMT_BCSR4, CSP_BFMT_COUNT) = range(8)
BFMT_NAMES = ("csr", "sell32", "sell128", "dia", "bcsr2", "bcsr3", "bcsr4")
CSP_BATCH_TUNE_MODEL, CSP_BATCH_TUNE_DEVICE = 0, 1
CSP_BATCH_FWD, CSP_BATCH_ADJ = 1, 2
CSP_BV_X, CSP_BV_Y, CSP_BV_YBAR, CSP_BV_XBAR, CSP_BV_ABAR = range(5)


class matrixInfo(C.Structure):
    _fields_ = [("width", C.c_int), ("height", C.c_int), ("nnz", C.c_int)]


class dia_matrix(C.Structure):
    _fields_ = [("matinfo", matrixInfo), ("dia_num", C.c_int), ("dia_length", C.c_int),
                ("dia_length_aligned", C.c_int), ("dia_offsets", IP), ("dia_data", FP)]


class bdia_matrix(C.Structure):
    _fields_ = [("matinfo", matrixInfo), ("bdia_band_num", C.c_int), ("bdia_length", C.c_int),
                ("bdia_length_aligned", C.c_int), ("bdia_offsets", IP), ("bdia_bptr", IP), ("bdia_data", FP)]


class ell_matrix(C.Structure):
    _fields_ = [("matinfo", matrixInfo), ("ell_num", C.c_int), ("ell_height_aligned", C.c_int),
                ("ell_col_id", IP), ("ell_data", FP)]


class sell_matrix(C.Structure):
    _fields_ = [("matinfo", matrixInfo), ("sell_slice_height", C.c_uint), ("sell_slice_num", C.c_int),
                ("sell_slice_ptr", IP), ("sell_col_id", IP), ("sell_data", FP)]


class coo_matrix(C.Structure):
    _fields_ = [("matinfo", matrixInfo), ("coo_row_id", IP), ("coo_col_id", IP), ("coo_data", FP)]


class csr_matrix(C.Structure):
    _fields_ = [("matinfo", matrixInfo), ("csr_row_ptr", IP), ("csr_col_id", IP), ("csr_data", FP)]


class bcsr_matrix(C.Structure):
    _fields_ = [("matinfo", matrixInfo), ("bcsr_bwidth", C.c_uint), ("bcsr_bheight", C.c_uint),
                ("bcsr_row_num", C.c_int), ("bcsr_aligned_size", C.c_int), ("bcsr_block_num", C.c_int),
                ("bcsr_row_ptr", IP), ("bcsr_col_id", IP), ("bcsr_data", FP)]


class bell_matrix(C.Structure):
    _fields_ = [("matinfo", matrixInfo), ("bell_bwidth", C.c_uint), ("bell_bheight", C.c_uint),
                ("bell_row_num", C.c_int), ("bell_block_num", C.c_int), ("bell_height_aligned", C.c_int),
                ("bell_float4_aligned", C.c_int), ("bell_col_id", IP), ("bell_data", FP)]


class b4csr_matrix(C.Structure):
    _fields_ = [("matinfo", matrixInfo), ("b4csr_bwidth", C.c_uint), ("b4csr_bheight", C.c_uint),
                ("b4csr_row_num", C.c_int), ("b4csr_aligned_size", C.c_int), ("b4csr_block_num", C.c_int),
                ("b4csr_row_ptr", IP), ("b4csr_col_id", IP), ("b4csr_data", FP)]


class b4ell_matrix(C.Structure):
    _fields_ = [("matinfo", matrixInfo), ("b4ell_bwidth", C.c_uint), ("b4ell_bheight", C.c_uint),
                ("b4ell_row_num", C.c_int), ("b4ell_block_num", C.c_int), ("b4ell_height_aligned", C.c_int),
                ("b4ell_float4_aligned", C.c_int), ("b4ell_col_id", IP), ("b4ell_data", FP)]


class sbell_matrix(C.Structure):
    _fields_ = [("matinfo", matrixInfo), ("sbell_bwidth", C.c_uint), ("sbell_bheight", C.c_uint),
                ("sbell_slice_height", C.c_uint), ("sbell_slice_num", C.c_int), ("sbell_row_num", C.c_int),
                ("sbell_slice_ptr", IP), ("sbell_col_id", IP), ("sbell_data", FP)]


class cocktail(C.Structure):
    _fields_ = (
        [(f"ifuse{n}", C.c_bool) for n in ("bdia", "dia", "sbell", "bell", "bcsr", "sell", "ell", "csr", "coo")]
        + [(f"{n}_meth_num", C.c_int) for n in ("bdia", "dia", "sbell", "bell", "bcsr", "sell", "ell", "csr", "coo")]
        + [("csr_group_num", C.c_int), ("coo_group_num", C.c_int),
           ("mat_width", C.c_int), ("mat_height", C.c_int), ("mat_nnz", C.c_int),
           ("bdia", bdia_matrix), ("dia", dia_matrix), ("sbell", sbell_matrix), ("bell", b4ell_matrix),
           ("bcsr", b4csr_matrix), ("sell", sell_matrix), ("ell", ell_matrix), ("csr", csr_matrix),
           ("coo", coo_matrix)]
    )


class csp_analyze_opts(C.Structure):
    _fields_ = [("mode", C.c_int), ("bench_path", C.c_char_p), ("verbose", C.c_int), ("cache_path", C.c_char_p),
                ("flags", C.c_int)]


class csp_batch_opts(C.Structure):
    _fields_ = [("flags", C.c_int), ("format", C.c_int), ("tune", C.c_int), ("cache_path", C.c_char_p)]


class csp_batch_features(C.Structure):
    _fields_ = [("rows", C.c_int), ("cols", C.c_int), ("nnz", C.c_int), ("max_row", C.c_int), ("ndiag", C.c_int),
                ("dia_slots", C.c_longlong), ("sell_slots", C.c_longlong * 2), ("bcsr_blocks", C.c_longlong * 3),
                ("feasible", C.c_uint), ("model_format", C.c_int), ("signature", C.c_ulonglong)]


class csp_bandwidth_report(C.Structure):
    _fields_ = [("launch_us", C.c_double), ("copy_gbs", C.c_double), ("gather_gbs", C.c_double),
                ("gather_per_s", C.c_double)]


class csp_report(C.Structure):
    _fields_ = [("method", C.c_int), ("gflops", C.c_double), ("gbytes", C.c_double), ("ms", C.c_double),
                ("l2_distance", C.c_double), ("max_diff", C.c_double), ("max_ratio_diff", C.c_double),
                ("group_num", C.c_int)]


# ----------------------------------------------------------------------------------
# pointer <-> numpy helpers
# ----------------------------------------------------------------------------------
def as_ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


def to_numpy(ptr, n: int, dtype) -> np.ndarray:
    """Copy n elements behind a struct pointer into a new numpy array."""
    n = int(n)
    if n <= 0 or not ptr:
        return np.zeros(0, dtype=dtype)
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True)


class COO:
    """A coo_matrix whose arrays are owned by numpy (kept alive by this object)."""

    def __init__(self, height: int, width: int, row, col, val):
        self.row = np.ascontiguousarray(row, dtype=np.int32).copy()
        self.col = np.ascontiguousarray(col, dtype=np.int32).copy()
        self.val = np.ascontiguousarray(val, dtype=np.float32).copy()
        self.height, self.width = int(height), int(width)
        self.s = coo_matrix()
        self.s.matinfo.width = self.width
        self.s.matinfo.height = self.height
        self.s.matinfo.nnz = int(self.row.size)
        self.s.coo_row_id = as_ptr(self.row, C.c_int)
        self.s.coo_col_id = as_ptr(self.col, C.c_int)
        self.s.coo_data = as_ptr(self.val, C.c_float)
        # the struct holds the arrays its pointers reference: ref() of a temporary COO
        # (`COO(...).ref()` passed straight to a call) keeps them alive through the call
        self.s._arrays = (self.row, self.col, self.val)

    @property
    def nnz(self) -> int:
        return int(self.row.size)

    def ref(self):
        return C.byref(self.s)


def _declare(lib):
    P = C.POINTER
    sig = {
        "csp_error_string": (C.c_char_p, [C.c_int]),
        "csp_last_error": (C.c_char_p, []),
        "csp_version": (C.c_char_p, []),
        "csp_aligned_length": (C.c_int, [C.c_int, C.c_int]),
        "csp_if_sorted_coo": (C.c_int, [P(coo_matrix)]),
        "csp_sort_coo": (C.c_int, [P(coo_matrix)]),
        "csp_coo2csr": (C.c_int, [P(coo_matrix), P(csr_matrix)]),
        "csp_csr2coo": (C.c_int, [P(csr_matrix), P(coo_matrix)]),
        "csp_coo2ell": (C.c_int, [P(coo_matrix), P(ell_matrix), C.c_int, C.c_int]),
        "csp_ell2coo": (C.c_int, [P(ell_matrix), P(coo_matrix)]),
        "csp_coo2sell": (C.c_int, [P(coo_matrix), P(sell_matrix), C.c_uint]),
        "csp_coo2dia": (C.c_int, [P(coo_matrix), P(dia_matrix), C.c_int]),
        "csp_dia2coo": (C.c_int, [P(dia_matrix), P(coo_matrix)]),
        "csp_coo2bdia": (C.c_int, [P(coo_matrix), P(bdia_matrix), C.c_int]),
        "csp_bdia2coo": (C.c_int, [P(bdia_matrix), P(coo_matrix)]),
        "csp_coo2bcsr": (C.c_int, [P(coo_matrix), P(bcsr_matrix), C.c_uint, C.c_uint, C.c_int]),
        "csp_bcsr2coo": (C.c_int, [P(bcsr_matrix), P(coo_matrix)]),
        "csp_coo2bell": (C.c_int, [P(coo_matrix), P(bell_matrix), C.c_uint, C.c_uint, C.c_int, C.c_int]),
        "csp_bell2coo": (C.c_int, [P(bell_matrix), P(coo_matrix)]),
        "csp_rearrange_bell_4col": (C.c_int, [P(bell_matrix), C.c_int]),
        "csp_coo2b4csr": (C.c_int, [P(coo_matrix), P(b4csr_matrix), C.c_uint, C.c_uint, C.c_int]),
        "csp_coo2b4ell": (C.c_int, [P(coo_matrix), P(b4ell_matrix), C.c_uint, C.c_uint, C.c_int, C.c_int]),
        "csp_coo2sbell": (C.c_int, [P(coo_matrix), P(sbell_matrix), C.c_uint, C.c_uint, C.c_uint]),
        "csp_pad_csr": (C.c_int, [P(csr_matrix), P(csr_matrix), C.c_int]),
        "csp_analyze_matrix": (C.c_int, [P(coo_matrix), P(cocktail), P(csp_analyze_opts)]),
        "csp_init_mat_kernels": (C.c_int, [P(cocktail), FP, FP, C.c_int, P(C.c_void_p)]),
        "csp_do_spmv": (C.c_int, [C.c_void_p, C.c_int]),
        "csp_iterate": (C.c_int, [C.c_void_p, C.c_int]),
        "csp_benchmark_tables": (C.c_int, [C.c_char_p, C.c_int]),
        "csp_init_mat_kernels_ex": (C.c_int, [P(cocktail), FP, FP, C.c_int, C.c_int, P(C.c_void_p)]),
        "csp_init_bcsr_kernels": (C.c_int, [P(bcsr_matrix), FP, FP, C.c_int, C.c_int, P(C.c_void_p)]),
        "csp_synchronize": (C.c_int, [C.c_void_p]),
        "csp_cpy_vector_from_cpu": (C.c_int, [C.c_void_p, FP, C.c_int]),
        "csp_cpy_vector_from_gpu": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
        "csp_cpy_result_from_cpu": (C.c_int, [C.c_void_p, FP, C.c_int]),
        "csp_cpy_result_from_gpu": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
        "csp_cpy_result_to_cpu": (C.c_int, [C.c_void_p, FP, C.c_int]),
        "csp_cpy_result_to_gpu": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
        "csp_free_mat_kernels": (C.c_int, [C.c_void_p]),
        "csp_get_vec_device_ptr": (C.c_int, [C.c_void_p, P(C.c_void_p)]),
        "csp_get_res_device_ptr": (C.c_int, [C.c_void_p, P(C.c_void_p)]),
        "csp_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
        "csp_get_stream": (C.c_int, [C.c_void_p, P(C.c_void_p)]),
        "csp_launches_per_spmv": (C.c_int, [C.c_void_p, P(C.c_int)]),
        "csp_device_bytes": (C.c_int, [C.c_void_p, P(C.c_size_t)]),
        "csp_evaluate": (C.c_int, [P(cocktail), FP, FP, FP, C.c_int, P(csp_report)]),
        "csp_spmv_all": (C.c_int, [P(coo_matrix), C.c_int, C.c_int, P(csp_report)]),
        "csp_read_mmf": (C.c_int, [C.c_char_p, P(coo_matrix)]),
        "csp_read_mmf_ex": (C.c_int, [C.c_char_p, P(coo_matrix), C.c_int]),
        "csp_sort_coo_device": (C.c_int, [P(coo_matrix)]),
        "csp_coo2dia_device": (C.c_int, [P(coo_matrix), P(dia_matrix), C.c_int]),
        "csp_coo2bdia_device": (C.c_int, [P(coo_matrix), P(bdia_matrix), C.c_int]),
        "csp_coo2bcsr_device": (C.c_int, [P(coo_matrix), P(bcsr_matrix), C.c_uint, C.c_uint, C.c_int]),
        "csp_autotune_choice": (C.c_char_p, []),
        "csp_bandwidth_test": (C.c_int, [C.c_size_t, C.c_int, P(csp_bandwidth_report)]),
        "csp_spmv_adjoint": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
        "csp_adjoint_slots": (C.c_int, [C.c_void_p, P(C.c_size_t)]),
        "csp_adjoint_pattern": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
        "csp_coo_spmv_noalloc": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.c_void_p, C.c_void_p]),
        "csp_batch_features_of": (C.c_int, [P(coo_matrix), C.c_int, P(csp_batch_features)]),
        "csp_batch_create": (C.c_int, [P(P(coo_matrix)), C.c_int, P(csp_batch_opts), P(C.c_void_p)]),
        "csp_batch_free": (C.c_int, [C.c_void_p]),
        "csp_batch_layout": (C.c_int, [C.c_void_p, P(C.c_longlong), P(C.c_longlong), P(C.c_longlong)]),
        "csp_batch_formats_adjoint": (C.c_int, [C.c_void_p, P(C.c_int)]),
        "csp_batch_formats": (C.c_int, [C.c_void_p, IP]),
        "csp_batch_device_ptrs": (C.c_int, [C.c_void_p, P(C.c_void_p), P(C.c_void_p), P(C.c_void_p), P(C.c_void_p),
                                            P(C.c_void_p)]),
        "csp_batch_copy": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
        "csp_batch_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
        "csp_batch_get_stream": (C.c_void_p, [C.c_void_p]),
        "csp_batch_run": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
        "csp_batch_run_plain": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int]),
        "csp_batch_synchronize": (C.c_int, [C.c_void_p]),
        "csp_batch_launches": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
        "csp_batch_device_bytes": (C.c_size_t, [C.c_void_p]),
        "csp_batch_pattern": (C.c_int, [C.c_void_p, C.c_int, IP, IP]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    for fmt in ("coo", "csr", "ell", "sell", "dia", "bdia", "bcsr", "bell", "b4csr", "b4ell", "sbell"):
        cls = {"coo": coo_matrix, "csr": csr_matrix, "ell": ell_matrix, "sell": sell_matrix, "dia": dia_matrix,
               "bdia": bdia_matrix, "bcsr": bcsr_matrix, "bell": bell_matrix, "b4csr": b4csr_matrix,
               "b4ell": b4ell_matrix, "sbell": sbell_matrix}[fmt]
        for pre in ("csp_init_", "csp_free_"):
            fn = getattr(lib, f"{pre}{fmt}_matrix")
            fn.restype = None
            fn.argtypes = [P(cls)]
    for pre in ("csp_init_cocktail", "csp_free_cocktail"):
        fn = getattr(lib, pre)
        fn.restype = None
        fn.argtypes = [P(cocktail)]
    for drv in ("csr_scalar", "csr_vector", "bdia", "dia", "ell", "sell", "coo", "bell", "bcsr", "sbell"):
        fn = getattr(lib, f"csp_spmv_{drv}")
        fn.restype = C.c_int
        fn.argtypes = [P(coo_matrix), C.c_int, P(csp_report)]
    return lib


_lib = None


def lib():
    """The loaded libclspmv_b200.so.  Raises if the library has not been built:
    there is no fallback implementation."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing; build it with `make -C clspmv_b200/csrc` "
                "(or __graft_entry__.build()).  There is no CPU fallback.")
        _lib = _declare(C.CDLL(LIB_PATH))
    return _lib


class CspError(RuntimeError):
    def __init__(self, code: int, where: str):
        l = lib()
        super().__init__(f"{where}: {l.csp_error_string(code).decode()} ({l.csp_last_error().decode()})")
        self.code = code


def check(code: int, where: str = "csp"):
    if code != CSP_OK:
        raise CspError(code, where)
    return code
