"""Loads the test oracles (oracle/liboracle.so, oracle/_ref/libclspmv_ref.so) and
wraps them for the tests.  Test infrastructure only."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from clspmv_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE = os.path.join(ROOT, "oracle", "liboracle.so")
REF = os.path.join(ROOT, "oracle", "_ref", "libclspmv_ref.so")
REF_BENCH = os.path.join(ROOT, "oracle", "_ref", "clSpMV_NV")

_orc = None
_ref = None
IP, FP, DP = C.POINTER(C.c_int), C.POINTER(C.c_float), C.POINTER(C.c_double)


def oracle_lib():
    global _orc
    if _orc is None:
        if not os.path.exists(ORACLE):
            raise RuntimeError("oracle/liboracle.so missing: run `make -C oracle`")
        l = C.CDLL(ORACLE)
        l.orc_csr_spmv_f64.argtypes = [C.c_int, C.c_int, IP, IP, FP, FP, FP, C.c_double, C.c_int, DP, DP]
        l.orc_csr_value_grad_f32.argtypes = [C.c_int, IP, IP, FP, FP, FP]
        l.orc_max_rel_err.argtypes = [C.c_int, FP, DP, DP, IP]
        l.orc_max_rel_err.restype = C.c_double
        l.orc_csr_spmv_f32.argtypes = [C.c_int, IP, IP, FP, FP, FP]
        l.orc_coo_spmv_f32.argtypes = [C.c_int, IP, IP, FP, FP, FP]
        l.orc_two_vec_compare.argtypes = [C.c_int, FP, FP, DP]
        _orc = l
    return _orc


def ref_lib():
    """The reference's own host code (compiled from its sources), or None."""
    global _ref
    if _ref is None:
        if not os.path.exists(REF):
            return None
        l = C.CDLL(REF)
        P = C.POINTER
        for name, args in {
            "ref_if_sorted_coo": [P(capi.coo_matrix)], "ref_sort_coo": [P(capi.coo_matrix)],
            "ref_coo2csr": [P(capi.coo_matrix), P(capi.csr_matrix)],
            "ref_coo2ell": [P(capi.coo_matrix), P(capi.ell_matrix), C.c_int, C.c_int],
            "ref_ell2coo": [P(capi.ell_matrix), P(capi.coo_matrix)],
            "ref_coo2sell": [P(capi.coo_matrix), P(capi.sell_matrix), C.c_uint],
            "ref_coo2dia": [P(capi.coo_matrix), P(capi.dia_matrix), C.c_int],
            "ref_dia2coo": [P(capi.dia_matrix), P(capi.coo_matrix)],
            "ref_coo2bdia": [P(capi.coo_matrix), P(capi.bdia_matrix), C.c_int],
            "ref_bdia2coo": [P(capi.bdia_matrix), P(capi.coo_matrix)],
            "ref_coo2bcsr": [P(capi.coo_matrix), P(capi.bcsr_matrix), C.c_uint, C.c_uint, C.c_int],
            "ref_bcsr2coo": [P(capi.bcsr_matrix), P(capi.coo_matrix)],
            "ref_coo2bell": [P(capi.coo_matrix), P(capi.bell_matrix), C.c_uint, C.c_uint, C.c_int, C.c_int],
            "ref_bell2coo": [P(capi.bell_matrix), P(capi.coo_matrix)],
            "ref_coo2b4csr": [P(capi.coo_matrix), P(capi.b4csr_matrix), C.c_uint, C.c_uint, C.c_int],
            "ref_coo2b4ell": [P(capi.coo_matrix), P(capi.b4ell_matrix), C.c_uint, C.c_uint, C.c_int, C.c_int],
            "ref_coo2sbell": [P(capi.coo_matrix), P(capi.sbell_matrix), C.c_uint, C.c_uint, C.c_uint],
            "ref_pad_csr": [P(capi.csr_matrix), P(capi.csr_matrix), C.c_int],
            "ref_rearrange_bell_4col": [P(capi.bell_matrix), C.c_int],
            "ref_dia_spmv": [P(capi.dia_matrix), FP, FP, C.c_int],
            "ref_bdia_spmv": [P(capi.bdia_matrix), FP, FP, C.c_int],
            "ref_ell_spmv": [P(capi.ell_matrix), FP, FP, C.c_int],
            "ref_sell_spmv": [P(capi.sell_matrix), FP, FP, C.c_int],
            "ref_sbell_spmv": [P(capi.sbell_matrix), FP, FP, C.c_int],
            "ref_coo_spmv": [P(capi.coo_matrix), FP, FP, C.c_int],
            "ref_csr_spmv": [P(capi.csr_matrix), FP, FP, C.c_int],
            "ref_bcsr_spmv": [P(capi.bcsr_matrix), FP, FP, C.c_int],
            "ref_bell_spmv": [P(capi.bell_matrix), FP, FP, C.c_int],
            "ref_analyze_matrix": [P(capi.coo_matrix), P(capi.cocktail), C.c_int],
            "ref_free_cocktail": [P(capi.cocktail)],
            "ref_read_mmf": [C.c_char_p, P(capi.coo_matrix)],
            "ref_free": [C.c_void_p],
        }.items():
            fn = getattr(l, name)
            fn.argtypes = args
        for name in ("ref_if_sorted_coo", "ref_sort_coo", "ref_coo2dia", "ref_coo2bdia", "ref_coo2b4csr",
                     "ref_coo2b4ell", "ref_coo2sbell"):
            getattr(l, name).restype = C.c_int
        _ref = l
    return _ref


# The per-row FP32 bound the parity tests apply: |y_i - yhat_i| <= TOL * bound_i with
# bound_i = sum_j |a_ij x_j| + Y0_WEIGHT * |y0_i|, i.e. 1e-5 * sum_j |a_ij x_j| plus
# 2^-23 * |y0_i| for the final FP32 add of the accumulated vector.
TOL = 1e-5
Y0_WEIGHT = 2.0 ** -23 / TOL


def fp64_spmv(h, w, rp, col, val, x, y0=None, transpose=False, y0_weight=Y0_WEIGHT):
    """FP64 reference product y0 + A x (or A^T x) and the per-row error scale
    sum_j |a_ij x_j| + y0_weight * |y0_i|."""
    l = oracle_lib()
    rp = np.ascontiguousarray(rp, np.int32)
    col = np.ascontiguousarray(col, np.int32)
    val = np.ascontiguousarray(val, np.float32)
    x = np.ascontiguousarray(x, np.float32)
    n_out = w if transpose else h
    y0p = None
    if y0 is not None:
        y0 = np.ascontiguousarray(y0, np.float32)
        y0p = y0.ctypes.data_as(FP)
    out = np.zeros(n_out, np.float64)
    bound = np.zeros(n_out, np.float64)
    l.orc_csr_spmv_f64(h, w, rp.ctypes.data_as(IP), col.ctypes.data_as(IP), val.ctypes.data_as(FP),
                       x.ctypes.data_as(FP), y0p, float(y0_weight), 1 if transpose else 0, out.ctypes.data_as(DP),
                       bound.ctypes.data_as(DP))
    return out, bound


def y0_term(y0, adds: int = 1):
    """The bound's share for an accumulated vector y0 that `adds` FP32 additions update."""
    return Y0_WEIGHT * adds * np.abs(np.asarray(y0, np.float64))


def max_rel_err(y, yhat, bound):
    l = oracle_lib()
    y = np.ascontiguousarray(y, np.float32)
    worst = C.c_int()
    e = l.orc_max_rel_err(y.size, y.ctypes.data_as(FP), yhat.ctypes.data_as(DP), bound.ctypes.data_as(DP),
                          C.byref(worst))
    return e, worst.value
