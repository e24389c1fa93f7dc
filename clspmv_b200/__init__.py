"""clspmv_b200 -- B200-native Cocktail SpMV (y += A*x) behind the clSpMV interface.

Python host mirror of the reference's C++ API for the hot path
(clSpMV_NV/include/spmv_cocktail.h:111-175, analyze.h:257, spmv_*.h:7):

    coo = COO(height, width, row, col, val)        # coo_matrix<int, float>
    mat = analyze_matrix(coo)                        # analyze.cpp:3704 analyze_matrix
    h = init_mat_kernels(mat, vec, res)              # spmv_cocktail.cpp:1593
    h.cpy_result_from_cpu(res)                       # :1562
    h.do_spmv(1)                                     # :1091  res += A * vec
    h.cpy_vector_from_gpu(h.res_ptr, n)              # :1513
    y = h.cpy_result_to_cpu()                        # :1578
    h.free()                                         # :1616 free_mat_kernels

Everything runs through libclspmv_b200.so (hand-written sm_100a CUDA); there is no
CPU fallback: a missing library or device raises.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi
from .capi import (COO, CSP_ANALYZE_AUTOTUNE, CSP_ANALYZE_REFERENCE, CSP_FLAG_ADJOINT, CSP_FLAG_BF16,
                   CSP_FLAG_L2_PERSIST, CSP_FLAG_TENSOR_CORES, CSP_METH_XPANEL,
                   CSP_FLAG_GRAPH, CSP_FLAG_USE_TEX, CspError, check, lib, to_numpy)

__all__ = ["COO", "Cocktail", "Handle", "analyze_matrix", "init_mat_kernels", "spmv_all", "evaluate",
           "CspError", "CSP_FLAG_BF16", "CSP_FLAG_GRAPH", "CSP_FLAG_USE_TEX", "CSP_FLAG_ADJOINT",
           "CSP_FLAG_L2_PERSIST", "CSP_FLAG_TENSOR_CORES", "CSP_METH_XPANEL", "benchmark_tables",
           "CSP_ANALYZE_REFERENCE", "CSP_ANALYZE_AUTOTUNE", "lib", "Batch"]

from .batch import Batch  # noqa: E402

FORMATS = ("bdia", "dia", "sbell", "bell", "bcsr", "sell", "ell", "csr", "coo")


class Cocktail:
    """A cocktail<int, int, float>: one optional sub-matrix per format.  Arrays
    written by the library (conversions, analyzer) are released by free()."""

    def __init__(self, height: int = 0, width: int = 0, nnz: int = 0):
        self.s = capi.cocktail()
        lib().csp_init_cocktail(C.byref(self.s))
        self.s.mat_width, self.s.mat_height, self.s.mat_nnz = int(width), int(height), int(nnz)
        self._keep = []   # numpy arrays referenced by borrowed struct pointers
        self._owned = True

    @classmethod
    def single(cls, fmt: str, coo: COO, method: int = 0, **kw) -> "Cocktail":
        """A cocktail holding the whole matrix in one format, converted by the
        library (coo2csr, coo2ell, ...).  kw: alignment, ellnum, slice_height,
        bwidth, bheight."""
        c = cls(coo.height, coo.width, coo.nnz)
        L = lib()
        s = c.s
        al = kw.get("alignment", 32)
        if fmt == "csr":
            check(L.csp_coo2csr(coo.ref(), C.byref(s.csr)), "coo2csr")
        elif fmt == "ell":
            check(L.csp_coo2ell(coo.ref(), C.byref(s.ell), al, kw.get("ellnum", 0)), "coo2ell")
        elif fmt == "sell":
            check(L.csp_coo2sell(coo.ref(), C.byref(s.sell), kw.get("slice_height", 32)), "coo2sell")
        elif fmt == "dia":
            check(L.csp_coo2dia(coo.ref(), C.byref(s.dia), al), "coo2dia")
        elif fmt == "bdia":
            check(L.csp_coo2bdia(coo.ref(), C.byref(s.bdia), al), "coo2bdia")
        elif fmt == "bell":
            check(L.csp_coo2b4ell(coo.ref(), C.byref(s.bell), kw.get("bwidth", 4), kw.get("bheight", 1), al,
                                  kw.get("ellnum", 0)), "coo2b4ell")
        elif fmt == "bcsr":
            check(L.csp_coo2b4csr(coo.ref(), C.byref(s.bcsr), kw.get("bwidth", 4), kw.get("bheight", 1), al),
                  "coo2b4csr")
        elif fmt == "sbell":
            check(L.csp_coo2sbell(coo.ref(), C.byref(s.sbell), kw.get("bwidth", 4), kw.get("bheight", 1),
                                  kw.get("slice_height", 32)), "coo2sbell")
        elif fmt == "coo":
            # borrow the caller's arrays (sorted); not freed by the library
            check(L.csp_sort_coo(coo.ref()) if not L.csp_if_sorted_coo(coo.ref()) else 0, "sort_coo")
            s.coo = coo.s
            c._keep.append(coo)
            c._borrowed_coo = True
        else:
            raise ValueError(fmt)
        setattr(s, f"ifuse{fmt}", True)
        setattr(s, f"{fmt}_meth_num", int(method))
        return c

    def uses(self):
        return [f for f in FORMATS if getattr(self.s, f"ifuse{f}")]

    def ref(self):
        return C.byref(self.s)

    def free(self):
        if self._owned:
            if getattr(self, "_borrowed_coo", False):
                self.s.coo = capi.coo_matrix()
            lib().csp_free_cocktail(C.byref(self.s))
            self._owned = False

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def analyze_matrix(coo: COO, mode: int = CSP_ANALYZE_REFERENCE, bench_path: str | None = None,
                   verbose: int = 0, cache_path: str | None = None, flags: int = 0) -> Cocktail:
    """Partition `coo` into per-format sub-matrices (analyze.cpp:3704).  `coo` may be
    sorted in place, as in the reference.  mode=CSP_ANALYZE_AUTOTUNE measures candidate
    partitions on the device instead of predicting from the clSpMV tables."""
    c = Cocktail()
    opts = capi.csp_analyze_opts(mode, bench_path.encode() if bench_path else None, verbose,
                                 cache_path.encode() if cache_path else None, flags)
    check(lib().csp_analyze_matrix(coo.ref(), c.ref(), C.byref(opts)), "analyze_matrix")
    if mode == CSP_ANALYZE_AUTOTUNE:
        c.choice = lib().csp_autotune_choice().decode()
    return c


class Handle:
    """Device engine of one cocktail (cocktail_gpu + cocktail_kernels of the reference)."""

    def __init__(self, mat: Cocktail | None, vec: np.ndarray | None = None, res: np.ndarray | None = None,
                 flags: int = 0, nrhs: int = 1, bcsr=None):
        """A handle over `mat` (a Cocktail), or over a generic BCSR struct `bcsr`
        (csp_init_bcsr_kernels).  With nrhs > 1, vec is width x nrhs and res height x nrhs,
        row-major."""
        self._mat = mat if mat is not None else bcsr
        self.nrhs = int(nrhs)
        v = None if vec is None else np.ascontiguousarray(vec, dtype=np.float32)
        r = None if res is None else np.ascontiguousarray(res, dtype=np.float32)
        vp = None if v is None else capi.as_ptr(v, C.c_float)
        rp = None if r is None else capi.as_ptr(r, C.c_float)
        h = C.c_void_p()
        if bcsr is not None:
            self.width, self.height = int(bcsr.matinfo.width), int(bcsr.matinfo.height)
            check(lib().csp_init_bcsr_kernels(C.byref(bcsr), vp, rp, self.nrhs, int(flags), C.byref(h)),
                  "init_bcsr_kernels")
        else:
            self.width, self.height = int(mat.s.mat_width), int(mat.s.mat_height)
            check(lib().csp_init_mat_kernels_ex(mat.ref(), vp, rp, self.nrhs, int(flags), C.byref(h)),
                  "init_mat_kernels")
        self.h = h

    def do_spmv(self, ntimes: int = 1):
        check(lib().csp_do_spmv(self.h, int(ntimes)), "do_spmv")

    def iterate(self, iterations: int):
        """eval.cpp:19 example() on the device: `iterations` times res += A*vec; vec = res."""
        check(lib().csp_iterate(self.h, int(iterations)), "iterate")

    def synchronize(self):
        check(lib().csp_synchronize(self.h), "synchronize")

    def cpy_vector_from_cpu(self, vec: np.ndarray):
        v = np.ascontiguousarray(vec, dtype=np.float32)
        check(lib().csp_cpy_vector_from_cpu(self.h, capi.as_ptr(v, C.c_float), v.size), "cpy_vector_from_cpu")

    def cpy_vector_from_gpu(self, dptr: int, n: int):
        check(lib().csp_cpy_vector_from_gpu(self.h, C.c_void_p(dptr), int(n)), "cpy_vector_from_gpu")

    def cpy_result_from_cpu(self, res: np.ndarray):
        r = np.ascontiguousarray(res, dtype=np.float32)
        check(lib().csp_cpy_result_from_cpu(self.h, capi.as_ptr(r, C.c_float), r.size), "cpy_result_from_cpu")

    def cpy_result_from_gpu(self, dptr: int, n: int):
        check(lib().csp_cpy_result_from_gpu(self.h, C.c_void_p(dptr), int(n)), "cpy_result_from_gpu")

    def cpy_result_to_cpu(self, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty(self.height * self.nrhs, dtype=np.float32)
        check(lib().csp_cpy_result_to_cpu(self.h, capi.as_ptr(out, C.c_float), out.size), "cpy_result_to_cpu")
        return out

    def cpy_result_to_gpu(self, dptr: int, n: int):
        check(lib().csp_cpy_result_to_gpu(self.h, C.c_void_p(dptr), int(n)), "cpy_result_to_gpu")

    @property
    def vec_ptr(self) -> int:
        p = C.c_void_p()
        check(lib().csp_get_vec_device_ptr(self.h, C.byref(p)), "vec ptr")
        return int(p.value)

    @property
    def res_ptr(self) -> int:
        p = C.c_void_p()
        check(lib().csp_get_res_device_ptr(self.h, C.byref(p)), "res ptr")
        return int(p.value)

    def set_stream(self, stream_ptr: int | None):
        check(lib().csp_set_stream(self.h, C.c_void_p(stream_ptr) if stream_ptr else None), "set_stream")

    @property
    def stream(self) -> int:
        p = C.c_void_p()
        check(lib().csp_get_stream(self.h, C.byref(p)), "get_stream")
        return int(p.value or 0)

    @property
    def launches_per_spmv(self) -> int:
        n = C.c_int()
        check(lib().csp_launches_per_spmv(self.h, C.byref(n)), "launches")
        return n.value

    @property
    def device_bytes(self) -> int:
        n = C.c_size_t()
        check(lib().csp_device_bytes(self.h, C.byref(n)), "device_bytes")
        return n.value

    # --- adjoint (handle built with CSP_FLAG_ADJOINT) ---
    def spmv_adjoint(self, ybar_ptr: int, xbar_ptr: int | None = None, abar_ptr: int | None = None):
        """xbar += A^T ybar and abar = ybar[row] * x[col] per stored slot (device pointers)."""
        check(lib().csp_spmv_adjoint(self.h, C.c_void_p(ybar_ptr), C.c_void_p(xbar_ptr) if xbar_ptr else None,
                                     C.c_void_p(abar_ptr) if abar_ptr else None), "spmv_adjoint")

    @property
    def adjoint_slots(self) -> int:
        n = C.c_size_t()
        check(lib().csp_adjoint_slots(self.h, C.byref(n)), "adjoint_slots")
        return n.value

    def adjoint_pattern(self, rows_ptr: int, cols_ptr: int):
        check(lib().csp_adjoint_pattern(self.h, C.c_void_p(rows_ptr), C.c_void_p(cols_ptr)), "adjoint_pattern")

    def free(self):
        if self.h:
            lib().csp_free_mat_kernels(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def benchmark_tables(clspmv_path: str, level: int = 1) -> None:
    """Write the analyzer's calibration tables, measured on this GPU, under
    clspmv_path/benchmark (the reference's bench_* programs; csp_benchmark_tables).
    analyze_matrix(coo, bench_path=clspmv_path) then partitions from them."""
    check(lib().csp_benchmark_tables(clspmv_path.encode(), int(level)), "benchmark_tables")


def init_mat_kernels(mat: Cocktail, vec=None, res=None, flags: int = 0) -> Handle:
    return Handle(mat, vec, res, flags)


def _report(r: capi.csp_report) -> dict:
    return {k: getattr(r, k) for k, _ in capi.csp_report._fields_}


def spmv_all(coo: COO, method: int, ntimes: int = 20) -> dict:
    """spmv_all method 1-10 (spmv_all.cpp:196): best kernel variant of one format."""
    r = capi.csp_report()
    check(lib().csp_spmv_all(coo.ref(), int(method), int(ntimes), C.byref(r)), f"spmv_all {method}")
    return _report(r)


def evaluate(mat: Cocktail, vec, res, coores, ntimes: int = 1000) -> dict:
    """Check one SpMV against `coores` and time `ntimes` (spmv_cocktail.cpp:1434)."""
    v = np.ascontiguousarray(vec, dtype=np.float32)
    r = np.ascontiguousarray(res, dtype=np.float32)
    c = np.ascontiguousarray(coores, dtype=np.float32)
    rep = capi.csp_report()
    check(lib().csp_evaluate(mat.ref(), capi.as_ptr(v, C.c_float), capi.as_ptr(r, C.c_float),
                             capi.as_ptr(c, C.c_float), int(ntimes), C.byref(rep)), "evaluate")
    return _report(rep)
