"""Batched SpMV: many matrices in one persistent launch (csp_batch_* in clspmv.h).

    b = Batch([coo0, coo1, ...], flags=CSP_FLAG_ADJOINT | CSP_FLAG_GRAPH, tune=CSP_BATCH_TUNE_DEVICE)
    b.copy_in(CSP_BV_X, x_all); b.copy_in(CSP_BV_YBAR, ybar_all)
    b.run(CSP_BATCH_FWD | CSP_BATCH_ADJ)          # one kernel launch
    y_all = b.copy_out(CSP_BV_Y)

Vectors are the concatenation of the matrices' vectors in batch order; `layout()`
returns the offsets.  No counterpart in the reference, whose engine serves one
cocktail at a time (spmv_cocktail.h:111-175).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi
from .capi import (BFMT_NAMES, CSP_BATCH_ADJ, CSP_BATCH_FWD, CSP_BATCH_TUNE_DEVICE, CSP_BATCH_TUNE_MODEL,
                   CSP_BFMT_AUTO, CSP_BV_ABAR, CSP_BV_X, CSP_BV_XBAR, CSP_BV_Y, CSP_BV_YBAR, COO, check, lib)

__all__ = ["Batch", "features", "BFMT_NAMES", "CSP_BATCH_FWD", "CSP_BATCH_ADJ", "CSP_BATCH_TUNE_MODEL",
           "CSP_BATCH_TUNE_DEVICE", "CSP_BFMT_AUTO", "CSP_BV_X", "CSP_BV_Y", "CSP_BV_YBAR", "CSP_BV_XBAR",
           "CSP_BV_ABAR"]


def features(coo: COO, flags: int = 0) -> dict:
    """csp_batch_features_of: the structure figures the format choice uses."""
    f = capi.csp_batch_features()
    check(lib().csp_batch_features_of(coo.ref(), int(flags), C.byref(f)), "batch_features_of")
    return {"rows": f.rows, "cols": f.cols, "nnz": f.nnz, "max_row": f.max_row, "ndiag": f.ndiag,
            "dia_slots": f.dia_slots, "sell_slots": list(f.sell_slots), "bcsr_blocks": list(f.bcsr_blocks),
            "feasible": f.feasible, "model_format": f.model_format, "signature": f.signature}


class Batch:
    """A csp_batch over a list of COO matrices."""

    def __init__(self, mats: list[COO], flags: int = 0, fmt: int = CSP_BFMT_AUTO,
                 tune: int = CSP_BATCH_TUNE_MODEL, cache_path: str | None = None):
        self.mats = list(mats)
        self.n = len(self.mats)
        arr = (C.POINTER(capi.coo_matrix) * self.n)(*[C.pointer(m.s) for m in self.mats])
        o = capi.csp_batch_opts(int(flags), int(fmt), int(tune), cache_path.encode() if cache_path else None)
        h = C.c_void_p()
        check(lib().csp_batch_create(arr, self.n, C.byref(o), C.byref(h)), "batch_create")
        self.h = h
        off = [(C.c_longlong * (self.n + 1))() for _ in range(3)]
        check(lib().csp_batch_layout(self.h, off[0], off[1], off[2]), "batch_layout")
        self.x_off, self.y_off, self.abar_off = (np.array(list(a), dtype=np.int64) for a in off)
        f = (C.c_int * self.n)()
        check(lib().csp_batch_formats(self.h, f), "batch_formats")
        self.formats = list(f)
        self.formats_adjoint = None
        if flags & capi.CSP_FLAG_ADJOINT:
            ft = (C.c_int * self.n)()
            check(lib().csp_batch_formats_adjoint(self.h, ft), "batch_formats_adjoint")
            self.formats_adjoint = list(ft)

    def _len(self, which: int) -> int:
        if which in (CSP_BV_X, CSP_BV_XBAR):
            return int(self.x_off[-1])
        if which in (CSP_BV_Y, CSP_BV_YBAR):
            return int(self.y_off[-1])
        return int(self.abar_off[-1])

    def copy_in(self, which: int, host: np.ndarray):
        a = np.ascontiguousarray(host, dtype=np.float32)
        if a.size != self._len(which):
            raise ValueError(f"vector {which}: {a.size} entries, expected {self._len(which)}")
        check(lib().csp_batch_copy(self.h, int(which), a.ctypes.data_as(C.c_void_p), None), "batch_copy")
        lib().csp_batch_synchronize(self.h)

    def copy_out(self, which: int) -> np.ndarray:
        out = np.empty(self._len(which), dtype=np.float32)
        check(lib().csp_batch_copy(self.h, int(which), None, out.ctypes.data_as(C.c_void_p)), "batch_copy")
        return out

    def device_ptrs(self) -> dict:
        p = [C.c_void_p() for _ in range(5)]
        check(lib().csp_batch_device_ptrs(self.h, *[C.byref(q) for q in p]), "batch_device_ptrs")
        return dict(zip(("x", "y", "ybar", "xbar", "abar"), (q.value or 0 for q in p)))

    def run(self, what: int = CSP_BATCH_FWD, ntimes: int = 1):
        check(lib().csp_batch_run(self.h, int(what), int(ntimes)), "batch_run")

    def run_plain(self, what: int = CSP_BATCH_FWD, ntimes: int = 1, lanes: int = 0):
        check(lib().csp_batch_run_plain(self.h, int(what), int(ntimes), int(lanes)), "batch_run_plain")

    def synchronize(self):
        check(lib().csp_batch_synchronize(self.h), "batch_synchronize")

    def set_stream(self, stream_ptr: int | None):
        check(lib().csp_batch_set_stream(self.h, C.c_void_p(stream_ptr or 0)), "batch_set_stream")

    def launches(self, what: int, plain: bool = False) -> int:
        return int(lib().csp_batch_launches(self.h, int(what), int(bool(plain))))

    def device_bytes(self) -> int:
        return int(lib().csp_batch_device_bytes(self.h))

    def pattern(self, i: int) -> tuple[np.ndarray, np.ndarray]:
        n = int(self.abar_off[i + 1] - self.abar_off[i])
        rows = np.empty(n, dtype=np.int32)
        cols = np.empty(n, dtype=np.int32)
        check(lib().csp_batch_pattern(self.h, int(i), capi.as_ptr(rows, C.c_int), capi.as_ptr(cols, C.c_int)),
              "batch_pattern")
        return rows, cols

    def free(self):
        if self.h:
            lib().csp_batch_free(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass
