"""torch.autograd binding of the Cocktail SpMV, for verification only.

    op = SpMVOperator(height, width, rows, cols)             # the sparsity pattern (COO)
    y = CocktailSpMV.apply(x, y0, values, op)                 # y = y0 + A(values) x
    backward:  x.grad      = A^T ybar                 (csp_spmv_adjoint, transposed parts)
               y0.grad     = ybar
               values.grad = ybar[row_e] * x[col_e]   (csp_spmv_adjoint's value gradients,
                                                       mapped from stored slots to entries)

`values` holds one value per COO entry of the pattern.  Each forward builds a handle
(CSP_FLAG_ADJOINT) from the pattern and the given values, in the format the operator
names: "auto" (the on-device autotuner), a (format, method) pair for
Cocktail.single, or "gbcsr" with a block shape (csp_init_bcsr_kernels).  The
library's stream and torch's are synchronized at the boundary, which is fine for
checking and not meant for speed.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import (COO, CSP_ANALYZE_AUTOTUNE, CSP_FLAG_ADJOINT, Cocktail, Handle, analyze_matrix, capi)


class SpMVOperator:
    """The pattern (height, width, rows, cols) of a sparse matrix and the storage its
    handles use."""

    def __init__(self, height: int, width: int, rows, cols, fmt="auto", block=(3, 3)):
        self.height, self.width = int(height), int(width)
        self.rows = np.ascontiguousarray(rows, np.int32)
        self.cols = np.ascontiguousarray(cols, np.int32)
        self.fmt = fmt
        self.block = block
        self._keep = []

    def handle(self, values: np.ndarray) -> Handle:
        """A CSP_FLAG_ADJOINT handle of the matrix with these entry values."""
        coo = COO(self.height, self.width, self.rows.copy(), self.cols.copy(),
                  np.ascontiguousarray(values, np.float32))
        if self.fmt == "gbcsr":
            b = capi.bcsr_matrix()
            capi.check(capi.lib().csp_coo2bcsr(coo.ref(), C.byref(b), int(self.block[0]), int(self.block[1]), 32),
                       "coo2bcsr")
            h = Handle(None, None, None, CSP_FLAG_ADJOINT, bcsr=b)
            capi.lib().csp_free_bcsr_matrix(C.byref(b))
            return h
        if self.fmt == "auto":
            mat = analyze_matrix(coo, mode=CSP_ANALYZE_AUTOTUNE)
        else:
            name, method = self.fmt
            mat = Cocktail.single(name, coo, method)
        h = Handle(mat, None, None, CSP_FLAG_ADJOINT)
        mat.free()
        return h

    def entry_gradient(self, abar: torch.Tensor, srows: torch.Tensor, scols: torch.Tensor) -> torch.Tensor:
        """Gradient per COO entry from the per-slot gradients: every slot of an entry's
        (row, col) holds ybar[row] * x[col], so each entry takes the value of any one."""
        dev = abar.device
        ok = srows >= 0
        w = max(self.width, 1)
        skey = srows[ok].long() * w + scols[ok].long()
        sval = abar[ok]
        skey, order = torch.sort(skey)
        sval = sval[order]
        ekey = torch.from_numpy(self.rows.astype(np.int64) * w + self.cols).to(dev)
        idx = torch.searchsorted(skey, ekey).clamp_(max=max(skey.numel() - 1, 0))
        if skey.numel() == 0 or not torch.equal(skey[idx], ekey):
            raise RuntimeError("a matrix entry has no stored slot")
        return sval[idx]


class CocktailSpMV(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x: torch.Tensor, y0: torch.Tensor, values: torch.Tensor, op: SpMVOperator):
        handle = op.handle(values.detach().float().cpu().numpy())
        x = x.detach().contiguous().float()
        y0 = y0.detach().contiguous().float()
        torch.cuda.current_stream(x.device).synchronize()
        handle.cpy_vector_from_gpu(x.data_ptr(), handle.width)
        handle.cpy_result_from_gpu(y0.data_ptr(), handle.height)
        handle.do_spmv(1)
        y = torch.empty(handle.height, dtype=torch.float32, device=x.device)
        handle.cpy_result_to_gpu(y.data_ptr(), handle.height)
        handle.synchronize()
        ctx.handle = handle
        ctx.op = op
        return y

    @staticmethod
    def backward(ctx, ybar: torch.Tensor):
        h, op = ctx.handle, ctx.op
        ybar = ybar.detach().contiguous().float()
        xbar = torch.zeros(h.width, dtype=torch.float32, device=ybar.device)
        torch.cuda.current_stream(ybar.device).synchronize()
        h.spmv_adjoint(ybar.data_ptr(), xbar.data_ptr(), None)
        abar, rows, cols = value_gradient(h, ybar)
        gvals = op.entry_gradient(abar, rows, cols)
        h.free()
        return xbar, ybar, gvals, None


def value_gradient(handle: Handle, ybar: torch.Tensor):
    """(abar, rows, cols): abar[s] = ybar[rows[s]] * x[cols[s]] over the stored slots."""
    n = handle.adjoint_slots
    dev = ybar.device
    abar = torch.empty(n, dtype=torch.float32, device=dev)
    rows = torch.empty(n, dtype=torch.int32, device=dev)
    cols = torch.empty(n, dtype=torch.int32, device=dev)
    ybar = ybar.detach().contiguous().float()
    torch.cuda.current_stream(dev).synchronize()
    handle.spmv_adjoint(ybar.data_ptr(), None, abar.data_ptr())
    handle.adjoint_pattern(rows.data_ptr(), cols.data_ptr())
    handle.synchronize()
    return abar, rows, cols
