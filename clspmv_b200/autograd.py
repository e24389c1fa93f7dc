"""torch.autograd binding of the Cocktail SpMV, for verification only.

    y = CocktailSpMV.apply(x, y0, handle)       # y = y0 + A x   (csp_do_spmv)
    backward: x.grad = A^T ybar  (csp_spmv_adjoint), y0.grad = ybar

The handle must be built with CSP_FLAG_ADJOINT.  The gradient with respect to the
stored values is not an autograd input (the values live in the handle); it is
available as value_gradient(handle, ybar) in the handle's stored-slot order.  The
library's stream and torch's are synchronized at the boundary, which is fine for
checking and not meant for speed.
"""
from __future__ import annotations

import torch

from . import Handle


class CocktailSpMV(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x: torch.Tensor, y0: torch.Tensor, handle: Handle):
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
        return y

    @staticmethod
    def backward(ctx, ybar: torch.Tensor):
        h = ctx.handle
        ybar = ybar.detach().contiguous().float()
        xbar = torch.zeros(h.width, dtype=torch.float32, device=ybar.device)
        torch.cuda.current_stream(ybar.device).synchronize()
        h.spmv_adjoint(ybar.data_ptr(), xbar.data_ptr(), None)
        h.synchronize()
        return xbar, ybar, None


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
