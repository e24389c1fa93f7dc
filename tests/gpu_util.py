"""Helpers for the GPU parity tests: run a cocktail on the device through the C ABI
and check it against the FP64 oracle with the per-row bound
|y_i - yhat_i| <= 1e-5 * sum_j |a_ij x_j| + 2^-23 * |y0_i| (per SpMV)."""
from __future__ import annotations

import numpy as np

from clspmv_b200 import COO, Cocktail, Handle
from clspmv_b200.matrices import csr_from_coo
from tests import _oracle

TOL = _oracle.TOL  # FP32 per-row tolerance relative to sum |a_ij x_j|


def run(mat: Cocktail, x, y0, ntimes: int = 1, flags: int = 0):
    h = Handle(mat, x, y0, flags)
    try:
        h.do_spmv(ntimes)
        return h.cpy_result_to_cpu()
    finally:
        h.free()


def row_sorted(h, w, r, c, v):
    """The COO sorted by (row, col); returned as is when it already is."""
    if r.size > 1:
        key = r.astype(np.int64) * max(w, 1) + c
        if np.any(key[1:] < key[:-1]):
            order = np.lexsort((c, r))
            return r[order], c[order], v[order]
    return r, c, v


def oracle(case, x, y0, ntimes=1):
    h, w, r, c, v = case
    r, c, v = row_sorted(h, w, r, c, v)
    rp = csr_from_coo(h, r)
    y = y0.astype(np.float32)
    out, bound = None, None
    yhat = y0.astype(np.float64)
    tot_bound = _oracle.y0_term(y0, ntimes)
    for _ in range(ntimes):
        out, bound = _oracle.fp64_spmv(h, w, rp, c, v, x, None)
        yhat = yhat + out
        tot_bound = tot_bound + bound
    return yhat, tot_bound


def check(case, y, x, y0, ntimes=1, tol=TOL):
    yhat, bound = oracle(case, x, y0, ntimes)
    err, worst = _oracle.max_rel_err(y, yhat, bound)
    assert err <= tol, f"max per-row error {err:.3e} at row {worst} (tolerance {tol})"
    return err


def vecs(h, w, seed=7):
    rng = np.random.default_rng(seed)
    return rng.uniform(-1, 1, w).astype(np.float32), rng.uniform(-1, 1, h).astype(np.float32)


def coo_of(case):
    h, w, r, c, v = case
    return COO(h, w, r, c, v)
