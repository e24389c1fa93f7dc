"""Several right-hand sides (SpMM): Y += A X with X, Y row-major, on CSR parts and on
generic BCSR handles (3x3 blocks, the FEM case), FP32 and BF16 values, against the FP64
oracle column by column."""
import ctypes as C

import numpy as np
import pytest

from clspmv_b200 import CSP_FLAG_BF16, Cocktail, Handle, capi, matrices as M
from clspmv_b200.matrices import csr_from_coo
from tests import _oracle
from tests.gpu_util import TOL, coo_of
from tests.test_gpu_bf16 import bf16_round

pytestmark = pytest.mark.gpu

CASES = {
    "zipf": M.zipf_rows(20_000, seed=81, max_len=2000),
    "block3": M.block_3x3(4000, deg=(10, 30), band=200, seed=82),
    "block4": M.block_3x3(1500, deg=(4, 10), band=50, seed=83, bs=4),
}


def _check_cols(case, Y, X, Y0, k, values=None, tol=TOL):
    h, w, r, c, v = case
    if values is not None:
        v = values
    rp = csr_from_coo(h, r)
    Y = Y.reshape(h, k)
    for j in range(k):
        yhat, bound = _oracle.fp64_spmv(h, w, rp, c, v, np.ascontiguousarray(X[:, j]), np.ascontiguousarray(Y0[:, j]))
        err, row = _oracle.max_rel_err(np.ascontiguousarray(Y[:, j]), yhat, bound)
        assert err <= tol, f"column {j}: error {err:.3e} at row {row}"


def _xy(h, w, k, seed=9):
    rng = np.random.default_rng(seed)
    return rng.uniform(-1, 1, (w, k)).astype(np.float32), rng.uniform(-1, 1, (h, k)).astype(np.float32)


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("k", [2, 3, 8, 32, 40])
def test_csr_spmm(name, k):
    case = CASES[name]
    h, w = case[0], case[1]
    X, Y0 = _xy(h, w, k)
    mat = Cocktail.single("csr", coo_of(case), 2)
    hd = Handle(mat, X, Y0, nrhs=k)
    hd.do_spmv(1)
    Y = hd.cpy_result_to_cpu()
    hd.free()
    _check_cols(case, Y, X, Y0, k)


@pytest.mark.parametrize("name,bs", [("block3", 3), ("block4", 4), ("zipf", 2)])
@pytest.mark.parametrize("k", [1, 8, 32, 33])
@pytest.mark.parametrize("bf16", [False, True])
def test_generic_bcsr_spmm(name, bs, k, bf16):
    case = CASES[name]
    h, w, r, c, v = case
    b = capi.bcsr_matrix()
    assert capi.lib().csp_coo2bcsr(coo_of(case).ref(), C.byref(b), bs, bs, 32) == 0
    X, Y0 = _xy(h, w, k)
    flags = CSP_FLAG_BF16 if bf16 else 0
    hd = Handle(None, X, Y0, flags=flags, nrhs=k, bcsr=b)
    hd.do_spmv(1)
    Y = hd.cpy_result_to_cpu()
    hd.free()
    capi.lib().csp_free_bcsr_matrix(C.byref(b))
    _check_cols(case, Y, X, Y0, k, values=bf16_round(v) if bf16 else None)


def test_spmm_rejects_other_formats():
    case = CASES["zipf"]
    mat = Cocktail.single("coo", coo_of(case), 0)
    with pytest.raises(Exception, match="CSP_EUNSUP"):
        Handle(mat, None, None, nrhs=4)


def _ragged(h, w, long_row, seed):
    """Rows of 0-39 entries, 30 % of them empty, one row of `long_row` entries; h is not
    a multiple of 2, 3 or 4, so the last block row is partial."""
    rng = np.random.default_rng(seed)
    lens = np.where(rng.random(h) < 0.3, 0, rng.integers(1, 40, h))
    lens[h // 2] = long_row
    rows, cols = [], []
    for i, n in enumerate(lens):
        if n:
            rows.append(np.full(n, i, np.int32))
            cols.append(np.sort(rng.choice(w, n, replace=False)).astype(np.int32))
    r = np.concatenate(rows)
    return h, w, r, np.concatenate(cols), rng.standard_normal(r.size).astype(np.float32)


# 1,021 entries in one row: with 1x1 blocks exactly the largest work item of the single
# right-hand-side kernel; 1,500: too long for one item (the row-per-group kernel runs)
RAGGED = {"ragged": _ragged(10_007, 9_001, 1021, 84), "ragged_long": _ragged(10_007, 9_001, 1500, 85)}


@pytest.mark.parametrize("name", sorted(RAGGED))
@pytest.mark.parametrize("bs", [1, 2, 3, 4])
@pytest.mark.parametrize("k", [1, 8])
@pytest.mark.parametrize("bf16", [False, True])
def test_generic_bcsr_ragged(name, bs, k, bf16):
    """Empty block rows, a partial last block row and item-sized block rows."""
    case = RAGGED[name]
    h, w, r, c, v = case
    b = capi.bcsr_matrix()
    assert capi.lib().csp_coo2bcsr(coo_of(case).ref(), C.byref(b), bs, bs, 32) == 0
    X, Y0 = _xy(h, w, k, seed=10)
    hd = Handle(None, X, Y0, flags=CSP_FLAG_BF16 if bf16 else 0, nrhs=k, bcsr=b)
    hd.do_spmv(1)
    Y = hd.cpy_result_to_cpu()
    hd.free()
    capi.lib().csp_free_bcsr_matrix(C.byref(b))
    _check_cols(case, Y, X, Y0, k, values=bf16_round(v) if bf16 else None)


TENSOR_CASES = {**CASES, **RAGGED}


@pytest.mark.parametrize("name,bs", [("block3", 3), ("block4", 4), ("zipf", 2), ("zipf", 1), ("ragged", 3),
                                     ("ragged_long", 4), ("ragged", 2)])
@pytest.mark.parametrize("k", [32, 64, 33])
@pytest.mark.parametrize("bf16", [False, True])
def test_generic_bcsr_spmm_tensor_cores(name, bs, k, bf16):
    """CSP_FLAG_TENSOR_CORES: the mma.sync path for k a multiple of 32 (k = 33 keeps the
    CUDA-core kernel), including empty and partial block rows and odd block counts."""
    from clspmv_b200 import CSP_FLAG_TENSOR_CORES
    case = TENSOR_CASES[name]
    h, w, r, c, v = case
    b = capi.bcsr_matrix()
    assert capi.lib().csp_coo2bcsr(coo_of(case).ref(), C.byref(b), bs, bs, 32) == 0
    X, Y0 = _xy(h, w, k, seed=11)
    flags = CSP_FLAG_TENSOR_CORES | (CSP_FLAG_BF16 if bf16 else 0)
    hd = Handle(None, X, Y0, flags=flags, nrhs=k, bcsr=b)
    hd.do_spmv(1)
    Y = hd.cpy_result_to_cpu()
    hd.free()
    capi.lib().csp_free_bcsr_matrix(C.byref(b))
    _check_cols(case, Y, X, Y0, k, values=bf16_round(v) if bf16 else None)
