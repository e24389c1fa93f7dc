"""The on-device autotuner (CSP_ANALYZE_AUTOTUNE): the partition it picks computes the
right product, and a second call on the same pattern is served from the cache."""
import os

import numpy as np
import pytest

from clspmv_b200 import CSP_ANALYZE_AUTOTUNE, analyze_matrix, matrices as M
from tests.gpu_util import check, coo_of, run, vecs
from tests.test_analyzer_parity import _stencil9, _uniform_rows

pytestmark = pytest.mark.gpu

CASES = {
    "zipf_100k": M.zipf_rows(100_000, seed=51, max_len=5000),
    "stencil24": M.stencil_27(24, seed=52),
    "stencil9_256": _stencil9(256),
    "block4": M.block_3x3(8000, deg=(4, 10), band=100, seed=53, bs=4),
    "block3": M.block_3x3(8000, deg=(10, 30), band=300, seed=54),
    "uniform16": _uniform_rows(60_000, 16, 55),
    "laplacian128": M.laplacian_2d(128),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_autotuned_partition_is_correct(name, tmp_path):
    case = CASES[name]
    cache = str(tmp_path / "tune.txt")
    mat = analyze_matrix(coo_of(case), mode=CSP_ANALYZE_AUTOTUNE, cache_path=cache)
    assert mat.choice
    x, y0 = vecs(case[0], case[1])
    check(case, run(mat, x, y0), x, y0)
    # second call on the same pattern: served from the cache, same choice
    again = analyze_matrix(coo_of(case), mode=CSP_ANALYZE_AUTOTUNE, cache_path=cache)
    assert again.choice == mat.choice
    lines = open(cache).read().split("\n")
    assert sum(1 for ln in lines if ln.strip()) == 1
    check(case, run(again, x, y0), x, y0)


def test_dense_blocks_get_a_generic_bcsr_candidate(tmp_path):
    """A matrix of dense 3x3 blocks (no b4 shape holds it): the autotuner's candidates are
    the generic block layouts and plain CSR, and the winner runs in the Cocktail engine."""
    case = CASES["block3"]
    mat = analyze_matrix(coo_of(case), mode=CSP_ANALYZE_AUTOTUNE, verbose=1)
    assert mat.choice.startswith("gbcsr") or mat.choice == "csr2", mat.choice
    x, y0 = vecs(case[0], case[1])
    check(case, run(mat, x, y0), x, y0)


@pytest.mark.parametrize("bs", [2, 3, 4])
def test_cocktail_generic_bcsr_part(bs):
    """CSP_METH_GENERIC_BCSR: a generic BCSR in the cocktail's bcsr member, forward with one
    and several right-hand sides (CUDA cores and tensor cores), FP32 and BF16 values,
    and the adjoint (A^T ybar and the value gradients on the caller's layout)."""
    import ctypes as C

    import torch

    from clspmv_b200 import (CSP_FLAG_ADJOINT, CSP_FLAG_BF16, CSP_FLAG_TENSOR_CORES, Cocktail, Handle, capi)
    from clspmv_b200.autograd import value_gradient
    from tests import _oracle
    from tests.test_gpu_adjoint import _xbar_ref
    from tests.test_gpu_bf16 import bf16_round
    from tests.test_gpu_spmm import _check_cols, _xy
    case = CASES["block3"]
    h, w, r, c, v = case
    mat = Cocktail(h, w, r.size)
    L = capi.lib()
    assert L.csp_coo2bcsr(coo_of(case).ref(), C.cast(C.byref(mat.s.bcsr), C.POINTER(capi.bcsr_matrix)), bs, bs, 32) == 0
    mat.s.ifusebcsr = True
    mat.s.bcsr_meth_num = capi.CSP_METH_GENERIC_BCSR
    x, y0 = vecs(h, w)
    for fl in (0, CSP_FLAG_BF16):
        yv = run(mat, x, y0, flags=fl)
        check((h, w, r, c, bf16_round(v) if fl else v), yv, x, y0)
    for k, fl in ((8, 0), (32, 0), (32, CSP_FLAG_TENSOR_CORES), (32, CSP_FLAG_TENSOR_CORES | CSP_FLAG_BF16)):
        X, Y0 = _xy(h, w, k, seed=13)
        hd = Handle(mat, X, Y0, flags=fl, nrhs=k)
        hd.do_spmv(1)
        Y = hd.cpy_result_to_cpu()
        hd.free()
        _check_cols(case, Y, X, Y0, k, values=bf16_round(v) if fl & CSP_FLAG_BF16 else None)
    hd = Handle(mat, x, y0, CSP_FLAG_ADJOINT)
    ybar = np.random.default_rng(3).uniform(-1, 1, h).astype(np.float32)
    dy = torch.from_numpy(ybar).cuda()
    dx = torch.zeros(w, device="cuda")
    hd.spmv_adjoint(dy.data_ptr(), dx.data_ptr())
    hd.synchronize()
    want, bound = _xbar_ref(case, ybar)
    err, row = _oracle.max_rel_err(dx.cpu().numpy(), want, bound)
    assert err <= 1e-5, f"xbar error {err:.3e} at {row}"
    abar, rows, cols = value_gradient(hd, dy)
    abar, rows, cols = abar.cpu().numpy(), rows.cpu().numpy(), cols.cpu().numpy()
    ok = rows >= 0
    assert np.array_equal(abar[ok], (ybar[rows[ok]] * x[cols[ok]]).astype(np.float32))
    assert np.all(abar[~ok] == 0)
    key = np.unique(r.astype(np.int64) * w + c)
    assert np.isin(key, rows[ok].astype(np.int64) * w + cols[ok]).all()
    hd.free()
    mat.free()


@pytest.mark.parametrize("choice", ["coo4+csr16", "coo8+csr16", "coo16+csr16", "coo8+csr2"])
def test_coo_split_candidates(choice, tmp_path):
    """The short-row split (rows of at most t entries as a COO part, the rest as a CSR
    part with the x-panel or adaptive kernel), forced through the decision cache: the
    first call records the pattern's key, the edited cache then names the candidate."""
    case = CASES["zipf_100k"]
    cache = str(tmp_path / "tune.txt")
    analyze_matrix(coo_of(case), mode=CSP_ANALYZE_AUTOTUNE, cache_path=cache)
    key = open(cache).read().split()[0]
    with open(cache, "w") as f:
        f.write(f"{key} {choice} 0.0\n")
    mat = analyze_matrix(coo_of(case), mode=CSP_ANALYZE_AUTOTUNE, cache_path=cache)
    assert mat.choice == choice
    x, y0 = vecs(case[0], case[1])
    check(case, run(mat, x, y0), x, y0)
