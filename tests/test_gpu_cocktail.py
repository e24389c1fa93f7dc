"""The Cocktail engine end to end on the device: analyzer partitions (several formats
in one handle) through csp_init_mat_kernels / csp_do_spmv, the reference's example()
loop (y = A^k x with cpy_vector_from_gpu, clSpMV_NV/src/eval.cpp:19), csp_evaluate and
the spmv_all drivers, each against the FP64 oracle."""
import ctypes as C
import os

import numpy as np
import pytest

from clspmv_b200 import COO, Cocktail, Handle, analyze_matrix, capi, evaluate, matrices as M, spmv_all
from clspmv_b200.matrices import csr_from_coo
from tests import _oracle
from tests.gpu_util import TOL, check, coo_of, run, vecs
from tests.test_analyzer_parity import _plus_noise, _stencil9, _uniform_rows

pytestmark = pytest.mark.gpu

CASES = {
    "laplacian128_dia": M.laplacian_2d(128),
    "stencil9_bdia": _stencil9(256),
    "laplacian_noise_ell_coo": _plus_noise(M.laplacian_2d(256), 20000, 1),
    "block4_bell": M.block_3x3(20_000, deg=(4, 10), band=100, seed=7, bs=4),
    "block8_sbell": M.block_3x3(5000, deg=(3, 8), band=50, seed=6, bs=8),
    "zipf_ell_coo": M.zipf_rows(200_000, seed=8, max_len=3000),
    "stencil24_dia": M.stencil_27(24),
    "uniform_ell": _uniform_rows(50_000, 16, 2),
}


def _analyze(case):
    return analyze_matrix(coo_of(case), bench_path=_oracle.REF_BENCH)


@pytest.fixture(scope="module", autouse=True)
def _tables():
    if not os.path.isdir(os.path.join(_oracle.REF_BENCH, "benchmark")):
        pytest.skip("calibration tables not built (make -C oracle)")


@pytest.mark.parametrize("name", sorted(CASES))
def test_analyzed_cocktail_spmv(name):
    case = CASES[name]
    mat = _analyze(case)
    x, y0 = vecs(case[0], case[1])
    y = run(mat, x, y0)
    check(case, y, x, y0)
    y = run(mat, x, y0, ntimes=2, flags=capi.CSP_FLAG_GRAPH)
    check(case, y, x, y0, ntimes=2)


@pytest.mark.parametrize("name", ["laplacian_noise_ell_coo", "stencil9_bdia"])
def test_example_power_loop(name):
    """eval.cpp:19 example(): res is never cleared, x <- res after every SpMV."""
    case = CASES[name]
    h, w, r, c, v = case
    mat = _analyze(case)
    x, y0 = vecs(h, w)
    x = x * 0.1
    y0 = y0 * 0.1
    hd = Handle(mat, x, y0)
    hd.cpy_result_from_cpu(y0)
    for _ in range(3):
        hd.do_spmv(1)
        hd.cpy_vector_from_gpu(hd.res_ptr, h)
    y = hd.cpy_result_to_cpu()
    hd.free()
    rp = csr_from_coo(h, r)
    yx = x.astype(np.float64)
    yy = y0.astype(np.float64)
    bx, by = np.abs(yx), np.abs(yy)
    dense_abs = None
    for _ in range(3):
        prod, _ = _oracle.fp64_spmv(h, w, rp, c, v, yx.astype(np.float32), None)
        babs, _ = _oracle.fp64_spmv(h, w, rp, c, np.abs(v), bx.astype(np.float32), None)
        yy = yy + prod
        by = by + babs
        yx, bx = yy.copy(), by.copy()
    err = np.max(np.abs(y - yy) / np.maximum(by, 1e-30))
    assert err <= 4 * TOL, err


def test_evaluate_reports_match():
    case = CASES["laplacian_noise_ell_coo"]
    h, w, r, c, v = case
    mat = _analyze(case)
    x, y0 = vecs(h, w)
    coores = y0.astype(np.float32).copy()
    np.add.at(coores, r, (v * x[c]).astype(np.float32))
    rep = evaluate(mat, x, y0, coores, ntimes=20)
    assert rep["ms"] > 0 and rep["gflops"] > 0
    # the reference's max relative difference (util.cpp:93) blows up on rows that cancel
    # to ~0, so the check is normwise: ||y - y_coo|| <= 1e-5 * ||y_coo||
    assert rep["l2_distance"] <= 1e-5 * np.linalg.norm(coores.astype(np.float64)), rep


@pytest.mark.parametrize("method", range(1, 11))
def test_spmv_all_drivers(method):
    """spmv_all methods 1-10 on a banded-block matrix every format can hold."""
    case = M.block_3x3(3000, deg=(3, 6), band=8, seed=9, bs=4)
    coo = coo_of(case)
    if method in (3, 4):
        case = M.laplacian_2d(96)
        coo = coo_of(case)
    rep = spmv_all(coo, method, ntimes=5)
    assert rep["method"] >= 0 and rep["ms"] > 0
    # x = 1, y = 0 against the serial COO result (util.cpp:93 two_vec_compare numbers);
    # normwise, since the reference's relative form is ill-conditioned on cancelling rows
    h, w, r, c, v = case
    ycoo = np.zeros(h)
    np.add.at(ycoo, r, v.astype(np.float64))
    assert rep["l2_distance"] <= 1e-5 * np.linalg.norm(ycoo), (method, rep)
