"""Parity at the benchmark configurations' full sizes, through the same calls bench.py
times, against the FP64 oracle with the per-row bound
|y_i - yhat_i| <= 1e-5 * sum_j |a_ij x_j| + 2^-23 * |y0_i|:

  C1  128x128 Laplacian, autotuned Cocktail (graph replay);
  C2  10^6 Zipf(2) rows: the autotuned Cocktail and the x-panel layout forced;
  C3  160^3 27-point stencil: autotuned forward, xbar = A^T ybar and the value
      gradients abar = ybar_i x_j on the stored pattern;
  C4  500,000 block rows of 3x3 blocks in the generic BCSR layout: 1, 8 and 32
      right-hand sides, FP32 and BF16 values (BF16 against the BF16-rounded matrix);
  C5  the 512-matrix uneven batch, device-tuned formats, one persistent launch:
      forward, then forward + value gradients + adjoint.

Each configuration's matrix is generated once per module (seeded, as in bench.py)."""
import ctypes as C

import numpy as np
import pytest
import torch

from clspmv_b200 import (COO, CSP_ANALYZE_AUTOTUNE, CSP_FLAG_ADJOINT, CSP_FLAG_BF16, CSP_FLAG_GRAPH,
                         CSP_METH_XPANEL, Batch, Cocktail, Handle, analyze_matrix, capi, matrices as M)
from clspmv_b200.batch import (CSP_BATCH_ADJ, CSP_BATCH_FWD, CSP_BATCH_TUNE_DEVICE, CSP_BV_ABAR, CSP_BV_X,
                               CSP_BV_XBAR, CSP_BV_Y, CSP_BV_YBAR)
from clspmv_b200.matrices import csr_from_coo
from tests import _oracle
from tests.gpu_util import TOL, oracle
from tests.test_gpu_bf16 import bf16_round

pytestmark = pytest.mark.gpu


def _vectors(h, w, seed=1):
    rng = np.random.default_rng(seed)
    return rng.uniform(-1, 1, w).astype(np.float32), rng.uniform(-1, 1, h).astype(np.float32)


def _check(case, y, x, y0, what):
    yhat, bound = oracle(case, x, y0)
    err, row = _oracle.max_rel_err(y, yhat, bound)
    assert err <= TOL, f"{what}: per-row error {err:.3e} at row {row}"
    return err


def _check_grad(ybar, x, rows, cols, g, what):
    ok = rows >= 0
    assert np.all(g[~ok] == 0.0), f"{what}: gradient written into padding slots"
    want = ybar[rows[ok]].astype(np.float64) * x[cols[ok]].astype(np.float64)
    err = np.abs(g[ok].astype(np.float64) - want)
    assert np.all(err <= 2.0 ** -24 * np.abs(want)), f"{what}: value gradient off by {err.max():.3e}"


@pytest.fixture(scope="module")
def laplacian():
    return M.laplacian_2d(128)


@pytest.fixture(scope="module")
def zipf():
    return M.zipf_rows(1_000_000, 2.0, 10_000, seed=0)


@pytest.fixture(scope="module")
def stencil():
    return M.stencil_27(160)


@pytest.fixture(scope="module")
def block():
    return M.block_3x3(500_000)


def _cocktail_run(case, mat, flags=0):
    h, w = case[0], case[1]
    x, y0 = _vectors(h, w)
    hd = Handle(mat, x, y0, flags)
    hd.do_spmv(1)
    y = hd.cpy_result_to_cpu()
    hd.free()
    return _check(case, y, x, y0, getattr(mat, "choice", "cocktail"))


def test_c1_laplacian_autotuned_graph(laplacian):
    mat = analyze_matrix(COO(*laplacian), mode=CSP_ANALYZE_AUTOTUNE)
    _cocktail_run(laplacian, mat, CSP_FLAG_GRAPH)
    mat.free()


def test_c2_zipf_autotuned(zipf):
    mat = analyze_matrix(COO(*zipf), mode=CSP_ANALYZE_AUTOTUNE)
    _cocktail_run(zipf, mat)
    mat.free()


@pytest.mark.parametrize("fmt", ["csr", "coo"])
def test_c2_zipf_xpanel(zipf, fmt):
    """The x-panel layout on the full matrix: 1,000,000 columns in 27 shared-memory panels."""
    mat = Cocktail.single(fmt, COO(*zipf), CSP_METH_XPANEL)
    _cocktail_run(zipf, mat)
    mat.free()


def test_c3_stencil_forward_and_adjoint(stencil):
    h, w, r, c, v = stencil
    mat = analyze_matrix(COO(*stencil), mode=CSP_ANALYZE_AUTOTUNE)
    x, y0 = _vectors(h, w)
    hd = Handle(mat, x, y0, CSP_FLAG_ADJOINT)
    hd.do_spmv(1)
    _check(stencil, hd.cpy_result_to_cpu(), x, y0, f"forward ({mat.choice})")
    ybar = np.random.default_rng(3).uniform(-1, 1, h).astype(np.float32)
    xbar0 = np.random.default_rng(4).uniform(-1, 1, w).astype(np.float32)
    dy = torch.from_numpy(ybar).cuda()
    dx = torch.from_numpy(xbar0).cuda()
    da = torch.zeros(hd.adjoint_slots, device="cuda")
    hd.spmv_adjoint(dy.data_ptr(), dx.data_ptr(), da.data_ptr())
    hd.synchronize()
    want, bound = _oracle.fp64_spmv(h, w, csr_from_coo(h, r), c, v, ybar, xbar0, transpose=True)
    err, row = _oracle.max_rel_err(dx.cpu().numpy(), want, bound)
    assert err <= TOL, f"xbar error {err:.3e} at {row}"
    rows = torch.empty(hd.adjoint_slots, dtype=torch.int32, device="cuda")
    cols = torch.empty_like(rows)
    hd.adjoint_pattern(rows.data_ptr(), cols.data_ptr())
    _check_grad(ybar, x, rows.cpu().numpy(), cols.cpu().numpy(), da.cpu().numpy(), "stencil abar")
    hd.free()
    mat.free()


@pytest.fixture(scope="module")
def block_bcsr(block):
    coo = COO(*block)
    b = capi.bcsr_matrix()
    capi.check(capi.lib().csp_coo2bcsr(coo.ref(), C.byref(b), 3, 3, 32), "coo2bcsr")
    yield b
    capi.lib().csp_free_bcsr_matrix(C.byref(b))


@pytest.mark.parametrize("bf16", [False, True], ids=["fp32", "bf16"])
@pytest.mark.parametrize("k,tensor", [(1, False), (8, False), (32, False), (32, True)],
                         ids=["k1", "k8", "k32", "k32_tensor"])
def test_c4_block_generic_bcsr(block, block_bcsr, k, tensor, bf16):
    from clspmv_b200 import CSP_FLAG_TENSOR_CORES
    h, w, r, c, v = block
    rng = np.random.default_rng(9 + k)
    X = rng.uniform(-1, 1, (w, k)).astype(np.float32)
    Y0 = rng.uniform(-1, 1, (h, k)).astype(np.float32)
    flags = (CSP_FLAG_BF16 if bf16 else 0) | (CSP_FLAG_TENSOR_CORES if tensor else 0)
    hd = Handle(None, X, Y0, flags=flags, nrhs=k, bcsr=block_bcsr)
    hd.do_spmv(1)
    Y = hd.cpy_result_to_cpu().reshape(h, k)
    hd.free()
    vals = bf16_round(v) if bf16 else v
    rp = csr_from_coo(h, r)
    for j in range(k):
        yhat, bound = _oracle.fp64_spmv(h, w, rp, c, vals, np.ascontiguousarray(X[:, j]),
                                        np.ascontiguousarray(Y0[:, j]))
        err, row = _oracle.max_rel_err(np.ascontiguousarray(Y[:, j]), yhat, bound)
        assert err <= TOL, f"k={k} column {j}: error {err:.3e} at row {row}"


@pytest.fixture(scope="module")
def batch():
    gen = M.batch_mixed(512)
    return [m[1:] for m in gen]


def test_c5_batch_forward_and_adjoint(batch):
    mats = batch
    coos = [COO(*m) for m in mats]
    bt = Batch(coos, flags=CSP_FLAG_ADJOINT | CSP_FLAG_GRAPH, tune=CSP_BATCH_TUNE_DEVICE)
    hs, ws = [m[0] for m in mats], [m[1] for m in mats]
    rng = np.random.default_rng(3)
    x = rng.uniform(-1, 1, sum(ws)).astype(np.float32)
    y0 = rng.uniform(-1, 1, sum(hs)).astype(np.float32)
    ybar = rng.uniform(-1, 1, sum(hs)).astype(np.float32)
    xbar0 = rng.uniform(-1, 1, sum(ws)).astype(np.float32)
    xo, yo = np.concatenate([[0], np.cumsum(ws)]), np.concatenate([[0], np.cumsum(hs)])

    def load():
        bt.copy_in(CSP_BV_X, x)
        bt.copy_in(CSP_BV_Y, y0)
        bt.copy_in(CSP_BV_YBAR, ybar)
        bt.copy_in(CSP_BV_XBAR, xbar0)

    def check(both):
        y = bt.copy_out(CSP_BV_Y)
        xbar = bt.copy_out(CSP_BV_XBAR)
        abar = bt.copy_out(CSP_BV_ABAR) if both else None
        for i, (h, w, r, c, v) in enumerate(mats):
            xs, ys = slice(int(xo[i]), int(xo[i + 1])), slice(int(yo[i]), int(yo[i + 1]))
            _check(mats[i], y[ys], x[xs], y0[ys], f"matrix {i} forward")
            if not both:
                assert np.array_equal(xbar[xs], xbar0[xs])
                continue
            rp = csr_from_coo(h, r)
            want, bound = _oracle.fp64_spmv(h, w, rp, c, v, ybar[ys], xbar0[xs], transpose=True)
            err, row = _oracle.max_rel_err(xbar[xs], want, bound)
            assert err <= TOL, f"matrix {i}: xbar error {err:.3e} at {row}"
            rows, cols = bt.pattern(i)
            _check_grad(ybar[ys], x[xs], rows, cols, abar[int(bt.abar_off[i]):int(bt.abar_off[i + 1])],
                        f"matrix {i} abar")

    load()
    bt.run(CSP_BATCH_FWD)
    check(False)
    load()
    bt.run(CSP_BATCH_FWD | CSP_BATCH_ADJ)
    check(True)
    bt.free()
