"""Adjoint on the device: xbar = A^T ybar against the FP64 oracle's transposed
product, value gradients against ybar_i x_j on the exported pattern, FP64 central
finite differences of f(x, a) = ybar^T A(a) x on the 27-point stencil at 32^3, and
the torch.autograd binding."""
import numpy as np
import pytest
import torch

from clspmv_b200 import CSP_FLAG_ADJOINT, COO, Cocktail, Handle, analyze_matrix, matrices as M
from clspmv_b200 import capi
from clspmv_b200.autograd import CocktailSpMV, SpMVOperator, value_gradient
from clspmv_b200.matrices import csr_from_coo
from tests import _oracle
from tests.cases import small_cases
from tests.gpu_util import TOL, coo_of, vecs
from tests.test_analyzer_parity import _plus_noise, _stencil9

pytestmark = pytest.mark.gpu

SMALL = small_cases()
CASES = {
    "stencil32": M.stencil_27(32, seed=71),
    "stencil9": _stencil9(128),
    "zipf": M.zipf_rows(30_000, seed=72, max_len=3000),
    "block4": M.block_3x3(2000, deg=(3, 8), band=40, seed=73, bs=4),
    "rect_wide": SMALL["rect_wide"],
    "rect_tall": SMALL["rect_tall"],
    "lap_noise": _plus_noise(M.laplacian_2d(96), 3000, 2),
}
VARIANTS = [("dia", 1), ("bdia", 1), ("csr", 2), ("coo", 0), ("csr", 16), ("coo", 16), ("ell", 1), ("sell", 0),
            ("bcsr", 0), ("sbell", 0), ("bell", 0)]


def _xbar_ref(case, ybar):
    h, w, r, c, v = case
    order = np.lexsort((c, r))
    r, c, v = r[order], c[order], v[order]
    return _oracle.fp64_spmv(h, w, csr_from_coo(h, r), c, v, ybar, None, transpose=True)


def _handle(mat, x, y0):
    return Handle(mat, x, y0, CSP_FLAG_ADJOINT)


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("variant", VARIANTS, ids=lambda v: f"{v[0]}{v[1]}")
def test_transposed_product(name, variant):
    fmt, m = variant
    case = CASES[name]
    h, w = case[0], case[1]
    kw = {"bwidth": 4, "bheight": 4} if fmt in ("bcsr", "sbell", "bell") else {}
    if fmt in ("dia", "bdia") and (name not in ("stencil32", "stencil9", "lap_noise")):
        pytest.skip("diagonal formats only for banded inputs")
    if fmt in ("bcsr", "sbell", "bell", "ell") and name in ("zipf",):
        pytest.skip("padding")
    try:
        mat = Cocktail.single(fmt, coo_of(case), m, **kw)
    except Exception as e:
        if "CSP_EFORMAT" in str(e):
            pytest.skip(str(e))
        raise
    x, y0 = vecs(h, w)
    ybar = np.random.default_rng(3).uniform(-1, 1, h).astype(np.float32)
    hd = _handle(mat, x, y0)
    dy = torch.from_numpy(ybar).cuda()
    xbar0 = np.random.default_rng(4).uniform(-1, 1, w).astype(np.float32)
    dx = torch.from_numpy(xbar0).cuda()
    hd.spmv_adjoint(dy.data_ptr(), dx.data_ptr())
    hd.synchronize()
    want, bound = _xbar_ref(case, ybar)
    bound = bound + _oracle.y0_term(xbar0)
    err, row = _oracle.max_rel_err(dx.cpu().numpy(), want + xbar0, bound)
    assert err <= TOL, f"xbar error {err:.3e} at {row}"
    abar, rows, cols = value_gradient(hd, dy)
    abar, rows, cols = abar.cpu().numpy(), rows.cpu().numpy(), cols.cpu().numpy()
    valid = rows >= 0
    expect = np.where(valid, ybar[np.maximum(rows, 0)] * x[np.maximum(cols, 0)], 0.0).astype(np.float32)
    assert np.array_equal(abar, expect)
    # every stored nonzero is covered exactly once by a valid slot
    hh, ww, r, c, v = case
    key = np.sort(r.astype(np.int64) * ww + c)
    got = np.sort(rows[valid].astype(np.int64) * ww + cols[valid])
    assert np.all(np.isin(key, got))
    hd.free()


def test_finite_differences_stencil32():
    """FP64 central differences of f(x, a) = ybar^T (A(a) x) on the 32^3 stencil."""
    case = CASES["stencil32"]
    h, w, r, c, v = case
    mat = analyze_matrix(COO(h, w, r, c, v), mode=1)   # autotuned partition
    rng = np.random.default_rng(5)
    x = rng.uniform(-1, 1, w).astype(np.float32)
    ybar = rng.uniform(-1, 1, h).astype(np.float32)
    hd = Handle(mat, x, None, CSP_FLAG_ADJOINT)
    dy = torch.from_numpy(ybar).cuda()
    xbar = torch.zeros(w, device="cuda")
    hd.spmv_adjoint(dy.data_ptr(), xbar.data_ptr())
    hd.synchronize()
    xbar = xbar.cpu().numpy().astype(np.float64)
    rp = csr_from_coo(h, r)

    def f(xx, vals):
        out, _ = _oracle.fp64_spmv(h, w, rp, c, vals.astype(np.float32), xx.astype(np.float32), None)
        return float(np.dot(ybar.astype(np.float64), out))

    for k in range(3):
        d = rng.uniform(-1, 1, w)
        eps = 1e-3
        fd = (f(x + eps * d, v) - f(x - eps * d, v)) / (2 * eps)
        assert abs(fd - np.dot(xbar, d)) <= 1e-4 * (abs(fd) + np.abs(xbar).dot(np.abs(d))), (k, fd, np.dot(xbar, d))
    hd.free()


def _value_fd_check(case, hd, x, ybar, nsample=40, seed=8):
    """FP64 central differences of f(a) = ybar^T (A(a) x) over a sample of the matrix's
    entries against the device value gradients of the slots holding them."""
    h, w, r, c, v = case
    rp = csr_from_coo(h, r)
    dy = torch.from_numpy(ybar).cuda()
    abar, rows, cols = value_gradient(hd, dy)
    abar, rows, cols = abar.cpu().numpy(), rows.cpu().numpy(), cols.cpu().numpy()
    ok = rows >= 0
    skey = rows[ok].astype(np.int64) * w + cols[ok]
    sval = abar[ok]

    def f(vals):
        out, _ = _oracle.fp64_spmv(h, w, rp, c, vals.astype(np.float32), x, None)
        return float(np.dot(ybar.astype(np.float64), out))

    rng = np.random.default_rng(seed)
    eps = 2.0 ** -6   # exact in FP32 next to values of order 1
    for e in rng.choice(r.size, size=min(nsample, r.size), replace=False):
        vp, vm = v.copy(), v.copy()
        vp[e] += eps
        vm[e] -= eps
        fd = (f(vp) - f(vm)) / (2 * eps)
        have = sval[skey == int(r[e]) * w + int(c[e])]
        assert have.size >= 1, f"entry {e} has no stored slot"
        scale = abs(float(ybar[r[e]]) * float(x[c[e]])) + 1e-30
        assert np.all(np.abs(have.astype(np.float64) - fd) <= 1e-5 * scale + 1e-7 * abs(fd)), (e, fd, have)


def test_value_finite_differences_stencil32():
    """The value gradients of the autotuned stencil partition against FP64 central
    differences that perturb one matrix value at a time."""
    case = CASES["stencil32"]
    h, w, r, c, v = case
    mat = analyze_matrix(COO(h, w, r, c, v), mode=1)
    rng = np.random.default_rng(5)
    x = rng.uniform(-1, 1, w).astype(np.float32)
    ybar = rng.uniform(-1, 1, h).astype(np.float32)
    hd = Handle(mat, x, None, CSP_FLAG_ADJOINT)
    _value_fd_check(case, hd, x, ybar)
    hd.free()


BLOCK_CASES = {"block3": M.block_3x3(3000, deg=(4, 12), band=100, seed=74),
               "block2_ragged": M.block_3x3(2001, deg=(1, 6), band=30, seed=75),   # 6,003 rows: ragged as 2x2
               "block4": CASES["block4"]}


@pytest.mark.parametrize("name,bs", [("block3", 3), ("block2_ragged", 2), ("block4", 4), ("block3", 1)])
def test_generic_bcsr_adjoint(name, bs):
    """csp_init_bcsr_kernels with CSP_FLAG_ADJOINT: xbar = A^T ybar against the oracle,
    value gradients on the caller's BCSR layout, and FP64 central differences over the
    values."""
    import ctypes as C
    case = BLOCK_CASES[name]
    h, w, r, c, v = case
    b = capi.bcsr_matrix()
    assert capi.lib().csp_coo2bcsr(coo_of(case).ref(), C.byref(b), bs, bs, 32) == 0
    x, y0 = vecs(h, w)
    hd = Handle(None, x, y0, CSP_FLAG_ADJOINT, bcsr=b)
    aligned, nblk, rp_b = b.bcsr_aligned_size, b.bcsr_block_num, b.bcsr_row_ptr
    bcol = np.ctypeslib.as_array(b.bcsr_col_id, shape=(max(nblk, 1),))[:nblk].copy()
    brp = np.ctypeslib.as_array(rp_b, shape=(b.bcsr_row_num + 1,)).copy()
    capi.lib().csp_free_bcsr_matrix(C.byref(b))
    assert hd.adjoint_slots == aligned * bs * bs
    ybar = np.random.default_rng(3).uniform(-1, 1, h).astype(np.float32)
    xbar0 = np.random.default_rng(4).uniform(-1, 1, w).astype(np.float32)
    dy = torch.from_numpy(ybar).cuda()
    dx = torch.from_numpy(xbar0).cuda()
    hd.spmv_adjoint(dy.data_ptr(), dx.data_ptr())
    hd.synchronize()
    want, bound = _xbar_ref(case, ybar)
    err, row = _oracle.max_rel_err(dx.cpu().numpy(), want + xbar0, bound + _oracle.y0_term(xbar0))
    assert err <= TOL, f"xbar error {err:.3e} at {row}"
    abar, rows, cols = value_gradient(hd, dy)
    abar, rows, cols = abar.cpu().numpy(), rows.cpu().numpy(), cols.cpu().numpy()
    # slot (e, j) of the caller's layout: row brow(j) * bs + e / bs, column col[j] + e % bs
    brow = np.repeat(np.arange(brp.size - 1), np.diff(brp))
    e_i, j_i = np.divmod(np.arange(aligned * bs * bs), aligned)
    want_r = np.where(j_i < nblk, brow[np.minimum(j_i, max(nblk - 1, 0))] * bs + e_i // bs, -1)
    want_c = np.where(j_i < nblk, bcol[np.minimum(j_i, max(nblk - 1, 0))] + e_i % bs, -1)
    inside = (want_r >= 0) & (want_r < h) & (want_c < w)
    assert np.array_equal(rows, np.where(inside, want_r, -1))
    assert np.array_equal(cols[inside], want_c[inside])
    expect = np.where(inside, ybar[np.maximum(rows, 0)] * x[np.maximum(cols, 0)], 0.0).astype(np.float32)
    assert np.array_equal(abar, expect)
    _value_fd_check(case, hd, x, ybar)
    hd.free()


@pytest.mark.parametrize("variant", [("bcsr", 0), ("sbell", 0), ("bell", 0)], ids=lambda v: v[0])
def test_b4_block_value_finite_differences(variant):
    """Value gradients of the b4 block layouts against FP64 central differences."""
    case = CASES["block4"]
    h, w, r, c, v = case
    mat = Cocktail.single(variant[0], coo_of(case), variant[1], bwidth=4, bheight=4)
    rng = np.random.default_rng(12)
    x = rng.uniform(-1, 1, w).astype(np.float32)
    ybar = rng.uniform(-1, 1, h).astype(np.float32)
    hd = Handle(mat, x, None, CSP_FLAG_ADJOINT)
    _value_fd_check(case, hd, x, ybar)
    hd.free()


@pytest.mark.parametrize("fmt", ["auto", ("csr", 2), ("coo", 16), "gbcsr"], ids=["auto", "csr2", "coo16", "gbcsr"])
def test_autograd_binding(fmt):
    """CocktailSpMV with x, y0 and the matrix values as autograd inputs."""
    case = CASES["lap_noise"] if fmt != "gbcsr" else BLOCK_CASES["block3"]
    h, w, r, c, v = case
    op = SpMVOperator(h, w, r, c, fmt=fmt, block=(3, 3))
    rng = np.random.default_rng(6)
    x = torch.from_numpy(rng.uniform(-1, 1, w).astype(np.float32)).cuda().requires_grad_(True)
    y0 = torch.from_numpy(rng.uniform(-1, 1, h).astype(np.float32)).cuda().requires_grad_(True)
    vals = torch.from_numpy(v.copy()).cuda().requires_grad_(True)
    ybar = torch.from_numpy(rng.uniform(-1, 1, h).astype(np.float32)).cuda()
    y = CocktailSpMV.apply(x, y0, vals, op)
    gx, gy0, gv = torch.autograd.grad(y, (x, y0, vals), ybar)
    want_y, bound = _oracle.fp64_spmv(h, w, csr_from_coo(h, r), c, v, x.detach().cpu().numpy(),
                                      y0.detach().cpu().numpy())
    err, _ = _oracle.max_rel_err(y.detach().cpu().numpy(), want_y, bound)
    assert err <= TOL
    want_x, bx = _xbar_ref(case, ybar.cpu().numpy())
    err, _ = _oracle.max_rel_err(gx.cpu().numpy(), want_x, bx)
    assert err <= TOL
    assert torch.equal(gy0, ybar)
    xn, yn = x.detach().cpu().numpy(), ybar.cpu().numpy()
    want_v = yn[r].astype(np.float64) * xn[c].astype(np.float64)
    assert np.all(np.abs(gv.cpu().numpy() - want_v) <= 2.0 ** -24 * np.abs(want_v))
