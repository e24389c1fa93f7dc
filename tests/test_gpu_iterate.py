"""The solver loop of the reference's example() (clSpMV_NV/src/eval.cpp:19-50) on the
device (csp_iterate: res += A*vec, then vec = res, `iterations` times), against the
same loop driven call by call through do_spmv + cpy_vector_from_gpu and against an
FP64 iteration; and the L2 persistence flag, which must not change any bit."""
import numpy as np
import pytest

from clspmv_b200 import CSP_FLAG_GRAPH, CSP_FLAG_L2_PERSIST, COO, Cocktail, Handle, matrices as M
from clspmv_b200.matrices import csr_from_coo
from tests import _oracle
from tests.gpu_util import TOL, coo_of, vecs

pytestmark = pytest.mark.gpu


def _scaled(case, f):
    h, w, r, c, v = case
    return h, w, r, c, (v * f).astype(np.float32)


CASES = {
    "laplacian32": _scaled(M.laplacian_2d(32), 0.1),
    "zipf": _scaled(M.zipf_rows(20_000, seed=41, max_len=2000), 0.05),
}


def _manual(mat, x, y0, k, flags=0):
    hd = Handle(mat, x, y0, flags)
    n = hd.height
    for _ in range(k):
        hd.do_spmv(1)
        hd.cpy_vector_from_gpu(hd.res_ptr, n)
    y = hd.cpy_result_to_cpu()
    hd.free()
    return y


def _iterated(mat, x, y0, k, flags=0):
    hd = Handle(mat, x, y0, flags)
    hd.iterate(k)
    y = hd.cpy_result_to_cpu()
    hd.free()
    return y


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("fmt,method", [("csr", 2), ("csr", 16), ("coo", 0)])
@pytest.mark.parametrize("k", [1, 3, 37])
@pytest.mark.parametrize("graph", [False, True])
def test_iterate_matches_call_by_call_loop(name, fmt, method, k, graph):
    case = CASES[name]
    h, w = case[0], case[1]
    mat = Cocktail.single(fmt, coo_of(case), method)
    x, y0 = vecs(h, w, seed=5)
    flags = CSP_FLAG_GRAPH if graph else 0
    a = _iterated(mat, x, y0, k, flags)
    b = _manual(mat, x, y0, k)
    assert a.tobytes() == b.tobytes()   # same kernels in the same order: identical bits


@pytest.mark.parametrize("name", sorted(CASES))
def test_iterate_against_fp64(name):
    """Three iterations against FP64; the per-row bound is the same recurrence run on
    |A|, |x|, |y| (so it covers the growth of every term), times the FP32 tolerance."""
    case = CASES[name]
    h, w, r, c, v = case
    order = np.lexsort((c, r))
    r, c, v = r[order], c[order], v[order]
    rp = csr_from_coo(h, r)
    mat = Cocktail.single("csr", coo_of(case), 16)
    x, y0 = vecs(h, w, seed=6)
    k = 3
    got = _iterated(mat, x, y0, k)
    xs, ys = x.astype(np.float64), y0.astype(np.float64)
    xa, ya = np.abs(xs), np.abs(ys)
    for _ in range(k):
        p, _ = _oracle.fp64_spmv(h, w, rp, c, v, xs, None)
        pa, _ = _oracle.fp64_spmv(h, w, rp, c, np.abs(v), xa, None)
        ys = ys + p
        ya = ya + pa
        xs, xa = ys.copy(), ya.copy()
    err = np.abs(got - ys) / np.maximum(ya, 1e-30)
    assert err.max() <= k * TOL, err.max()


def test_iterate_rejects_rectangular():
    case = (30, 40, np.array([0, 5], np.int32), np.array([1, 39], np.int32), np.array([1.0, 2.0], np.float32))
    mat = Cocktail.single("csr", COO(*case), 2)
    hd = Handle(mat, None, None)
    with pytest.raises(Exception, match="CSP_EINVAL"):
        hd.iterate(2)
    hd.free()


@pytest.mark.parametrize("fmt,method", [("csr", 16), ("coo", 0), ("csr", 2)])
@pytest.mark.parametrize("graph", [False, True])
def test_l2_persist_changes_no_bit(fmt, method, graph):
    case = CASES["zipf"]
    h, w = case[0], case[1]
    mat = Cocktail.single(fmt, coo_of(case), method)
    x, y0 = vecs(h, w, seed=7)
    base = CSP_FLAG_GRAPH if graph else 0
    a = _iterated(mat, x, y0, 2, base)
    b = _iterated(mat, x, y0, 2, base | CSP_FLAG_L2_PERSIST)
    assert a.tobytes() == b.tobytes()
