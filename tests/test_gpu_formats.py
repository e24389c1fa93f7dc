"""GPU parity of every format kernel and variant against the FP64 oracle, through the
C ABI (csp_init_mat_kernels / csp_do_spmv / csp_cpy_result_to_cpu)."""
import numpy as np
import pytest

from clspmv_b200 import Cocktail, matrices as M
from tests.cases import small_cases
from tests.gpu_util import check, coo_of, run, vecs

pytestmark = pytest.mark.gpu

CASES = small_cases()
def _long_rows(seed=24):
    """A few very long rows among short ones: 3 rows of 150,000 entries in 2,000 x 200,000."""
    rng = np.random.default_rng(seed)
    h, w = 2000, 200_000
    lens = rng.integers(0, 9, h)
    lens[[0, 777, 1999]] = 150_000
    rows = np.repeat(np.arange(h), lens)
    cols = np.concatenate([np.sort(rng.choice(w, k, replace=False)) for k in lens])
    vals = rng.standard_normal(rows.size).astype(np.float32)
    return h, w, rows.astype(np.int32), cols.astype(np.int32), vals


MEDIUM = {
    "long_rows": _long_rows(),
    "zipf_100k": M.zipf_rows(100_000, seed=21, max_len=6000),
    "stencil24": M.stencil_27(24, seed=22),
    "block3_5k": M.block_3x3(5000, deg=(10, 30), band=300, seed=23),
    "laplacian128": M.laplacian_2d(128),
}
ALL = {**CASES, **MEDIUM}

VARIANTS = (
    [("csr", m, {}) for m in range(7)]
    + [("coo", 0, {})]
    + [("csr", 16, {}), ("coo", 16, {})]
    + [("ell", m, {}) for m in (0, 1)]
    + [("sell", 0, {"slice_height": 32}), ("sell", 1, {"slice_height": 128}), ("sell", 2, {"slice_height": 32}),
       ("sell", 0, {"slice_height": 5})]
    + [("bell", 0, {"bwidth": bw, "bheight": bh}) for bw in (4, 8) for bh in (1, 2, 4, 8)]
    + [("sbell", 0, {"bwidth": bw, "bheight": bh}) for bw in (4, 8) for bh in (1, 2, 4, 8)]
    + [("bcsr", m, {"bwidth": bw, "bheight": bh}) for bw in (4, 8) for bh in (1, 2, 4, 8) for m in (0, 1)]
)
DIAG = [("dia", m, {}) for m in range(4)] + [("bdia", m, {}) for m in range(5)]


def _id(v):
    fmt, m, kw = v
    return f"{fmt}{m}" + "".join(f"-{k[0]}{val}" for k, val in kw.items())


@pytest.mark.parametrize("name", sorted(ALL))
@pytest.mark.parametrize("variant", VARIANTS, ids=_id)
def test_flat_and_block(name, variant):
    fmt, method, kw = variant
    case = ALL[name]
    h, w = case[0], case[1]
    if fmt in ("bell", "sbell", "bcsr") and name in ("zipf_100k", "long_rows") and kw.get("bheight", 1) * kw.get("bwidth", 4) > 8:
        pytest.skip("block padding of a random matrix exceeds the memory-object limit")
    if fmt in ("ell", "bell") and name == "long_rows":
        pytest.skip("ELL padding of 150,000-entry rows: 1.2 GB of zeros")
    try:
        mat = Cocktail.single(fmt, coo_of(case), method, **kw)
    except Exception as e:  # the reference refuses some block shapes (MAX_MEM_OBJ)
        if "CSP_EFORMAT" in str(e):
            pytest.skip(str(e))
        raise
    x, y0 = vecs(h, w)
    y = run(mat, x, y0)
    check(case, y, x, y0)


@pytest.mark.parametrize("name", sorted(ALL))
@pytest.mark.parametrize("variant", DIAG, ids=_id)
def test_diagonal(name, variant):
    fmt, method, kw = variant
    case = ALL[name]
    h, w = case[0], case[1]
    if h > w:
        pytest.skip("DIA needs rows within the diagonal length")
    try:
        mat = Cocktail.single(fmt, coo_of(case), method, **kw)
    except Exception as e:
        if "CSP_EFORMAT" in str(e):
            pytest.skip("too much padding for DIA (the reference refuses it too)")
        raise
    x, y0 = vecs(h, w)
    y = run(mat, x, y0)
    check(case, y, x, y0)


@pytest.mark.parametrize("fmt,method", [("csr", 2), ("coo", 0), ("sell", 0), ("csr", 0), ("csr", 16), ("coo", 16)])
def test_accumulates_over_repeated_spmv(fmt, method):
    """do_spmv(3) computes y0 + 3*A*x (the reference's accumulate semantics)."""
    case = MEDIUM["zipf_100k"]
    mat = Cocktail.single(fmt, coo_of(case), method)
    x, y0 = vecs(case[0], case[1])
    y = run(mat, x, y0, ntimes=3)
    check(case, y, x, y0, ntimes=3)


def test_graph_replay_matches_eager():
    from clspmv_b200 import CSP_FLAG_GRAPH
    case = MEDIUM["zipf_100k"]
    mat = Cocktail.single("coo", coo_of(case), 0)
    x, y0 = vecs(case[0], case[1])
    a = run(mat, x, y0, ntimes=4)
    b = run(mat, x, y0, ntimes=4, flags=CSP_FLAG_GRAPH)
    assert a.tobytes() == b.tobytes()  # deterministic kernels: identical bits


def test_deterministic_bits():
    case = MEDIUM["zipf_100k"]
    for fmt, m in (("csr", 2), ("coo", 0), ("csr", 0)):
        mat = Cocktail.single(fmt, coo_of(case), m)
        x, y0 = vecs(case[0], case[1])
        assert run(mat, x, y0).tobytes() == run(mat, x, y0).tobytes()
