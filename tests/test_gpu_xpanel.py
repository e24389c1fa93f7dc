"""The x-panel kernel choice (CSP_METH_XPANEL on a CSR or COO part): x staged in
shared memory by column panels, one partial sum per run of a row inside a 128-entry
tile, merged per row.  Edge cases of the layout against the FP64 oracle: runs that end
exactly on tile boundaries, empty panels, entries only in the last (partial) panel,
a one-column matrix, rows spread over every panel; plus determinism and graph replay."""
import numpy as np
import pytest

from clspmv_b200 import CSP_FLAG_GRAPH, Cocktail, Handle, matrices as M
from tests.gpu_util import check, coo_of, run, vecs

pytestmark = pytest.mark.gpu

XP = 16
PANEL = 32768


def _case(rows, cols, h, w, seed=0):
    rows = np.asarray(rows, np.int32)
    cols = np.asarray(cols, np.int32)
    order = np.lexsort((cols, rows))
    v = np.random.default_rng(seed).standard_normal(rows.size).astype(np.float32)
    return h, w, rows[order], cols[order], v


def _tile_edges():
    # row 0: exactly one tile in panel 0; row 1: two tiles; row 2: 129 entries (one
    # run ends one entry into the next tile); rows 3..: one entry each
    rows, cols = [], []
    for r, k in ((0, 128), (1, 256), (2, 129)):
        rows += [r] * k
        cols += list(range(k))
    for r in range(3, 40):
        rows.append(r)
        cols.append(r * 7)
    return _case(rows, cols, 40, 40_000)


def _last_panel_only():
    w = 2 * PANEL + 5
    rng = np.random.default_rng(3)
    rows = rng.integers(0, 300, 2000)
    cols = 2 * PANEL + rng.integers(0, 5, 2000)
    key = np.unique(rows.astype(np.int64) * w + cols)
    return _case(key // w, key % w, 300, w)


def _empty_middle_panels():
    w = 6 * PANEL
    rng = np.random.default_rng(4)
    rows = rng.integers(0, 5000, 40_000)
    cols = np.where(rng.random(40_000) < 0.5, rng.integers(0, PANEL, 40_000), rng.integers(5 * PANEL, w, 40_000))
    key = np.unique(rows.astype(np.int64) * w + cols)
    return _case(key // w, key % w, 5000, w)


def _one_column():
    return _case(np.arange(1000), np.zeros(1000), 1000, 1)


def _all_panels_dense_rows():
    # 8 rows of 20,000 entries over 300,000 columns: every row has runs in all 10 panels
    rng = np.random.default_rng(5)
    rows, cols = [], []
    for r in range(8):
        c = np.sort(rng.choice(300_000, 20_000, replace=False))
        rows.append(np.full(c.size, r))
        cols.append(c)
    return _case(np.concatenate(rows), np.concatenate(cols), 8, 300_000)


CASES = {
    "tile_edges": _tile_edges(),
    "last_panel_only": _last_panel_only(),
    "empty_middle_panels": _empty_middle_panels(),
    "one_column": _one_column(),
    "dense_rows": _all_panels_dense_rows(),
    "zipf_wide": M.zipf_rows(120_000, seed=91, max_len=5000),
}


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("fmt", ["csr", "coo"])
def test_xpanel_parity(name, fmt):
    case = CASES[name]
    h, w = case[0], case[1]
    mat = Cocktail.single(fmt, coo_of(case), XP)
    x, y0 = vecs(h, w, seed=11)
    y = run(mat, x, y0, ntimes=2)
    check(case, y, x, y0, ntimes=2)


def test_xpanel_two_launches_and_graph_bits():
    case = CASES["zipf_wide"]
    mat = Cocktail.single("csr", coo_of(case), XP)
    x, y0 = vecs(case[0], case[1], seed=12)
    hd = Handle(mat, x, y0)
    assert hd.launches_per_spmv == 2
    hd.free()
    a = run(mat, x, y0, ntimes=4)
    b = run(mat, x, y0, ntimes=4, flags=CSP_FLAG_GRAPH)
    c = run(mat, x, y0, ntimes=4)
    assert a.tobytes() == b.tobytes() == c.tobytes()


def test_xpanel_rejects_several_rhs():
    case = CASES["tile_edges"]
    mat = Cocktail.single("csr", coo_of(case), XP)
    with pytest.raises(Exception, match="CSP_EUNSUP"):
        Handle(mat, None, None, nrhs=4)
