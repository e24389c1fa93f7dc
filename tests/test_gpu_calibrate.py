"""B200 calibration tables (csp_benchmark_tables): the ten .ben files in the layout the
reference's bench_* programs write (clSpMV_NV/src/bench_*.cpp), readable by the
reference-mode analyzer, which then partitions matrices whose SpMVs match the FP64
oracle."""
import numpy as np
import pytest

from clspmv_b200 import COO, CSP_ANALYZE_REFERENCE, analyze_matrix, benchmark_tables, matrices as M
from tests.gpu_util import check, coo_of, run, vecs

pytestmark = pytest.mark.gpu

# integer fields, GFLOPS columns (the analyzer's method counts, analyze.h)
LAYOUT = {"overhead.ben": (2, 1), "dia.ben": (2, 4), "bdia.ben": (2, 5), "ell.ben": (2, 2), "sell.ben": (2, 2),
          "csr.ben": (3, 2), "coo.ben": (3, 1), "bcsr.ben": (4, 1), "bell.ben": (4, 2), "sbell.ben": (4, 1)}
SHAPES = [(1, 4), (2, 4), (4, 4), (8, 4), (1, 8), (2, 8), (4, 8), (8, 8)]   # (bh, bw) in the analyzer's order


@pytest.fixture(scope="module")
def tables(tmp_path_factory):
    d = tmp_path_factory.mktemp("clspmv")
    benchmark_tables(str(d), 0)
    return d


def _rows(path):
    return [ln.split() for ln in path.read_text().splitlines() if ln.strip()]


@pytest.mark.parametrize("name", sorted(LAYOUT))
def test_table_layout(tables, name):
    ni, nd = LAYOUT[name]
    rows = _rows(tables / "benchmark" / name)
    assert rows, name
    for r in rows:
        assert len(r) == ni + nd, r
        assert all(int(v) > 0 for v in r[:ni]), r
        assert all(float(v) > 0.0 for v in r[ni:]), r
    if name in ("bcsr.ben", "bell.ben", "sbell.ben"):
        seen = []
        for r in rows:
            s = (int(r[0]), int(r[1]))
            if not seen or seen[-1] != s:
                seen.append(s)
        assert seen == SHAPES


CASES = {
    "laplacian": M.laplacian_2d(64),
    "zipf": M.zipf_rows(30_000, seed=31, max_len=3000),
    "stencil": M.stencil_27(20, seed=32),
    "block4": M.block_3x3(3000, deg=(4, 10), band=60, seed=33, bs=4),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_reference_analyzer_on_b200_tables(tables, name):
    case = CASES[name]
    h, w = case[0], case[1]
    mat = analyze_matrix(coo_of(case), mode=CSP_ANALYZE_REFERENCE, bench_path=str(tables))
    assert mat.uses(), "empty partition"
    x, y0 = vecs(h, w, seed=3)
    y = run(mat, x, y0)
    check(case, y, x, y0)
    mat.free()
