"""The committed B200 calibration tables (clspmv_b200/tables_b200, written by
csp_benchmark_tables on a B200) have the reference's table layout and drive the
reference-mode analyzer on the CPU: every nonzero lands in exactly one sub-matrix."""
import os

import numpy as np
import pytest

from clspmv_b200 import CSP_ANALYZE_REFERENCE, analyze_matrix, matrices as M
from tests.gpu_util import coo_of

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TABLES = os.path.join(ROOT, "clspmv_b200", "tables_b200")
LAYOUT = {"overhead.ben": 3, "dia.ben": 6, "bdia.ben": 7, "ell.ben": 4, "sell.ben": 4, "csr.ben": 5, "coo.ben": 4,
          "bcsr.ben": 5, "bell.ben": 6, "sbell.ben": 5}


@pytest.mark.parametrize("name", sorted(LAYOUT))
def test_table_columns(name):
    rows = [ln.split() for ln in open(os.path.join(TABLES, "benchmark", name)) if ln.strip()]
    assert rows
    assert all(len(r) == LAYOUT[name] for r in rows)


def _stored_nnz(mat):
    s = mat.s
    n = 0
    for f in mat.uses():
        n += getattr(s, f).matinfo.nnz
    return n


@pytest.mark.parametrize("name,case", [("laplacian", M.laplacian_2d(48)), ("zipf", M.zipf_rows(8000, seed=3, max_len=800)),
                                       ("stencil", M.stencil_27(12, seed=4)),
                                       ("block4", M.block_3x3(800, deg=(4, 8), band=30, seed=5, bs=4))])
def test_reference_analyzer_with_b200_tables(name, case):
    mat = analyze_matrix(coo_of(case), mode=CSP_ANALYZE_REFERENCE, bench_path=TABLES)
    assert mat.uses()
    assert _stored_nnz(mat) >= case[2].size   # padded formats may store explicit zeros
    mat.free()
