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
