"""Partition parity: csp_analyze_matrix (CSP_ANALYZE_REFERENCE) against the reference's
own analyze_matrix (clSpMV_NV/src/analyze.cpp:3704, compiled from its sources) with the
reference's calibration tables: same formats used, same kernel variants and work-group
counts, and byte-identical sub-matrices."""
import ctypes as C
import os

import numpy as np
import pytest

from clspmv_b200 import COO, capi, matrices as M
from tests import _oracle
from tests.cases import small_cases
from tests.fmt_extract import assert_same, extract

FORMATS = [("bdia", "bdia"), ("dia", "dia"), ("sbell", "sbell"), ("bell", "b4ell"), ("bcsr", "b4csr"),
           ("sell", "sell"), ("ell", "ell"), ("csr", "csr"), ("coo", "coo")]


def _banded_blocks(n=4096, seed=31):
    """Dense 4x4 blocks near the diagonal plus scattered entries: exercises the block peel."""
    rng = np.random.default_rng(seed)
    rows, cols = [], []
    for br in range(n // 4):
        for bc in {br, min(br + 1, n // 4 - 1), max(br - 3, 0)}:
            for a in range(4):
                for b in range(4):
                    if rng.random() < 0.9:
                        rows.append(4 * br + a)
                        cols.append(4 * bc + b)
    rows += list(rng.integers(0, n, n))
    cols += list(rng.integers(0, n, n))
    r, c = np.array(rows), np.array(cols)
    key = np.unique(r.astype(np.int64) * n + c)
    r, c = (key // n).astype(np.int32), (key % n).astype(np.int32)
    return n, n, r, c, rng.standard_normal(r.size).astype(np.float32)


def _uniform_rows(n, k, seed):
    rng = np.random.default_rng(seed)
    rows = np.repeat(np.arange(n), k)
    cols = rng.integers(0, n, n * k)
    key = np.unique(rows.astype(np.int64) * n + cols)
    r, c = (key // n).astype(np.int32), (key % n).astype(np.int32)
    return n, n, r, c, rng.standard_normal(r.size).astype(np.float32)


def _stencil9(g, seed=0):
    rng = np.random.default_rng(seed)
    n = g * g
    k = np.arange(n)
    i, j = k // g, k % g
    cols = []
    for di in (-1, 0, 1):
        for dj in (-1, 0, 1):
            ok = (i + di >= 0) & (i + di < g) & (j + dj >= 0) & (j + dj < g)
            cols.append(np.where(ok, k + di * g + dj, -1))
    cols = np.stack(cols, 1)
    mask = cols >= 0
    r = np.repeat(k, mask.sum(1)).astype(np.int32)
    return n, n, r, cols[mask].astype(np.int32), rng.uniform(0.5, 1.5, r.size).astype(np.float32)


def _plus_noise(case, k, seed):
    h, w, r, c, v = case
    rng = np.random.default_rng(seed)
    r2 = np.concatenate([r, rng.integers(0, h, k)])
    c2 = np.concatenate([c, rng.integers(0, w, k)])
    v2 = np.concatenate([v, rng.standard_normal(k).astype(np.float32)])
    key, idx = np.unique(r2.astype(np.int64) * w + c2, return_index=True)
    return h, w, (key // w).astype(np.int32), (key % w).astype(np.int32), v2[idx]


def _cases():
    cases = dict(small_cases())
    cases.update({
        "laplacian128": M.laplacian_2d(128),
        "zipf_20k": M.zipf_rows(20_000, seed=33, max_len=2000),
        "stencil12": M.stencil_27(12, seed=34),
        "block3_2k": M.block_3x3(2000, deg=(10, 30), band=100, seed=35),
        "banded_blocks": _banded_blocks(),
        "block8": M.block_3x3(300, deg=(4, 9), band=30, seed=36, bs=8),
        # larger inputs reaching the other extraction paths under the shipped tables
        "stencil9_512_bdia": _stencil9(512),                          # BDIA, 3 bands
        "laplacian256_noise_ell_coo": _plus_noise(M.laplacian_2d(256), 20000, 1),   # ELL + COO
        "uniform16_ell": _uniform_rows(100_000, 16, 2),               # ELL
        "block4_bell": M.block_3x3(20_000, deg=(4, 10), band=100, seed=7, bs=4),      # BELL 4x4
        "block8_sbell": M.block_3x3(5000, deg=(3, 8), band=50, seed=6, bs=8),         # SBELL 4x8
        "zipf_200k_ell_coo": M.zipf_rows(200_000, seed=8, max_len=3000),              # ELL + COO
        "stencil48_dia": M.stencil_27(48),                            # DIA, 27 diagonals
    })
    return cases


CASES = _cases()


@pytest.fixture(scope="module")
def bench_path():
    p = _oracle.REF_BENCH
    if not os.path.isdir(os.path.join(p, "benchmark")):
        pytest.skip("reference calibration tables not built (make -C oracle)")
    return p


@pytest.mark.parametrize("name", sorted(CASES))
def test_partition_matches_reference(L, ref, bench_path, name):
    h, w, r, c, v = CASES[name]
    os.environ["CLSPMVPATH"] = bench_path
    a, b = COO(h, w, r, c, v), COO(h, w, r, c, v)
    # the reference analyzer expects sorted input (ReadMMF sorts)
    assert ref.ref_sort_coo(b.ref()) == 1
    mine, theirs = capi.cocktail(), capi.cocktail()
    opts = capi.csp_analyze_opts(capi.CSP_ANALYZE_REFERENCE, bench_path.encode(), 0, None)
    assert L.csp_analyze_matrix(a.ref(), C.byref(mine), C.byref(opts)) == 0, L.csp_last_error()
    ref.ref_analyze_matrix(b.ref(), C.byref(theirs), 1)
    used = []
    for f, ext in FORMATS:
        assert getattr(mine, f"ifuse{f}") == getattr(theirs, f"ifuse{f}"), f"{name}: ifuse{f}"
        if getattr(theirs, f"ifuse{f}"):
            used.append(f)
            assert getattr(mine, f"{f}_meth_num") == getattr(theirs, f"{f}_meth_num"), f"{name}: {f}_meth_num"
            assert_same(extract(ext, getattr(mine, f)), extract(ext, getattr(theirs, f)), f"{name}.{f}")
    if theirs.ifusecsr:
        assert mine.csr_group_num == theirs.csr_group_num
    if theirs.ifusecoo:
        assert mine.coo_group_num == theirs.coo_group_num
    assert (mine.mat_width, mine.mat_height, mine.mat_nnz) == (theirs.mat_width, theirs.mat_height, theirs.mat_nnz)
    # every nonzero lands in exactly one part
    total = sum(getattr(mine, f).matinfo.nnz for f in used)
    assert total == b.nnz, (name, used, total, b.nnz)
    L.csp_free_cocktail(C.byref(mine))
    ref.ref_free_cocktail(C.byref(theirs))


def test_laplacian_partition_is_dia(L, bench_path):
    """The 128x128 5-point Laplacian becomes DIA with 5 diagonals under the shipped tables."""
    h, w, r, c, v = M.laplacian_2d(128)
    a = COO(h, w, r, c, v)
    mine = capi.cocktail()
    opts = capi.csp_analyze_opts(0, bench_path.encode(), 0, None)
    assert L.csp_analyze_matrix(a.ref(), C.byref(mine), C.byref(opts)) == 0
    assert mine.ifusedia and not mine.ifusecsr and mine.dia.dia_num == 5
    assert list(np.ctypeslib.as_array(mine.dia.dia_offsets, (5,))) == [-128, -1, 0, 1, 128]
    L.csp_free_cocktail(C.byref(mine))


def test_missing_tables_is_an_error(L):
    a = COO(3, 3, [0, 1, 2], [0, 1, 2], [1, 2, 3])
    mine = capi.cocktail()
    opts = capi.csp_analyze_opts(0, b"/nonexistent", 0, None)
    assert L.csp_analyze_matrix(a.ref(), C.byref(mine), C.byref(opts)) == capi.CSP_EIO
