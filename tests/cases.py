"""Small seeded matrices for the parity tests: regular, irregular, empty rows,
rectangular, banded, blocked, unsorted and duplicated inputs."""
from __future__ import annotations

import numpy as np

from clspmv_b200 import matrices as M


def _random(h, w, density, seed, empty_rows=(), first_nonempty=True):
    rng = np.random.default_rng(seed)
    mask = rng.random((h, w)) < density
    for r in empty_rows:
        mask[r, :] = False
    if first_nonempty:
        mask[0, rng.integers(0, w)] = True
    r, c = np.nonzero(mask)
    v = rng.standard_normal(r.size).astype(np.float32)
    return h, w, r.astype(np.int32), c.astype(np.int32), v


def _banded(n, offsets, seed, drop=0.0):
    rng = np.random.default_rng(seed)
    rows, cols = [], []
    for o in offsets:
        r = np.arange(max(0, -o), min(n, n - o))
        keep = rng.random(r.size) >= drop
        rows.append(r[keep])
        cols.append(r[keep] + o)
    r = np.concatenate(rows)
    c = np.concatenate(cols)
    order = np.lexsort((c, r))
    r, c = r[order], c[order]
    v = rng.uniform(0.5, 1.5, r.size).astype(np.float32)
    return n, n, r.astype(np.int32), c.astype(np.int32), v


def _shuffled(case, seed):
    h, w, r, c, v = case
    p = np.random.default_rng(seed).permutation(r.size)
    return h, w, r[p].copy(), c[p].copy(), v[p].copy()


def _with_duplicates(case, seed, k=7):
    h, w, r, c, v = case
    rng = np.random.default_rng(seed)
    idx = rng.integers(0, r.size, k)
    r2 = np.concatenate([r, r[idx]])
    c2 = np.concatenate([c, c[idx]])
    v2 = np.concatenate([v, rng.standard_normal(k).astype(np.float32)])
    p = rng.permutation(r2.size)
    return h, w, r2[p].copy(), c2[p].copy(), v2[p].copy()


def small_cases():
    """name -> (height, width, row, col, val); rows sorted unless the name says otherwise."""
    cases = {
        "laplacian8": M.laplacian_2d(8),
        "laplacian32": M.laplacian_2d(32),
        "random_irregular": _random(203, 177, 0.03, 1, empty_rows=(5, 6, 7, 100, 202)),
        "random_dense_rows": _random(64, 64, 0.4, 2),
        "rect_wide": _random(37, 300, 0.05, 3),
        "rect_tall": _random(300, 41, 0.05, 4),
        "zipf_small": M.zipf_rows(1500, seed=5, max_len=400),
        "banded": _banded(257, [-9, -8, -1, 0, 1, 2, 3, 40], 6, drop=0.1),
        "stencil6": M.stencil_27(6, seed=7),
        "block3_small": M.block_3x3(70, deg=(3, 8), band=20, seed=8),
        "block_like_4": M.block_3x3(40, deg=(2, 6), band=10, seed=9, bs=4),
        "one_by_one": (1, 1, np.array([0], np.int32), np.array([0], np.int32), np.array([2.5], np.float32)),
        "single_row": (1, 90, np.zeros(5, np.int32), np.array([3, 10, 11, 50, 89], np.int32),
                       np.arange(1, 6, dtype=np.float32)),
        "single_col": (90, 1, np.array([0, 4, 5, 88, 89], np.int32), np.zeros(5, np.int32),
                       np.arange(1, 6, dtype=np.float32)),
    }
    cases["unsorted_random"] = _shuffled(cases["random_irregular"], 10)
    cases["unsorted_stencil"] = _shuffled(cases["stencil6"], 11)
    return cases


def duplicate_cases():
    base = small_cases()
    return {"dup_random": _with_duplicates(base["random_irregular"], 12),
            "dup_banded": _with_duplicates(base["banded"], 13)}
