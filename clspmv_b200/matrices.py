"""Seeded synthetic matrices with the shapes of the benchmark workloads.

The reference measures on matrices from a public sparse-matrix collection that is
not available here (clSpMV_NV/matrix/README; the one shipped MTX file is absent), so
these generators stand in for it with the sizes and value distributions the
workloads name.  Every generator returns a row-major sorted COO as numpy arrays
(row, col, val) plus (height, width); all draws come from numpy.random.default_rng.
"""
from __future__ import annotations

import numpy as np


def laplacian_2d(nx: int = 128):
    """5-point Laplacian on an nx-by-nx grid, natural ordering: 4 on the diagonal,
    -1 to the four neighbours.  nx = 128 gives 16,384 rows and 81,408 nonzeros."""
    n = nx * nx
    k = np.arange(n, dtype=np.int64)
    i, j = k // nx, k % nx
    offs = [(-nx, i > 0), (-1, j > 0), (0, np.ones(n, bool)), (1, j < nx - 1), (nx, i < nx - 1)]
    cols = np.stack([np.where(m, k + o, -1) for o, m in offs], axis=1)
    vals = np.stack([np.where(m, 4.0 if o == 0 else -1.0, 0.0) for o, m in offs], axis=1)
    mask = cols >= 0
    row = np.repeat(k, mask.sum(axis=1)).astype(np.int32)
    return n, n, row, cols[mask].astype(np.int32), vals[mask].astype(np.float32)


def _dedup_uniform_cols(rng, rows, cols, low, high):
    """Redraw columns until no row repeats one (uniform without replacement per row).
    rows must be sorted; low/high are per-entry inclusive/exclusive bounds."""
    span = int(cols.max()) + 1 if low is None and cols.size else 0
    while True:
        if low is None:
            # one int64 key sort: the same order as lexsort((cols, rows)), equal keys are equal pairs
            span = max(span, int(high))
            key = np.sort(rows.astype(np.int64) * span + cols)
            rows, cols = key // span, key % span
        else:
            order = np.lexsort((cols, rows))
            rows, cols = rows[order], cols[order]
            low, high = low[order], high[order]
        dup = np.zeros(rows.size, bool)
        dup[1:] = (rows[1:] == rows[:-1]) & (cols[1:] == cols[:-1])
        nd = int(dup.sum())
        if nd == 0:
            return rows, cols
        if low is None:
            cols[dup] = rng.integers(0, high, nd)
        else:
            cols[dup] = rng.integers(low[dup], high[dup])


def zipf_rows(n: int = 1_000_000, s: float = 2.0, max_len: int = 10_000, seed: int = 0):
    """n-by-n matrix whose row lengths are Zipf(s) clipped to [1, max_len]; columns
    uniform without replacement within each row; values N(0, 1)."""
    rng = np.random.default_rng(seed)
    lens = np.clip(rng.zipf(s, n), 1, max_len).astype(np.int64)
    rows = np.repeat(np.arange(n, dtype=np.int64), lens)
    cols = rng.integers(0, n, rows.size)
    rows, cols = _dedup_uniform_cols(rng, rows, cols, None, n)
    vals = rng.standard_normal(rows.size).astype(np.float32)
    return n, n, rows.astype(np.int32), cols.astype(np.int32), vals


def stencil_27(g: int = 160, seed: int = 0):
    """27-point stencil on a g^3 grid: row k couples to k + dz*g^2 + dy*g + dx for
    dz, dy, dx in {-1, 0, 1} when the neighbour lies inside the grid (out-of-grid
    couplings are absent); values U(0.5, 1.5).  g = 160: 4,096,000 rows,
    478^3 = 109,215,352 nonzeros on 27 diagonals."""
    rng = np.random.default_rng(seed)
    n = g * g * g
    k = np.arange(n, dtype=np.int64)
    z, y, x = k // (g * g), (k // g) % g, k % g
    cols = np.empty((n, 27), dtype=np.int64)
    t = 0
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                ok = ((z + dz >= 0) & (z + dz < g) & (y + dy >= 0) & (y + dy < g) & (x + dx >= 0) & (x + dx < g))
                cols[:, t] = np.where(ok, k + dz * g * g + dy * g + dx, -1)
                t += 1
    mask = cols >= 0
    counts = mask.sum(axis=1)
    col = cols[mask].astype(np.int32)
    del cols
    row = np.repeat(k.astype(np.int32), counts)
    val = rng.uniform(0.5, 1.5, col.size).astype(np.float32)
    return n, n, row, col, val


def block_3x3(nbr: int = 500_000, deg=(10, 30), band: int = 2000, seed: int = 0, bs: int = 3):
    """Block-structured FEM-like matrix: nbr block rows of dense bs-by-bs blocks,
    block-row degree uniform in [deg[0], deg[1]] (capped by the band where the matrix
    is smaller), block columns distinct and uniform within +-band of the diagonal
    block, clamped to the matrix; values N(0, 1)."""
    rng = np.random.default_rng(seed)
    i = np.arange(nbr, dtype=np.int64)
    lo_r = np.maximum(i - band, 0)
    hi_r = np.minimum(i + band, nbr - 1) + 1
    d = np.minimum(rng.integers(deg[0], deg[1] + 1, nbr), hi_r - lo_r)
    brow = np.repeat(i, d)
    lo, hi = lo_r[brow], hi_r[brow]
    bcol = rng.integers(lo, hi)
    brow, bcol = _dedup_uniform_cols(rng, brow, bcol, lo, hi)
    nb = brow.size
    vals = rng.standard_normal((nb, bs, bs)).astype(np.float32)
    a = np.arange(bs, dtype=np.int64)
    rows = (bs * brow[:, None, None] + a[None, :, None] + np.zeros(bs, np.int64)[None, None, :]).ravel()
    cols = (bs * bcol[:, None, None] + np.zeros(bs, np.int64)[None, :, None] + a[None, None, :]).ravel()
    order = np.lexsort((cols, rows))
    n = bs * nbr
    return n, n, rows[order].astype(np.int32), cols[order].astype(np.int32), vals.ravel()[order]


def vector(n: int, seed: int = 1, low: float = -1.0, high: float = 1.0):
    """Dense vector ~ U(low, high), FP32."""
    return np.random.default_rng(seed).uniform(low, high, n).astype(np.float32)


def csr_from_coo(height: int, row: np.ndarray):
    """Row pointer of a row-sorted COO."""
    rp = np.zeros(height + 1, dtype=np.int64)
    np.cumsum(np.bincount(row, minlength=height), out=rp[1:])
    return rp.astype(np.int32)


def laplacian_sq(nx: int, ny: int):
    """L @ L for the 5-point Laplacian L on an nx-by-ny grid: the 13-point
    squared-Laplacian stencil (20 on the diagonal, -8 to the four neighbours, 2 to
    the four diagonal neighbours, 1 two steps along an axis, interior rows), the
    Laplacian family at about 12 nonzeros per row."""
    import scipy.sparse as sp

    def lap1(k):
        return sp.diags([-np.ones(k - 1), 2.0 * np.ones(k), -np.ones(k - 1)], [-1, 0, 1])

    L = (sp.kron(sp.identity(ny), lap1(nx)) + sp.kron(lap1(ny), sp.identity(nx))).tocsr()
    A = (L @ L).tocoo()
    order = np.lexsort((A.col, A.row))
    n = nx * ny
    return n, n, A.row[order].astype(np.int32), A.col[order].astype(np.int32), A.data[order].astype(np.float32)


BATCH_KINDS = ("laplacian", "zipf", "block")


def batch_mixed(count: int = 512, lo: int = 1_000, hi: int = 200_000, seed: int = 0, first: int = 0,
                n: int | None = None):
    """Uneven batch: `count` matrices with row counts log-uniform in [lo, hi], each
    drawn by seed from one of three generators at about 12 nonzeros per row --
    the squared Laplacian (laplacian_sq on a near-square grid), Zipf(1.85) row
    lengths clipped to [1, min(10000, n / 4)] (zipf_rows), or 3x3 blocks with block-row
    degree uniform in [2, 6] (block_3x3, band +-2000 block columns).  Only matrices
    [first, first + n) are built (a shard of the list; all of them by default): every
    matrix's parameters are drawn in list order, so matrix i is the same in every shard
    layout.  Returns a list of (kind, height, width, row, col, val)."""
    rng = np.random.default_rng(seed)
    stop = count if n is None else min(count, first + n)
    out = []
    for i in range(stop):
        rows = int(round(np.exp(rng.uniform(np.log(lo), np.log(hi)))))
        kind = BATCH_KINDS[int(rng.integers(0, 3))]
        s = int(rng.integers(0, 2**31 - 1))
        if i < first:
            continue
        if kind == "laplacian":
            nx = max(3, int(np.sqrt(rows)))
            ny = max(3, rows // nx)
            out.append((kind,) + laplacian_sq(nx, ny))
        elif kind == "zipf":
            out.append((kind,) + zipf_rows(rows, s=1.85, max_len=min(10_000, max(1, rows // 4)), seed=s))
        else:
            out.append((kind,) + block_3x3(max(2, rows // 3), deg=(2, 6), band=2000, seed=s))
    return out


def shard(total: int, world: int, rank: int) -> tuple[int, int]:
    """(first, count) of rank's contiguous share of `total` independent units, the
    first total % world ranks taking one more."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of {world}")
    base, extra = divmod(total, world)
    return rank * base + min(rank, extra), base + (1 if rank < extra else 0)
