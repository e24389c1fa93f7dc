"""Reads every field and array of a format struct into numpy, for byte-exact
comparison between the product's conversions and the reference's."""
from __future__ import annotations

import numpy as np

from clspmv_b200 import capi
from clspmv_b200.capi import to_numpy

I32, F32 = np.int32, np.float32


def _info(s):
    return (s.matinfo.width, s.matinfo.height, s.matinfo.nnz)


def extract(fmt: str, s) -> dict:
    d = {"matinfo": _info(s)}
    if fmt == "coo":
        n = s.matinfo.nnz
        d.update(row=to_numpy(s.coo_row_id, n, I32), col=to_numpy(s.coo_col_id, n, I32),
                 val=to_numpy(s.coo_data, n, F32))
    elif fmt == "csr":
        h = s.matinfo.height
        rp = to_numpy(s.csr_row_ptr, h + 1, I32)
        n = int(rp[-1]) if rp.size else 0
        d.update(rp=rp, col=to_numpy(s.csr_col_id, n, I32), val=to_numpy(s.csr_data, n, F32))
    elif fmt == "ell":
        n = s.ell_num * s.ell_height_aligned
        d.update(ell_num=s.ell_num, hal=s.ell_height_aligned, col=to_numpy(s.ell_col_id, n, I32),
                 val=to_numpy(s.ell_data, n, F32))
    elif fmt == "sell":
        sp = to_numpy(s.sell_slice_ptr, s.sell_slice_num + 1, I32)
        n = int(sp[-1])
        d.update(sh=s.sell_slice_height, num=s.sell_slice_num, sp=sp, col=to_numpy(s.sell_col_id, n, I32),
                 val=to_numpy(s.sell_data, n, F32))
    elif fmt == "dia":
        d.update(num=s.dia_num, length=s.dia_length, al=s.dia_length_aligned,
                 off=to_numpy(s.dia_offsets, s.dia_num, I32),
                 val=to_numpy(s.dia_data, s.dia_num * s.dia_length_aligned, F32))
    elif fmt == "bdia":
        bp = to_numpy(s.bdia_bptr, s.bdia_band_num + 1, I32)
        nd = int(bp[-1]) if bp.size else 0
        d.update(num=s.bdia_band_num, length=s.bdia_length, al=s.bdia_length_aligned,
                 off=to_numpy(s.bdia_offsets, s.bdia_band_num, I32), bptr=bp,
                 val=to_numpy(s.bdia_data, nd * s.bdia_length_aligned, F32))
    elif fmt == "bcsr":
        bs = s.bcsr_bwidth * s.bcsr_bheight
        d.update(bw=s.bcsr_bwidth, bh=s.bcsr_bheight, rows=s.bcsr_row_num, al=s.bcsr_aligned_size,
                 nb=s.bcsr_block_num, rp=to_numpy(s.bcsr_row_ptr, s.bcsr_row_num + 1, I32),
                 col=to_numpy(s.bcsr_col_id, s.bcsr_block_num, I32),
                 val=to_numpy(s.bcsr_data, s.bcsr_aligned_size * bs, F32))
    elif fmt == "bell":
        bs = s.bell_bwidth * s.bell_bheight
        n = s.bell_height_aligned * s.bell_block_num
        d.update(bw=s.bell_bwidth, bh=s.bell_bheight, rows=s.bell_row_num, nb=s.bell_block_num,
                 hal=s.bell_height_aligned, col=to_numpy(s.bell_col_id, n, I32),
                 val=to_numpy(s.bell_data, n * bs, F32))
    elif fmt == "b4csr":
        bw4 = s.b4csr_bwidth // 4
        d.update(bw=s.b4csr_bwidth, bh=s.b4csr_bheight, rows=s.b4csr_row_num, al=s.b4csr_aligned_size,
                 nb=s.b4csr_block_num, rp=to_numpy(s.b4csr_row_ptr, s.b4csr_row_num + 1, I32),
                 col=to_numpy(s.b4csr_col_id, s.b4csr_block_num, I32),
                 val=to_numpy(s.b4csr_data, s.b4csr_aligned_size * s.b4csr_bheight * bw4, F32))
    elif fmt == "b4ell":
        bw4, bh, nbr = s.b4ell_bwidth // 4, s.b4ell_bheight, s.b4ell_row_num
        hal, f4, k = s.b4ell_height_aligned, s.b4ell_float4_aligned, s.b4ell_block_num
        col = to_numpy(s.b4ell_col_id, hal * k, I32).reshape(k, hal)[:, :nbr]
        # only the first 4*row_num entries of each f4-long segment are defined (the
        # reference leaves the alignment tail uninitialised)
        val = to_numpy(s.b4ell_data, f4 * bh * bw4 * k, F32).reshape(-1, f4)[:, :4 * nbr]
        d.update(bw=s.b4ell_bwidth, bh=bh, rows=nbr, nb=k, hal=hal, f4=f4, col=col, val=val)
    elif fmt == "sbell":
        sp = to_numpy(s.sbell_slice_ptr, s.sbell_slice_num + 1, I32)
        n = int(sp[-1])
        bs = s.sbell_bwidth * s.sbell_bheight
        sh = s.sbell_slice_height
        col = to_numpy(s.sbell_col_id, n, I32)
        # column ids of the block rows past sbell_row_num in the last slice are left
        # uninitialised by the reference analyzer (analyze.cpp:1819): not compared
        for sl in range(s.sbell_slice_num):
            first = sl * sh
            if first + sh > s.sbell_row_num:
                width = (sp[sl + 1] - sp[sl]) // sh if sh else 0
                for lr in range(max(s.sbell_row_num - first, 0), sh):
                    col[sp[sl] + lr + np.arange(width) * sh] = 0
        d.update(bw=s.sbell_bwidth, bh=s.sbell_bheight, sh=sh, num=s.sbell_slice_num,
                 rows=s.sbell_row_num, sp=sp, col=col, val=to_numpy(s.sbell_data, n * bs, F32))
    else:
        raise ValueError(fmt)
    return d


def assert_same(a: dict, b: dict, what: str = ""):
    assert a.keys() == b.keys(), what
    for k in a:
        x, y = a[k], b[k]
        if isinstance(x, np.ndarray):
            assert x.shape == y.shape, f"{what}.{k}: shape {x.shape} vs {y.shape}"
            # byte-exact (also distinguishes -0.0 / NaN payloads)
            assert x.tobytes() == y.tobytes(), f"{what}.{k}: first diff at {np.flatnonzero(x != y)[:5]}"
        else:
            assert x == y, f"{what}.{k}: {x} vs {y}"


STRUCT = {"coo": capi.coo_matrix, "csr": capi.csr_matrix, "ell": capi.ell_matrix, "sell": capi.sell_matrix,
          "dia": capi.dia_matrix, "bdia": capi.bdia_matrix, "bcsr": capi.bcsr_matrix, "bell": capi.bell_matrix,
          "b4csr": capi.b4csr_matrix, "b4ell": capi.b4ell_matrix, "sbell": capi.sbell_matrix}
