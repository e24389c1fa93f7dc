"""Host side of the batched path, without a GPU: the structure figures the format
choice uses (csp_batch_features_of) against numpy, the byte model's choice, the
sparsity signature shared by matrices of one structure class, and the refusal of
csp_batch_create when no device is visible."""
import numpy as np
import pytest
import torch

from clspmv_b200 import COO, CSP_FLAG_BF16, CspError, matrices as M
from clspmv_b200.batch import Batch, features
from clspmv_b200.capi import (CSP_BFMT_BCSR2, CSP_BFMT_COUNT, CSP_BFMT_CSR, CSP_BFMT_DIA, CSP_BFMT_SELL32,
                              CSP_BFMT_SELL128, CSP_ENODEV)
from tests.cases import duplicate_cases, small_cases

CASES = dict(small_cases())
CASES.update(duplicate_cases())
CASES["lap_sq"] = M.laplacian_sq(30, 21)
CASES["block"] = M.block_3x3(300, deg=(2, 6), band=50, seed=4)
CASES["zipf"] = M.zipf_rows(3000, s=1.85, max_len=700, seed=4)


def _expected(case, bf16=False):
    h, w, r, c, v = case
    nnz = r.size
    lens = np.bincount(r, minlength=h) if h else np.zeros(0, np.int64)
    offs = np.unique(c.astype(np.int64) - r)
    ndiag = offs.size if offs.size <= 64 else -1
    f = {"rows": h, "cols": w, "nnz": nnz, "max_row": int(lens.max()) if h else 0, "ndiag": ndiag,
         "dia_slots": ndiag * ((h + 31) // 32 * 32) if ndiag >= 0 else 0}
    sell = []
    for H in (32, 128):
        pad = np.zeros(((h + H - 1) // H) * H, np.int64)
        pad[:h] = lens
        sell.append(int(pad.reshape(-1, H).max(axis=1).sum() * H) if h else 0)
    f["sell_slots"] = sell
    blocks = []
    for b in (2, 3, 4):
        key = np.unique((r.astype(np.int64) // b) * (w + b) + (c - c % b))
        blocks.append(int(key.size))
    f["bcsr_blocks"] = blocks
    lim, sell_lim = 1.5 * nnz + 64, 2.0 * nnz + 64
    feas = 1 << CSP_BFMT_CSR
    if nnz:
        if sell[0] <= sell_lim:
            feas |= 1 << CSP_BFMT_SELL32
        if sell[1] <= sell_lim:
            feas |= 1 << CSP_BFMT_SELL128
        if ndiag >= 0 and ndiag * h <= lim:
            feas |= 1 << CSP_BFMT_DIA
        for b in (2, 3, 4):
            if blocks[b - 2] * b * b <= lim:
                feas |= 1 << (CSP_BFMT_BCSR2 + b - 2)
    f["feasible"] = feas
    es = 2.0 if bf16 else 4.0
    cost = {CSP_BFMT_CSR: 2 * ((es + 4) * nnz + 4 * h) + 4 * nnz,
            CSP_BFMT_SELL32: (2 * (es + 4) + 4) * sell[0], CSP_BFMT_SELL128: (2 * (es + 4) + 4) * sell[1],
            CSP_BFMT_DIA: (2 * es + 4) * f["dia_slots"]}
    for b in (2, 3, 4):
        cost[CSP_BFMT_BCSR2 + b - 2] = 2 * (4 + es * b * b) * blocks[b - 2] + 4 * b * b * blocks[b - 2]
    best = CSP_BFMT_CSR
    for fmt in range(CSP_BFMT_COUNT):
        if feas & (1 << fmt) and cost[fmt] < cost[best]:
            best = fmt
    f["model_format"] = best
    return f


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("bf16", [False, True])
def test_features_match_numpy(name, bf16):
    got = features(COO(*CASES[name]), CSP_FLAG_BF16 if bf16 else 0)
    want = _expected(CASES[name], bf16)
    for k, v in want.items():
        assert got[k] == v, f"{name}: {k} = {got[k]}, expected {v}"


def test_model_picks_the_structure():
    assert features(COO(*CASES["lap_sq"]))["model_format"] == CSP_BFMT_DIA
    assert features(COO(*CASES["block"]))["model_format"] == CSP_BFMT_BCSR2 + 1
    assert features(COO(*CASES["zipf"]))["model_format"] == CSP_BFMT_CSR


def test_signature_classes():
    a = features(COO(*M.laplacian_sq(40, 40)))["signature"]
    b = features(COO(*M.laplacian_sq(41, 41)))["signature"]
    c = features(COO(*M.block_3x3(540, deg=(2, 6), band=50, seed=1)))["signature"]
    d = features(COO(*M.laplacian_sq(40, 40)), CSP_FLAG_BF16)["signature"]
    assert a == b and a != c and a != d


def test_unsorted_input_gives_the_same_features():
    base = features(COO(*CASES["random_irregular"]))
    shuffled = features(COO(*CASES["unsorted_random"]))
    for k in ("nnz", "ndiag", "dia_slots", "sell_slots", "bcsr_blocks", "feasible", "signature"):
        assert base[k] == shuffled[k]


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-device path")
def test_create_without_device():
    with pytest.raises(CspError) as e:
        Batch([COO(*CASES["lap_sq"])])
    assert e.value.code == CSP_ENODEV
