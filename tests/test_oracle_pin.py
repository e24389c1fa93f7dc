"""Pins the oracle (oracle/oracle.c) before it is trusted: its serial products must
equal the reference's own serial SpMVs (clSpMV_NV/include/spmv_serial.h, compiled from
its sources) bit for bit, and the committed golden fixtures generated from the
reference (tests/golden/make_golden.py)."""
import ctypes as C
import glob
import hashlib
import json
import os

import numpy as np
import pytest

from clspmv_b200 import COO, capi
from tests import _oracle
from tests.cases import small_cases
from tests.fmt_extract import STRUCT, extract

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FP = C.POINTER(C.c_float)
IP = C.POINTER(C.c_int)
CASES = small_cases()


def _p(a, t=C.c_float):
    return a.ctypes.data_as(C.POINTER(t))


def _vecs(h, w, seed=3):
    rng = np.random.default_rng(seed)
    return rng.uniform(-1, 1, w).astype(np.float32), rng.uniform(-1, 1, h).astype(np.float32)


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLD, "*.npz"))), ids=os.path.basename)
def test_oracle_matches_golden(orc, path):
    g = np.load(path)
    h, w = int(g["height"]), int(g["width"])
    rp = np.zeros(h + 1, np.int32)
    np.cumsum(np.bincount(g["row"], minlength=h), out=rp[1:])
    y = g["y0"].copy()
    orc.orc_csr_spmv_f32(h, _p(rp, C.c_int), _p(g["col"], C.c_int), _p(g["val"]), _p(g["x"]), _p(y))
    assert y.tobytes() == g["y_csr"].tobytes()
    y = g["y0"].copy()
    orc.orc_coo_spmv_f32(g["row"].size, _p(g["row"], C.c_int), _p(g["col"], C.c_int), _p(g["val"]), _p(g["x"]), _p(y))
    assert y.tobytes() == g["y_coo"].tobytes()


def test_golden_conversions_match_product(L):
    """The product's conversions reproduce the reference digests recorded in tests/golden."""
    meta = json.load(open(os.path.join(GOLD, "conversions.json")))
    fn = {"csr": "csp_coo2csr", "ell": "csp_coo2ell", "sell": "csp_coo2sell", "bcsr": "csp_coo2bcsr",
          "bell": "csp_coo2bell", "b4csr": "csp_coo2b4csr", "b4ell": "csp_coo2b4ell", "sbell": "csp_coo2sbell",
          "dia": "csp_coo2dia", "bdia": "csp_coo2bdia"}
    checked = 0
    for name, digests in meta["digests"].items():
        g = np.load(os.path.join(GOLD, f"{name}.npz"))
        for key, want in digests.items():
            fmt = key[:key.index("[")]
            args = tuple(json.loads(key[key.index("["):]))
            src = COO(int(g["height"]), int(g["width"]), g["row"], g["col"], g["val"])
            s = STRUCT[fmt]()
            rc = getattr(L, fn[fmt])(src.ref(), C.byref(s), *args)
            if want == "refused":
                assert rc == capi.CSP_EFORMAT, (name, key)
                continue
            assert rc == 0, (name, key, L.csp_last_error())
            d = extract(fmt, s)
            h = hashlib.sha256()
            for k in sorted(d):
                v = d[k]
                h.update(k.encode())
                h.update(v.tobytes() if isinstance(v, np.ndarray) else repr(v).encode())
            assert h.hexdigest() == want, (name, key)
            checked += 1
    assert checked >= 50


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_serial_equals_reference_serial(orc, ref, name):
    """orc_csr/coo_spmv_f32 keep the reference's summation order: identical bits."""
    h, w, r, c, v = CASES[name]
    x, y0 = _vecs(h, w)
    a, b = COO(h, w, r, c, v), COO(h, w, r, c, v)
    csr = capi.csr_matrix()
    ref.ref_coo2csr(b.ref(), C.byref(csr))
    ya, yb = y0.copy(), y0.copy()
    rp = _oracle_rp = np.ctypeslib.as_array(csr.csr_row_ptr, (h + 1,)).copy()
    col = np.ctypeslib.as_array(csr.csr_col_id, (max(int(rp[-1]), 1),))[: rp[-1]].copy()
    val = np.ctypeslib.as_array(csr.csr_data, (max(int(rp[-1]), 1),))[: rp[-1]].copy()
    orc.orc_csr_spmv_f32(h, _p(rp, C.c_int), _p(col, C.c_int), _p(val), _p(x), _p(ya))
    ref.ref_csr_spmv(C.byref(csr), _p(x), _p(yb), w)
    assert ya.tobytes() == yb.tobytes()
    ya, yb = y0.copy(), y0.copy()
    orc.orc_coo_spmv_f32(b.nnz, _p(b.row, C.c_int), _p(b.col, C.c_int), _p(b.val), _p(x), _p(ya))
    ref.ref_coo_spmv(b.ref(), _p(x), _p(yb), w)
    assert ya.tobytes() == yb.tobytes()


def test_fp64_oracle_against_numpy(orc):
    h, w, r, c, v = CASES["random_irregular"]
    x, y0 = _vecs(h, w)
    rp = np.zeros(h + 1, np.int32)
    np.cumsum(np.bincount(r, minlength=h), out=rp[1:])
    out, bound = _oracle.fp64_spmv(h, w, rp, c, v, x, y0)
    dense = np.zeros((h, w))
    dense[r, c] = v
    want = y0.astype(np.float64) + dense @ x.astype(np.float64)
    assert np.allclose(out, want, rtol=0, atol=1e-12)
    assert np.allclose(bound, _oracle.Y0_WEIGHT * np.abs(y0) + np.abs(dense) @ np.abs(x.astype(np.float64)), atol=1e-12)
    outt, _ = _oracle.fp64_spmv(h, w, rp, c, v, y0, None, transpose=True)
    assert np.allclose(outt, dense.T @ y0.astype(np.float64), atol=1e-12)


def test_error_metric_flags_planted_mistake(orc):
    """A mistake planted in a result is caught by the per-row bound."""
    h, w, r, c, v = CASES["laplacian32"]
    x, y0 = _vecs(h, w)
    rp = np.zeros(h + 1, np.int32)
    np.cumsum(np.bincount(r, minlength=h), out=rp[1:])
    out, bound = _oracle.fp64_spmv(h, w, rp, c, v, x, y0)
    y = out.astype(np.float32)
    e, _ = _oracle.max_rel_err(y, out, bound)
    assert e < 1e-6
    y[17] += 1e-3
    e, worst = _oracle.max_rel_err(y, out, bound)
    assert e > 1e-5 and worst == 17


@pytest.mark.parametrize("name", ["laplacian32", "banded", "stencil6", "block3_small", "random_irregular"])
def test_format_serial_products_bitexact(orc, ref, name):
    """The reference's per-format serial SpMVs equal the oracle's restatements."""
    h, w, r, c, v = CASES[name]
    x, y0 = _vecs(h, w)
    # ELL
    for fmt, conv, args, rs in (("ell", "ref_coo2ell", (32, 0), "ref_ell_spmv"),
                                ("sell", "ref_coo2sell", (32,), "ref_sell_spmv"),
                                ("bcsr", "ref_coo2bcsr", (3, 3, 32), "ref_bcsr_spmv"),
                                ("bell", "ref_coo2bell", (4, 2, 32, 0), "ref_bell_spmv"),
                                ("sbell", "ref_coo2sbell", (4, 2, 32), "ref_sbell_spmv"),
                                ("dia", "ref_coo2dia", (32,), "ref_dia_spmv"),
                                ("bdia", "ref_coo2bdia", (32,), "ref_bdia_spmv")):
        if fmt in ("dia", "bdia") and h > w:
            continue
        src = COO(h, w, r, c, v)
        s = STRUCT[fmt]()
        ok = getattr(ref, conv)(src.ref(), C.byref(s), *args)
        if fmt in ("dia", "bdia", "sbell") and ok == 0:
            continue
        d = extract(fmt, s)
        yr = np.concatenate([y0, np.zeros(4096, np.float32)])
        getattr(ref, rs)(C.byref(s), _p(x), _p(yr), w)
        yo = np.concatenate([y0, np.zeros(4096, np.float32)])
        if fmt == "ell":
            orc.orc_ell_spmv_f32(h, d["ell_num"], d["hal"], _p(d["col"], C.c_int), _p(d["val"]), _p(x), _p(yo))
        elif fmt == "sell":
            orc.orc_sell_spmv_f32(h, C.c_uint(d["sh"]), d["num"], _p(d["sp"], C.c_int), _p(d["col"], C.c_int),
                                  _p(d["val"]), _p(x), _p(yo))
        elif fmt == "bcsr":
            orc.orc_bcsr_spmv_f32(h, d["rows"], C.c_uint(d["bw"]), C.c_uint(d["bh"]), d["al"], _p(d["rp"], C.c_int),
                                  _p(d["col"], C.c_int), _p(d["val"]), _p(x), w, _p(yo))
        elif fmt == "bell":
            orc.orc_bell_spmv_f32(d["rows"], d["nb"], C.c_uint(d["bw"]), C.c_uint(d["bh"]), d["hal"],
                                  _p(d["col"], C.c_int), _p(d["val"]), _p(x), _p(yo))
        elif fmt == "sbell":
            orc.orc_sbell_spmv_f32(h, w, C.c_uint(d["bw"]), C.c_uint(d["bh"]), C.c_uint(d["sh"]), d["num"],
                                   _p(d["sp"], C.c_int), _p(d["col"], C.c_int), _p(d["val"]), _p(x), _p(yo))
        elif fmt == "dia":
            orc.orc_dia_spmv_f32(d["num"], d["al"], _p(d["off"], C.c_int), _p(d["val"]), _p(x), w, _p(yo))
        elif fmt == "bdia":
            orc.orc_bdia_spmv_f32(d["num"], d["al"], _p(d["off"], C.c_int), _p(d["bptr"], C.c_int), _p(d["val"]),
                                  _p(x), w, _p(yo))
        assert yo.tobytes() == yr.tobytes(), (name, fmt)
