"""csp_read_mmf against the reference's ReadMMF (clSpMV_NV/src/fileio.cpp:10): same
dimensions, same sorted entries, symmetric expansion and pattern values."""
import ctypes as C

import numpy as np
import pytest

from clspmv_b200 import capi
from tests.fmt_extract import assert_same, extract


def _write(path, field, sym, h, w, entries):
    with open(path, "w") as f:
        f.write(f"%%MatrixMarket matrix coordinate {field} {sym}\n% a comment line\n%\n")
        f.write(f"{h} {w} {len(entries)}\n")
        for r, c, v in entries:
            f.write(f"{r + 1} {c + 1}" + ("" if field == "pattern" else f" {v:.9g}") + "\n")


@pytest.mark.parametrize("field,sym", [("real", "general"), ("pattern", "general"), ("real", "symmetric"),
                                       ("pattern", "symmetric")])
def test_read_mmf_matches_reference(L, ref, tmp_path, field, sym):
    rng = np.random.default_rng(7)
    h = w = 300
    mask = rng.random((h, w)) < 0.02
    if sym == "symmetric":
        mask = np.tril(mask)
        np.fill_diagonal(mask, True)
    r, c = np.nonzero(mask)
    p = rng.permutation(r.size)            # unsorted file order
    entries = [(int(r[i]), int(c[i]), float(rng.standard_normal())) for i in p]
    path = str(tmp_path / "m.mtx")
    _write(path, field, sym, h, w, entries)
    a, b = capi.coo_matrix(), capi.coo_matrix()
    assert L.csp_read_mmf(path.encode(), C.byref(a)) == 0, L.csp_last_error()
    ref.ref_read_mmf(path.encode(), C.byref(b))
    assert_same(extract("coo", a), extract("coo", b), f"{field}/{sym}")


def test_read_mmf_errors(L, tmp_path):
    m = capi.coo_matrix()
    assert L.csp_read_mmf(str(tmp_path / "missing.mtx").encode(), C.byref(m)) == capi.CSP_EIO
    bad = tmp_path / "bad.mtx"
    bad.write_text("%%MatrixMarket matrix coordinate real general\n3 3 2\n1 1 1.0\n")
    assert L.csp_read_mmf(str(bad).encode(), C.byref(m)) == capi.CSP_EIO
