"""Byte-exact parity of the product's host conversions (libclspmv_b200.so, csp_coo2*)
with the reference's own conversions (clSpMV_NV/include/matrix_storage.h, compiled
from its sources into oracle/_ref) on the same inputs."""
import ctypes as C

import numpy as np
import pytest

from clspmv_b200 import COO, capi
from tests.cases import duplicate_cases, small_cases
from tests.fmt_extract import STRUCT, assert_same, extract

CASES = small_cases()
DUPS = duplicate_cases()

# (format, product function, reference function, extra args)
CONVERSIONS = [
    ("csr", "csp_coo2csr", "ref_coo2csr", ()),
    ("ell", "csp_coo2ell", "ref_coo2ell", (32, 0)),
    ("ell", "csp_coo2ell", "ref_coo2ell", (7, 0)),
    ("sell", "csp_coo2sell", "ref_coo2sell", (32,)),
    ("sell", "csp_coo2sell", "ref_coo2sell", (128,)),
    ("sell", "csp_coo2sell", "ref_coo2sell", (5,)),
    ("bcsr", "csp_coo2bcsr", "ref_coo2bcsr", (3, 3, 32)),
    ("bcsr", "csp_coo2bcsr", "ref_coo2bcsr", (4, 2, 32)),
    ("bcsr", "csp_coo2bcsr", "ref_coo2bcsr", (8, 8, 16)),
    ("bell", "csp_coo2bell", "ref_coo2bell", (3, 3, 32, 0)),
    ("bell", "csp_coo2bell", "ref_coo2bell", (4, 1, 32, 0)),
] + [("b4csr", "csp_coo2b4csr", "ref_coo2b4csr", (bw, bh, 32)) for bw in (4, 8) for bh in (1, 2, 4, 8)] \
  + [("b4ell", "csp_coo2b4ell", "ref_coo2b4ell", (bw, bh, 32, 0)) for bw in (4, 8) for bh in (1, 2, 4, 8)] \
  + [("sbell", "csp_coo2sbell", "ref_coo2sbell", (bw, bh, 32)) for bw in (4, 8) for bh in (1, 2, 4, 8)]


def _coo(case):
    h, w, r, c, v = case
    return COO(h, w, r, c, v)


def _run_pair(L, ref, fmt, pf, rf, args, case):
    a, b = _coo(case), _coo(case)
    sa, sb = STRUCT[fmt](), STRUCT[fmt]()
    rc = getattr(L, pf)(a.ref(), C.byref(sa), *args)
    rr = getattr(ref, rf)(b.ref(), C.byref(sb), *args)
    return a, b, sa, sb, rc, rr


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("conv", CONVERSIONS, ids=lambda c: f"{c[1]}{c[3]}")
def test_conversion_bytes(L, ref, name, conv):
    fmt, pf, rf, args = conv
    if fmt == "sell" and name.startswith("unsorted"):
        pytest.skip("the reference coo2sell reads its input as row-sorted without sorting it "
                    "(matrix_storage.h:1414-1431); unsorted input is undefined there")
    a, b, sa, sb, rc, rr = _run_pair(L, ref, fmt, pf, rf, args, CASES[name])
    if fmt in ("b4csr", "b4ell", "sbell") and rr == 0:
        assert rc == capi.CSP_EFORMAT
        return
    assert rc == capi.CSP_OK, L.csp_last_error()
    assert_same(extract(fmt, sa), extract(fmt, sb), f"{name}/{pf}{args}")
    # the input COO is sorted in place by both sides the same way
    assert_same(extract("coo", a.s), extract("coo", b.s), f"{name}/input")


@pytest.mark.parametrize("name", sorted(CASES))
def test_dia_bdia_bytes(L, ref, name):
    h, w = CASES[name][0], CASES[name][1]
    for fmt, pf, rf in (("dia", "csp_coo2dia", "ref_coo2dia"), ("bdia", "csp_coo2bdia", "ref_coo2bdia")):
        if h > w:
            continue  # rows beyond the DIA length: undefined behaviour in the reference
        a, b, sa, sb, rc, rr = _run_pair(L, ref, fmt, pf, rf, (32,), CASES[name])
        if rr == 0:
            # too much padding: both refuse, with the same diagonal count reported
            assert rc == capi.CSP_EFORMAT
            if fmt == "dia":
                assert (sa.dia_num, sa.dia_length_aligned) == (sb.dia_num, sb.dia_length_aligned)
            continue
        assert rc == capi.CSP_OK, L.csp_last_error()
        assert_same(extract(fmt, sa), extract(fmt, sb), f"{name}/{fmt}")


@pytest.mark.parametrize("name", sorted(CASES))
def test_sort_coo_bytes(L, ref, name):
    a, b = _coo(CASES[name]), _coo(CASES[name])
    assert L.csp_sort_coo(a.ref()) == capi.CSP_OK
    assert ref.ref_sort_coo(b.ref()) == 1
    assert_same(extract("coo", a.s), extract("coo", b.s), name)
    assert L.csp_if_sorted_coo(a.ref()) == ref.ref_if_sorted_coo(b.ref()) == 1


@pytest.mark.parametrize("name", sorted(DUPS))
def test_duplicates_follow_reference(L, ref, name):
    """Duplicate (row, col) entries: same order after sorting, same winner in DIA."""
    a, b = _coo(DUPS[name]), _coo(DUPS[name])
    assert L.csp_sort_coo(a.ref()) == capi.CSP_OK
    assert ref.ref_sort_coo(b.ref()) == 1
    assert_same(extract("coo", a.s), extract("coo", b.s), name)
    for fmt, pf, rf, args in (("csr", "csp_coo2csr", "ref_coo2csr", ()), ("dia", "csp_coo2dia", "ref_coo2dia", (32,)),
                              ("bcsr", "csp_coo2bcsr", "ref_coo2bcsr", (4, 4, 32))):
        a, b, sa, sb, rc, rr = _run_pair(L, ref, fmt, pf, rf, args, DUPS[name])
        if fmt == "dia" and rr == 0:
            continue
        assert rc == 0
        assert_same(extract(fmt, sa), extract(fmt, sb), f"{name}/{fmt}")


@pytest.mark.parametrize("name", ["laplacian32", "random_irregular", "zipf_small", "stencil6"])
def test_pad_csr_bytes(L, ref, name):
    a, b = _coo(CASES[name]), _coo(CASES[name])
    ca, cb = capi.csr_matrix(), capi.csr_matrix()
    assert L.csp_coo2csr(a.ref(), C.byref(ca)) == 0
    ref.ref_coo2csr(b.ref(), C.byref(cb))
    for al in (4, 3, 8):
        pa, pb = capi.csr_matrix(), capi.csr_matrix()
        assert L.csp_pad_csr(C.byref(ca), C.byref(pa), al) == 0
        ref.ref_pad_csr(C.byref(cb), C.byref(pb), al)
        assert_same(extract("csr", pa), extract("csr", pb), f"{name}/pad{al}")


@pytest.mark.parametrize("name", ["laplacian32", "random_irregular", "banded", "block3_small", "stencil6"])
def test_back_to_coo(L, ref, name):
    """dia2coo / bdia2coo / ell2coo / bcsr2coo / bell2coo agree with the reference."""
    for fmt, to, conv, args, rconv in (("ell", "ell2coo", "coo2ell", (32, 0), "ref_coo2ell"),
                                       ("bcsr", "bcsr2coo", "coo2bcsr", (3, 3, 32), "ref_coo2bcsr"),
                                       ("bell", "bell2coo", "coo2bell", (4, 2, 32, 0), "ref_coo2bell"),
                                       ("dia", "dia2coo", "coo2dia", (32,), "ref_coo2dia"),
                                       ("bdia", "bdia2coo", "coo2bdia", (32,), "ref_coo2bdia")):
        a, b, sa, sb, rc, rr = _run_pair(L, ref, fmt, f"csp_{conv}", rconv, args, CASES[name])
        if fmt in ("dia", "bdia") and rr == 0:
            continue
        oa, ob = capi.coo_matrix(), capi.coo_matrix()
        assert getattr(L, f"csp_{to}")(C.byref(sa), C.byref(oa)) == 0, L.csp_last_error()
        getattr(ref, f"ref_{to}")(C.byref(sb), C.byref(ob))
        assert_same(extract("coo", oa), extract("coo", ob), f"{name}/{to}")


def test_invalid_input_is_an_error_not_a_crash(L):
    bad = COO(4, 4, [0, 1, 9], [0, 1, 2], [1, 2, 3])   # row 9 outside a 4x4 matrix
    s = capi.csr_matrix()
    assert L.csp_coo2csr(bad.ref(), C.byref(s)) == capi.CSP_EINVAL
    assert b"outside" in L.csp_last_error()
    ok = COO(4, 4, [0, 1, 2], [0, 1, 2], [1, 2, 3])
    e = capi.ell_matrix()
    assert L.csp_coo2ell(ok.ref(), C.byref(e), 32, 0) == 0
    e2 = capi.ell_matrix()
    two = COO(2, 4, [0, 0, 1], [0, 1, 2], [1, 2, 3])
    assert L.csp_coo2ell(two.ref(), C.byref(e2), 32, 1) == capi.CSP_EINVAL   # ellnum below the longest row


@pytest.mark.parametrize("name", ["laplacian32", "random_irregular", "block3_small", "stencil6"])
@pytest.mark.parametrize("shape", [(4, 1), (4, 2), (8, 2), (8, 4)], ids=lambda s: f"{s[0]}x{s[1]}")
@pytest.mark.parametrize("alignment", [32, 7])
def test_rearrange_bell_4col_bytes(L, ref, name, shape, alignment):
    """util.cpp:273 rearrange_bell_4col on coo2bell output: float4 data layout and /4
    column ids byte-identical to the reference's, except the alignment slots between
    4 * row_num and float4_aligned, which the reference leaves uninitialized (malloc) and
    this library zeroes."""
    bw, bh = shape
    a, b = _coo(CASES[name]), _coo(CASES[name])
    sa, sb = capi.bell_matrix(), capi.bell_matrix()
    assert L.csp_coo2bell(a.ref(), C.byref(sa), bw, bh, 32, 0) == 0
    ref.ref_coo2bell(b.ref(), C.byref(sb), bw, bh, 32, 0)
    assert L.csp_rearrange_bell_4col(C.byref(sa), alignment) == 0
    ref.ref_rearrange_bell_4col(C.byref(sb), alignment)
    for s in (sa, sb):
        assert s.bell_float4_aligned == -(-4 * s.bell_row_num // alignment) * alignment
    f4, rows, ell, w4 = sa.bell_float4_aligned, sa.bell_row_num, sa.bell_block_num, bw // 4
    ncol = sa.bell_height_aligned * ell
    ca = np.ctypeslib.as_array(sa.bell_col_id, shape=(max(ncol, 1),))[:ncol]
    cb = np.ctypeslib.as_array(sb.bell_col_id, shape=(max(ncol, 1),))[:ncol]
    assert np.array_equal(ca, cb)
    n = f4 * bh * w4 * ell
    da = np.ctypeslib.as_array(sa.bell_data, shape=(max(n, 1),))[:n].reshape(ell, w4, bh, f4)
    db = np.ctypeslib.as_array(sb.bell_data, shape=(max(n, 1),))[:n].reshape(ell, w4, bh, f4)
    defined = np.arange(f4) < 4 * rows
    assert da[..., defined].tobytes() == db[..., defined].tobytes()
    assert np.all(da[..., ~defined] == 0)
    bad = capi.bell_matrix()
    bad.bell_bwidth = 3
    assert L.csp_rearrange_bell_4col(C.byref(bad), 32) == capi.CSP_EINVAL
