"""csp_coo2dia_device / csp_coo2bdia_device / csp_coo2bcsr_device: the DIA, BDIA and
generic BCSR layout builds on the device (matrix_storage.h:937 coo2dia, :1185 coo2bdia,
:1595 coo2bcsr) against the product's host
builds, which tests/test_formats_parity.py pins byte for byte to the reference's own
conversions.  Same bytes without duplicate (row, col) entries, the same errors at the
same entry, and with duplicates the last entry in input order."""
import ctypes as C
import time

import numpy as np
import pytest

from clspmv_b200 import COO, capi, matrices as M
from tests.cases import duplicate_cases, small_cases
from tests.fmt_extract import STRUCT, assert_same, extract

pytestmark = pytest.mark.gpu

CASES = small_cases()
DUPS = duplicate_cases()
BCSR_SHAPES = [(3, 3, 32), (4, 2, 32), (8, 8, 16), (1, 1, 1), (2, 5, 7)]


def _both(L, fmt, host_fn, case, args):
    a, b = COO(*case), COO(*case)
    sa, sb = STRUCT[fmt](), STRUCT[fmt]()
    rd = getattr(L, host_fn + "_device")(a.ref(), C.byref(sa), *args)
    ed = L.csp_last_error()
    rh = getattr(L, host_fn)(b.ref(), C.byref(sb), *args)
    eh = L.csp_last_error()
    return a, b, sa, sb, (rd, ed), (rh, eh)


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("alignment", [32, 1, 5])
def test_dia_device_bytes(L, name, alignment):
    a, b, sa, sb, (rd, ed), (rh, eh) = _both(L, "dia", "csp_coo2dia", CASES[name], (alignment,))
    assert rd == rh, (ed, eh)
    if rh == capi.CSP_OK:
        assert_same(extract("dia", sa), extract("dia", sb), f"{name}/dia{alignment}")
    else:
        assert ed == eh
        assert (sa.dia_length, sa.matinfo.nnz) == (sb.dia_length, sb.matinfo.nnz)
        if b"padding" in eh:
            assert (sa.dia_num, sa.dia_length_aligned) == (sb.dia_num, sb.dia_length_aligned)


@pytest.mark.parametrize("name", sorted(CASES))
def test_bdia_device_bytes(L, name):
    a, b, sa, sb, (rd, ed), (rh, eh) = _both(L, "bdia", "csp_coo2bdia", CASES[name], (32,))
    assert rd == rh, (ed, eh)
    if rh == capi.CSP_OK:
        assert_same(extract("bdia", sa), extract("bdia", sb), f"{name}/bdia")
    else:
        assert ed == eh


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("shape", BCSR_SHAPES, ids=lambda s: "x".join(map(str, s)))
def test_bcsr_device_bytes(L, name, shape):
    a, b, sa, sb, (rd, ed), (rh, eh) = _both(L, "bcsr", "csp_coo2bcsr", CASES[name], shape)
    assert rd == rh == capi.CSP_OK, (ed, eh)
    assert_same(extract("bcsr", sa), extract("bcsr", sb), f"{name}/bcsr{shape}")
    # both sort an unsorted input in place the same way
    assert_same(extract("coo", a.s), extract("coo", b.s), f"{name}/input")


def _last_wins(r, c, v):
    """(row, col) -> value of its last entry in the given order."""
    out = {}
    for i in range(r.size):
        out[(int(r[i]), int(c[i]))] = v[i]
    return out


@pytest.mark.parametrize("name", sorted(DUPS))
def test_dia_device_duplicates(L, name):
    """The host DIA build also keeps the last duplicate in input order: same bytes."""
    a, b, sa, sb, (rd, ed), (rh, eh) = _both(L, "dia", "csp_coo2dia", DUPS[name], (32,))
    assert rd == rh, (ed, eh)
    if rh == capi.CSP_OK:
        assert_same(extract("dia", sa), extract("dia", sb), name)


@pytest.mark.parametrize("name", sorted(DUPS))
def test_bcsr_device_duplicates(L, name):
    """Same blocks as the host build; every stored element is the last entry (in the
    row-sorted input order) at its position."""
    a, b, sa, sb, (rd, ed), (rh, eh) = _both(L, "bcsr", "csp_coo2bcsr", DUPS[name], (3, 3, 32))
    assert rd == rh == capi.CSP_OK, (ed, eh)
    da, db = extract("bcsr", sa), extract("bcsr", sb)
    for k in ("rows", "al", "nb", "rp"):
        assert np.array_equal(np.asarray(da[k]), np.asarray(db[k])), k
    co = extract("coo", a.s)
    want = _last_wins(np.asarray(co["row"]), np.asarray(co["col"]), np.asarray(co["val"]))
    rp, cid, data, al = np.asarray(da["rp"]), np.asarray(da["col"]), np.asarray(da["val"]), int(da["al"])
    assert np.array_equal(cid, np.asarray(db["col"]))
    got = {}
    for br in range(int(da["rows"])):
        for j in range(rp[br], rp[br + 1]):
            for q in range(9):
                rr, cc = 3 * br + q // 3, int(cid[j]) + q % 3
                if (rr, cc) in want:
                    got[(rr, cc)] = data[q * al + j]
    assert got.keys() == want.keys()
    for k in want:
        assert np.float32(got[k]).tobytes() == np.float32(want[k]).tobytes(), k


def test_empty_and_edge(L):
    for h, w in ((1, 1), (5, 3), (3, 5)):
        case = (h, w, np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros(0, np.float32))
        _, _, sa, sb, (rd, _), (rh, _) = _both(L, "dia", "csp_coo2dia", case, (32,))
        assert rd == rh == capi.CSP_OK
        assert_same(extract("dia", sa), extract("dia", sb), f"empty dia {h}x{w}")
        _, _, sa, sb, (rd, _), (rh, _) = _both(L, "bcsr", "csp_coo2bcsr", case, (3, 3, 32))
        assert rd == rh == capi.CSP_OK
        assert_same(extract("bcsr", sa), extract("bcsr", sb), f"empty bcsr {h}x{w}")
    # a zero block size is refused before any device work
    a = COO(2, 2, np.array([0], np.int32), np.array([1], np.int32), np.array([1.0], np.float32))
    assert L.csp_coo2bcsr_device(a.ref(), C.byref(capi.bcsr_matrix()), 0, 3, 32) == capi.CSP_EINVAL


@pytest.mark.parametrize("kind", ["stencil", "block"])
def test_full_size_layouts(L, kind):
    """The C3 stencil (160^3, 109 M entries) as DIA and the C4 3x3-block matrix as
    generic BCSR 3x3, built on the device and on the host: same bytes."""
    if kind == "stencil":
        case, fmt, fn, args = M.stencil_27(160), "dia", "csp_coo2dia", (32,)
    else:
        case, fmt, fn, args = M.block_3x3(500_000), "bcsr", "csp_coo2bcsr", (3, 3, 32)
    a, b = COO(*case), COO(*case)
    sa, sb = STRUCT[fmt](), STRUCT[fmt]()
    w = COO(4, 4, np.arange(4, dtype=np.int32), np.arange(4, dtype=np.int32), np.ones(4, np.float32))
    assert getattr(L, fn + "_device")(w.ref(), C.byref(STRUCT[fmt]()), *args) == 0   # context and modules loaded
    t0 = time.perf_counter()
    assert getattr(L, fn + "_device")(a.ref(), C.byref(sa), *args) == 0, L.csp_last_error()
    t1 = time.perf_counter()
    assert getattr(L, fn)(b.ref(), C.byref(sb), *args) == 0, L.csp_last_error()
    t2 = time.perf_counter()
    assert_same(extract(fmt, sa), extract(fmt, sb), kind)
    print(f"{kind}: {fmt} build on the device {t1 - t0:.2f} s (copies included), on the host {t2 - t1:.2f} s")
