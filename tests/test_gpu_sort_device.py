"""csp_sort_coo_device and csp_read_mmf_ex(CSP_MMF_SORT_ON_DEVICE): the COO sort by
(row, col) on the device.  Without duplicate (row, col) entries it gives the host sort
(csp_sort_coo, the reference's order) byte for byte; with duplicates, equal entries keep
their input order.  MatrixMarket files read with the device sort match the reference's
ReadMMF (clSpMV_NV/src/fileio.cpp:10)."""
import ctypes as C
import time

import numpy as np
import pytest

from clspmv_b200 import COO, capi
from tests.fmt_extract import assert_same, extract
from tests.test_mmf import _write

pytestmark = pytest.mark.gpu


def _random_coo(h, w, nnz, seed, unique=True):
    rng = np.random.default_rng(seed)
    if unique:
        key = np.unique(rng.integers(0, h * w, int(nnz * 1.1) + 8, dtype=np.int64))[:nnz]
        rng.shuffle(key)
        r, c = (key // w).astype(np.int32), (key % w).astype(np.int32)
    else:
        r = rng.integers(0, h, nnz).astype(np.int32)
        c = rng.integers(0, w, nnz).astype(np.int32)
    return r, c, rng.standard_normal(r.size).astype(np.float32)


def _device_sorted(h, w, r, c, v):
    coo = COO(h, w, r.copy(), c.copy(), v.copy())
    assert capi.lib().csp_sort_coo_device(coo.ref()) == 0, capi.lib().csp_last_error()
    return extract("coo", coo.s)


@pytest.mark.parametrize("h,w,nnz", [(1, 1, 1), (7, 9, 2), (64, 64, 4095), (128, 64, 4096), (200, 300, 4097),
                                     (100_000, 100_000, 1_000_003), (1, 5_000_000, 3_000_000),
                                     (5_000_000, 1, 3_000_000), ((1 << 31) - 1, (1 << 31) - 1, 70_001)])
def test_device_sort_matches_host_sort(h, w, nnz):
    r, c, v = _random_coo(h, w, min(nnz, h * w), seed=nnz % 97)
    got = _device_sorted(h, w, r, c, v)
    host = COO(h, w, r.copy(), c.copy(), v.copy())
    assert capi.lib().csp_sort_coo(host.ref()) == 0
    assert_same(got, extract("coo", host.s), f"{h}x{w} nnz={r.size}")
    order = np.lexsort((c, r))
    assert np.array_equal(np.asarray(got["row"]), r[order])
    assert np.array_equal(np.asarray(got["col"]), c[order])


def test_device_sort_is_stable_on_duplicates():
    h, w = 300, 200
    r, c, v = _random_coo(h, w, 200_000, seed=5, unique=False)
    got = _device_sorted(h, w, r, c, v)
    order = np.lexsort((c, r))   # numpy's lexsort is stable: ties keep input order
    assert np.array_equal(np.asarray(got["row"]), r[order])
    assert np.array_equal(np.asarray(got["col"]), c[order])
    assert np.array_equal(np.asarray(got["val"]).view(np.uint32), v[order].view(np.uint32))


def test_device_sort_large():
    h = w = 4_000_000
    r, c, v = _random_coo(h, w, 40_000_000, seed=11)
    coo = COO(h, w, r.copy(), c.copy(), v.copy())
    t0 = time.perf_counter()
    assert capi.lib().csp_sort_coo_device(coo.ref()) == 0
    dt = time.perf_counter() - t0
    order = np.lexsort((c, r))
    got = extract("coo", coo.s)
    assert np.array_equal(np.asarray(got["row"]), r[order])
    assert np.array_equal(np.asarray(got["col"]), c[order])
    assert np.array_equal(np.asarray(got["val"]).view(np.uint32), v[order].view(np.uint32))
    print(f"device sort of {r.size} entries: {dt:.3f} s including the copies")


@pytest.mark.parametrize("field,sym", [("real", "general"), ("pattern", "symmetric"), ("real", "symmetric")])
def test_read_mmf_device_sort_matches_reference(L, ref, tmp_path, field, sym):
    rng = np.random.default_rng(9)
    h = w = 400
    mask = rng.random((h, w)) < 0.03
    if sym == "symmetric":
        mask = np.tril(mask)
        np.fill_diagonal(mask, True)
    r, c = np.nonzero(mask)
    p = rng.permutation(r.size)
    entries = [(int(r[i]), int(c[i]), float(rng.standard_normal())) for i in p]
    path = str(tmp_path / "m.mtx")
    _write(path, field, sym, h, w, entries)
    a, b = capi.coo_matrix(), capi.coo_matrix()
    assert L.csp_read_mmf_ex(path.encode(), C.byref(a), capi.CSP_MMF_SORT_ON_DEVICE) == 0, L.csp_last_error()
    ref.ref_read_mmf(path.encode(), C.byref(b))
    assert_same(extract("coo", a), extract("coo", b), f"{field}/{sym}")
