"""CSP_ANALYZE_ON_DEVICE: the reference-table partitioner with its counting passes
(nonzeros per diagonal, blocks per block row for the eight b4 shapes) on the device
gives the partition the host passes give, byte for byte, on the analyzer parity inputs
and on the full-size 10^6 Zipf, 160^3 stencil and 3x3-block matrices."""
import ctypes as C
import os
import time

import pytest

from clspmv_b200 import COO, capi, matrices as M
from tests import _oracle
from tests.fmt_extract import assert_same, extract
from tests.test_analyzer_parity import CASES, FORMATS

pytestmark = pytest.mark.gpu


def _partition(L, case, flags):
    h, w, r, c, v = case
    a = COO(h, w, r, c, v)
    mat = capi.cocktail()
    opts = capi.csp_analyze_opts(capi.CSP_ANALYZE_REFERENCE, _oracle.REF_BENCH.encode(), 0, None, flags)
    t0 = time.perf_counter()
    assert L.csp_analyze_matrix(a.ref(), C.byref(mat), C.byref(opts)) == 0, L.csp_last_error()
    return mat, time.perf_counter() - t0


def _same(L, case, name):
    host, th = _partition(L, case, 0)
    dev, td = _partition(L, case, capi.CSP_ANALYZE_ON_DEVICE)
    for f, ext in FORMATS:
        assert getattr(dev, f"ifuse{f}") == getattr(host, f"ifuse{f}"), f"{name}: ifuse{f}"
        if getattr(host, f"ifuse{f}"):
            assert getattr(dev, f"{f}_meth_num") == getattr(host, f"{f}_meth_num"), f"{name}: {f}_meth_num"
            assert_same(extract(ext, getattr(dev, f)), extract(ext, getattr(host, f)), f"{name}.{f}")
    assert (dev.csr_group_num, dev.coo_group_num) == (host.csr_group_num, host.coo_group_num)
    L.csp_free_cocktail(C.byref(host))
    L.csp_free_cocktail(C.byref(dev))
    return th, td


@pytest.fixture(scope="module", autouse=True)
def _tables():
    if not os.path.isdir(os.path.join(_oracle.REF_BENCH, "benchmark")):
        pytest.skip("reference calibration tables not built (make -C oracle)")


@pytest.mark.parametrize("name", sorted(CASES))
def test_device_counts_give_the_host_partition(L, name):
    _same(L, CASES[name], name)


@pytest.mark.parametrize("name", ["zipf_1m", "stencil_160", "block3_500k"])
def test_device_counts_full_size(L, name):
    case = {"zipf_1m": lambda: M.zipf_rows(1_000_000, 2.0, 10_000, seed=0),
            "stencil_160": lambda: M.stencil_27(160),
            "block3_500k": lambda: M.block_3x3(500_000)}[name]()
    th, td = _same(L, case, name)
    print(f"{name}: reference-table analysis {th:.2f} s with host counts, {td:.2f} s with device counts")
