"""The C ABI library loads without a GPU and exports every function the public
headers declare; calls that need a device fail with CSP_ENODEV, not a crash."""
import ctypes as C
import glob
import os
import re

import numpy as np

from clspmv_b200 import COO, Cocktail, capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "csp", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(csp_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_every_declared_symbol_is_exported(L):
    names = declared_functions()
    assert len(names) > 60
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_struct_sizes_match_reference_layout():
    # cocktail<int,int,float>: 9 bools, 11+3 ints, then 9 sub-structs (LP64)
    assert C.sizeof(capi.coo_matrix) == 40
    assert C.sizeof(capi.csr_matrix) == 40
    assert C.sizeof(capi.dia_matrix) == 40
    assert C.sizeof(capi.bdia_matrix) == 48
    assert C.sizeof(capi.b4ell_matrix) == 56
    assert C.sizeof(capi.sbell_matrix) == 56


def test_version_and_errors(L):
    assert b"sm_100a" in L.csp_version()
    assert L.csp_error_string(capi.CSP_EFORMAT) == b"CSP_EFORMAT"
    assert L.csp_aligned_length(33, 32) == 64


def test_device_calls_fail_cleanly_without_gpu(L):
    import torch
    if torch.cuda.is_available():
        return
    coo = COO(3, 3, [0, 1, 2], [0, 1, 2], [1, 2, 3])
    mat = Cocktail.single("csr", coo)
    h = C.c_void_p()
    x = np.ones(3, np.float32)
    rc = L.csp_init_mat_kernels(mat.ref(), capi.as_ptr(x, C.c_float), None, 0, C.byref(h))
    assert rc in (capi.CSP_ENODEV, capi.CSP_ECUDA)
    assert not h.value


def test_device_setup_calls_refuse_without_gpu(L):
    """The device sort and the device layout builds check for a device before any work:
    CSP_ENODEV, and the input COO (which the builds may sort in place) unchanged."""
    import torch
    if torch.cuda.is_available():
        return
    from tests.fmt_extract import extract
    r = np.array([2, 0, 1], np.int32)
    c = np.array([1, 0, 2], np.int32)
    v = np.array([3.0, 1.0, 2.0], np.float32)
    for fn, st, args in (("csp_sort_coo_device", None, ()), ("csp_coo2dia_device", capi.dia_matrix, (32,)),
                         ("csp_coo2bdia_device", capi.bdia_matrix, (32,)),
                         ("csp_coo2bcsr_device", capi.bcsr_matrix, (3, 3, 32))):
        coo = COO(3, 3, r.copy(), c.copy(), v.copy())
        before = extract("coo", coo.s)
        call = getattr(L, fn)
        if st is None:
            rc = call(coo.ref())
        else:
            out = st()
            rc = call(coo.ref(), C.byref(out), *args)
        assert rc == capi.CSP_ENODEV, (fn, rc)
        after = extract("coo", coo.s)
        assert all(np.array_equal(np.asarray(before[k]), np.asarray(after[k])) for k in ("row", "col", "val")), fn


def test_temporary_coo_outlives_the_call(L):
    """`COO(...).ref()` passed straight to a conversion: the struct keeps the arrays its
    pointers reference alive through the call (large arrays, whose memory would
    otherwise go back to the system at once)."""
    rng = np.random.default_rng(5)
    h, w, nnz = 200_000, 150_000, 1_000_000
    r = np.sort(rng.integers(0, h, nnz)).astype(np.int32)
    c = rng.integers(0, w, nnz).astype(np.int32)
    v = rng.standard_normal(nnz).astype(np.float32)
    ref = COO(h, w, r, c, v).ref()   # the COO itself is gone after this line
    # freed arrays of these sizes would be handed out again here, and overwritten
    junk = [np.full(nnz, 0x7fffffff, np.int32) for _ in range(2)] + [np.full(nnz, np.nan, np.float32)]
    csr = capi.csr_matrix()
    assert L.csp_coo2csr(ref, C.byref(csr)) == 0
    del junk
    rp = np.ctypeslib.as_array(csr.csr_row_ptr, (h + 1,)).copy()
    assert rp[-1] == nnz
    assert np.array_equal(np.diff(rp), np.bincount(r, minlength=h))
    L.csp_free_csr_matrix(C.byref(csr))
