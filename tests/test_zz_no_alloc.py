"""csp_coo_spmv_noalloc: the SpMV entry point for callers that cannot allocate device
memory (a framework allocator owns the device, or cudaMalloc is forbidden in their
loop).  The caller passes device arrays it already owns; the library uses only its
fixed scratch array.  Its result must match the regular engine (csp_init_mat_kernels +
csp_do_spmv) within the per-row tolerance the parity tests use, on two calls in a row
(the scratch array keeps the previous call's contents).

This file is collected last so a failure here does not stop the rest of the suite."""
import ctypes as C

import numpy as np
import pytest

from clspmv_b200 import Cocktail, Handle, capi, matrices as M
from tests.gpu_util import TOL, coo_of, oracle

pytestmark = pytest.mark.gpu


def _cases():
    # nnz deliberately not a multiple of the 128-entry tile; long rows span many warps
    h, w, r, c, v = M.zipf_rows(30_011, seed=41, max_len=5000)
    assert r.size % 128 != 0
    yield "zipf", (h, w, r, c, v)
    h, w, r, c, v = M.laplacian_2d(37)
    yield "laplacian", (h, w, r, c, v)


@pytest.mark.parametrize("name,case", list(_cases()), ids=lambda v: v if isinstance(v, str) else "")
def test_noalloc_matches_engine_twice(name, case):
    import torch
    L = capi.lib()
    h, w, r, c, v = case
    rng = np.random.default_rng(5)
    x = rng.uniform(-1, 1, w).astype(np.float32)
    y0 = rng.uniform(-1, 1, h).astype(np.float32)

    # regular engine, one and two SpMVs
    mat = Cocktail.single("coo", coo_of(case), 0)
    eng = Handle(mat, x, y0)
    eng.do_spmv(1)
    want1 = eng.cpy_result_to_cpu()
    eng.do_spmv(1)
    want2 = eng.cpy_result_to_cpu()
    eng.free()

    # caller-owned device buffers (the caller allocates; the entry point does not)
    dev = torch.device("cuda", 0)
    d_row = torch.from_numpy(r.astype(np.int32)).to(dev)
    d_col = torch.from_numpy(c.astype(np.int32)).to(dev)
    d_val = torch.from_numpy(v.astype(np.float32)).to(dev)
    d_x = torch.from_numpy(x).to(dev)
    d_y = torch.from_numpy(y0.copy()).to(dev)
    stream = torch.cuda.current_stream(dev)
    got = []
    for _ in range(2):
        rc = L.csp_coo_spmv_noalloc(h, w, r.size, d_row.data_ptr(), d_col.data_ptr(), d_val.data_ptr(),
                                    d_x.data_ptr(), d_y.data_ptr(), stream.cuda_stream)
        assert rc == capi.CSP_OK, L.csp_last_error()
        torch.cuda.synchronize()
        got.append(d_y.cpu().numpy().copy())

    for k, (g, want) in enumerate(zip(got, (want1, want2)), start=1):
        _, bound = oracle(case, x, y0, ntimes=k)
        diff = np.abs(g.astype(np.float64) - want.astype(np.float64))
        worst = float(np.max(diff / np.maximum(bound, 1e-30)))
        assert worst <= TOL, f"call {k}: no-alloc result differs from the engine by {worst:.3e} of the row bound"


def test_noalloc_rejects_oversize_and_misaligned():
    import torch
    L = capi.lib()
    rc = L.csp_coo_spmv_noalloc(10, 10, capi.CSP_NOALLOC_MAX_NNZ + 1, None, None, None, None, None, None)
    assert rc == capi.CSP_EINVAL and b"no-allocation limit" in L.csp_last_error()
    buf = torch.zeros(64, dtype=torch.int32, device="cuda")
    f = torch.zeros(64, dtype=torch.float32, device="cuda")
    rc = L.csp_coo_spmv_noalloc(4, 4, 8, buf.data_ptr() + 4, buf.data_ptr(), f.data_ptr(), f.data_ptr(), f.data_ptr(), None)
    assert rc == capi.CSP_EINVAL and b"aligned" in L.csp_last_error()
