"""csp_coo_spmv_noalloc: the SpMV entry point for callers that cannot allocate device
memory (a framework allocator owns the device, or cudaMalloc is forbidden in their
loop).  The caller passes device arrays it already owns; the library uses only its
fixed scratch array.  Its result must agree with the FP64 oracle within the per-row
bound the parity tests use (1e-5 * sum_j |a_ij x_j| + 2^-23 * |y0_i| per call) and
with the regular engine (csp_init_mat_kernels + csp_do_spmv) on two calls in a row
(the scratch array keeps the previous call's contents), and the calls must leave the
device's free memory unchanged.

This file is collected last so a failure here does not stop the rest of the suite."""
import numpy as np
import pytest

from clspmv_b200 import Cocktail, Handle, capi, matrices as M
from tests import _oracle
from tests.gpu_util import TOL, coo_of, oracle

pytestmark = pytest.mark.gpu

MAX_NNZ = capi.CSP_NOALLOC_MAX_NNZ


def _rows_of_lengths(lengths, width, seed):
    """Row-sorted COO whose row i holds lengths[i] entries with distinct random columns."""
    rng = np.random.default_rng(seed)
    lengths = np.asarray(lengths, np.int64)
    h = lengths.size
    r = np.repeat(np.arange(h, dtype=np.int64), lengths)
    c = np.empty(r.size, np.int64)
    o = 0
    for ln in lengths:
        c[o:o + ln] = np.sort(rng.choice(width, size=int(ln), replace=False))
        o += ln
    v = rng.standard_normal(r.size).astype(np.float32)
    return h, width, r.astype(np.int32), c.astype(np.int32), v


def _cases():
    # nnz deliberately not a multiple of the 128-entry tile; long rows span many warps
    h, w, r, c, v = M.zipf_rows(30_011, seed=41, max_len=5000)
    assert r.size % 128 != 0
    yield "zipf", (h, w, r, c, v)
    yield "laplacian", M.laplacian_2d(37)
    yield "nnz1", (3, 4, np.array([1], np.int32), np.array([2], np.int32), np.array([1.5], np.float32))
    yield "nnz5", _rows_of_lengths([2, 0, 3], 7, seed=1)
    # 1024 entries: a row ends exactly at entry 512, where the second warp's chunk starts
    yield "chunk_edge", _rows_of_lengths([300, 212, 100, 412], 2000, seed=2)
    # one row of 1,500 entries covers three warp chunks and part of a fourth
    yield "row_spans_chunks", _rows_of_lengths([7, 1500, 3, 600], 4000, seed=3)


def _device(*arrays):
    import torch
    dev = torch.device("cuda", 0)
    return [torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in arrays]


def _call(L, h, w, nnz, d_row, d_col, d_val, d_x, d_y, stream):
    rc = L.csp_coo_spmv_noalloc(h, w, nnz, d_row.data_ptr(), d_col.data_ptr(), d_val.data_ptr(),
                                d_x.data_ptr(), d_y.data_ptr(), stream)
    assert rc == capi.CSP_OK, L.csp_last_error()


def _check_oracle(case, y, x, y0, ntimes):
    yhat, bound = oracle(case, x, y0, ntimes)
    err, row = _oracle.max_rel_err(y, yhat, bound)
    assert err <= TOL, f"call {ntimes}: per-row error {err:.3e} at row {row} against the FP64 oracle"


@pytest.mark.parametrize("name,case", list(_cases()), ids=lambda v: v if isinstance(v, str) else "")
def test_noalloc_matches_oracle_and_engine_twice(name, case):
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
    d_row, d_col, d_val, d_x, d_y = _device(r.astype(np.int32), c.astype(np.int32), v.astype(np.float32), x, y0.copy())
    stream = torch.cuda.current_stream().cuda_stream
    got = []
    for _ in range(2):
        _call(L, h, w, r.size, d_row, d_col, d_val, d_x, d_y, stream)
        torch.cuda.synchronize()
        got.append(d_y.cpu().numpy().copy())

    for k, (g, want) in enumerate(zip(got, (want1, want2)), start=1):
        _check_oracle(case, g, x, y0, k)
        _, bound = oracle(case, x, y0, ntimes=k)
        diff = np.abs(g.astype(np.float64) - want.astype(np.float64))
        worst = float(np.max(diff / np.maximum(bound, 1e-30)))
        assert worst <= 2 * TOL, f"call {k}: no-alloc result differs from the engine by {worst:.3e} of the row bound"


def test_noalloc_at_the_entry_limit():
    """nnz = 2^25 exactly: 65,536 warp chunks, the last of them full, every scratch pair used."""
    import torch
    L = capi.lib()
    h, per_row = 1 << 20, 32
    assert h * per_row == MAX_NNZ
    rng = np.random.default_rng(11)
    w = 1 << 20
    r = np.repeat(np.arange(h, dtype=np.int32), per_row)
    c = rng.integers(0, w, r.size, dtype=np.int32)
    v = rng.standard_normal(r.size, dtype=np.float32)
    x = rng.uniform(-1, 1, w).astype(np.float32)
    y0 = rng.uniform(-1, 1, h).astype(np.float32)
    d_row, d_col, d_val, d_x, d_y = _device(r, c, v, x, y0.copy())
    stream = torch.cuda.current_stream().cuda_stream
    for k in (1, 2):
        _call(L, h, w, r.size, d_row, d_col, d_val, d_x, d_y, stream)
        torch.cuda.synchronize()
        _check_oracle((h, w, r, c, v), d_y.cpu().numpy(), x, y0, k)


def test_noalloc_skips_out_of_range_ids():
    """Row ids -1 (first) and >= height (last) and column ids -1 and >= width are skipped."""
    import torch
    L = capi.lib()
    h, w = 6, 9
    r = np.array([-1, -1, 0, 0, 2, 2, 2, 5, 6, 6, 7], np.int32)
    c = np.array([0, 3, 1, -1, 0, 9, 8, 4, 0, 2, 1], np.int32)
    v = np.arange(1, r.size + 1, dtype=np.float32)
    x = np.linspace(-1, 1, w).astype(np.float32)
    y0 = np.linspace(0.5, 2.0, h).astype(np.float32)
    ok = (r >= 0) & (r < h) & (c >= 0) & (c < w)
    case = (h, w, r[ok], c[ok], v[ok])
    d_row, d_col, d_val, d_x, d_y = _device(r, c, v, x, y0.copy())
    _call(L, h, w, r.size, d_row, d_col, d_val, d_x, d_y, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    _check_oracle(case, d_y.cpu().numpy(), x, y0, 1)


def test_noalloc_allocates_nothing():
    """After a first call (which looks the scratch address up), further calls leave the
    device's free memory exactly as it was."""
    import torch
    L = capi.lib()
    h, w, r, c, v = M.zipf_rows(50_000, seed=13, max_len=4000)
    x = np.random.default_rng(1).uniform(-1, 1, w).astype(np.float32)
    d_row, d_col, d_val, d_x, d_y = _device(r, c, v, x, np.zeros(h, np.float32))
    stream = torch.cuda.current_stream().cuda_stream
    _call(L, h, w, r.size, d_row, d_col, d_val, d_x, d_y, stream)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(5):
        _call(L, h, w, r.size, d_row, d_col, d_val, d_x, d_y, stream)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, f"device free memory changed by {free0 - free1} bytes across the calls"


def test_noalloc_rejects_bad_arguments():
    import torch
    L = capi.lib()
    rc = L.csp_coo_spmv_noalloc(10, 10, MAX_NNZ + 1, None, None, None, None, None, None)
    assert rc == capi.CSP_EINVAL and b"no-allocation limit" in L.csp_last_error()
    buf = torch.zeros(64, dtype=torch.int32, device="cuda")
    f = torch.zeros(64, dtype=torch.float32, device="cuda")
    g = torch.zeros(64, dtype=torch.float32, device="cuda")
    rc = L.csp_coo_spmv_noalloc(4, 4, 8, buf.data_ptr() + 4, buf.data_ptr(), f.data_ptr(), f.data_ptr(), g.data_ptr(), None)
    assert rc == capi.CSP_EINVAL and b"aligned" in L.csp_last_error()
    # x and y the same array, and overlapping ranges of one buffer
    rc = L.csp_coo_spmv_noalloc(4, 4, 8, buf.data_ptr(), buf.data_ptr(), f.data_ptr(), g.data_ptr(), g.data_ptr(), None)
    assert rc == capi.CSP_EINVAL and b"overlap" in L.csp_last_error()
    rc = L.csp_coo_spmv_noalloc(8, 8, 8, buf.data_ptr(), buf.data_ptr(), f.data_ptr(), g.data_ptr(),
                                g.data_ptr() + 16, None)
    assert rc == capi.CSP_EINVAL and b"overlap" in L.csp_last_error()
