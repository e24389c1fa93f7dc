"""Batched persistent execution on the device (csp_batch_*): forward y += A x,
adjoint xbar += A^T ybar and value gradients abar = ybar (x) x on every stored slot,
for every batch format, the byte-model and device-tuned format choices, CUDA-graph
replay, BF16 values and the per-matrix plain CSR path, each matrix checked against
the FP64 oracle with the per-row bound |y_i - yhat_i| <= 1e-5 * sum_j |a_ij x_j| + 2^-23 * |y0_i|."""
import numpy as np
import pytest

from clspmv_b200 import COO, CSP_FLAG_ADJOINT, CSP_FLAG_BF16, CSP_FLAG_GRAPH, CspError, matrices as M
from clspmv_b200.batch import (BFMT_NAMES, CSP_BATCH_ADJ, CSP_BATCH_FWD, CSP_BATCH_TUNE_DEVICE, CSP_BFMT_AUTO,
                               CSP_BV_ABAR, CSP_BV_X, CSP_BV_XBAR, CSP_BV_Y, CSP_BV_YBAR, Batch, features)
from clspmv_b200.capi import CSP_BFMT_CSR, CSP_BFMT_DIA, CSP_BFMT_SELL32, CSP_BFMT_SELL128, CSP_EFORMAT, CSP_EUNSUP
from clspmv_b200.matrices import csr_from_coo
from tests import _oracle
from tests.cases import duplicate_cases, small_cases
from tests.gpu_util import TOL

pytestmark = pytest.mark.gpu

BOTH = CSP_BATCH_FWD | CSP_BATCH_ADJ


def _cases():
    c = dict(small_cases())
    c.update(duplicate_cases())
    for i, (kind, *case) in enumerate(M.batch_mixed(12, lo=300, hi=20_000, seed=5)):
        c[f"mixed{i}_{kind}"] = tuple(case)
    c["long_rows"] = M.zipf_rows(20_000, s=1.3, max_len=6000, seed=31)
    c["lap_sq"] = M.laplacian_sq(37, 29)
    c["empty"] = (50, 60, np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros(0, np.float32))
    return c


CASES = _cases()


def _bf16(v):
    u = np.asarray(v, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def _merged(case):
    """Duplicates summed in FP32 (DIA and BCSR store one slot per position)."""
    h, w, r, c, v = case
    key = r.astype(np.int64) * max(w, 1) + c
    order = np.argsort(key, kind="stable")
    uk, first = np.unique(key[order], return_index=True)
    acc = np.zeros(uk.size, np.float32)
    for k in range(order.size):   # sequential FP32 sums, in input order per position
        acc[np.searchsorted(uk, key[order[k]])] += v[order[k]]
    return h, w, (uk // max(w, 1)).astype(np.int32), (uk % max(w, 1)).astype(np.int32), acc


def _oracle_all(case, x, y0, ybar, xbar0, vals=None, case_t=None, vals_t=None):
    """FP64 references of y0 + A x and xbar0 + A^T ybar; the transposed product uses
    case_t / vals_t (the matrix as the A^T part stores it) where given."""
    def prod(cs, vv, vec, transpose):
        h, w, r, c, v = cs
        if vv is not None:
            v = vv
        order = np.lexsort((c, r))
        r, c, v = r[order], c[order], v[order]
        return _oracle.fp64_spmv(h, w, csr_from_coo(h, r), c, v, vec, None, transpose=transpose)
    fy, by = prod(case, vals, x, False)
    fx, bx = prod(case_t if case_t is not None else case, vals_t if case_t is not None else vals, ybar, True)
    return (y0 + fy, _oracle.y0_term(y0) + by), (xbar0 + fx, _oracle.y0_term(xbar0) + bx)


def _err(y, ref):
    yhat, bound = ref
    if y.size == 0:
        return 0.0
    e, _ = _oracle.max_rel_err(y, yhat, bound)
    return e


class Run:
    """A batch with random vectors loaded, and the oracle per matrix."""

    def __init__(self, names, flags=CSP_FLAG_ADJOINT, fmt=CSP_BFMT_AUTO, tune=0, cache_path=None, seed=3):
        self.names = names
        self.cases = [CASES[n] for n in names]
        self.coos = [COO(*cs) for cs in self.cases]
        self.b = Batch(self.coos, flags=flags, fmt=fmt, tune=tune, cache_path=cache_path)
        self.adjoint = bool(flags & CSP_FLAG_ADJOINT)
        rng = np.random.default_rng(seed)
        nx, ny = int(self.b.x_off[-1]), int(self.b.y_off[-1])
        self.x = rng.uniform(-1, 1, nx).astype(np.float32)
        self.y0 = rng.uniform(-1, 1, ny).astype(np.float32)
        self.ybar = rng.uniform(-1, 1, ny).astype(np.float32)
        self.xbar0 = rng.uniform(-1, 1, nx).astype(np.float32)
        self.load()

    def load(self):
        self.b.copy_in(CSP_BV_X, self.x)
        self.b.copy_in(CSP_BV_Y, self.y0)
        if self.adjoint:
            self.b.copy_in(CSP_BV_YBAR, self.ybar)
            self.b.copy_in(CSP_BV_XBAR, self.xbar0)

    def sl(self, off, i):
        return slice(int(off[i]), int(off[i + 1]))

    def check(self, what=BOTH, bf16=False, tol=TOL):
        y = self.b.copy_out(CSP_BV_Y)
        xbar = self.b.copy_out(CSP_BV_XBAR) if what & CSP_BATCH_ADJ else None
        abar = self.b.copy_out(CSP_BV_ABAR) if what & CSP_BATCH_ADJ else None
        worst = 0.0
        for i, (name, case) in enumerate(zip(self.names, self.cases)):
            xs, ys = self.sl(self.b.x_off, i), self.sl(self.b.y_off, i)
            vals = vals_t = case_t = None
            if bf16:
                # DIA and BCSR parts store duplicates summed, then rounded to BF16
                flat = (CSP_BFMT_CSR, CSP_BFMT_SELL32, CSP_BFMT_SELL128)
                fa = self.b.formats[i]
                ft = self.b.formats_adjoint[i] if self.b.formats_adjoint else fa
                case_t = _merged(case) if ft not in flat else case
                if fa not in flat:
                    case = _merged(case)
                vals, vals_t = _bf16(case[4]), _bf16(case_t[4])
            ry, rx = _oracle_all(case, self.x[xs], self.y0[ys], self.ybar[ys], self.xbar0[xs], vals, case_t, vals_t)
            if what & CSP_BATCH_FWD:
                e = _err(y[ys], ry)
                assert e <= tol, f"{name} ({BFMT_NAMES[self.b.formats[i]]}): forward error {e:.3e}"
                worst = max(worst, e)
            else:
                assert np.array_equal(y[ys], self.y0[ys]), f"{name}: y changed by an adjoint-only run"
            if what & CSP_BATCH_ADJ:
                e = _err(xbar[xs], rx)
                assert e <= tol, f"{name} ({BFMT_NAMES[self.b.formats[i]]}): adjoint error {e:.3e}"
                worst = max(worst, e)
                self.check_grad(i, abar[self.sl(self.b.abar_off, i)])
        return worst

    def check_grad(self, i, g):
        name, case = self.names[i], self.cases[i]
        h, w, r, c, v = case
        rows, cols = self.b.pattern(i)
        assert rows.size == g.size
        pad = rows < 0
        assert np.all(g[pad] == 0.0), f"{name}: gradient written into padding slots"
        rr, cc = rows[~pad], cols[~pad]
        xs, ys = self.sl(self.b.x_off, i), self.sl(self.b.y_off, i)
        want = self.ybar[ys][rr].astype(np.float64) * self.x[xs][cc].astype(np.float64)
        err = np.abs(g[~pad].astype(np.float64) - want)
        assert np.all(err <= 1e-6 * np.abs(want) + 1e-38), f"{name}: value gradient off by {err.max():.3e}"
        # CSR and SELL store exactly the matrix's entries; DIA and BCSR also store the
        # zeros inside their diagonals and blocks, so their slots cover the entries
        have = np.unique(rr.astype(np.int64) * max(w, 1) + cc)
        exp = np.unique(r.astype(np.int64) * max(w, 1) + c)
        if self.b.formats[i] in (CSP_BFMT_CSR, CSP_BFMT_SELL32, CSP_BFMT_SELL128):
            assert np.array_equal(have, exp), f"{name}: stored pattern differs from the matrix"
            assert rr.size == r.size
        else:
            assert np.isin(exp, have).all(), f"{name}: an entry has no stored slot"
            assert np.unique(rr.astype(np.int64) * max(w, 1) + cc).size == rr.size, f"{name}: a slot repeats"


def _feasible(fmt):
    return [n for n, cs in CASES.items() if features(COO(*cs))["feasible"] & (1 << fmt)]


@pytest.mark.parametrize("fmt", range(7), ids=list(BFMT_NAMES))
def test_forced_format(fmt):
    names = _feasible(fmt)
    assert names, f"no case is feasible for {BFMT_NAMES[fmt]}"
    run = Run(names, fmt=fmt)
    assert all(f == fmt for f in run.b.formats)
    assert run.b.launches(BOTH) == 1
    run.b.run(BOTH)
    run.check(BOTH)


def test_model_choice_and_directions():
    names = list(CASES)
    run = Run(names)
    model = [features(COO(*CASES[n]))["model_format"] for n in names]
    assert run.b.formats == model
    assert len(run.b.formats_adjoint) == len(names)
    run.b.run(CSP_BATCH_FWD)
    run.check(CSP_BATCH_FWD)
    xbar = run.b.copy_out(CSP_BV_XBAR)
    assert np.array_equal(xbar, run.xbar0), "a forward-only run changed xbar"
    run.load()
    run.b.run(CSP_BATCH_ADJ)
    run.check(CSP_BATCH_ADJ)


def test_repeated_runs_accumulate():
    names = ["long_rows", "lap_sq", "zipf_small", "empty", "single_row"]
    run = Run(names, fmt=CSP_BFMT_CSR)
    run.b.run(CSP_BATCH_FWD, 3)
    y = run.b.copy_out(CSP_BV_Y)
    for i, case in enumerate(run.cases):
        ys, xs = run.sl(run.b.y_off, i), run.sl(run.b.x_off, i)
        h, w, r, c, v = case
        order = np.lexsort((c, r))
        out, bound = _oracle.fp64_spmv(h, w, csr_from_coo(h, r[order]), c[order], v[order], run.x[xs], None)
        e = _err(y[ys], (run.y0[ys] + 3 * out, _oracle.y0_term(run.y0[ys], 3) + 3 * bound))
        assert e <= TOL


def test_graph_replay_is_deterministic():
    names = list(CASES)
    a = Run(names, flags=CSP_FLAG_ADJOINT)
    a.b.run(BOTH)
    ref = [a.b.copy_out(k) for k in (CSP_BV_Y, CSP_BV_XBAR, CSP_BV_ABAR)]
    g = Run(names, flags=CSP_FLAG_ADJOINT | CSP_FLAG_GRAPH)
    for _ in range(2):
        g.load()
        g.b.run(BOTH)
        out = [g.b.copy_out(k) for k in (CSP_BV_Y, CSP_BV_XBAR, CSP_BV_ABAR)]
        for p, q in zip(ref, out):
            assert np.array_equal(p, q), "graph replay differs from a direct launch"
    g.check(BOTH)


def test_device_tuning_and_cache(tmp_path):
    names = [n for n in CASES if n.startswith("mixed")] + ["lap_sq", "long_rows", "block3_small"]
    cache = str(tmp_path / "batch.cache")
    run = Run(names, tune=CSP_BATCH_TUNE_DEVICE, cache_path=cache)
    feas = [features(COO(*CASES[n]))["feasible"] for n in names]
    assert all(f & (1 << fmt) for f, fmt in zip(feas, run.b.formats))
    lines = open(cache).read().split("\n")
    assert any(" batch " in ln for ln in lines)
    run.b.run(BOTH)
    run.check(BOTH)
    again = Batch(run.coos, flags=CSP_FLAG_ADJOINT, tune=CSP_BATCH_TUNE_DEVICE, cache_path=cache)
    assert again.formats == run.b.formats
    again.free()


def test_bf16_values():
    names = list(CASES)
    run = Run(names, flags=CSP_FLAG_ADJOINT | CSP_FLAG_BF16)
    run.b.run(BOTH)
    run.check(BOTH, bf16=True)


def test_plain_csr_launches():
    names = list(CASES)
    run = Run(names, fmt=CSP_BFMT_CSR)
    nonempty = sum(1 for cs in run.cases if cs[0] > 0)
    assert run.b.launches(CSP_BATCH_FWD, plain=True) == nonempty
    for lanes in (0, 1, 32):
        run.load()
        run.b.run_plain(BOTH, 1, lanes)
        run.check(BOTH)


def test_errors():
    coos = [COO(*CASES["zipf_small"]), COO(*CASES["lap_sq"])]
    with pytest.raises(CspError) as e:
        Batch(coos, fmt=CSP_BFMT_DIA)
    assert e.value.code == CSP_EFORMAT
    b = Batch(coos)
    with pytest.raises(CspError) as e:
        b.run(CSP_BATCH_ADJ)
    assert e.value.code == CSP_EUNSUP
    b.free()
    b = Batch([COO(*CASES["lap_sq"])], fmt=CSP_BFMT_DIA)
    with pytest.raises(CspError) as e:
        b.run_plain(CSP_BATCH_FWD)
    assert e.value.code == CSP_EUNSUP
    b.free()
