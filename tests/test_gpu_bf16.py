"""BF16 value storage (CSP_FLAG_BF16): values rounded to BF16 on upload, FP32
accumulation.  Against the FP64 oracle evaluated on the same BF16-rounded values the
per-row bound is the FP32 one; against the original FP32 values the error is the
BF16 quantization (~2^-9 relative), reported and bounded."""
import numpy as np
import pytest

from clspmv_b200 import CSP_FLAG_BF16, Cocktail, matrices as M
from tests.gpu_util import check, coo_of, oracle, run, vecs
from tests import _oracle

pytestmark = pytest.mark.gpu


def bf16_round(v):
    """Round-to-nearest-even FP32 -> BF16 -> FP32."""
    u = np.ascontiguousarray(v, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


CASES = {
    "zipf": M.zipf_rows(50_000, seed=61, max_len=4000),
    "stencil": M.stencil_27(20, seed=62),
    "block4": M.block_3x3(3000, deg=(4, 10), band=50, seed=63, bs=4),
}
VARIANTS = [("csr", 2, {}), ("csr", 0, {}), ("coo", 0, {}), ("csr", 16, {}), ("coo", 16, {}), ("ell", 1, {}), ("sell", 0, {}), ("dia", 1, {}),
            ("bdia", 1, {}), ("bdia", 0, {}), ("bcsr", 0, {"bwidth": 4, "bheight": 4}),
            ("bell", 0, {"bwidth": 4, "bheight": 4}), ("sbell", 0, {"bwidth": 4, "bheight": 4})]


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("variant", VARIANTS, ids=lambda v: f"{v[0]}{v[1]}")
def test_bf16_storage(name, variant):
    fmt, m, kw = variant
    case = CASES[name]
    h, w, r, c, v = case
    if fmt in ("dia", "bdia") and name != "stencil":
        pytest.skip("DIA only for the banded case")
    if fmt == "ell" and name == "zipf":
        pytest.skip("ELL padding of Zipf rows")
    if fmt in ("bcsr", "bell", "sbell") and name != "block4":
        pytest.skip("block formats only for the blocked case")
    mat = Cocktail.single(fmt, coo_of(case), m, **kw)
    x, y0 = vecs(h, w)
    y = run(mat, x, y0, flags=CSP_FLAG_BF16)
    rounded = (h, w, r, c, bf16_round(v))
    check(rounded, y, x, y0)                       # kernel error: FP32 accumulation
    yhat, bound = oracle(case, x, y0)              # storage error vs the FP32 matrix
    err, _ = _oracle.max_rel_err(y, yhat, bound)
    assert err <= 2.0 ** -8, err
