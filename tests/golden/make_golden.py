"""Generates the golden fixtures in this directory from the reference's own host code
(oracle/_ref/libclspmv_ref.so, compiled from the reference sources by oracle/Makefile).

    python tests/golden/make_golden.py

For each small seeded case it records the inputs, the reference's serial CSR and COO
products (spmv_serial.h:199 csr_spmv, :184 coo_spmv) and a SHA-256 digest of every
array the reference conversions produce.  The fixtures let the oracle and the product
conversions be checked where the reference tree is absent.
"""
import ctypes as C
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from clspmv_b200 import COO, capi  # noqa: E402
from tests import _oracle  # noqa: E402
from tests.cases import small_cases  # noqa: E402
from tests.fmt_extract import STRUCT, extract  # noqa: E402

CASES = ["laplacian8", "random_irregular", "banded", "block3_small", "stencil6", "zipf_small", "rect_wide"]
CONVS = [("csr", "ref_coo2csr", ()), ("ell", "ref_coo2ell", (32, 0)), ("sell", "ref_coo2sell", (32,)),
         ("sell", "ref_coo2sell", (128,)), ("bcsr", "ref_coo2bcsr", (3, 3, 32)), ("bell", "ref_coo2bell", (4, 2, 32, 0)),
         ("b4csr", "ref_coo2b4csr", (8, 2, 32)), ("b4ell", "ref_coo2b4ell", (4, 4, 32, 0)),
         ("sbell", "ref_coo2sbell", (4, 2, 32)), ("dia", "ref_coo2dia", (32,)), ("bdia", "ref_coo2bdia", (32,))]


def digest(d: dict) -> str:
    h = hashlib.sha256()
    for k in sorted(d):
        v = d[k]
        h.update(k.encode())
        h.update(v.tobytes() if isinstance(v, np.ndarray) else repr(v).encode())
    return h.hexdigest()


def conv_key(fmt, args):
    return f"{fmt}{list(args)}"


def main():
    ref = _oracle.ref_lib()
    assert ref is not None, "build oracle/_ref first (make -C oracle)"
    cases = small_cases()
    meta = {}
    for name in CASES:
        h, w, r, c, v = cases[name]
        rng = np.random.default_rng(100)
        x = rng.uniform(-1, 1, w).astype(np.float32)
        y0 = rng.uniform(-1, 1, h).astype(np.float32)
        coo = COO(h, w, r, c, v)
        csr = capi.csr_matrix()
        ref.ref_coo2csr(coo.ref(), C.byref(csr))
        y_csr = y0.copy()
        ref.ref_csr_spmv(C.byref(csr), capi.as_ptr(x, C.c_float), capi.as_ptr(y_csr, C.c_float), w)
        y_coo = y0.copy()
        ref.ref_coo_spmv(coo.ref(), capi.as_ptr(x, C.c_float), capi.as_ptr(y_coo, C.c_float), w)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), height=h, width=w, row=r, col=c, val=v, x=x, y0=y0,
                            y_csr=y_csr, y_coo=y_coo)
        digests = {}
        for fmt, fn, args in CONVS:
            if fmt in ("dia", "bdia") and h > w:
                continue
            src = COO(h, w, r, c, v)
            s = STRUCT[fmt]()
            ok = getattr(ref, fn)(src.ref(), C.byref(s), *args)
            if fmt in ("dia", "bdia", "b4csr", "b4ell", "sbell") and ok == 0:
                digests[conv_key(fmt, args)] = "refused"
                continue
            digests[conv_key(fmt, args)] = digest(extract(fmt, s))
        meta[name] = digests
    with open(os.path.join(HERE, "conversions.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "conversions": [[f, list(a)] for f, _, a in CONVS],
                   "digests": meta}, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
