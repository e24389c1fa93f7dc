"""The spmv_all / spmv_cocktail commands (clSpMV_NV/src/spmv_all.cpp:158, eval.cpp:93)
built on the library, and spmv_all method 0 (bandwidth / launch overhead)."""
import ctypes as C
import os
import subprocess

import pytest

from clspmv_b200 import capi, matrices as M
from tests import _oracle

pytestmark = pytest.mark.gpu
BIN = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "clspmv_b200", "bin")


def _mtx(path, case):
    h, w, r, c, v = case
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n")
        f.write(f"{h} {w} {r.size}\n")
        for a, b, x in zip(r, c, v):
            f.write(f"{a + 1} {b + 1} {x:.9g}\n")


def test_bandwidth_probe():
    rep = capi.csp_bandwidth_report()
    assert capi.lib().csp_bandwidth_test(256 << 20, 1 << 20, C.byref(rep)) == 0
    assert rep.copy_gbs > 1000 and rep.gather_per_s > 1e9 and 0 < rep.launch_us < 100


@pytest.mark.parametrize("method", [0, 1, 2, 4, 5, 6, 9])
def test_spmv_all_cli(tmp_path, method):
    path = str(tmp_path / "lap.mtx")
    _mtx(path, M.laplacian_2d(64))
    out = subprocess.run([os.path.join(BIN, "spmv_all"), path, str(method), "5"], capture_output=True, text=True,
                         timeout=120)
    assert out.returncode == 0, out.stderr
    assert ("GB/s" in out.stdout)


@pytest.mark.parametrize("tables", [True, False])
def test_spmv_cocktail_cli(tmp_path, tables):
    path = str(tmp_path / "z.mtx")
    _mtx(path, M.zipf_rows(5000, seed=3, max_len=500))
    env = dict(os.environ)
    env.pop("CLSPMVPATH", None)
    if tables:
        if not os.path.isdir(os.path.join(_oracle.REF_BENCH, "benchmark")):
            pytest.skip("calibration tables not built")
        env["CLSPMVPATH"] = _oracle.REF_BENCH
    out = subprocess.run([os.path.join(BIN, "spmv_cocktail"), path], capture_output=True, text=True, timeout=300,
                         env=env)
    assert out.returncode == 0, out.stderr
    assert "Partition (" + ("reference tables" if tables else "autotuned") in out.stdout
    assert "GFLOPS" in out.stdout


def test_gather_rate_probe():
    """The standalone random-gather probe (clspmv_b200/bin/gather_rates, not part of the
    library) reports positive L2 and shared-memory rates (cluster -1 only where the
    device has no thread-block clusters)."""
    import json
    out = subprocess.run([os.path.join(BIN, "gather_rates")], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    r = json.loads(out.stdout)
    assert r["l2_per_s"] > 0 and r["shared_per_s"] > 0
    assert r["cluster_per_s"] > 0 or r["cluster_per_s"] == -1.0
