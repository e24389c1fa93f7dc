"""bench.py's output contract, checked on the host: the reference arm (the reference's
serial csr_spmv, compiled from its own sources into oracle/_ref) prints one JSON line
with the same metric, unit and keys as this library's arm; this library's arm has no CPU path and fails without a
GPU; the per-partition DRAM traffic files that feed `roofline.traffic` are well formed."""
import glob
import json
import os
import re
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(args, timeout=600):
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], cwd=ROOT,
                          capture_output=True, text=True, timeout=timeout)


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libclspmv_ref.so")),
                    reason="oracle/_ref not built")
def test_reference_arm_line():
    p = _run(["--impl", "reference", "--workload", "laplacian", "--steps", "3", "--warmup", "3"])
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    sys.path.insert(0, ROOT)
    import bench
    assert d["impl"] == "reference"
    assert d["metric"] == bench.METRIC   # the same metric as this library's arm
    assert d["unit"] == "GB/s" and d["higher_is_better"] is True
    assert d["n_gpus"] == 1 and d["steps"] == 3 and d["warmup"] == 3
    assert d["value"] > 0 and d["ms_per_step"] > 0
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    assert d["config"]["workload"].startswith("laplacian")


def test_own_arm_has_no_cpu_path():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    p = _run(["--workload", "laplacian", "--steps", "3", "--warmup", "3"])
    assert p.returncode != 0
    assert not [ln for ln in p.stdout.splitlines() if ln.startswith("{")]


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(ROOT, "profiles", "traffic_*.json"))),
                         ids=os.path.basename)
def test_traffic_files(path):
    d = json.load(open(path))
    src = d.pop("source")
    assert d, "no partition entries"
    for part, nbytes in d.items():
        assert isinstance(part, str) and part
        assert isinstance(nbytes, int) and nbytes > 0
    # the summary the figure comes from is committed beside it
    m = re.search(r"profiles/[\w.]+\.md", src)
    assert m and os.path.exists(os.path.join(ROOT, m.group(0)))
