#!/usr/bin/env python
"""Cocktail SpMV throughput on B200: HBM GB/s and fraction of the HBM roofline.

Default workload (the irregular-row benchmark): a 1,000,000 x 1,000,000 matrix with
Zipf(2) row lengths clipped to [1, 10,000], uniform distinct columns per row, N(0,1)
FP32 values, x ~ U(-1, 1), y = A*x + y (accumulate, as in clSpMV).  Synthetic and
seeded (the reference's public matrix collection is not available offline).

One step = one forward SpMV of the whole matrix through the autotuned Cocktail
engine.  `value` is algorithmic GB/s (values + indices + x + y read/write, no
padding counted) over the CUDA-event time of the SpMV kernels, inputs resident in
HBM; L2 (126 MB, larger than this working set) is flushed before every timed SpMV by
a 256 MB write followed by a 256 MB read of another buffer, so neither the workload's
data nor the flush's own dirty lines (whose write-back would land inside the timed
region) are left in L2.  `e2e` is the same metric through the C ABI with host buffers:
H2D of x and y, the SpMV, D2H of y, every step.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload zipf|laplacian|stencil|block] [--tune-cache FILE]

With --impl reference the reference's own CPU SpMV (clSpMV_NV/include/spmv_serial.h
csr_spmv, compiled from the reference sources into oracle/_ref) runs on the same
workload on the host (it is single-threaded).  Under torchrun every rank runs an
independent replica (weak scaling, no collective on the data path).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "SpMV HBM GB/s & % of roofline; fwd+adjoint time, autotuned vs plain CSR"
L2_FLUSH_BYTES = 256 << 20


def _peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def make_workload(name: str):
    from clspmv_b200 import matrices as M
    if name == "zipf":
        h, w, r, c, v = M.zipf_rows(1_000_000, 2.0, 10_000, seed=0)
        desc = "zipf_rows n=1,000,000 s=2.0 len<=10,000 FP32"
    elif name == "laplacian":
        h, w, r, c, v = M.laplacian_2d(128)
        desc = "laplacian_2d 128x128 (16,384 rows) FP32"
    elif name == "stencil":
        h, w, r, c, v = M.stencil_27(160)
        desc = "stencil_27 160^3 (4,096,000 rows) FP32"
    elif name == "block":
        h, w, r, c, v = M.block_3x3(500_000)
        desc = "block_3x3 500,000 block rows FP32"
    else:
        raise ValueError(name)
    x = M.vector(w, seed=1)
    y0 = M.vector(h, seed=2)
    return desc, (h, w, r, c, v), x, y0


def algorithmic_bytes(h, w, nnz, value_bytes=4, ndiag=None):
    """Minimum bytes per SpMV, no padding counted: values + indices of the structure class
    + x once + y read and written.  CSR class: column ids and row pointers; DIA class
    (ndiag given): one offset per diagonal."""
    if ndiag is not None:
        return value_bytes * nnz + 4 * ndiag + 4 * w + 8 * h
    return value_bytes * nnz + 4 * nnz + 4 * (h + 1) + 4 * w + 8 * h


def workload_bytes(name, case):
    """Algorithmic bytes of one SpMV of a workload: banded matrices are counted in the DIA
    class (their natural storage), the others in the CSR class."""
    h, w, r, c, v = case
    if name in ("stencil", "laplacian"):
        return algorithmic_bytes(h, w, int(r.size), ndiag=int(np.unique(c.astype(np.int64) - r).size))
    return algorithmic_bytes(h, w, int(r.size))


class ClockSampler:
    """nvidia-smi SM clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [t.strip() for t in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
            except ValueError:
                continue
            for nm, val in zip(names, p[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_reference_spmv_time(case, x, y0, budget_s: float, min_reps: int = 2):
    """Times the reference's serial csr_spmv (oracle/_ref) -- or, where that was not
    built, the oracle's restatement of it -- over whole SpMVs for about budget_s."""
    from clspmv_b200 import capi
    from clspmv_b200.matrices import csr_from_coo
    from tests import _oracle
    h, w, r, c, v = case
    rp = csr_from_coo(h, r)
    ref = _oracle.ref_lib()
    y = y0.copy()
    FP = C.POINTER(C.c_float)
    if ref is not None:
        s = capi.csr_matrix()
        s.matinfo.width, s.matinfo.height, s.matinfo.nnz = w, h, r.size
        s.csr_row_ptr = rp.ctypes.data_as(C.POINTER(C.c_int))
        s.csr_col_id = c.ctypes.data_as(C.POINTER(C.c_int))
        s.csr_data = v.ctypes.data_as(FP)
        fn = lambda: ref.ref_csr_spmv(C.byref(s), x.ctypes.data_as(FP), y.ctypes.data_as(FP), w)  # noqa: E731
        kind = "reference"
    else:
        orc = _oracle.oracle_lib()
        fn = lambda: orc.orc_csr_spmv_f32(h, rp.ctypes.data_as(C.POINTER(C.c_int)),  # noqa: E731
                                          c.ctypes.data_as(C.POINTER(C.c_int)), v.ctypes.data_as(FP),
                                          x.ctypes.data_as(FP), y.ctypes.data_as(FP))
        kind = "port"
    fn()  # warm-up
    times = []
    t_end = time.perf_counter() + budget_s
    while len(times) < min_reps or time.perf_counter() < t_end:
        t0 = time.perf_counter()
        fn()
        times.append(time.perf_counter() - t0)
    return statistics.median(times), len(times), kind


def run_reference_arm(args, desc, case, x, y0):
    h, w, r, c, v = case
    ab = workload_bytes(args.workload, case)
    # one step = one whole serial SpMV on one host core; W warm-ups, K timed
    t_step, reps, kind = cpu_reference_spmv_time(case, x, y0, budget_s=0.0, min_reps=args.warmup + args.steps)
    gbs = ab / t_step / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": gbs, "unit": "GB/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_step * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": desc, "nnz": int(r.size), "path": "clSpMV serial csr_spmv (spmv_serial.h:199)"},
        "cpu_baseline": {"value": gbs, "unit": "GB/s", "cores": 1, "kind": kind,
                         "sample": f"{reps} whole SpMVs of the workload on one host core (the reference path is serial)"},
        "e2e": {"value": gbs, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="zipf", choices=["zipf", "laplacian", "stencil", "block"])
    ap.add_argument("--cpu-budget", type=float, default=10.0, help="seconds of CPU-baseline sampling")
    ap.add_argument("--tune-cache", default=None,
                    help="autotuner decision file: a pattern decided in an earlier run is rebuilt without "
                         "timing candidates (used to profile the bench's own partition)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        desc, case, x, y0 = make_workload(args.workload)
        run_reference_arm(args, desc, case, x, y0)
        return

    import torch
    import torch.distributed as dist
    from clspmv_b200 import COO, Cocktail, Handle
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))

    desc, case, x, y0 = make_workload(args.workload)
    h, w, r, c, v = case
    nnz = int(r.size)
    ab = workload_bytes(args.workload, case)
    # a dedicated stream: the library and torch (flush, events) must launch on the same one
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    flush_w = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    flush_r = torch.ones(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    flush_sink = torch.empty(1, dtype=torch.float32, device="cuda")

    def flush_l2():
        flush_w.zero_()
        torch.sum(flush_r, dim=0, out=flush_sink[0])

    def time_handle(hd: Handle, steps: int, warmup: int):
        hd.set_stream(stream.cuda_stream)
        for _ in range(warmup):
            hd.do_spmv(1)
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for e0, e1 in evs:
            flush_l2()
            e0.record(stream)
            hd.do_spmv(1)
            e1.record(stream)
        torch.cuda.synchronize()
        return [e0.elapsed_time(e1) for e0, e1 in evs]

    # --- the library's on-device autotuner picks the Cocktail partition ---
    from clspmv_b200 import CSP_ANALYZE_AUTOTUNE, analyze_matrix
    coo = COO(h, w, r, c, v)
    best_mat = analyze_matrix(coo, mode=CSP_ANALYZE_AUTOTUNE, cache_path=args.tune_cache)
    best_key = best_mat.choice
    best = Handle(best_mat, x, y0)
    # plain single-format CSR on the same GPU: one warp per row (the reference's vector
    # kernel design, spmv_all method 2) and one thread per row (method 1); the faster
    plain = {}
    for m_ in (0, 4):
        pm = Cocktail.single("csr", coo, m_)
        ph = Handle(pm, x, y0)
        plain[f"csr{m_}"] = (statistics.median(time_handle(ph, 10, 3)), pm, ph)
    plain_key = min(plain, key=lambda k: plain[k][0])
    for k_, (_, pm, ph) in plain.items():
        if k_ != plain_key:
            ph.free()
    _, _, plain_hd = plain[plain_key]

    # --- timed region: K SpMVs, L2 flushed before each, CUDA events on the launching stream ---
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    times = time_handle(best, args.steps, args.warmup)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    total_ms = float(sum(times))
    if world > 1:
        t = torch.tensor([total_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
        dist.barrier()
    ms_step = total_ms / args.steps
    plain_times = time_handle(plain_hd, max(10, args.steps // 2), 3)

    # --- e2e through the C ABI with pinned host buffers ---
    xp = torch.from_numpy(x).pin_memory()
    y0p = torch.from_numpy(y0).pin_memory()
    yout = torch.empty(h, dtype=torch.float32).pin_memory()
    from clspmv_b200 import capi
    L = capi.lib()
    FP = C.POINTER(C.c_float)
    xptr = C.cast(C.c_void_p(xp.data_ptr()), FP)
    y0ptr = C.cast(C.c_void_p(y0p.data_ptr()), FP)
    yptr = C.cast(C.c_void_p(yout.data_ptr()), FP)

    def e2e_step():
        capi.check(L.csp_cpy_vector_from_cpu(best.h, xptr, w))
        capi.check(L.csp_cpy_result_from_cpu(best.h, y0ptr, h))
        capi.check(L.csp_do_spmv(best.h, 1))
        capi.check(L.csp_cpy_result_to_cpu(best.h, yptr, h))

    for _ in range(args.warmup):
        e2e_step()
    torch.cuda.synchronize()
    e_times = []
    for _ in range(args.steps):
        flush_l2()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        e2e_step()
        e1.record(stream)
        torch.cuda.synchronize()
        e_times.append(e0.elapsed_time(e1))
    e2e_ms = sum(e_times) / len(e_times)
    if world > 1:
        t = torch.tensor([e2e_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())

    peak, peak_kind = _peak()
    kernel_gbs = ab / (statistics.mean(times) * 1e-3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", f"traffic_{args.workload}.json")
    if os.path.exists(tpath):
        try:
            traffic = json.load(open(tpath)).get(best_key)
        except Exception:
            traffic = None

    value = world * ab / (ms_step * 1e-3) / 1e9
    e2e_gbs = world * ab / (e2e_ms * 1e-3) / 1e9
    plain_gbs = ab / (statistics.median(plain_times) * 1e-3) / 1e9
    line = None
    if rank == 0:
        cpu_t, cpu_reps, cpu_kind = cpu_reference_spmv_time(case, x, y0, budget_s=args.cpu_budget)
        line = {
            "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": desc, "nnz": nnz, "algorithmic_bytes_per_spmv": ab,
                       "partition": best_key,
                       "plain_csr": {"kernel": plain_key, "gb_s": plain_gbs},
                       "speedup_vs_plain_csr": statistics.median(plain_times) / ms_step,
                       "l2": "256 MB write then 256 MB read of another buffer between timed SpMVs (working set < L2)",
                       "parallelism": f"replicas x{world}"},
            "roofline": {"bound": "hbm", "achieved": kernel_gbs, "peak": peak, "unit": "GB/s",
                         "frac": kernel_gbs / peak, "peak_source": peak_kind, "traffic": traffic},
            "cpu_baseline": {"value": ab / cpu_t / 1e9, "unit": "GB/s", "cores": 1, "kind": cpu_kind,
                             "sample": f"{cpu_reps} whole serial csr_spmv runs of the same matrix (~{args.cpu_budget:.0f} s)"},
            "e2e": {"value": e2e_gbs, "unit": "GB/s", "h2d_bytes_per_step": 4 * (w + h), "d2h_bytes_per_step": 4 * h},
            "gpu_launches": args.steps * best.launches_per_spmv,
            "clocks": clocks,
        }
    best.free()
    plain_hd.free()
    best_mat.free()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line))


if __name__ == "__main__":
    main()
