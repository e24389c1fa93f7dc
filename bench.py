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

The other workloads are the remaining benchmark configurations, one JSON line each,
with their further legs in `config.legs`:
  laplacian  128x128 5-point Laplacian (0.85 MB, L2-resident): back-to-back graph
             replays, no flush (per-SpMV latency is the meaningful number);
  stencil    160^3 27-point stencil: forward plus the adjoint (xbar = A^T ybar and the
             value gradients);
  block      3x3-block FEM matrix, 500,000 block rows, in the generic BCSR layout:
             one right-hand side in FP32 and BF16, 8 and 32 right-hand sides;
  batch      512 matrices of uneven size in one persistent launch (formats from the
             on-device autotuner): forward, forward + adjoint, and the same work as
             per-matrix plain CSR launches.
Every workload also times plain single-format CSR on the same GPU.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload zipf|laplacian|stencil|block|batch] [--tune-cache FILE]

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


WORKLOADS = ["zipf", "laplacian", "stencil", "block", "batch"]


def make_workload(name: str, scale: float = 1.0):
    """(description, list of matrices (h, w, row, col, val), x, y0); for the batch the
    vectors are the matrices' vectors concatenated in order.  scale < 1 shrinks the
    workload (rows, grid edge, block rows or matrix count) for profiling runs."""
    from clspmv_b200 import matrices as M
    if name == "batch":
        mats = [m[1:] for m in M.batch_mixed(max(1, int(round(512 * scale))))]
        W = sum(m[1] for m in mats)
        H = sum(m[0] for m in mats)
        return ("batch_mixed 512 matrices, rows log-uniform in [1,000, 200,000], Laplacian / Zipf / 3x3-block, FP32",
                mats, M.vector(W, seed=1), M.vector(H, seed=2))
    if name == "zipf":
        case = M.zipf_rows(max(1000, int(1_000_000 * scale)), 2.0, 10_000, seed=0)
        desc = "zipf_rows n=1,000,000 s=2.0 len<=10,000 FP32"
    elif name == "laplacian":
        case = M.laplacian_2d(max(8, int(round(128 * scale ** 0.5))))
        desc = "laplacian_2d 128x128 (16,384 rows) FP32"
    elif name == "stencil":
        case = M.stencil_27(max(8, int(round(160 * scale ** (1.0 / 3.0)))))
        desc = "stencil_27 160^3 (4,096,000 rows) FP32"
    elif name == "block":
        case = M.block_3x3(max(1000, int(500_000 * scale)))
        desc = "block_3x3 500,000 block rows (3x3 blocks, block-row degree U[10,30], band +-2000) FP32"
    else:
        raise ValueError(name)
    return desc, [case], M.vector(case[1], seed=1), M.vector(case[0], seed=2)


def algorithmic_bytes(h, w, nnz, value_bytes=4, ndiag=None):
    """Minimum bytes per SpMV, no padding counted: values + indices of the structure class
    + x once + y read and written.  CSR class: column ids and row pointers; DIA class
    (ndiag given): one offset per diagonal."""
    if ndiag is not None:
        return value_bytes * nnz + 4 * ndiag + 4 * w + 8 * h
    return value_bytes * nnz + 4 * nnz + 4 * (h + 1) + 4 * w + 8 * h


def workload_bytes(name, mats, k=1, value_bytes=4):
    """Algorithmic bytes of one SpMV of a workload: banded matrices in the DIA class (their
    natural storage), 3x3-block matrices in the block class, the others in the CSR class;
    k right-hand sides multiply the vector terms."""
    tot = 0
    for h, w, r, c, v in mats:
        nnz = int(r.size)
        if name in ("stencil", "laplacian"):
            nd = int(np.unique(c.astype(np.int64) - r).size)
            tot += value_bytes * nnz + 4 * nd + k * (4 * w + 8 * h)
        elif name == "block":
            nb = nnz // 9
            tot += value_bytes * nnz + 4 * nb + 4 * (h // 3 + 1) + k * (4 * w + 8 * h)
        else:
            tot += value_bytes * nnz + 4 * nnz + 4 * (h + 1) + k * (4 * w + 8 * h)
    return tot


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


def cpu_reference_spmv_time(mats, x, y0, budget_s: float, min_reps: int = 2):
    """Times the reference's serial csr_spmv (oracle/_ref) -- or, where that was not
    built, the oracle's restatement of it -- over whole SpMVs of every matrix of the
    workload (x and y0 hold the matrices' vectors one after another) for about budget_s."""
    from clspmv_b200 import capi
    from clspmv_b200.matrices import csr_from_coo
    from tests import _oracle
    ref = _oracle.ref_lib()
    orc = None if ref is not None else _oracle.oracle_lib()
    FP = C.POINTER(C.c_float)
    IP = C.POINTER(C.c_int)
    calls, keep = [], []
    xo = yo = 0
    y = y0.copy()
    for h, w, r, c, v in mats:
        rp = csr_from_coo(h, r)
        xs, ys = x[xo:xo + w], y[yo:yo + h]
        keep += [rp, xs, ys]
        if ref is not None:
            s = capi.csr_matrix()
            s.matinfo.width, s.matinfo.height, s.matinfo.nnz = w, h, r.size
            s.csr_row_ptr = rp.ctypes.data_as(IP)
            s.csr_col_id = c.ctypes.data_as(IP)
            s.csr_data = v.ctypes.data_as(FP)
            keep.append(s)
            calls.append((ref.ref_csr_spmv, (C.byref(s), xs.ctypes.data_as(FP), ys.ctypes.data_as(FP), w)))
        else:
            calls.append((orc.orc_csr_spmv_f32, (h, rp.ctypes.data_as(IP), c.ctypes.data_as(IP), v.ctypes.data_as(FP),
                                                 xs.ctypes.data_as(FP), ys.ctypes.data_as(FP))))
        xo += w
        yo += h

    def fn():
        for f, a in calls:
            f(*a)

    kind = "reference" if ref is not None else "port"
    fn()  # warm-up
    times = []
    t_end = time.perf_counter() + budget_s
    while len(times) < min_reps or time.perf_counter() < t_end:
        t0 = time.perf_counter()
        fn()
        times.append(time.perf_counter() - t0)
    return statistics.median(times), len(times), kind


def run_reference_arm(args, desc, mats, x, y0):
    ab = workload_bytes(args.workload, mats)
    # one step = one whole serial SpMV (of every matrix) on one host core; W warm-ups, K timed
    t_step, reps, kind = cpu_reference_spmv_time(mats, x, y0, budget_s=0.0, min_reps=args.warmup + args.steps)
    gbs = ab / t_step / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": gbs, "unit": "GB/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_step * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": desc, "nnz": int(sum(m[2].size for m in mats)),
                   "path": "clSpMV serial csr_spmv (spmv_serial.h:199)"},
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
    ap.add_argument("--workload", default="zipf", choices=WORKLOADS)
    ap.add_argument("--cpu-budget", type=float, default=10.0, help="seconds of CPU-baseline sampling")
    ap.add_argument("--scale", type=float, default=1.0,
                    help="shrink the workload (profiling runs only; the benchmark configuration is 1.0)")
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
        desc, mats, x, y0 = make_workload(args.workload, args.scale)
        run_reference_arm(args, desc, mats, x, y0)
        return

    import torch
    import torch.distributed as dist
    from clspmv_b200 import (COO, CSP_ANALYZE_AUTOTUNE, CSP_FLAG_ADJOINT, CSP_FLAG_BF16, CSP_FLAG_GRAPH, Cocktail,
                             Handle, analyze_matrix, capi)
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))

    wl = args.workload
    desc, mats, x, y0 = make_workload(wl, args.scale)
    if args.scale != 1.0:
        desc += f" (scaled x{args.scale:g} for profiling)"
    nnz = int(sum(m[2].size for m in mats))
    ab = workload_bytes(wl, mats)
    # a dedicated stream: the library and torch (flush, events) must launch on the same one
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    flush_w = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    flush_r = torch.ones(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    flush_sink = torch.empty(1, dtype=torch.float32, device="cuda")
    l2_resident = wl == "laplacian"   # 0.85 MB: flushing would only time a cold start

    def flush_l2():
        flush_w.zero_()
        torch.sum(flush_r, dim=0, out=flush_sink[0])

    def time_fn(fn, steps: int, warmup: int):
        """CUDA-event milliseconds of `steps` calls of fn on the stream, L2 flushed before
        each (back to back, without flushing, for the L2-resident workload)."""
        for _ in range(warmup):
            fn()
        if l2_resident:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(steps):
                fn()
            e1.record(stream)
            torch.cuda.synchronize()
            return [e0.elapsed_time(e1) / steps] * steps
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for e0, e1 in evs:
            flush_l2()
            e0.record(stream)
            fn()
            e1.record(stream)
        torch.cuda.synchronize()
        return [e0.elapsed_time(e1) for e0, e1 in evs]

    def gbs(nbytes, ms):
        return nbytes / (ms * 1e-3) / 1e9

    legs = {}
    keep = []
    coo = COO(*mats[0]) if wl != "batch" else None

    # --- the measured path: one step = one forward SpMV of the workload ---
    if wl == "batch":
        from clspmv_b200 import Batch
        from clspmv_b200.batch import (BFMT_NAMES, CSP_BATCH_ADJ, CSP_BATCH_FWD, CSP_BATCH_TUNE_DEVICE, CSP_BV_X,
                                       CSP_BV_Y, CSP_BV_YBAR)
        coos = [COO(*m) for m in mats]
        bt = Batch(coos, flags=CSP_FLAG_ADJOINT | CSP_FLAG_GRAPH, tune=CSP_BATCH_TUNE_DEVICE,
                   cache_path=args.tune_cache)
        bt.set_stream(stream.cuda_stream)
        bt.copy_in(CSP_BV_X, x)
        bt.copy_in(CSP_BV_Y, y0)
        bt.copy_in(CSP_BV_YBAR, np.random.default_rng(3).uniform(-1, 1, bt._len(CSP_BV_YBAR)).astype(np.float32))
        step = lambda: bt.run(CSP_BATCH_FWD)  # noqa: E731
        launches = bt.launches(CSP_BATCH_FWD)
        partition = "batch: " + ", ".join(f"{n} x{bt.formats.count(i)}" for i, n in enumerate(BFMT_NAMES)
                                          if bt.formats.count(i))
        best = None
    elif wl == "block":
        b = capi.bcsr_matrix()
        capi.check(capi.lib().csp_coo2bcsr(coo.ref(), C.byref(b), 3, 3, 32), "coo2bcsr")
        keep.append(b)
        best = Handle(None, x, y0, bcsr=b)
        best.set_stream(stream.cuda_stream)
        step = lambda: best.do_spmv(1)  # noqa: E731
        launches = best.launches_per_spmv
        partition = "bcsr3x3 (generic BCSR, adaptive kernel)"
    else:
        best_mat = analyze_matrix(coo, mode=CSP_ANALYZE_AUTOTUNE, cache_path=args.tune_cache)
        keep.append(best_mat)
        flags = CSP_FLAG_ADJOINT if wl == "stencil" else (CSP_FLAG_GRAPH if l2_resident else 0)
        best = Handle(best_mat, x, y0, flags)
        best.set_stream(stream.cuda_stream)
        step = lambda: best.do_spmv(1)  # noqa: E731
        launches = best.launches_per_spmv
        partition = best_mat.choice

    # --- timed region: K steps, CUDA events on the launching stream ---
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    times = time_fn(step, args.steps, args.warmup)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    total_ms = float(sum(times))
    if world > 1:
        t = torch.tensor([total_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
        dist.barrier()
    ms_step = total_ms / args.steps
    reps = max(10, args.steps // 2)

    # --- further legs of the configuration ---
    if wl == "stencil":
        h, w = mats[0][0], mats[0][1]
        ybar = torch.rand(h, device="cuda") * 2 - 1
        xbar = torch.zeros(w, device="cuda")
        abar = torch.zeros(best.adjoint_slots, device="cuda")
        n = int(mats[0][2].size)
        b_abar = 4 * n + 4 * 27 + 4 * w + 4 * h
        t_x = statistics.median(time_fn(lambda: best.spmv_adjoint(ybar.data_ptr(), xbar.data_ptr(), None), reps, 3))
        t_a = statistics.median(time_fn(lambda: best.spmv_adjoint(ybar.data_ptr(), None, abar.data_ptr()), reps, 3))
        t_b = statistics.median(time_fn(lambda: best.spmv_adjoint(ybar.data_ptr(), xbar.data_ptr(), abar.data_ptr()),
                                        reps, 3))
        legs["adjoint_xbar"] = {"ms": t_x, "gb_s": gbs(ab, t_x)}
        legs["adjoint_abar"] = {"ms": t_a, "gb_s": gbs(b_abar, t_a)}
        legs["adjoint_both"] = {"ms": t_b, "gb_s": gbs(ab + b_abar, t_b)}
        legs["fwd_plus_adjoint"] = {"ms": ms_step + t_b, "gb_s": gbs(2 * ab + b_abar, ms_step + t_b),
                                    "frac": gbs(2 * ab + b_abar, ms_step + t_b) / _peak()[0]}
    if wl == "block":
        h, w = mats[0][0], mats[0][1]
        hb = Handle(None, x, y0, flags=CSP_FLAG_BF16, bcsr=keep[0])
        hb.set_stream(stream.cuda_stream)
        t = statistics.median(time_fn(lambda: hb.do_spmv(1), reps, 3))
        legs["k1_bf16"] = {"ms": t, "gb_s": gbs(workload_bytes(wl, mats, 1, 2), t)}
        hb.free()
        rng = np.random.default_rng(9)
        for k in (8, 32):
            X = rng.uniform(-1, 1, (w, k)).astype(np.float32)
            Y0 = rng.uniform(-1, 1, (h, k)).astype(np.float32)
            hk = Handle(None, X, Y0, nrhs=k, bcsr=keep[0])
            hk.set_stream(stream.cuda_stream)
            t = statistics.median(time_fn(lambda: hk.do_spmv(1), reps, 3))
            legs[f"k{k}"] = {"ms": t, "gb_s": gbs(workload_bytes(wl, mats, k), t),
                             "gflop_s": 2.0 * nnz * k / (t * 1e-3) / 1e9}
            hk.free()
            pm = Cocktail.single("csr", coo, 0)
            pk = Handle(pm, X, Y0, nrhs=k)
            pk.set_stream(stream.cuda_stream)
            t = statistics.median(time_fn(lambda: pk.do_spmv(1), reps, 3))
            legs[f"k{k}_plain_csr"] = {"ms": t}
            pk.free()
            pm.free()
    if wl == "batch":
        t_fa = statistics.median(time_fn(lambda: bt.run(CSP_BATCH_FWD | CSP_BATCH_ADJ), reps, 3))
        b_fa = 2 * ab + 4 * nnz
        legs["fwd_plus_adjoint"] = {"ms": t_fa, "gb_s": gbs(b_fa, t_fa), "frac": gbs(b_fa, t_fa) / _peak()[0]}
        # the same matrices with every one in CSR: one persistent launch, and per-matrix plain launches
        from clspmv_b200.capi import CSP_BFMT_CSR
        bc = Batch(coos, flags=CSP_FLAG_ADJOINT | CSP_FLAG_GRAPH, fmt=CSP_BFMT_CSR)
        bc.set_stream(stream.cuda_stream)
        bc.copy_in(CSP_BV_X, x)
        t_cf = statistics.median(time_fn(lambda: bc.run(CSP_BATCH_FWD), reps, 3))
        legs["all_csr_fwd_one_launch"] = {"ms": t_cf, "gb_s": gbs(ab, t_cf)}
        plain_reps = 5
        t_pf = statistics.median(time_fn(lambda: bc.run_plain(CSP_BATCH_FWD), plain_reps, 2))
        t_pfa = statistics.median(time_fn(lambda: bc.run_plain(CSP_BATCH_FWD | CSP_BATCH_ADJ), plain_reps, 2))
        legs["plain_fwd_per_matrix_csr"] = {"ms": t_pf, "launches": bc.launches(CSP_BATCH_FWD, plain=True)}
        legs["plain_fwd_plus_adjoint_per_matrix_csr"] = {"ms": t_pfa}
        bc.free()
        plain_ms, plain_key = t_pf, "per-matrix plain CSR launches"
    else:
        # plain single-format CSR on the same GPU: warp per row and thread per row; the faster
        plain_ms, plain_key = None, None
        for m_ in (0, 4):
            pm = Cocktail.single("csr", coo, m_)
            ph = Handle(pm, x, y0, CSP_FLAG_GRAPH if l2_resident else 0)
            ph.set_stream(stream.cuda_stream)
            t = statistics.median(time_fn(lambda: ph.do_spmv(1), reps, 3))
            if plain_ms is None or t < plain_ms:
                plain_ms, plain_key = t, f"csr{m_}"
            ph.free()
            pm.free()

    # --- e2e through the C ABI with pinned host buffers ---
    L = capi.lib()
    FP = C.POINTER(C.c_float)
    xp = torch.from_numpy(x).pin_memory()
    y0p = torch.from_numpy(y0).pin_memory()
    yout = torch.empty(y0.size, dtype=torch.float32).pin_memory()
    xptr = C.cast(C.c_void_p(xp.data_ptr()), FP)
    y0ptr = C.cast(C.c_void_p(y0p.data_ptr()), FP)
    yptr = C.cast(C.c_void_p(yout.data_ptr()), FP)
    if wl == "batch":
        def e2e_step():
            capi.check(L.csp_batch_copy(bt.h, CSP_BV_X, xptr, None), "batch_copy")
            capi.check(L.csp_batch_copy(bt.h, CSP_BV_Y, y0ptr, None), "batch_copy")
            bt.run(CSP_BATCH_FWD)
            capi.check(L.csp_batch_copy(bt.h, CSP_BV_Y, None, yptr), "batch_copy")
    else:
        def e2e_step():
            capi.check(L.csp_cpy_vector_from_cpu(best.h, xptr, x.size), "cpy_vector_from_cpu")
            capi.check(L.csp_cpy_result_from_cpu(best.h, y0ptr, y0.size), "cpy_result_from_cpu")
            capi.check(L.csp_do_spmv(best.h, 1), "do_spmv")
            capi.check(L.csp_cpy_result_to_cpu(best.h, yptr, y0.size), "cpy_result_to_cpu")
    for _ in range(args.warmup):
        e2e_step()
    torch.cuda.synchronize()
    e_times = []
    for _ in range(args.steps):
        if not l2_resident:
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
    tpath = os.path.join(ROOT, "profiles", f"traffic_{wl}.json")
    if os.path.exists(tpath):
        try:
            traffic = json.load(open(tpath)).get(partition)
        except Exception:
            traffic = None
    value = world * ab / (ms_step * 1e-3) / 1e9
    e2e_gbs = world * ab / (e2e_ms * 1e-3) / 1e9
    line = None
    if rank == 0:
        cpu_t, cpu_reps, cpu_kind = cpu_reference_spmv_time(mats, x, y0, budget_s=args.cpu_budget)
        l2_note = ("L2-resident working set (0.85 MB): back-to-back graph replays, no flush" if l2_resident else
                   "256 MB write then 256 MB read of another buffer between timed SpMVs")
        line = {
            "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": desc, "nnz": nnz, "algorithmic_bytes_per_spmv": ab, "partition": partition,
                       "gflop_s": 2.0 * nnz / (ms_step * 1e-3) / 1e9,
                       "plain_csr": {"kernel": plain_key, "ms": plain_ms, "gb_s": gbs(ab, plain_ms)},
                       "speedup_vs_plain_csr": plain_ms / ms_step,
                       "legs": legs, "l2": l2_note, "parallelism": f"replicas x{world}"},
            "roofline": {"bound": "hbm", "achieved": kernel_gbs, "peak": peak, "unit": "GB/s",
                         "frac": kernel_gbs / peak, "peak_source": peak_kind, "traffic": traffic},
            "cpu_baseline": {"value": ab / cpu_t / 1e9, "unit": "GB/s", "cores": 1, "kind": cpu_kind,
                             "sample": f"{cpu_reps} whole serial csr_spmv runs of the workload (~{args.cpu_budget:.0f} s)"},
            "e2e": {"value": e2e_gbs, "unit": "GB/s", "h2d_bytes_per_step": 4 * (x.size + y0.size),
                    "d2h_bytes_per_step": 4 * y0.size},
            "gpu_launches": args.steps * launches,
            "clocks": clocks,
        }
    if best is not None:
        best.free()
    else:
        bt.free()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line))


if __name__ == "__main__":
    main()
