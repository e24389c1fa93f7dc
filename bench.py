#!/usr/bin/env python
"""Cocktail SpMV on B200: HBM GB/s, fraction of the HBM roofline, forward + adjoint
time, autotuned against plain CSR on the same GPU.

Headline (the default `--workload batch`): the batched uneven workload, 512 matrices
with row counts log-uniform in [1,000, 200,000], each drawn by seed from the
Laplacian-family, Zipf-row and 3x3-block generators at about 12 nonzeros per row,
FP32, each with its own x, y and ybar.  One step = forward y += A x, value gradients
abar = ybar (x) x on the stored pattern and adjoint xbar += A^T ybar for every matrix
in ONE persistent kernel launch (a CUDA graph replay), formats chosen per matrix by
the on-device autotuner.  `value` is algorithmic GB/s of that step (values + indices
+ vectors of A and of A^T, plus the gradient store; no padding counted) over the
CUDA-event time on the launching stream, inputs resident in HBM.  Between timed steps
L2 is cleared by a 256 MB write followed by a 256 MB read of another buffer (the
batch's 2 GB per pass is far larger than the 126 MB L2 in any case).  The baseline on
the same GPU is the same work as per-matrix plain CSR launches.

The other benchmark configurations run in the same process and are reported in
`config.legs`, each with its own roofline fraction, plain-CSR time on the same GPU,
reference-CPU baseline and FP64 error:
  c1_laplacian  128x128 5-point Laplacian (0.85 MB, L2-resident): back-to-back graph
                replays, no flush (per-SpMV latency is the meaningful number);
  c2_zipf       10^6 x 10^6, Zipf(2) row lengths clipped to [1, 10,000], forward;
  c3_stencil    160^3 27-point stencil: forward, xbar = A^T ybar and the value
                gradients;
  c4_block      3x3-block FEM matrix, 500,000 block rows, autotuned Cocktail (the
                generic 3x3 BCSR is among its candidates): one right-hand side in
                FP32 and BF16 values, 8 and 32 right-hand sides (CUDA cores and
                tensor cores).
All matrices are synthetic and seeded (the reference's public matrix collection is
not available offline).

Errors: each configuration is run once more with y = 0 (and xbar = 0) and compared
with an FP64 product computed here with scipy: max over rows of
|y_i - yhat_i| / sum_j |a_ij x_j| (the per-row FP32 bound is 1e-5).  Where the
reference CPU path runs (cpu_baseline), its own FP32 result is compared the same way
and by ulp distance.

`e2e` is the headline step through the C ABI with pinned host buffers: H2D of x, y,
ybar and xbar, the step, D2H of y and xbar, every step, split into H2D, kernel and D2H
milliseconds.  The value gradients stay in HBM (as a training step's gradients do);
their read-back is timed separately and reported beside e2e.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload batch|laplacian|zipf|stencil|block] [--no-legs]
                  [--scale S] [--tune-cache FILE]

With --impl reference the reference's own CPU SpMV (clSpMV_NV/include/spmv_serial.h
csr_spmv, compiled from the reference sources into oracle/_ref) runs the headline
step on the host: csr_spmv over every matrix and over its explicit transpose, plus
the value-gradient loop (which the reference lacks; the oracle's C loop), on all host
threads, each thread taking whole matrices or row ranges.  Under torchrun every rank
runs an independent replica of the headline (weak scaling, no collective on the data
path) and the legs are skipped.
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
from concurrent.futures import ThreadPoolExecutor

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "SpMV HBM GB/s & % of roofline; fwd+adjoint time, autotuned vs plain CSR"
L2_FLUSH_BYTES = 256 << 20
WORKLOADS = ["batch", "laplacian", "zipf", "stencil", "block"]
LEG_NAMES = {"laplacian": "c1_laplacian", "zipf": "c2_zipf", "stencil": "c3_stencil", "block": "c4_block"}
FP = C.POINTER(C.c_float)
IP = C.POINTER(C.c_int)


def _peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


# ---------------------------------------------------------------------------
# workloads and their algorithmic bytes
# ---------------------------------------------------------------------------
CLASS_OF = {"laplacian": "dia", "stencil": "dia", "block": "block", "zipf": "csr"}


def make_workload(name: str, scale: float = 1.0, world: int = 1, rank: int = 0):
    """(description, list of matrices (h, w, row, col, val), x, y0, structure class of
    each matrix); for the batch the vectors are the matrices' vectors concatenated in
    order.  scale < 1 shrinks the workload (rows, grid edge, block rows or matrix count)
    for profiling runs.  With world > 1 the batch is a list of world * 512 matrices and
    this rank builds its shard of 512 (matrix.shard): rank 0's shard is the 1-GPU batch."""
    from clspmv_b200 import matrices as M
    if name == "batch":
        per = max(1, int(round(512 * scale)))
        first, n = M.shard(per * world, world, rank)
        gen = M.batch_mixed(per * world, first=first, n=n)
        mats = [m[1:] for m in gen]
        kinds = [CLASS_OF[m[0]] for m in gen]
        del gen
        W = sum(m[1] for m in mats)
        H = sum(m[0] for m in mats)
        return ("batch_mixed 512 matrices, rows log-uniform in [1,000, 200,000], Laplacian / Zipf / 3x3-block, FP32",
                mats, M.vector(W, seed=1 + rank), M.vector(H, seed=2 + rank), kinds)
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
    return desc, [case], M.vector(case[1], seed=1), M.vector(case[0], seed=2), [CLASS_OF[name]]


def matrix_bytes(kind: str, h: int, w: int, r, c, k: int = 1, value_bytes: int = 4) -> int:
    """Algorithmic bytes of one SpMV y = A x + y of one matrix: values + indices of its
    structure class + k * (x once + y read and written); no padding counted.  Banded
    matrices count in the DIA class (one offset per diagonal), 3x3-block matrices in the
    block class (one column per block + block-row pointers), the rest in the CSR class."""
    nnz = int(r.size)
    vec = k * (4 * w + 8 * h)
    if kind == "dia":
        nd = int(np.unique(c.astype(np.int64) - r).size) if nnz else 0
        return value_bytes * nnz + 4 * nd + vec
    if kind == "block":
        return value_bytes * nnz + 4 * (nnz // 9) + 4 * (h // 3 + 1) + vec
    return value_bytes * nnz + 4 * nnz + 4 * (h + 1) + vec


def workload_bytes(mats, kinds, k=1, value_bytes=4):
    """Algorithmic bytes of one forward SpMV of a workload (every matrix once)."""
    return sum(matrix_bytes(kd, h, w, r, c, k, value_bytes) for kd, (h, w, r, c, v) in zip(kinds, mats))


def fwd_adjoint_bytes(fwd_bytes: int, nnz: int, value_bytes: int = 4) -> int:
    """Forward + adjoint of the same matrices: the forward pass (which also writes the
    value gradients, one store per entry) and the same-sized pass over A^T."""
    return 2 * fwd_bytes + value_bytes * nnz


# ---------------------------------------------------------------------------
# FP64 checks (scipy; independent of the test oracle)
# ---------------------------------------------------------------------------
def _scipy_csr(h, w, r, c, v):
    import scipy.sparse as sp
    from clspmv_b200.matrices import csr_from_coo
    order = None
    if r.size > 1 and (np.any(r[1:] < r[:-1])):
        order = np.lexsort((c, r))
    rr, cc, vv = (r, c, v) if order is None else (r[order], c[order], v[order])
    rp = csr_from_coo(h, rr)
    return sp.csr_matrix((vv.astype(np.float64), cc, rp), shape=(h, w))


def rel_err(y, yhat, scale):
    """max_i |y_i - yhat_i| / scale_i; rows with scale 0 must match exactly."""
    if y.size == 0:
        return 0.0
    d = np.abs(y.astype(np.float64) - yhat)
    z = scale == 0
    if np.any(d[z] != 0):
        return float("inf")
    with np.errstate(invalid="ignore", divide="ignore"):
        q = np.where(z, 0.0, d / np.where(z, 1.0, scale))
    return float(np.max(q))


def ulp_dist(a, b):
    """ulp distance between two FP32 arrays (max, median)."""
    def key(u):
        i = u.astype(np.float32).view(np.int32).astype(np.int64)
        return np.where(i < 0, -(i & 0x7FFFFFFF), i)
    d = np.abs(key(a) - key(b))
    return int(d.max()) if d.size else 0, float(np.median(d)) if d.size else 0.0


def fp64_products(mats, xs, transpose=False, values=None):
    """Per matrix (yhat, sum|a x|) in FP64; xs: the per-matrix input vectors."""
    out = []
    for i, (h, w, r, c, v) in enumerate(mats):
        A = _scipy_csr(h, w, r, c, v if values is None else values[i])
        if transpose:
            A = A.T.tocsr()
        x64 = xs[i].astype(np.float64)
        out.append((A @ x64, abs(A) @ np.abs(x64)))
    return out


def split(vec, sizes):
    offs = np.concatenate([[0], np.cumsum(sizes)])
    return [vec[int(offs[i]):int(offs[i + 1])] for i in range(len(sizes))]


def max_err(ys, refs):
    return max((rel_err(y, yh, s) for y, (yh, s) in zip(ys, refs)), default=0.0)


def bf16_round(v):
    u = np.asarray(v, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


# ---------------------------------------------------------------------------
# the reference's CPU path (test oracle; the CPU-baseline leg only)
# ---------------------------------------------------------------------------
class CpuReference:
    """The reference's serial csr_spmv (oracle/_ref, compiled from the reference
    sources) -- or, where that was not built, the oracle's C restatement of it -- over
    every matrix of a workload, on `threads` host threads.  Each matrix is cut into
    row ranges of about equal nonzeros; csr_spmv on a range is csr_spmv of those rows
    (row pointers are absolute), so the result is the serial one bit for bit.  With
    `adjoint`, each step also runs csr_spmv on the explicit transposes (built here with
    scipy, untimed) and the value-gradient loop abar_j = ybar_row * x_col (the oracle's
    C loop: the reference has no adjoint)."""

    def __init__(self, mats, x, y0, threads, adjoint=False, ybar=None):
        from clspmv_b200 import capi
        from clspmv_b200.matrices import csr_from_coo
        from tests import _oracle
        self.ref = _oracle.ref_lib()
        self.orc = _oracle.oracle_lib()
        self.kind = "reference" if self.ref is not None else "port"
        total = sum(int(m[2].size) for m in mats)
        # a thread per 256K nonzeros at least: below that, dispatch costs more than it saves
        self.threads = max(1, min(threads, total // (1 << 18)))
        self.keep = []
        hs = [m[0] for m in mats]
        ws = [m[1] for m in mats]
        self.y0 = y0
        self.y = y0.copy()
        xs, ys = split(x, ws), split(self.y, hs)
        tasks = []   # (nnz, fn, args)
        chunk = max(4096, total // (self.threads * 8))
        csrs = []
        for i, (h, w, r, c, v) in enumerate(mats):
            rp = csr_from_coo(h, r)
            cc = np.ascontiguousarray(c, np.int32)
            vv = np.ascontiguousarray(v, np.float32)
            csrs.append((h, w, rp, cc, vv))
            self.keep += [rp, cc, vv]
            tasks += self._spmv_tasks(capi, h, w, rp, cc, vv, xs[i], ys[i], chunk)
        if adjoint:
            import scipy.sparse as sp
            self.xbar = np.zeros(x.size, np.float32)
            xbs, ybs = split(self.xbar, ws), split(ybar, hs)
            self.abar = np.zeros(total, np.float32)
            goff = 0
            for i, (h, w, rp, cc, vv) in enumerate(csrs):
                T = sp.csr_matrix((vv, cc, rp), shape=(h, w)).T.tocsr()
                T.sort_indices()
                trp = T.indptr.astype(np.int32)
                tc = T.indices.astype(np.int32)
                tv = T.data.astype(np.float32)
                self.keep += [trp, tc, tv]
                tasks += self._spmv_tasks(capi, w, h, trp, tc, tv, ybs[i], xbs[i], chunk)
                g = self.abar[goff:goff + int(rp[-1])]
                goff += int(rp[-1])
                self.keep.append(g)
                for r0, r1 in self._ranges(rp, h, chunk):
                    tasks.append((int(rp[r1] - rp[r0]), self.orc.orc_csr_value_grad_f32,
                                  (r1 - r0, self._p(rp, r0, IP), self._p(cc, 0, IP), self._p(ybs[i], r0, FP),
                                   self._p(xs[i], 0, FP), self._p(g, 0, FP))))
        # longest-first onto the least-loaded thread
        tasks.sort(key=lambda t: -t[0])
        self.lists = [[] for _ in range(self.threads)]
        load = [0] * self.threads
        for t in tasks:
            k = load.index(min(load))
            self.lists[k].append(t[1:])
            load[k] += t[0] + 64
        self.pool = ThreadPoolExecutor(self.threads) if self.threads > 1 else None

    @staticmethod
    def _p(a, off, T):
        return C.cast(C.c_void_p(a.ctypes.data + a.itemsize * int(off)), T)

    @staticmethod
    def _ranges(rp, h, chunk):
        """Row ranges [r0, r1) of about `chunk` nonzeros each (at least one row)."""
        r0 = 0
        while r0 < h:
            r1 = int(np.searchsorted(rp, rp[r0] + chunk, side="right")) - 1
            r1 = min(h, max(r0 + 1, r1))
            yield r0, r1
            r0 = r1

    def _spmv_tasks(self, capi, h, w, rp, cc, vv, x, y, chunk):
        out = []
        for r0, r1 in self._ranges(rp, h, chunk):
            nz = int(rp[r1] - rp[r0])
            if self.ref is not None:
                s = capi.csr_matrix()
                s.matinfo.width, s.matinfo.height, s.matinfo.nnz = w, r1 - r0, nz
                s.csr_row_ptr = self._p(rp, r0, IP)
                s.csr_col_id = self._p(cc, 0, IP)
                s.csr_data = self._p(vv, 0, FP)
                self.keep.append(s)
                out.append((nz, self.ref.ref_csr_spmv, (C.byref(s), self._p(x, 0, FP), self._p(y, r0, FP), w)))
            else:
                out.append((nz, self.orc.orc_csr_spmv_f32, (r1 - r0, self._p(rp, r0, IP), self._p(cc, 0, IP),
                                                            self._p(vv, 0, FP), self._p(x, 0, FP), self._p(y, r0, FP))))
        return out

    @staticmethod
    def _run_list(lst):
        for f, a in lst:
            f(*a)

    def step(self):
        if self.pool is None:
            self._run_list(self.lists[0])
        else:
            list(self.pool.map(self._run_list, self.lists))

    def time(self, budget_s: float, min_reps: int = 2, warmup: int = 1):
        for _ in range(warmup):
            self.step()
        times = []
        t_end = time.perf_counter() + budget_s
        while len(times) < min_reps or time.perf_counter() < t_end:
            t0 = time.perf_counter()
            self.step()
            times.append(time.perf_counter() - t0)
        return statistics.median(times), len(times)

    def result_from_zero(self):
        """One forward pass from y = 0 (the FP32 result compared with the device's)."""
        self.y[:] = 0.0
        if hasattr(self, "xbar"):
            self.xbar[:] = 0.0
        self.step()
        return self.y.copy()

    def close(self):
        if self.pool is not None:
            self.pool.shutdown()


def cpu_baseline(mats, x, y0, nbytes, budget_s, adjoint=False, ybar=None, gpu_y=None, refs=None):
    """The cpu_baseline object of one configuration (and the reference's own error)."""
    cr = CpuReference(mats, x, y0, host_threads(), adjoint=adjoint, ybar=ybar)
    try:
        t, reps = cr.time(budget_s)
        out = {"value": nbytes / t / 1e9, "unit": "GB/s", "cores": cr.threads, "host_cores": os.cpu_count(),
               "kind": cr.kind, "ms": t * 1e3,
               "sample": (f"{reps} whole {'forward + adjoint ' if adjoint else ''}passes over the workload on "
                          f"{cr.threads} host threads (~{budget_s:.0f} s), each thread running the serial "
                          "csr_spmv on whole matrices or row ranges")}
        if gpu_y is not None and refs is not None:
            yr = cr.result_from_zero()
            hs = [m[0] for m in mats]
            out["max_rel_err"] = max_err(split(yr, hs), refs)
            mx, med = ulp_dist(gpu_y, yr)
            out["ulp_vs_device"] = {"max": mx, "median": med}
        return out
    finally:
        cr.close()


# ---------------------------------------------------------------------------
# device timing
# ---------------------------------------------------------------------------
class ClockSampler:
    """SM clocks and throttle reasons sampled during the timed region: NVML read every
    5 ms from a thread (the timed regions are tens of milliseconds), else nvidia-smi
    every 100 ms.  Read-only queries; nothing of the GPU's settings changes."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4))

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []
        self.thread = None
        self.nvml = None
        self.samples = []   # (sm MHz, reason bits)
        self.smax = None
        self.running = False

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            pr = torch.cuda.get_device_properties(self.device)
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.device)

    def _nvml_sample(self):
        nv, h = self.nvml
        try:
            bits = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
        except Exception:
            bits = nv.nvmlDeviceGetCurrentClocksThrottleReasons(h)
        self.samples.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)), int(bits)))

    def _nvml_loop(self):
        while self.running:
            try:
                self._nvml_sample()
            except Exception:
                return
            time.sleep(0.005)

    def start(self):
        try:
            self.nvml = self._nvml_handle()
            self.smax = float(self.nvml[0].nvmlDeviceGetMaxClockInfo(self.nvml[1], self.nvml[0].NVML_CLOCK_SM))
            self._nvml_sample()   # the first sample before the timed region starts
            self.running = True
            self.thread = threading.Thread(target=self._nvml_loop, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.nvml = None
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
        if self.nvml is not None:
            self.running = False
            self.thread.join(timeout=1)
            sm = [c for c, _ in self.samples]
            reasons = sorted({nm for _, bits in self.samples for nm, b in self.REASONS if bits & b})
            return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.smax, "reasons": reasons,
                    "samples": len(sm), "source": "NVML every 5 ms"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = [nm for nm, _ in self.REASONS]
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
                "samples": len(sm), "source": "nvidia-smi every 100 ms"}


class Device:
    """The launching stream, the L2 flush and CUDA-event timing."""

    def __init__(self, torch, local):
        self.torch = torch
        self.stream = torch.cuda.Stream()
        torch.cuda.set_stream(self.stream)
        self.flush_w = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
        self.flush_r = torch.ones(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
        self.flush_sink = torch.empty(1, dtype=torch.float32, device="cuda")
        self.local = local

    @property
    def sp(self):
        return self.stream.cuda_stream

    def flush_l2(self):
        self.flush_w.zero_()
        self.torch.sum(self.flush_r, dim=0, out=self.flush_sink[0])

    def time(self, fn, steps: int, warmup: int, l2_resident: bool = False):
        """CUDA-event milliseconds of `steps` calls of fn on the stream, L2 flushed before
        each (back to back, without flushing, for an L2-resident workload)."""
        torch = self.torch
        for _ in range(warmup):
            fn()
        if l2_resident:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(self.stream)
            for _ in range(steps):
                fn()
            e1.record(self.stream)
            torch.cuda.synchronize()
            return [e0.elapsed_time(e1) / steps] * steps
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for e0, e1 in evs:
            self.flush_l2()
            e0.record(self.stream)
            fn()
            e1.record(self.stream)
        torch.cuda.synchronize()
        return [e0.elapsed_time(e1) for e0, e1 in evs]

    def median(self, fn, reps=20, warmup=3, l2_resident=False):
        return statistics.median(self.time(fn, reps, warmup, l2_resident))


def gbs(nbytes, ms):
    return nbytes / (ms * 1e-3) / 1e9


def traffic_of(workload, partition):
    """ncu-measured DRAM bytes per launch of the dominant kernel (profiles/traffic_*.json),
    or None."""
    p = os.path.join(ROOT, "profiles", f"traffic_{workload}.json")
    try:
        return json.load(open(p)).get(partition)
    except Exception:
        return None


# ---------------------------------------------------------------------------
# the batch (headline)
# ---------------------------------------------------------------------------
def run_batch(dev, args, world, rank, with_cpu: bool):
    from clspmv_b200 import COO, CSP_FLAG_ADJOINT, CSP_FLAG_GRAPH, Batch, capi
    from clspmv_b200.batch import (BFMT_NAMES, CSP_BATCH_ADJ, CSP_BATCH_FWD, CSP_BATCH_TUNE_DEVICE, CSP_BV_ABAR,
                                   CSP_BV_X, CSP_BV_XBAR, CSP_BV_Y, CSP_BV_YBAR)
    from clspmv_b200.capi import CSP_BFMT_CSR
    torch = dev.torch
    desc, mats, x, y0, kinds = make_workload("batch", args.scale, world, rank)
    nnz = int(sum(m[2].size for m in mats))
    fwd_b = workload_bytes(mats, kinds)
    both_b = fwd_adjoint_bytes(fwd_b, nnz)
    hs, ws = [m[0] for m in mats], [m[1] for m in mats]
    ybar = np.random.default_rng(3).uniform(-1, 1, sum(hs)).astype(np.float32)
    coos = [COO(*m) for m in mats]
    t0 = time.perf_counter()
    bt = Batch(coos, flags=CSP_FLAG_ADJOINT | CSP_FLAG_GRAPH, tune=CSP_BATCH_TUNE_DEVICE, cache_path=args.tune_cache)
    setup_s = time.perf_counter() - t0
    bt.set_stream(dev.sp)
    xbar0 = np.zeros(sum(ws), np.float32)

    def load():
        bt.copy_in(CSP_BV_X, x)
        bt.copy_in(CSP_BV_Y, y0)
        bt.copy_in(CSP_BV_YBAR, ybar)
        bt.copy_in(CSP_BV_XBAR, xbar0)

    load()
    BOTH = CSP_BATCH_FWD | CSP_BATCH_ADJ
    step = lambda: bt.run(BOTH)  # noqa: E731
    partition = ("batch: " + ", ".join(f"{n} x{bt.formats.count(i)}" for i, n in enumerate(BFMT_NAMES)
                                       if bt.formats.count(i))
                 + "; transposes: " + ", ".join(f"{n} x{bt.formats_adjoint.count(i)}" for i, n in enumerate(BFMT_NAMES)
                                                if bt.formats_adjoint.count(i)))

    # --- timed region: K steps, CUDA events on the launching stream ---
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(dev.local)
    sampler.start()
    times = dev.time(step, args.steps, args.warmup)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    total_ms = float(sum(times))
    if world > 1:
        t = torch.tensor([total_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
        dist.barrier()
    ms_step = total_ms / args.steps

    out = {"desc": desc, "nnz": nnz, "setup_s": setup_s, "partition": partition, "ms_step": ms_step,
           "bytes": both_b, "fwd_bytes": fwd_b, "clocks": clocks, "launches": bt.launches(BOTH)}
    legs = {}
    reps = max(10, args.steps // 2)
    t_f = dev.median(lambda: bt.run(CSP_BATCH_FWD), reps)
    legs["forward"] = {"ms": t_f, "gb_s": gbs(fwd_b, t_f), "frac": gbs(fwd_b, t_f) / _peak()[0]}

    # --- errors: one step from y = 0, xbar = 0 against FP64 ---
    bt.copy_in(CSP_BV_Y, np.zeros_like(y0))
    bt.copy_in(CSP_BV_XBAR, xbar0)
    bt.run(BOTH)
    y_dev, xbar_dev, abar_dev = bt.copy_out(CSP_BV_Y), bt.copy_out(CSP_BV_XBAR), bt.copy_out(CSP_BV_ABAR)
    xs, ybs = split(x, ws), split(ybar, hs)
    refs_y = fp64_products(mats, xs)
    refs_x = fp64_products(mats, ybs, transpose=True)
    err_y = max_err(split(y_dev, hs), refs_y)
    err_x = max_err(split(xbar_dev, ws), refs_x)
    err_a = 0.0
    for i in range(len(mats)):
        rows, cols = bt.pattern(i)
        g = abar_dev[int(bt.abar_off[i]):int(bt.abar_off[i + 1])]
        ok = rows >= 0
        want = ybs[i][rows[ok]].astype(np.float64) * xs[i][cols[ok]].astype(np.float64)
        d = np.abs(g[ok].astype(np.float64) - want)
        aw = np.abs(want)
        if np.any(g[~ok] != 0) or np.any(d[aw == 0] != 0):
            err_a = float("inf")
        elif np.any(aw > 0):
            err_a = max(err_a, float(np.max(d[aw > 0] / aw[aw > 0])))
    out["errors"] = {"y_max_rel_err": err_y, "xbar_max_rel_err": err_x, "abar_max_rel_err": err_a,
                     "bound": "per row |err| <= 1e-5 * sum_j |a_ij x_j| (y), |a_ij ybar_i| (xbar); "
                              "abar relative to |ybar_i x_j|"}
    load()

    # --- the same matrices as per-matrix plain CSR (one launch per matrix and direction) ---
    bc = Batch(coos, flags=CSP_FLAG_ADJOINT | CSP_FLAG_GRAPH, fmt=CSP_BFMT_CSR)
    bc.set_stream(dev.sp)
    bc.copy_in(CSP_BV_X, x)
    bc.copy_in(CSP_BV_YBAR, ybar)
    t_cb = dev.median(lambda: bc.run(BOTH), reps)
    legs["all_csr_one_launch_fwd_plus_adjoint"] = {"ms": t_cb, "gb_s": gbs(both_b, t_cb)}
    t_pf = dev.median(lambda: bc.run_plain(CSP_BATCH_FWD), 5, 2)
    t_pb = dev.median(lambda: bc.run_plain(BOTH), 5, 2)
    legs["plain_csr_per_matrix_forward"] = {"ms": t_pf, "gb_s": gbs(fwd_b, t_pf),
                                            "launches": bc.launches(CSP_BATCH_FWD, plain=True)}
    out["plain"] = {"kernel": "per-matrix plain CSR-vector launches (forward, value gradients, A^T)",
                    "ms": t_pb, "gb_s": gbs(both_b, t_pb), "launches": bc.launches(BOTH, plain=True)}
    bc.free()

    # --- e2e through the C ABI with pinned host buffers ---
    L = capi.lib()
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()  # noqa: E731
    hx, hy0, hyb, hxb0 = pin(x), pin(y0), pin(ybar), pin(xbar0)
    hy = torch.empty(y0.size, dtype=torch.float32).pin_memory()
    hxb = torch.empty(xbar0.size, dtype=torch.float32).pin_memory()
    ha = torch.empty(int(bt.abar_off[-1]), dtype=torch.float32).pin_memory()
    ptr = lambda t: C.cast(C.c_void_p(t.data_ptr()), FP)  # noqa: E731

    def h2d():
        for which, src in ((CSP_BV_X, hx), (CSP_BV_Y, hy0), (CSP_BV_YBAR, hyb), (CSP_BV_XBAR, hxb0)):
            capi.check(L.csp_batch_copy(bt.h, which, ptr(src), None), "batch_copy")

    def d2h():
        for which, dst in ((CSP_BV_Y, hy), (CSP_BV_XBAR, hxb)):
            capi.check(L.csp_batch_copy(bt.h, which, None, ptr(dst)), "batch_copy")

    for _ in range(args.warmup):
        h2d()
        bt.run(BOTH)
        d2h()
    torch.cuda.synchronize()
    split_ms = []
    for _ in range(args.steps):
        dev.flush_l2()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        ev[0].record(dev.stream)
        h2d()
        ev[1].record(dev.stream)
        bt.run(BOTH)
        ev[2].record(dev.stream)
        d2h()
        ev[3].record(dev.stream)
        torch.cuda.synchronize()
        split_ms.append([ev[i].elapsed_time(ev[i + 1]) for i in range(3)])
    sm = np.mean(np.array(split_ms), axis=0)
    e2e_ms = float(sm.sum())
    # the value gradients' read-back, timed on its own (not part of the step: they stay in HBM)
    abar_ms = []
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(dev.stream)
        capi.check(L.csp_batch_copy(bt.h, CSP_BV_ABAR, None, ptr(ha)), "batch_copy")
        e1.record(dev.stream)
        torch.cuda.synchronize()
        abar_ms.append(e0.elapsed_time(e1))
    job_b = world * both_b
    if world > 1:
        t = torch.tensor([e2e_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
        tb = torch.tensor([both_b], dtype=torch.int64, device="cuda")
        dist.all_reduce(tb, op=dist.ReduceOp.SUM)   # the shards' bytes
        job_b = int(tb.item())
    out["e2e"] = {"value": job_b / (e2e_ms * 1e-3) / 1e9, "unit": "GB/s",
                  "h2d_bytes_per_step": 4 * (x.size + y0.size + ybar.size + xbar0.size),
                  "d2h_bytes_per_step": 4 * (y0.size + xbar0.size),
                  "ms_per_step": e2e_ms, "h2d_ms": float(sm[0]), "kernel_ms": float(sm[1]), "d2h_ms": float(sm[2]),
                  "path": "csp_batch_copy (x, y, ybar, xbar in from pinned host memory) + csp_batch_run + "
                          "csp_batch_copy (y, xbar out)",
                  "abar": {"bytes": 4 * int(bt.abar_off[-1]), "d2h_ms": statistics.median(abar_ms),
                           "note": "the value gradients stay in HBM for the caller's update, like a training "
                                   "step's gradients; their read-back is timed here, outside the step"}}
    out["legs"] = legs
    bt.free()
    if with_cpu:
        out["cpu"] = cpu_baseline(mats, x, y0, both_b, args.cpu_budget, adjoint=True, ybar=ybar,
                                  gpu_y=y_dev, refs=refs_y)
    return out


# ---------------------------------------------------------------------------
# single-matrix configurations (the legs)
# ---------------------------------------------------------------------------
def run_single(dev, name, args, with_cpu: bool, steps: int, warmup: int):
    from clspmv_b200 import (COO, CSP_ANALYZE_AUTOTUNE, CSP_FLAG_ADJOINT, CSP_FLAG_BF16, CSP_FLAG_GRAPH,
                             CSP_FLAG_TENSOR_CORES, Cocktail, Handle, analyze_matrix, capi)
    torch = dev.torch
    desc, mats, x, y0, kinds = make_workload(name, args.scale)
    h, w, r, c, v = mats[0]
    nnz = int(r.size)
    ab = workload_bytes(mats, kinds)
    l2_resident = name == "laplacian"
    coo = COO(*mats[0])
    keep = []
    out = {"desc": desc, "nnz": nnz, "bytes": ab}
    t0 = time.perf_counter()
    mat = analyze_matrix(coo, mode=CSP_ANALYZE_AUTOTUNE, cache_path=args.tune_cache)
    keep.append(mat)
    flags = CSP_FLAG_ADJOINT if name == "stencil" else (CSP_FLAG_GRAPH if l2_resident else 0)
    best = Handle(mat, x, y0, flags)
    partition = mat.choice
    out["setup_s"] = time.perf_counter() - t0
    out["analyzer_s"] = reference_tables_analysis_s(mats[0])
    best.set_stream(dev.sp)
    step = lambda: best.do_spmv(1)  # noqa: E731
    times = dev.time(step, steps, warmup, l2_resident)
    ms = float(np.mean(times))
    out.update({"partition": partition, "ms_step": ms, "launches": best.launches_per_spmv,
                "l2": ("L2-resident working set (0.85 MB): back-to-back graph replays, no flush" if l2_resident else
                       "256 MB write then 256 MB read of another buffer before each timed SpMV")})
    legs = {}
    reps = max(10, steps // 2)

    # --- error of one SpMV from y = 0 ---
    best.cpy_result_from_cpu(np.zeros_like(y0))
    best.do_spmv(1)
    y_dev = best.cpy_result_to_cpu()
    refs = fp64_products(mats, [x])
    errors = {"y_max_rel_err": max_err([y_dev], refs)}

    if name == "stencil":
        ybar = torch.rand(h, device="cuda") * 2 - 1
        xbar = torch.zeros(w, device="cuda")
        abar = torch.zeros(best.adjoint_slots, device="cuda")
        nd = 27
        b_abar = 4 * nnz + 4 * nd + 4 * w + 4 * h
        t_x = dev.median(lambda: best.spmv_adjoint(ybar.data_ptr(), xbar.data_ptr(), None), reps)
        t_a = dev.median(lambda: best.spmv_adjoint(ybar.data_ptr(), None, abar.data_ptr()), reps)
        t_b = dev.median(lambda: best.spmv_adjoint(ybar.data_ptr(), xbar.data_ptr(), abar.data_ptr()), reps)
        legs["adjoint_xbar"] = {"ms": t_x, "gb_s": gbs(ab, t_x), "frac": gbs(ab, t_x) / _peak()[0]}
        legs["adjoint_abar"] = {"ms": t_a, "gb_s": gbs(b_abar, t_a), "frac": gbs(b_abar, t_a) / _peak()[0]}
        legs["adjoint_both"] = {"ms": t_b, "gb_s": gbs(ab + b_abar, t_b)}
        legs["fwd_plus_adjoint"] = {"ms": ms + t_b, "gb_s": gbs(2 * ab + b_abar, ms + t_b),
                                    "frac": gbs(2 * ab + b_abar, ms + t_b) / _peak()[0]}
        xbar.zero_()
        best.spmv_adjoint(ybar.data_ptr(), xbar.data_ptr(), abar.data_ptr())
        torch.cuda.synchronize()
        ybh = ybar.cpu().numpy()
        errors["xbar_max_rel_err"] = max_err([xbar.cpu().numpy()], fp64_products(mats, [ybh], transpose=True))
        # value gradients: abar[slot] = ybar[row] * x[col] on the stored pattern
        rows = torch.empty(best.adjoint_slots, dtype=torch.int32, device="cuda")
        cols = torch.empty_like(rows)
        best.adjoint_pattern(rows.data_ptr(), cols.data_ptr())
        rr, cc, g = rows.cpu().numpy(), cols.cpu().numpy(), abar.cpu().numpy()
        ok = rr >= 0
        want = ybh[rr[ok]].astype(np.float64) * x[cc[ok]].astype(np.float64)
        aw = np.abs(want)
        d = np.abs(g[ok].astype(np.float64) - want)
        errors["abar_max_rel_err"] = float(np.max(d[aw > 0] / aw[aw > 0])) if np.any(aw > 0) else 0.0
        del rows, cols, abar, xbar
    if name == "block":
        # BF16 values and several right-hand sides on the same autotuned partition
        hb = Handle(mat, x, y0, flags=CSP_FLAG_BF16)
        hb.set_stream(dev.sp)
        t = dev.median(lambda: hb.do_spmv(1), reps)
        bb = workload_bytes(mats, kinds, 1, 2)
        legs["k1_bf16"] = {"ms": t, "gb_s": gbs(bb, t), "frac": gbs(bb, t) / _peak()[0]}
        hb.cpy_result_from_cpu(np.zeros_like(y0))
        hb.do_spmv(1)
        yb = hb.cpy_result_to_cpu()
        hb.free()
        errors["k1_bf16_vs_bf16_matrix_max_rel_err"] = max_err([yb], fp64_products(mats, [x], values=[bf16_round(v)]))
        errors["k1_bf16_vs_fp32_matrix_max_rel_err"] = max_err([yb], refs)
        rng = np.random.default_rng(9)
        A64 = _scipy_csr(h, w, r, c, v)
        A64b = _scipy_csr(h, w, r, c, bf16_round(v))
        for k in (8, 32):
            X = rng.uniform(-1, 1, (w, k)).astype(np.float32)
            Y0 = rng.uniform(-1, 1, (h, k)).astype(np.float32)
            X64 = X.astype(np.float64)
            Xabs = np.abs(X64)
            bk = workload_bytes(mats, kinds, k)
            bkb = workload_bytes(mats, kinds, k, 2)
            variants = [("", 0, bk, A64), ("_bf16", CSP_FLAG_BF16, bkb, A64b)]
            if k == 32:
                variants += [("_tensor_cores", CSP_FLAG_TENSOR_CORES, bk, A64),
                             ("_bf16_tensor_cores", CSP_FLAG_BF16 | CSP_FLAG_TENSOR_CORES, bkb, A64b)]
            for suffix, fl, nbytes, Aref in variants:
                hk = Handle(mat, X, Y0, flags=fl, nrhs=k)
                hk.set_stream(dev.sp)
                t = dev.median(lambda: hk.do_spmv(1), reps)
                legs[f"k{k}{suffix}"] = {
                    "ms": t, "gb_s": gbs(nbytes, t), "frac": gbs(nbytes, t) / _peak()[0],
                    "gflop_s": 2.0 * nnz * k / (t * 1e-3) / 1e9,
                    "path": ("generic BCSR SpMM on tensor cores (mma.sync m16n8k8, TF32 high/low split)"
                             if fl & CSP_FLAG_TENSOR_CORES else "generic BCSR SpMM on CUDA cores")}
                hk.cpy_result_from_cpu(np.zeros_like(Y0))
                hk.do_spmv(1)
                Y = hk.cpy_result_to_cpu()
                hk.free()
                errors[f"k{k}{suffix}_max_rel_err"] = rel_err(Y, (Aref @ X64).ravel(), (abs(Aref) @ Xabs).ravel())
            pm = Cocktail.single("csr", coo, 0)
            pk = Handle(pm, X, Y0, nrhs=k)
            pk.set_stream(dev.sp)
            t = dev.median(lambda: pk.do_spmv(1), reps)
            legs[f"k{k}_plain_csr"] = {"ms": t, "gb_s": gbs(bk, t)}
            pk.free()
            pm.free()
    out["errors"] = errors

    # --- plain single-format CSR on the same GPU: warp per row and thread per row; the faster ---
    plain_ms, plain_key = None, None
    for m_ in (0, 4):
        pm = Cocktail.single("csr", coo, m_)
        ph = Handle(pm, x, y0, CSP_FLAG_GRAPH if l2_resident else 0)
        ph.set_stream(dev.sp)
        t = dev.median(lambda: ph.do_spmv(1), reps, 3, l2_resident)
        if plain_ms is None or t < plain_ms:
            plain_ms, plain_key = t, f"csr{m_}"
        ph.free()
        pm.free()
    out["plain"] = {"kernel": plain_key, "ms": plain_ms, "gb_s": gbs(ab, plain_ms)}
    out["legs"] = legs
    best.free()
    for k in keep:
        if hasattr(k, "free"):
            k.free()
    if with_cpu:
        out["cpu"] = cpu_baseline(mats, x, y0, ab, args.cpu_budget, gpu_y=y_dev, refs=refs)
    return out


def reference_tables_analysis_s(case):
    """Wall seconds of the reference-table partitioner (csp_analyze_matrix,
    CSP_ANALYZE_REFERENCE) on this library's B200 calibration tables, with its counting
    passes on the device (CSP_ANALYZE_ON_DEVICE): the one-time setup a caller of the
    reference's analyze_matrix pays."""
    from clspmv_b200 import COO, capi
    tables = os.path.join(ROOT, "clspmv_b200", "tables_b200")
    a = COO(*case)
    mat = capi.cocktail()
    opts = capi.csp_analyze_opts(capi.CSP_ANALYZE_REFERENCE, tables.encode(), 0, None, capi.CSP_ANALYZE_ON_DEVICE)
    t0 = time.perf_counter()
    rc = capi.lib().csp_analyze_matrix(a.ref(), C.byref(mat), C.byref(opts))
    dt = time.perf_counter() - t0
    capi.lib().csp_free_cocktail(C.byref(mat))
    return dt if rc == 0 else None


def summarize_leg(res, peak):
    """A config.legs entry from a run_single/run_batch result."""
    leg = {"workload": res["desc"], "nnz": res["nnz"], "partition": res["partition"], "ms": res["ms_step"],
           "gb_s": gbs(res["bytes"], res["ms_step"]), "frac": gbs(res["bytes"], res["ms_step"]) / peak,
           "algorithmic_bytes": res["bytes"], "setup_s": res["setup_s"],
           "reference_tables_analysis_s": res.get("analyzer_s"), "errors": res["errors"],
           "plain_csr": res["plain"], "speedup_vs_plain_csr": res["plain"]["ms"] / res["ms_step"]}
    if "l2" in res:
        leg["l2"] = res["l2"]
    leg.update({k: v for k, v in res["legs"].items()})
    if "cpu" in res:
        leg["cpu_baseline"] = res["cpu"]
    return leg


# ---------------------------------------------------------------------------
# the reference arm
# ---------------------------------------------------------------------------
def run_reference_arm(args, world, rank):
    """The reference's own CPU SpMV on the headline step, all host threads."""
    if rank != 0:
        return
    wl = args.workload
    desc, mats, x, y0, kinds = make_workload(wl, args.scale)
    nnz = int(sum(m[2].size for m in mats))
    adjoint = wl == "batch"
    fwd_b = workload_bytes(mats, kinds)
    nbytes = fwd_adjoint_bytes(fwd_b, nnz) if adjoint else fwd_b
    ybar = np.random.default_rng(3).uniform(-1, 1, sum(m[0] for m in mats)).astype(np.float32)
    cr = CpuReference(mats, x, y0, host_threads(), adjoint=adjoint, ybar=ybar)
    try:
        for _ in range(args.warmup):
            cr.step()
        ts = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            cr.step()
            ts.append(time.perf_counter() - t0)
    finally:
        cr.close()
    t_step = statistics.median(ts)
    v = nbytes / t_step / 1e9
    what = ("csr_spmv over every matrix and its explicit transpose + the value-gradient loop" if wl == "batch"
            else "csr_spmv forward")
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "GB/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_step * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": desc, "nnz": nnz, "algorithmic_bytes_per_step": nbytes,
                   "step": "forward + adjoint" if adjoint else "forward",
                   "path": f"clSpMV serial csr_spmv (spmv_serial.h:199): {what}"},
        "cpu_baseline": {"value": v, "unit": "GB/s", "cores": cr.threads, "host_cores": os.cpu_count(),
                         "kind": cr.kind,
                         "sample": f"{args.steps} whole steps of the workload on {cr.threads} host threads"},
        "e2e": {"value": v, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ---------------------------------------------------------------------------
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="batch", choices=WORKLOADS)
    ap.add_argument("--no-legs", action="store_true", help="headline configuration only")
    ap.add_argument("--cpu-budget", type=float, default=4.0, help="seconds of CPU-baseline sampling per config")
    ap.add_argument("--scale", type=float, default=1.0,
                    help="shrink the workloads (profiling runs only; the benchmark configuration is 1.0)")
    ap.add_argument("--tune-cache", default=None,
                    help="autotuner decision file: a pattern decided in an earlier run is rebuilt without "
                         "timing candidates (used to profile the bench's own partition)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference_arm(args, world, rank)
        return

    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    dev = Device(torch, local)
    peak, peak_kind = _peak()
    wl = args.workload
    with_cpu = rank == 0 and world == 1
    t_start = time.perf_counter()

    if wl == "batch":
        res = run_batch(dev, args, world, rank, with_cpu)
        head_legs = dict(res["legs"])
        ms_step = res["ms_step"]
        e2e = res["e2e"]
        clocks = res["clocks"]
    else:
        # a single configuration as the headline: its own timed region
        torch.cuda.synchronize()
        sampler = ClockSampler(local)
        sampler.start()
        res = run_single(dev, wl, args, with_cpu, args.steps, args.warmup)
        clocks = sampler.stop()
        head_legs = dict(res["legs"])
        ms_step = res["ms_step"]
        e2e = None
    job_bytes = world * res["bytes"]
    if world > 1 and wl == "batch":
        # each rank ran its own shard of the matrix list: the job's bytes are their sum
        import torch.distributed as dist
        tb = torch.tensor([res["bytes"]], dtype=torch.int64, device="cuda")
        dist.all_reduce(tb, op=dist.ReduceOp.SUM)
        job_bytes = int(tb.item())
    value = job_bytes / (ms_step * 1e-3) / 1e9
    kernel_gbs = res["bytes"] / (ms_step * 1e-3) / 1e9

    legs = {}
    if not args.no_legs and world == 1:
        for name in ("laplacian", "zipf", "stencil", "block"):
            if name == wl:
                continue
            r = run_single(dev, name, args, with_cpu, 20, 3)
            legs[LEG_NAMES[name]] = summarize_leg(r, peak)
            del r

    if e2e is None:
        e2e = {"value": None, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
               "note": "e2e is measured on the batch headline"}
    line = None
    if rank == 0:
        partition = res["partition"]
        config = {"workload": res["desc"], "nnz": res["nnz"], "algorithmic_bytes_per_step": res["bytes"],
                  "step": ("forward + value gradients + adjoint of every matrix in one persistent launch "
                           "(CUDA graph)" if wl == "batch" else "one forward SpMV"),
                  "partition": partition, "setup_s": res["setup_s"],
                  "plain_csr": res["plain"], "speedup_vs_plain_csr": res["plain"]["ms"] / ms_step,
                  "errors": res["errors"], "legs": {**head_legs, **legs},
                  "l2": res.get("l2", "256 MB write then 256 MB read of another buffer before each timed step; "
                                      "the working set (GBs) also exceeds the 126 MB L2"),
                  "parallelism": (f"matrix shards x{world}: a {512 * world}-matrix batch, 512 per rank, no "
                                  "collective on the data path" if wl == "batch" and world > 1 else
                                  f"replicas x{world}"),
                  "bench_wall_s": None}
        line = {
            "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config,
            "roofline": {"bound": "hbm", "achieved": kernel_gbs, "peak": peak, "unit": "GB/s",
                         "frac": kernel_gbs / peak, "peak_source": peak_kind,
                         "traffic": traffic_of(wl, partition),
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per launch "
                                           f"(profiles/traffic_{wl}.json)"},
            "cpu_baseline": res.get("cpu"),
            "e2e": e2e,
            "gpu_launches": args.steps * res["launches"],
            "clocks": clocks,
        }
        config["bench_wall_s"] = time.perf_counter() - t_start
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line))


if __name__ == "__main__":
    main()
