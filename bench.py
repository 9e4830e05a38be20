#!/usr/bin/env python
"""Benchmark of the engine's headline workload: slog_pfaffian of one large skew
matrix, 2n = 4096, float64, A = (G - G^T)/2 with G ~ N(0, 1/2n) from seed 1
(seed 1 + rank on rank > 0), in matrices/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

A step is one pfb_slog_pfaffian call on a batch of independent matrices (as
many as the GPU factors concurrently: 8 at 2n = 4096) through the C ABI; the
batch-1 latency of each path is reported beside it.  `value` is the
split-precision path (int8 slices on the tcgen05 tensor cores, FP64 panel) when
it is available, else the FP64 path; the other path is timed in the same run
and reported beside it.  Multi-GPU runs are replicas (each rank factors its own
matrix, no collective): value = matrices of all ranks / max-over-ranks time.

--impl reference times the reference's own CPU implementation of the path,
src/pfaffian_cpu.cpp compiled unchanged (oracle/_ref/libref_cpu.so), with one
matrix per host thread per step, on rank 0 only.
"""
from __future__ import annotations

import argparse
import ctypes
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

METRIC = "matrices/s, split-precision vs FP64 slog_pfaffian on one B200 at <=1e-10 log err"
N_DEFAULT = 4096


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="engine", choices=["engine", "reference"])
    p.add_argument("--n", type=int, default=N_DEFAULT)
    p.add_argument("--dtype", default="float64", choices=["float64", "complex128"])
    p.add_argument("--mode", default="auto", choices=["auto", "split", "fp64"])
    p.add_argument("--batch", type=int, default=0, help="matrices per call (0: as many as run concurrently)")
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


# ----------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi clock / throttle samples while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            t0 = time.time()
            while not self.lines and time.time() - t0 < 10:   # sampling has begun
                time.sleep(0.01)
            self.lines.clear()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------- reference arm

def run_reference(args, rank, world):
    if rank != 0:
        return
    from oracle import oracle as O
    R = O.ref_cpu()
    if R is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libref_cpu.so was not built"}))
        return
    threads = min(os.cpu_count() or 1, 32)
    n = args.n
    A = O.config_large(n, seed=1)[0]
    batch = np.ascontiguousarray(np.broadcast_to(A, (threads, n, n)))
    out = np.empty(threads)

    def step():
        R.refcpu_pfaffian_batch(O._p(batch), threads, n, O._p(out), threads)

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = time.perf_counter() - t0
    value = threads * args.steps / dt
    sample = f"{threads} matrices of order {n} (one per host thread) per step"
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "matrices/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"slog_pfaffian 2n={n} float64, seed 1", "n": n, "batch": 1},
        "cpu_baseline": {"value": value, "unit": "matrices/s", "cores": threads, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": "matrices/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def cpu_baseline(n):
    """The reference's pfaffian_cpu on the host cores, a bounded sample."""
    from oracle import oracle as O
    R = O.ref_cpu()
    if R is None:
        return None
    threads = min(os.cpu_count() or 1, 32)
    A = O.config_large(n, seed=1)[0]
    batch = np.ascontiguousarray(np.broadcast_to(A, (threads, n, n)))
    out = np.empty(threads)
    t0 = time.perf_counter()
    R.refcpu_pfaffian_batch(O._p(batch), threads, n, O._p(out), threads)
    dt = time.perf_counter() - t0
    return {"value": threads / dt, "unit": "matrices/s", "cores": threads, "kind": "reference",
            "sample": f"{threads} matrices of order {n}, one per thread, src/pfaffian_cpu.cpp as shipped "
                      f"({dt:.1f} s)"}


# ----------------------------------------------------------------- engine arm

def auto_batch(n):
    """Matrices factored concurrently per call: as many panel clusters as the
    GPU runs at once (a cluster of ceil((n-64)/256) CTAs per matrix, at most one
    16-CTA cluster per GPC)."""
    cl = max(1, -(-(n - 64) // 256))
    return max(1, min(16, 128 // max(cl, 8) if cl >= 8 else 16))


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch
    import pfcuda_b200 as pf
    from pfcuda_b200 import _lib
    from oracle import oracle as O

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
        pg = dist

    n = args.n
    B = args.batch if args.batch > 0 else auto_batch(n)
    npdt = np.float64 if args.dtype == "float64" else np.complex128
    A_host = O.config_large(n, dtype=npdt, seed=1 + rank, B=B)
    A = torch.from_numpy(A_host).to(dev)
    tdt = A.dtype
    L = _lib.lib()
    stream = torch.cuda.current_stream(dev)
    dtc = {torch.float64: _lib.F64, torch.complex128: _lib.C128}[tdt]
    mc = {"split": _lib.MODE_SPLIT, "fp64": _lib.MODE_FP64}

    def available(mode):
        try:
            pf.slog_pfaffian_raw(A[:1], mode=mode)
            torch.cuda.synchronize()
            return True
        except _lib.PfbError as e:
            if e.status == 5:
                return False
            raise

    modes = ["split", "fp64"] if args.mode == "auto" else [args.mode]
    modes = [m for m in modes if available(m)]
    head = modes[0]
    ws = {m: torch.empty(pf.slog_workspace_bytes(tdt, B, n, m), dtype=torch.uint8, device=dev) for m in modes}
    la = torch.empty(B, dtype=torch.float64, device=dev)
    sg = torch.empty(B, dtype=tdt, device=dev)

    def step(mode, src=None, nb=B):
        X = src if src is not None else A
        st = L.pfb_slog_pfaffian(dtc, X.data_ptr(), nb, n, _lib.ROW_MAJOR, mc[mode], la.data_ptr(),
                                 sg.data_ptr(), ws[mode].data_ptr(), ws[mode].numel(), stream.cuda_stream)
        _lib.check(st, "pfb_slog_pfaffian")

    def barrier():
        if pg is not None:
            pg.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if pg is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        return t.item()

    def timed(mode, nb, k, clocks=None):
        for _ in range(args.warmup):
            step(mode, nb=nb)
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if clocks:
            clocks.start()
        e0.record(stream)
        for _ in range(k):
            step(mode, nb=nb)
        e1.record(stream)
        barrier()
        ck = clocks.stop() if clocks else None
        return max_over_ranks(e0.elapsed_time(e1) / k), ck

    results, results1 = {}, {}
    clocks = None
    for m in modes:
        cs = ClockSampler(local) if m == head else None
        ms, ck = timed(m, B, args.steps, cs)
        results[m] = ms
        if ck is not None:
            clocks = ck
        results1[m], _ = timed(m, 1, max(3, args.steps // 2))

    # accuracy of the headline path against the FP64 oracle (rank 0)
    step(head)
    torch.cuda.synchronize()
    acc = None
    if rank == 0:
        wl, ws_ = O.slog_pf(A_host)
        got_l, got_s = la.cpu().numpy(), sg.cpu().numpy()
        acc = {"max_log_rel_err": float(np.max(np.abs(got_l - wl) / np.abs(wl))),
               "max_log_abs_err": float(np.max(np.abs(got_l - wl))),
               "sign_equal": bool(np.all(np.abs(got_s - ws_) < 1e-10)), "matrices": int(B)}

    # per-kernel times of the headline path (a separate, instrumented call)
    nb = L.pfb_slog_panel_width(dtc, n)
    npan = (n - 1 + nb - 1) // nb
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(2 * npan)] for _ in range(2)]
    for e in evs[0] + evs[1]:
        e.record(stream)          # creates the CUDA events (torch creates them lazily)
    torch.cuda.synchronize()
    arr = [(ctypes.c_void_p * (2 * npan))(*[e.cuda_event for e in es]) for es in evs]
    tm = _lib.SlogTiming(ctypes.cast(arr[0], ctypes.POINTER(ctypes.c_void_p)),
                         ctypes.cast(arr[1], ctypes.POINTER(ctypes.c_void_p)), npan)
    st = L.pfb_slog_pfaffian_timed(dtc, A.data_ptr(), B, n, _lib.ROW_MAJOR, mc[head], la.data_ptr(),
                                   sg.data_ptr(), ws[head].data_ptr(), ws[head].numel(),
                                   stream.cuda_stream, ctypes.byref(tm))
    _lib.check(st, "pfb_slog_pfaffian_timed")
    torch.cuda.synchronize()
    panel_ms = sum(evs[0][2 * i].elapsed_time(evs[0][2 * i + 1]) for i in range(npan))
    upd_ms = sum(evs[1][2 * i].elapsed_time(evs[1][2 * i + 1]) for i in range(npan - 1))

    # end to end through the Python API: pinned host input -> device -> slog -> (log, sign) to host
    h_in = torch.from_numpy(A_host).pin_memory()
    d_in = torch.empty_like(A)
    h_log = torch.empty(B, dtype=torch.float64).pin_memory()
    h_sign = torch.empty(B, dtype=tdt).pin_memory()
    wsh = ws[head]

    def e2e_step():
        d_in.copy_(h_in, non_blocking=True)
        l2, s2 = pf.slog_pfaffian_raw(d_in, mode=head, workspace=wsh)
        h_log.copy_(l2, non_blocking=True)
        h_sign.copy_(s2, non_blocking=True)

    for _ in range(args.warmup):
        e2e_step()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        e2e_step()
    e1.record(stream)
    barrier()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / args.steps)

    if rank != 0:
        if pg is not None:
            pg.destroy_process_group()
        return

    ms = results[head]
    value = world * B / (ms * 1e-3)
    esz = A.element_size()
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    # trailing update, the kernel that carries the O(n^3) arithmetic: each of
    # its launches reads and writes the upper triangle of the trailing block in
    # FP64 once (algorithmic bytes 2 * m^2/2 * element size per matrix)
    upd_bytes = sum(2 * (m * m / 2.0) * esz for m in (n - nb * (i + 1) for i in range(npan - 1)) if m > 0) * B
    # panel: the panel rows are read and written once per panel
    panel_bytes = 2.0 * (n * n / 2.0) * esz * B
    dominant = "panel" if panel_ms >= upd_ms else "update"
    if dominant == "panel":
        achieved = panel_bytes / (panel_ms * 1e-3) / 1e9
        roof = {"kernel": "panel_kernel", "bound": "hbm", "achieved": achieved, "peak": hbm_peak,
                "unit": "GB/s", "frac": achieved / hbm_peak, "traffic": None,
                "note": "latency-bound (one cluster barrier and one global round trip per pivot pair); "
                        "algorithmic bytes = panel rows read and written once"}
    else:
        achieved = upd_bytes / (upd_ms * 1e-3) / 1e9
        roof = {"kernel": "split_update_kernel" if head == "split" else "gemm_fp64_kernel", "bound": "hbm",
                "achieved": achieved, "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
                "traffic": None, "note": "algorithmic bytes = FP64 read+write of the upper trailing block per launch"}
    line = {
        "metric": METRIC, "value": value, "unit": "matrices/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if tdt == torch.float64 else "c128",
        "data": "synthetic",
        "config": {"workload": f"slog_pfaffian of independent 2n={n} {args.dtype} matrices, seed 1 (+rank), "
                               f"{B} per call", "n": n, "batch": B, "mode": head, "panel_width": nb,
                   "l2": f"inputs {B * n * n * esz / 1e6:.0f} MB > 126 MB L2, re-read every step",
                   "parallelism": f"replicas x{world}"},
        "modes_ms_per_step": results,
        "split_over_fp64": (results["fp64"] / results["split"]) if len(results) == 2 else None,
        "batch1_ms": results1,
        "batch1_matrices_per_s": {m: 1e3 / v for m, v in results1.items()},
        "batch1_split_over_fp64": (results1["fp64"] / results1["split"]) if len(results1) == 2 else None,
        "accuracy": acc,
        "kernel_ms": {"panel": panel_ms, "update": upd_ms, "panels": npan},
        "roofline": roof,
        "e2e": {"value": world * B / (e2e_ms * 1e-3), "unit": "matrices/s",
                "h2d_bytes_per_step": B * n * n * esz, "d2h_bytes_per_step": B * (8 + esz)},
        "gpu_launches": args.steps * (2 + npan + (npan - 1)),
        "clocks": clocks,
    }
    if world == 1:
        line["cpu_baseline"] = cpu_baseline(n)
    print(json.dumps(line))
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
