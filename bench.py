#!/usr/bin/env python
"""Benchmark of the engine's headline workload: slog_pfaffian of one large skew
matrix, 2n = 4096, float64, A = (G - G^T)/2 with G ~ N(0, 1/2n) from seed 1
(seed 1 + rank on rank > 0), in matrices/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

A step is one pfb_slog_pfaffian call on a batch of independent matrices (as
many as the GPU factors concurrently: 7 at 2n = 4096) through the C ABI; the
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
    p.add_argument("--batch", type=int, default=0, help="matrices per call (0: four waves of concurrently resident panel clusters)")
    p.add_argument("--panel", default="table", choices=["table", "registers", "half_shared"],
                   help="panel form of the headline calls (table: the tuned table's choice)")
    p.add_argument("--epilogue", default="table", choices=["table", "roundtrip", "reduce", "direct"],
                   help="split-update epilogue of the headline calls (table: the tuned table's choice)")
    p.add_argument("--workloads", default="all",
                   choices=["all", "headline", "small", "ragged", "grad", "illcond"],
                   help="'all': the headline line plus the other workloads under 'workloads'; "
                        "a single name runs only that workload (for profiling)")
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
        "config": {"workload": f"slog_pfaffian of independent 2n={n} float64 matrices, seed 1 (+rank)",
                   "n": n, "batch": threads},
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


# ----------------------------------------------------------------- other workloads
#
# Each returns a dict that goes under "workloads" in the JSON line.  Inputs are
# built on the host from the seeded generators, copied to the device once, and
# every timed region brackets device work only (CUDA events on the launching
# stream); where a workload's inputs fit in L2 (126 MB), L2 is flushed between
# timed iterations by writing a 256 MB buffer, outside the timed events.

def _ev_time(torch, stream, fn, k, warmup, flush=None):
    """Mean device ms of fn() over k calls after warmup calls."""
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    if flush is None:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / k
    tot = 0.0
    for _ in range(k):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        tot += e0.elapsed_time(e1)
    return tot / k


def measure_peaks(torch, dev, stream):
    """FP64 and INT8 tensor-core denominators measured here with library GEMMs
    (torch.matmul float64 and torch._int_mm), for the roofline of the FP64 and
    split updates; MEASURED_PEAKS.json carries only HBM and bf16."""
    out = {}
    n = 4096
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    ms = _ev_time(torch, stream, lambda: torch.matmul(a, a), 5, 2)
    out["fp64_gemm_tflops"] = 2 * n ** 3 / (ms * 1e-3) / 1e12
    try:
        m = 8192
        b = torch.randint(-64, 64, (m, m), dtype=torch.int8, device=dev)
        ms = _ev_time(torch, stream, lambda: torch._int_mm(b, b), 5, 2)
        out["int8_gemm_tops"] = 2 * m ** 3 / (ms * 1e-3) / 1e12
    except RuntimeError as e:
        out["int8_gemm_tops"] = None
        out["int8_note"] = str(e).splitlines()[0]
    out["how"] = "torch.matmul float64 4096^3 and torch._int_mm int8 8192^3, mean of 5 after 2 warm-up"
    return out


def reference_gpu_baseline(torch, pf, _lib, O, dev, stream):
    """The reference's own CUDA kernels on this GPU (src/*.cu compiled unchanged
    for sm_100a into oracle/_ref/libref_gpu.so, driven the way its XLA handlers
    drive them, bindings/jax_bindings.cu:19-112), beside this engine on the same
    inputs: pf_sm_calc launched once per matrix on the 4096 x 32x32 float64
    batch (jax_bindings.cu:107-109), and the host-driven slog_pfaffian_lg
    (src/slog_pfaffian_lg.cu:151-211) on one matrix of order 1024 and 2048.
    A reported baseline, like cpu_baseline: no engine number comes from it."""
    import ctypes
    if not os.path.exists(O.REF_GPU_SO):
        return {"unavailable": "oracle/_ref/libref_gpu.so was not built"}
    R = ctypes.CDLL(O.REF_GPU_SO)
    R.refgpu_pfaffian_f64.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_void_p,
                                      ctypes.c_void_p]
    R.refgpu_slog_f64.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_void_p,
                                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    out = {}
    # the small path: the reference takes column-major matrices (pfcuda/cuda_api.py:50)
    Ah = O.config_small()
    Acm = torch.from_numpy(np.ascontiguousarray(np.swapaxes(Ah, -1, -2))).to(dev)
    B, n = Acm.shape[0], Acm.shape[-1]
    o_ref = torch.empty(B, dtype=torch.float64, device=dev)
    o_eng = torch.empty(B, dtype=torch.float64, device=dev)
    L = _lib.lib()
    ms_ref = _ev_time(torch, stream, lambda: R.refgpu_pfaffian_f64(Acm.data_ptr(), B, n, o_ref.data_ptr(),
                                                                   stream.cuda_stream), 3, 1)
    ms_eng = _ev_time(torch, stream, lambda: L.pfb_pfaffian(_lib.F64, Acm.data_ptr(), B, n, _lib.COL_MAJOR,
                                                           o_eng.data_ptr(), stream.cuda_stream), 10, 3)
    torch.cuda.synchronize()
    rel = float(torch.max(torch.abs(o_ref - o_eng) / torch.abs(o_eng)))
    out["pfaffian_4096x32_f64"] = {"reference_ms": ms_ref, "engine_ms": ms_eng, "speedup": ms_ref / ms_eng,
                                   "max_rel_diff": rel,
                                   "how": "reference: pf_sm_calc once per matrix (4096 launches); "
                                          "engine: pfb_pfaffian, one launch; same column-major buffer"}
    for nn in (1024, 2048):
        Al = O.config_large(nn, seed=1)[0]
        X = torch.from_numpy(np.ascontiguousarray(Al.T)).to(dev)[None].contiguous()
        tmp = torch.empty(nn * nn, dtype=torch.float64, device=dev)
        l_ref = torch.empty(1, dtype=torch.float64, device=dev)
        p_ref = torch.empty(1, dtype=torch.float64, device=dev)
        ms_ref = _ev_time(torch, stream, lambda: R.refgpu_slog_f64(X.data_ptr(), 1, nn, l_ref.data_ptr(),
                                                                   p_ref.data_ptr(), tmp.data_ptr(),
                                                                   stream.cuda_stream), 2, 1)
        res = {"reference_ms": ms_ref}
        for mode in ("split", "fp64"):
            ws = torch.empty(pf.slog_workspace_bytes(X.dtype, 1, nn, mode), dtype=torch.uint8, device=dev)
            ms = _ev_time(torch, stream, lambda: pf.slog_pfaffian_raw(X, mode, layout=_lib.COL_MAJOR,
                                                                      workspace=ws), 5, 2)
            la, _ = pf.slog_pfaffian_raw(X, mode, layout=_lib.COL_MAJOR, workspace=ws)
            res[f"engine_{mode}_ms"] = ms
            res[f"speedup_{mode}"] = ms_ref / ms
            res[f"log_diff_{mode}"] = float(torch.abs(la - l_ref)[0])
        out[f"slog_pfaffian_{nn}_f64_batch1"] = res
    out["note"] = ("the reference's large path copies one pivot to the host per pivot pair "
                   "(src/slog_pfaffian_lg.cu:178), so its time is bound by those round trips")
    return out


def wl_small(torch, pf, _lib, O, dev, stream, steps, warmup, hbm_peak):
    """4096 independent 32x32 float64 matrices (seed 0): pfb_pfaffian, one launch."""
    L = _lib.lib()
    Ah = O.config_small()
    A = torch.from_numpy(Ah).to(dev)
    out = torch.empty(A.shape[0], dtype=torch.float64, device=dev)
    B, n = A.shape[0], A.shape[-1]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def fn():
        _lib.check(L.pfb_pfaffian(_lib.F64, A.data_ptr(), B, n, _lib.ROW_MAJOR, out.data_ptr(),
                                  stream.cuda_stream), "pfb_pfaffian")

    ms = _ev_time(torch, stream, fn, max(steps, 10), warmup, flush)
    fn()
    got = out.cpu().numpy()
    want = O.pf_product(Ah, as_shipped=False)
    rel = np.abs(got - want) / np.abs(want)
    tri = (n * (n - 1) // 2) * 8 + 8          # strict upper triangle in, one value out
    full = n * n * 8 + 8
    ach_tri = B * tri / (ms * 1e-3) / 1e9
    return {
        "workload": "pfaffian of 4096 independent 32x32 float64 matrices, A=(G-G^T)/2, G~N(0,1), seed 0",
        "matrices_per_s": B / (ms * 1e-3), "ms_per_call": ms, "launches_per_call": 1,
        "l2": "256 MB written between timed calls (inputs 33.5 MB < L2)",
        "accuracy": {"max_rel_err_vs_fp64_oracle": float(rel.max())},
        "roofline": {"kernel": "pf_small_kernel", "bound": "hbm", "achieved": ach_tri, "peak": hbm_peak,
                     "unit": "GB/s", "frac": ach_tri / hbm_peak,
                     "achieved_full_read": B * full / (ms * 1e-3) / 1e9,
                     "note": "algorithmic bytes = strict upper triangle + result (3976 B per matrix); "
                             "the kernel reads whole rows (8200 B), reported as achieved_full_read"},
    }


def wl_ragged(torch, pf, _lib, O, dev, stream, steps, warmup):
    """2000 float32 + 2000 float64 matrices of even orders in [8, 512] (seed 2):
    one persistent launch (captured in a CUDA graph) against a per-size loop of
    the plain path (one batched pfb_slog_pfaffian call per (order, dtype))."""
    cfg = O.config_ragged()
    mats_h = cfg["float32"] + cfg["float64"]
    mats = [torch.from_numpy(M).to(dev) for M in mats_h]
    plan = pf.RaggedPlan(mats)
    plan.run()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        plan.run()
    ms_graph = _ev_time(torch, stream, g.replay, max(3, steps // 4), warmup)
    ms_launch = _ev_time(torch, stream, plan.run, max(3, steps // 4), warmup)
    g.replay()
    torch.cuda.synchronize()
    la, sg = plan.log.cpu().numpy(), plan.sign.cpu().numpy()

    # per-size loop of the plain path: stacked groups, one call each
    groups = {}
    for i, M in enumerate(mats_h):
        groups.setdefault((M.shape[0], M.dtype.name), []).append(i)
    stacks = []
    for (n, _), idx in sorted(groups.items()):
        X = torch.stack([mats[i] for i in idx])
        l_ = torch.empty(len(idx), dtype=torch.float64, device=dev)
        s_ = torch.empty(len(idx), dtype=X.dtype, device=dev)
        wsb = pf.slog_workspace_bytes(X.dtype, len(idx), n, "fp64")
        w_ = torch.empty(max(wsb, 1), dtype=torch.uint8, device=dev)
        stacks.append((X, n, l_, s_, w_, wsb))
    L = _lib.lib()
    dmap = {torch.float32: _lib.F32, torch.float64: _lib.F64}

    def loop():
        for X, n, l_, s_, w_, wsb in stacks:
            _lib.check(L.pfb_slog_pfaffian(dmap[X.dtype], X.data_ptr(), X.shape[0], n, _lib.ROW_MAJOR,
                                           _lib.MODE_FP64, l_.data_ptr(), s_.data_ptr(), w_.data_ptr(),
                                           wsb, stream.cuda_stream), "pfb_slog_pfaffian")

    ms_loop = _ev_time(torch, stream, loop, max(3, steps // 4), warmup)
    # accuracy against the FP64 oracle on every matrix (the float32 ones widened exactly)
    wl = np.empty(len(mats_h))
    wsg = np.empty(len(mats_h))
    for (n, _), idx in groups.items():
        l_, s_ = O.slog_pf(np.stack([mats_h[i].astype(np.float64) for i in idx]))
        wl[idx], wsg[idx] = l_, s_
    err = np.abs(la - wl) / np.maximum(np.abs(wl), 1e-300)
    flops = sum(M.shape[0] ** 3 / 3.0 for M in mats_h)
    cnt = len(mats_h)
    return {
        "workload": "ragged batch: 2000 float32 + 2000 float64 skew matrices, even orders uniform in [8, 512], "
                    "entries N(0, 1/2n), seed 2",
        "matrices_per_s": cnt / (ms_graph * 1e-3), "ms_per_call_graph": ms_graph,
        "ms_per_call_direct": ms_launch, "launches_per_call": 2,
        "per_size_loop": {"ms": ms_loop, "matrices_per_s": cnt / (ms_loop * 1e-3), "calls": len(stacks),
                          "how": "one batched pfb_slog_pfaffian (FP64 mode) per (order, dtype) group"},
        "speedup_vs_per_size_loop": ms_loop / ms_graph,
        "fp64_gflops": flops / (ms_graph * 1e-3) / 1e9,
        "accuracy": {"max_log_rel_err": float(err.max()), "sign_equal": bool(np.array_equal(sg, wsg))},
    }


def wl_grad(torch, pf, _lib, O, dev, stream, steps, warmup):
    """256 complex128 matrices of order 512 (seed 3), loss = sum log|Pf|:
    forward + adjoint in one pfb_slog_pfaffian_grad call."""
    Ah = O.config_grad()
    A = torch.from_numpy(Ah).to(dev)
    B, n = A.shape[0], A.shape[-1]
    res = {"workload": "VJP of sum log|Pf| over 256 complex128 matrices of order 512, A=(G-G^T)/2, "
                       "Re/Im N(0, 1/2n), seed 3"}
    ct = torch.ones(B, dtype=torch.float64, device=dev)
    for mode in ("fp64", "split"):
        ws = torch.empty(pf.grad_workspace_bytes(A.dtype, B, n, mode), dtype=torch.uint8, device=dev)

        def fn():
            pf.slog_pfaffian_grad(A, ct, mode=mode, workspace=ws)

        ms = _ev_time(torch, stream, fn, max(3, steps // 2), warmup)
        wsf = torch.empty(pf.slog_workspace_bytes(A.dtype, B, n, mode), dtype=torch.uint8, device=dev)
        msf = _ev_time(torch, stream, lambda: pf.slog_pfaffian_raw(A, mode, workspace=wsf),
                       max(3, steps // 2), warmup)
        res[mode] = {"matrices_per_s": B / (ms * 1e-3), "ms_per_call": ms, "forward_only_ms": msf}
    G = pf.slog_pfaffian_grad(A[:8], mode="split").cpu().numpy()
    want = O.slog_pf_vjp(Ah[:8])
    rel = np.linalg.norm((G - want).reshape(8, -1), axis=1) / np.linalg.norm(want.reshape(8, -1), axis=1)
    rng = np.random.default_rng(33)
    E = O.skew_normal(rng, 2, n, complex_=True)
    d = np.sum(G[:2] * E, axis=(-1, -2)).real
    fd = O.fd_slog(Ah[:2], E, h=1e-6)
    jvp = O.slog_pf_jvp(Ah[:2], E).real
    ms_inv = _ev_time(torch, stream, lambda: torch.linalg.inv(A), 3, 2)
    res.update({
        "accuracy": {"max_rel_frobenius_err_vs_half_inv_T": float(rel.max()),
                     "max_rel_err_vs_central_difference_h1e-6": float(np.max(np.abs(d - fd) / np.abs(fd))),
                     "max_rel_err_vs_reference_jvp_rule": float(np.max(np.abs(d - jvp) / np.abs(jvp))),
                     "checked": "8 matrices vs (1/2) inv(A)^T; 2 directional derivatives vs FD and the JVP rule"},
        "torch_linalg_inv_ms": ms_inv,
        "note": "torch_linalg_inv_ms is the general inverse alone (the reference's rule calls jnp.linalg.inv)",
    })
    return res


def wl_illcond(torch, pf, _lib, O, dev, stream, steps, warmup):
    """64 float32 and 64 float64 matrices of order 2048, A = Q blockdiag(s_k J) Q^T,
    s_k log-spaced in [1e-6, 1] (seed 4): split-precision forward and VJP error
    against the exact log|Pf| and the FP64 oracle."""
    Ah, exact_log, exact_sign, Qh = O.config_illcond(return_q=True)
    B, n = Ah.shape[0], Ah.shape[-1]
    G_exact = O.illcond_half_inv_t(Qh[:2])       # (1/2) A^-T from the construction
    res = {"workload": "ill-conditioned: 64 float32 and 64 float64 matrices, 2n=2048, "
                       "A = Q blockdiag(s_k J) Q^T, Q Haar, s_k logspace(-6, 0), seed 4"}
    for name, npdt in (("float64", np.float64), ("float32", np.float32)):
        A = torch.from_numpy(Ah.astype(npdt)).to(dev)
        ws = torch.empty(pf.slog_workspace_bytes(A.dtype, B, n, "split"), dtype=torch.uint8, device=dev)
        ms = _ev_time(torch, stream, lambda: pf.slog_pfaffian_raw(A, "split", workspace=ws),
                      max(2, steps // 4), min(warmup, 2))
        la, sg = pf.slog_pfaffian_raw(A, "split", workspace=ws)
        la, sg = la.cpu().numpy(), sg.cpu().numpy()
        sub = 4
        wl, wsg = O.slog_pf(Ah[:sub].astype(npdt).astype(np.float64))
        r = {"matrices_per_s": B / (ms * 1e-3), "ms_per_call": ms,
             "max_log_rel_err_vs_exact": float(np.max(np.abs(la - exact_log) / np.abs(exact_log))),
             "sign_equal_exact": bool(np.array_equal(np.sign(sg), exact_sign)),
             "max_log_rel_err_vs_fp64_oracle": float(np.max(np.abs(la[:sub] - wl) / np.abs(wl))),
             "oracle_matrices": sub}
        G = pf.slog_pfaffian_grad(A[:2], mode="split").cpu().numpy().astype(np.float64)

        def frob(X, Y):
            return float(np.max(np.linalg.norm((X - Y).reshape(2, -1), axis=1) /
                                np.linalg.norm(Y.reshape(2, -1), axis=1)))

        if npdt == np.float64:
            # the exact adjoint of the construction; bar 4 cond sqrt(n) u with u
            # the unit of the split update (sqrt(K) 2^(-7S), K = 64, S = 7); the
            # FP64 path's adjoint, with u = eps, beside it
            r["vjp_max_rel_frobenius_err_vs_exact"] = frob(G, G_exact)
            r["vjp_bar"] = 4 * 1e6 * np.sqrt(n) * np.sqrt(64) * 2.0 ** -49
            G64 = pf.slog_pfaffian_grad(A[:2], mode="fp64").cpu().numpy()
            r["vjp_fp64_max_rel_frobenius_err_vs_exact"] = frob(G64, G_exact)
            r["vjp_fp64_bar"] = 4 * 1e6 * np.sqrt(n) * np.finfo(np.float64).eps
        else:
            # the float32 matrices are the float64 ones rounded (cond 1e6), so the
            # exact adjoint is out of reach; compared with NumPy's FP64 inverse of
            # the rounded matrices, and the output is rounded to float32 once
            r["vjp_max_rel_frobenius_err_vs_numpy_inverse"] = frob(
                G, O.slog_pf_vjp(Ah[:2].astype(npdt).astype(np.float64)))
        res[name] = r
        del A, ws
        torch.cuda.empty_cache()
    res["note"] = ("float32 inputs are rounded from the float64 matrices, so their exact-value error "
                   "includes that rounding (cond ~ 1e6); the oracle column uses the rounded matrix")
    return res


# ----------------------------------------------------------------- engine arm

def _hbm_peak():
    """Measured copy bandwidth of this GPU type (MEASURED_PEAKS.json), else the
    pool's earlier measurement."""
    try:
        return float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"])
    except (OSError, ValueError, KeyError):
        return 6650.0


def _hbm_peak_source():
    try:
        json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]
        return "MEASURED_PEAKS.json hbm_gbs (measured)"
    except (OSError, ValueError, KeyError):
        return "fallback 6650 GB/s (MEASURED_PEAKS.json absent)"


# DRAM read+write bytes over algorithmic bytes per launch for kernel variants
# captured with ncu after the first captures quoted at the roofline block
# below: the reduce-add split epilogue at k0 = 640 of 2n = 4096, batch 2
# (145.6 MB against 184.1 MB), the configuration the table picks for the
# headline
TRAFFIC_RATIO_MEASURED = {"split_update_kernel_reduce": 0.79}


def auto_batch(n, dtype="float64"):
    """The saturating batch: four waves of the widest panel clusters (one
    cluster per matrix; pfb_slog_max_concurrent of them resident at once), at
    most 4 GB of input.  Later panels use smaller clusters, so more of them fit
    at once and a one-wave batch leaves most SMs idle there: at 2n = 4096
    float64 (7 clusters of 16 per wave) split mode runs 453, 555, 597 and 608
    matrices/s at 7, 14, 21 and 28 matrices per call."""
    from pfcuda_b200 import _lib
    dt = _lib.F64 if dtype == "float64" else _lib.C128
    m = int(_lib.lib().pfb_slog_max_concurrent(dt, n))
    if m <= 0:
        return 8
    elem = 8 if dtype == "float64" else 16
    cap = max(1, int(4e9 // (n * n * elem)))
    return max(1, min(4 * m, cap))


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

    stream0 = torch.cuda.current_stream(dev)
    single = {"small": wl_small, "ragged": wl_ragged, "grad": wl_grad, "illcond": wl_illcond}
    if args.workloads in single:
        kw = dict(torch=torch, pf=pf, _lib=_lib, O=O, dev=dev, stream=stream0, steps=args.steps,
                  warmup=args.warmup)
        if args.workloads == "small":
            kw["hbm_peak"] = _hbm_peak()
        r = single[args.workloads](**kw)
        if rank == 0:
            print(json.dumps({"workloads": {args.workloads: r}}))
        if pg is not None:
            pg.destroy_process_group()
        return

    n = args.n
    B = args.batch if args.batch > 0 else auto_batch(n, args.dtype)
    npdt = np.float64 if args.dtype == "float64" else np.complex128
    A_host = O.config_large(n, dtype=npdt, seed=1 + rank, B=B)
    A = torch.from_numpy(A_host).to(dev)
    tdt = A.dtype
    L = _lib.lib()
    stream = torch.cuda.current_stream(dev)
    dtc = {torch.float64: _lib.F64, torch.complex128: _lib.C128}[tdt]
    mc = {"split": _lib.MODE_SPLIT, "fp64": _lib.MODE_FP64}

    def available(mode):
        # a zero matrix: the mode's support is checked before any work, and the
        # factorisation stops at its first pivot
        try:
            pf.slog_pfaffian_raw(torch.zeros(1, 66, 66, dtype=tdt, device=dev), mode=mode)
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

    # the configuration overrides given on the command line (0: the tuned table's choice)
    over = _lib.SlogConfig({"table": 0, "registers": 1, "half_shared": 2}[args.panel], 0, 0,
                           {"table": 0, "roundtrip": 1, "reduce": 2, "direct": 3}[args.epilogue])
    over_p = ctypes.byref(over) if (over.panel or over.epilogue) else None

    def step(mode, src=None, nb=B):
        X = src if src is not None else A
        st = L.pfb_slog_pfaffian_ex(dtc, X.data_ptr(), nb, n, _lib.ROW_MAJOR, mc[mode], la.data_ptr(),
                                    sg.data_ptr(), ws[mode].data_ptr(), ws[mode].numel(), stream.cuda_stream,
                                    None, over_p)
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
    tuned = {m: pf.slog_config(tdt, B, n, m) for m in modes}
    tuned1 = {m: pf.slog_config(tdt, 1, n, m) for m in modes}

    # each panel form at the headline batch, split and FP64 (a few calls each)
    forms = {}
    variants = [("registers", "roundtrip"), ("half_shared", "roundtrip"), ("registers", "reduce"),
                ("half_shared", "reduce"), ("registers", "direct"), ("half_shared", "direct")]
    for m in modes:
        for form, epi in variants:
            if L.pfb_slog_max_concurrent_form(dtc, n, {"registers": 1, "half_shared": 2}[form]) <= 0:
                continue
            if m != "split" and epi != "roundtrip":
                continue
            if epi == "direct" and tdt != torch.float64:
                continue
            cfgx = {"panel": form, "epilogue": epi}

            def stepx(m=m, cfgx=cfgx):
                pf.slog_pfaffian_raw(A, mode=m, workspace=ws[m], config=cfgx)

            for _ in range(2):
                stepx()
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            kk = max(3, args.steps // 4)
            for _ in range(kk):
                stepx()
            e1.record(stream)
            barrier()
            forms[f"{m}_{form}" + (f"_{epi}" if m == "split" else "") + "_ms"] = \
                max_over_ranks(e0.elapsed_time(e1) / kk)

    # accuracy of the headline path against the FP64 oracle (rank 0)
    step(head)
    torch.cuda.synchronize()
    acc = None
    if rank == 0:
        wl, ws_ = O.slog_pf(A_host)
        got_l, got_s = la.cpu().numpy(), sg.cpu().numpy()
        acc = {"max_log_rel_err": float(np.max(np.abs(got_l - wl) / np.abs(wl))),
               "max_log_abs_err": float(np.max(np.abs(got_l - wl))), "matrices": int(B)}
        if np.iscomplexobj(got_s):
            # the sign of a complex matrix is a phase: its error is reported, not "equal"
            acc["max_phase_err"] = float(np.max(np.abs(got_s - ws_)))
        else:
            acc["sign_equal"] = bool(np.array_equal(got_s, ws_))

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
    st = L.pfb_slog_pfaffian_ex(dtc, A.data_ptr(), B, n, _lib.ROW_MAJOR, mc[head], la.data_ptr(),
                                sg.data_ptr(), ws[head].data_ptr(), ws[head].numel(),
                                stream.cuda_stream, ctypes.byref(tm), over_p)
    _lib.check(st, "pfb_slog_pfaffian_ex (timed)")
    torch.cuda.synchronize()
    panel_ms = sum(evs[0][2 * i].elapsed_time(evs[0][2 * i + 1]) for i in range(npan))
    upd_ms = sum(evs[1][2 * i].elapsed_time(evs[1][2 * i + 1]) for i in range(npan - 1))

    # end to end through the Python API: pinned host input -> device -> slog ->
    # (log, sign) to host, every step.  Pipelined as a user streaming batches
    # would run it: two device input buffers, the copy of step i+1 on a copy
    # stream overlapping the factorisation of step i on the compute stream.
    h_in = torch.from_numpy(A_host).pin_memory()
    d_in = [torch.empty_like(A), torch.empty_like(A)]
    h_log = [torch.empty(B, dtype=torch.float64).pin_memory() for _ in range(2)]
    h_sign = [torch.empty(B, dtype=tdt).pin_memory() for _ in range(2)]
    wsh = ws[head]
    cstream = torch.cuda.Stream(dev)
    copied = [torch.cuda.Event() for _ in range(2)]
    done = [torch.cuda.Event() for _ in range(2)]

    def e2e_run(k):
        for i in range(k):
            bb = i & 1
            with torch.cuda.stream(cstream):
                if i >= 2:
                    cstream.wait_event(done[bb])          # buffer bb is free once step i-2 is factored
                pf.upload_upper(h_in, out=d_in[bb])   # the triangle the engine reads
                copied[bb].record(cstream)
            stream.wait_event(copied[bb])
            l2, s2 = pf.slog_pfaffian_raw(d_in[bb], mode=head, workspace=wsh)
            h_log[bb].copy_(l2, non_blocking=True)
            h_sign[bb].copy_(s2, non_blocking=True)
            done[bb].record(stream)

    e2e_run(args.warmup)
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    cstream.wait_event(e0)                               # no copy starts before the timed region
    e2e_run(args.steps)
    e1.record(stream)
    barrier()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / args.steps)
    # the triangle upload leaves the rest of the device buffer stale; the
    # results must equal those of the whole matrix on the device, bit for bit
    l_ref, s_ref = pf.slog_pfaffian_raw(A, mode=head, workspace=wsh)
    torch.cuda.synchronize()
    last = (args.steps - 1) & 1
    e2e_same = bool(torch.equal(h_log[last], l_ref.cpu()) and torch.equal(h_sign[last], s_ref.cpu()))

    if rank != 0:
        if pg is not None:
            pg.destroy_process_group()
        return

    ms = results[head]
    value = world * B / (ms * 1e-3)
    # kernel launches per call: the library may run a batch as two ranges on two
    # streams, each with its own sequence of launches
    ranges = int(L.pfb_slog_stream_ranges(dtc, B, n, mc[head]))
    esz = A.element_size()
    hbm_peak = _hbm_peak()
    # trailing update, the kernel that carries the O(n^3) arithmetic: each of
    # its launches reads and writes the upper triangle of the trailing block in
    # FP64 once (algorithmic bytes 2 * m^2/2 * element size per matrix)
    upd_bytes = sum(2 * (m * m / 2.0) * esz for m in (n - nb * (i + 1) for i in range(npan - 1)) if m > 0) * B
    # panel: the panel rows are read and written once per panel
    panel_bytes = 2.0 * (n * n / 2.0) * esz * B
    dominant = "panel" if panel_ms >= upd_ms else "update"
    # DRAM read+write bytes over algorithmic bytes for one launch of each kernel,
    # from ncu captures (--set full) of 2n = 4096 float64, batch 2: panel_kernel
    # at k0 = 128 (19.44 MB against 8.13 MB: the interchanged row is read down a
    # column, a 32-byte sector per element), split_update_kernel and
    # gemm_dmma_kernel at k0 = 320 (177 / 175 MB against 228 MB: part of the
    # written tiles is still in L2 when the launch ends)
    traffic_ratio = {"panel_kernel": 2.39, "split_update_kernel": 0.78, "gemm_dmma_kernel": 0.77}
    traffic_ratio.update(TRAFFIC_RATIO_MEASURED)
    # the configuration the headline call ran: the command line's override, else the table's
    eff = dict(tuned[head])
    if args.panel != "table":
        eff["panel"] = args.panel
    if args.epilogue != "table":
        eff["epilogue"] = args.epilogue
    pk_name = "panel_hs_kernel" if eff["panel"] == "half_shared" else "panel_kernel"
    if dominant == "panel":
        achieved = panel_bytes / (panel_ms * 1e-3) / 1e9
        tr = traffic_ratio.get(pk_name)
        roof = {"kernel": pk_name, "bound": "hbm", "achieved": achieved, "peak": hbm_peak,
                "unit": "GB/s", "frac": achieved / hbm_peak,
                "traffic": tr * panel_bytes / npan if tr else None,
                "note": "latency-bound: 32 dependent pivot steps per launch, each a cluster barrier and a "
                        "global load of the interchanged row (8-11k cycles per step); algorithmic bytes = "
                        "panel rows read and written once; traffic per launch scaled from ncu"}
    else:
        kname = "split_update_kernel" if head == "split" else "gemm_dmma_kernel"
        tkey = kname + (f"_{eff.get('epilogue')}" if head == "split" and eff.get("epilogue") != "roundtrip"
                        else "")
        achieved = upd_bytes / (upd_ms * 1e-3) / 1e9
        tr = traffic_ratio.get(tkey)
        roof = {"kernel": kname, "variant": tkey, "bound": "hbm",
                "achieved": achieved, "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
                "traffic": tr * upd_bytes / max(npan - 1, 1) if tr else None,
                "note": "algorithmic bytes = FP64 read+write of the upper trailing block per launch; the "
                        "timed region includes the operand-slicing launch before each update; traffic per "
                        "launch scaled from ncu"}
    roof["peak_source"] = _hbm_peak_source()
    line = {
        "metric": METRIC, "value": value, "unit": "matrices/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if tdt == torch.float64 else "c128",
        "data": "synthetic",
        "config": {"workload": f"slog_pfaffian of independent 2n={n} {args.dtype} matrices, seed 1 (+rank)",
                   "n": n, "batch": B, "mode": head, "panel_width": nb,
                   "l2": f"inputs {B * n * n * esz / 1e6:.0f} MB > 126 MB L2, re-read every step",
                   "parallelism": f"replicas x{world}"},
        "tuned_config": tuned,
        "config_override": {"panel": args.panel, "epilogue": args.epilogue},
        "tuned_config_batch1": tuned1,
        "panel_forms_ms_per_step": forms,
        "modes_ms_per_step": results,
        "split_over_fp64": (results["fp64"] / results["split"]) if len(results) == 2 else None,
        "batch1_ms": results1,
        "batch1_matrices_per_s": {m: 1e3 / v for m, v in results1.items()},
        "batch1_split_over_fp64": (results1["fp64"] / results1["split"]) if len(results1) == 2 else None,
        "accuracy": acc,
        "kernel_ms": {"panel": panel_ms, "update": upd_ms, "panels": npan},
        "roofline": roof,
        "e2e": {"value": world * B / (e2e_ms * 1e-3), "unit": "matrices/s",
                "h2d_bytes_per_step": pf.upload_upper_bytes(tdt, B, n), "d2h_bytes_per_step": B * (8 + esz),
                "how": "per step: upload_upper of the pinned-host batch (the upper triangle of each "
                       "matrix, the part the engine reads, in 256-row rectangles) on a copy stream, then "
                       "slog_pfaffian_raw and the results back to pinned host memory; two device buffers "
                       "so the upload of step i+1 overlaps the factorisation of step i",
                "results_equal_device_path": e2e_same},
        "gpu_launches": args.steps * ranges * (2 + npan + (npan - 1) * (2 if head == "split" else 1)),
        "clocks": clocks,
    }
    if world == 1:
        line["cpu_baseline"] = cpu_baseline(n)
    if world == 1 and args.workloads == "all":
        # the other configurations, on the same GPU after the headline
        del A, ws, d_in
        torch.cuda.empty_cache()
        kw = dict(torch=torch, pf=pf, _lib=_lib, O=O, dev=dev, stream=stream, steps=args.steps,
                  warmup=args.warmup)
        line["peaks_measured_here"] = measure_peaks(torch, dev, stream)
        t0 = time.perf_counter()
        line["reference_gpu_baseline"] = reference_gpu_baseline(torch, pf, _lib, O, dev, stream)
        line["reference_gpu_baseline"]["wall_s"] = time.perf_counter() - t0
        wls = {}
        for name, fn in (("small", wl_small), ("ragged", wl_ragged), ("grad", wl_grad),
                         ("illcond", wl_illcond)):
            t0 = time.perf_counter()
            extra = {"hbm_peak": hbm_peak} if name == "small" else {}
            wls[name] = fn(**kw, **extra)
            wls[name]["wall_s"] = time.perf_counter() - t0
            torch.cuda.empty_cache()
        line["workloads"] = wls
    print(json.dumps(line))
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
