"""Test infrastructure: the reference's own GPU direct sum against this project's
on the same B200 and the same inputs.

    python oracle/ref_gpu_timing.py [--n 1000000] [--m 1000000] [--block 128]

Workload: the headline configuration's evaluation pass with a fixed bandwidth
(the reference's CudaDirectKde direct sum takes per-point masses and bandwidth
factors; unit factors here): 2-D Gaussian product kernel, h = (0.05, 0.05),
1,000,000 bimodal references with weights U[0.5, 1.5] (normalised), 1,000,000
uniform queries on [-3, 3]^2 -- 1e12 pair evaluations per call.

* reference: CudaDirectKde<2, float, GaussianProductKernel2d<float>>::
  unnormalized_eval (include/CudaDirectKde.h:176-215) built unmodified for sm_100a
  (oracle/_ref/libkde_ref_gpu.so). Each call uploads the kernel object, launches
  eval_kernel (one query per thread, `block` threads) and downloads the results,
  synchronously; CUDA events around the calls.
* ours: bbkde_eval_range_device (FP32-compensated pair sum) on device-resident
  inputs, CUDA events on the library's stream, and the per-launch kernel time.

Both are checked against the FP64 oracle on 1,024 queries. Prints one JSON line.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)
REF_GPU_SO = os.path.join(HERE, "_ref", "libkde_ref_gpu.so")


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=1_000_000)
    ap.add_argument("--m", type=int, default=1_000_000)
    ap.add_argument("--block", type=int, default=128)
    ap.add_argument("--reps", type=int, default=3)
    a = ap.parse_args()

    import torch
    import bbrcit_kde_b200 as bk
    from bbrcit_kde_b200 import workloads as W
    from bbrcit_kde_b200.parity import error_stats
    from oracle.pyoracle import Oracle

    if not os.path.exists(REF_GPU_SO):
        print(json.dumps({"unavailable": f"{REF_GPU_SO} not built"}))
        return 0
    wl = W.config2(n=a.n, m=a.m)
    wn = wl.weights / wl.weights.sum()
    n, m = len(wl.refs), len(wl.queries)
    h = (0.05, 0.05)
    dp = C.POINTER(C.c_double)
    lib = C.CDLL(REF_GPU_SO)
    lib.ref_gpu_direct.argtypes = [C.c_int, C.c_double, C.c_double, C.c_int64, dp, dp, dp,
                                   C.c_int64, dp, C.c_int, C.c_int, dp, dp]
    p = lambda x: np.ascontiguousarray(x, dtype=np.float64).ctypes.data_as(dp)  # noqa: E731
    refs = np.ascontiguousarray(wl.refs)
    qs = np.ascontiguousarray(wl.queries)
    ref_out = np.empty(m)
    ref_ms = C.c_double(0.0)
    torch.cuda.init()
    from bench import ClockSampler
    sampler = ClockSampler(0)
    sampler.start()
    rc = lib.ref_gpu_direct(W.GAUSS_PROD2D, h[0], h[1], n, p(refs), p(wn), None, m, p(qs),
                            a.block, a.reps, ref_out.ctypes.data_as(dp), C.byref(ref_ms))
    if rc != 0:
        print(json.dumps({"error": f"ref_gpu_direct returned {rc}"}))
        return 1

    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx = bk.Context(0)
    ctx.set_stream(stream.cuda_stream)
    desc = bk.kernel_desc(W.GAUSS_PROD2D, 2, h)
    ctx.upload(bk.REFERENCE, refs, mass=wn, weight=wn)
    ctx.upload(bk.QUERY, qs)
    out = torch.empty(m, dtype=torch.float64, device="cuda")
    kernel_ms, call_ms = [], []
    for i in range(3 + a.reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ctx.eval_range_device(desc, 0, n - 1, 0, m - 1, out.data_ptr())
        e1.record(stream)
        torch.cuda.synchronize()
        if i >= 3:
            call_ms.append(e0.elapsed_time(e1))
            kernel_ms.append(ctx.last_launch_stats()[0])
    ours = out.cpu().numpy()
    clocks = sampler.stop()
    ctx.close()

    sel = np.linspace(0, m - 1, 1024).astype(np.int64)
    want = Oracle().direct(W.GAUSS_PROD2D, 2, h, refs, wn, qs[sel])
    smi = subprocess.run(["nvidia-smi", "--query-gpu=name,clocks.sm,clocks.max.sm",
                          "--format=csv,noheader"], capture_output=True, text=True).stdout.strip()
    pairs = float(n) * m
    line = {
        "workload": f"2-D Gaussian product, h=(0.05,0.05), {n} refs x {m} queries, fixed "
                    f"bandwidth (1e12 pairs per call)",
        "reference_eval_kernel": {
            "ms_per_call": ref_ms.value, "evals_per_s": pairs / (ref_ms.value / 1e3),
            "block": a.block, "reps": a.reps,
            "timed": "CudaDirectKde::unnormalized_eval calls (kernel-object upload, "
                     "eval_kernel, results download), CUDA events",
            "error_vs_fp64": error_stats(ref_out[sel], want)},
        "ours_pair_sum": {
            "kernel_ms": float(np.mean(kernel_ms)), "call_ms": float(np.mean(call_ms)),
            "evals_per_s": pairs / (float(np.mean(call_ms)) / 1e3),
            "timed": "bbkde_eval_range_device calls (pair sum + FP64 combine), CUDA events",
            "error_vs_fp64": error_stats(ours[sel], want)},
        "speedup_call": ref_ms.value / float(np.mean(call_ms)),
        "gpu": smi,
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
