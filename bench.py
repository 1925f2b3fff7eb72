"""Benchmark of the direct kernel-density path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one "step"): the adaptive 2-D product-Gaussian KDE of the reference's
headline configuration -- 1,000,000 reference points from the seeded bimodal
mixture, weights U[0.5, 1.5], pilot bandwidth (0.05, 0.05), alpha = 0.5, then the
adapted density at 1,000,000 uniform queries over [-3, 3]^2:
  pilot pass  (KernelDensity::adapt_density)   N x N pair evaluations
  evaluation  (KernelDensity::direct_eval)     M x N pair evaluations
The unit of work is one pair evaluation ("kernel eval"). Synthetic, seeded data.

Lines printed by rank 0 (one JSON object):
  value    evals/s with inputs resident in HBM (device-timed, CUDA events on the
           library's stream, L2 flushed between timed steps, max over ranks).
  e2e      the same through the C ABI with pinned HOST buffers: every step uploads
           the points, runs pilot + evaluation and reads the densities back.
  roofline the pair-sum kernel against the MUFU (ex2) bound: SMs x 16 ex2/clk x clock.
  cpu_baseline  the reference's own CPU code (oracle/_ref, compiled from its
           headers) timed on this host's cores on a bounded query sample.

Multi-GPU: one process per GPU (torchrun); queries are independent, so each rank
evaluates its own query batch against the full reference set with no collective
in the data path ("scaling": "weak"); timings are reduced with MAX over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = ("2D KDE queries/s (kernel evals/s vs FP32 roofline), direct vs surrogate at "
          "stated rel err")
UNIT = "kernel evals/s"
MUFU_EX2_PER_CLK_PER_SM = 16
FP32_FMA_PER_CLK_PER_SM = 128
# FP32-pipe poly stride of each pair-sum launch shape (bbkde_launch_variants order):
# every k-th reference's exponentials on the FP32 pipe, 0 = all on MUFU.
VARIANT_POLY = [0, 0, 0, 0, 8, 8, 4, 8, 16, 32, 16]


def pair_sum_bound_per_clk_per_sm(poly: int, fma_cycles: float = 12.0) -> tuple[float, str]:
    """Pairs per clock per SM the packed Gaussian pair sum can reach. Per warp and
    per 64 pairs (two queries per packed instruction) the main path issues
    fma_cycles / 2 packed FP32 instructions (2 FMA-pipe cycles each: 12 cycles for
    the 2-D isotropic kernel, 8 in 1-D) and 2 MUFU.EX2 (8 cycles each on a
    4-lane-per-clock unit: 16 cycles); the polynomial exp2 costs 8 packed
    instructions (16 cycles) instead of the 2 MUFU operations. 4 SMSPs per SM."""
    mufu = 4 * 64 / (16.0 * (1 - 1 / poly)) if poly else 4 * 64 / 16.0
    fma = 4 * 64 / (fma_cycles + (16.0 / poly if poly else 0.0))
    bound = "sfu" if mufu <= fma else "fma"
    if poly:
        bound = "sfu+fma (exp2 split: MUFU and FP32 polynomial)"
    return min(mufu, fma), bound
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per full-size launch of
# the pair-sum kernel on this workload (the autotuned shape, 5 reference segments),
# from one ncu capture of the pilot and the evaluation launch (25.30 MB and 26.57 MB):
# profiles/pair_sum_f32x2_adaptive_gaussprod2d_1M.md.
TRAFFIC_BYTES_PER_LAUNCH = 25_936_000


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=1_000_000, help="reference points")
    ap.add_argument("--m", type=int, default=1_000_000, help="queries per rank")
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="target CPU time of the bounded CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--workload",
                    choices=["direct", "surrogate-grid", "plain-small", "cv-batch", "direct1d"],
                    default="direct",
                    help="direct: adaptive pilot + evaluation, 1M x 1M (the default); "
                         "surrogate-grid: 4M references on an 8192 x 8192 grid; "
                         "plain-small: 10k references on a 100 x 100 grid (latency); "
                         "cv-batch: 16 datasets x 64 x 64 bandwidths, one launch; "
                         "direct1d: 1-D Gaussian, 2^24 references x 2^24 queries")
    ap.add_argument("--cv-sets", type=int, default=16, help="cv-batch: datasets")
    ap.add_argument("--cv-size", type=int, default=0,
                    help="cv-batch: points per dataset (0: log-uniform in [1e4, 5e5])")
    ap.add_argument("--n1d", type=int, default=1 << 24, help="direct1d: references")
    ap.add_argument("--m1d", type=int, default=1 << 24, help="direct1d: queries per rank")
    ap.add_argument("--grid", type=int, default=8192, help="surrogate-grid: points per axis")
    ap.add_argument("--n-grid-ref", type=int, default=4_000_000,
                    help="surrogate-grid: reference points")
    ap.add_argument("--train-steps", type=int, default=30000)
    ap.add_argument("--no-plain", action="store_true",
                    help="surrogate-grid: skip the plain direct comparator (~1 min)")
    return ap.parse_args()


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def rank_queries(W, wl, rank: int, m: int):
    """Query batch of `rank`: rank 0 keeps the configuration's own queries, every
    other rank draws its own seeded batch from the same distribution (queries are
    independent, so ranks share no data-path collective)."""
    if rank == 0:
        return wl.queries
    rng = W.SplitMix64(W.SEED_BASE + 200 + rank)
    return W.f32(rng.uniform(2 * m, -3.0, 3.0).reshape(m, 2))


def max_over_ranks(dist, ms: float, device) -> float:
    """The job's time: the slowest rank's (all_reduce MAX); ms itself without dist."""
    if dist is None:
        return ms
    import torch
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank_step: float, steps: int, world: int, total_ms: float) -> float:
    """Units processed by all ranks divided by the (max-over-ranks) time."""
    return units_per_rank_step * steps * world / (total_ms / 1e3)


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return {}


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = os.path.join("/tmp", f"bbkde_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.close()
        sm, smax, power, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
                power.append(float(parts[3]))
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax),
                "power_w_max": max(power), "samples": len(sm), "reasons": sorted(reasons)}


def l2_flush(torch, buf):
    buf.zero_()   # 256 MB write > 126 MB L2


def cpu_reference_rate(wl, seconds: float, kind_pref: str = "reference"):
    """evals/s of the reference's CPU direct_eval on a bounded query sample."""
    from oracle.pyoracle import Oracle, Reference, nthreads_default
    threads = nthreads_default()
    n = len(wl.refs)
    dim = wl.dim
    if kind_pref == "reference" and Reference.available():
        ref = Reference()
        handle = ref.create(wl.kind, dim, wl.h, wl.refs, wl.weights)
        run = lambda q: ref.direct(handle, q, nthreads=threads)  # noqa: E731
        kind = "reference"
        cleanup = lambda: ref.destroy(handle)  # noqa: E731
    else:
        orc = Oracle()
        wn = wl.weights / wl.weights.sum()
        run = lambda q: orc.direct(wl.kind, dim, wl.h, wl.refs, wn, q, nthreads=threads)  # noqa
        kind = "port"
        cleanup = lambda: None  # noqa: E731
    # size the sample from a probe of at least ~0.5 s
    probe = max(threads, 8)
    while True:
        t0 = time.perf_counter()
        run(wl.queries[:probe])
        dt = time.perf_counter() - t0
        if dt >= 0.5 or probe >= len(wl.queries):
            break
        probe = min(len(wl.queries), probe * 4)
    per_q = dt / probe
    m = int(min(len(wl.queries), max(probe, seconds / max(per_q, 1e-9))))
    t0 = time.perf_counter()
    run(wl.queries[:m])
    dt = time.perf_counter() - t0
    cleanup()
    kname = {0: f"GaussianKernel<{dim},double>", 2: "GaussianProductKernel2d<double>"}.get(
        wl.kind, f"kind {wl.kind}")
    return {"value": m * n / dt, "unit": UNIT, "cores": threads, "kind": kind,
            "sample": f"direct_eval of {m} queries x {n} refs ({kname}), {threads} host "
                      f"threads, {dt:.1f} s"}


def run_reference_arm(a, world, rank):
    """The reference's own CPU direct_eval (oracle/_ref, all host threads) on the
    headline workload (config 2, the default) or on plain-small (config 1). The
    other workloads time their CPU baseline inside their own line."""
    if a.workload not in ("direct", "plain-small"):
        print(f"--impl reference times the direct and plain-small workloads; the "
              f"{a.workload} line carries its own cpu_baseline", file=sys.stderr)
        return 2
    if rank != 0:
        return 0
    from bbrcit_kde_b200 import workloads as W
    small = a.workload == "plain-small"
    wl = W.config1() if small else W.config2(n=a.n, m=a.m)
    per_step = max(1.0, a.cpu_seconds / 4)
    rates = []
    base = None
    for i in range(a.warmup + a.steps):
        r = cpu_reference_rate(wl, per_step)
        if i >= a.warmup:
            rates.append(r["value"])
        base = r
    value = float(np.median(rates))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": (len(wl.refs) * len(wl.queries) if small else 2.0 * a.n * a.m)
        / value * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded splitmix64 bimodal mixture)",
        "config": ({"workload": "plain 2-D Gaussian, 10k bimodal refs, h=0.1, 100x100 grid "
                                "on [-3,3)^2 (1e8 evals per call)"}
                   if small else workload_config(a)),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": base["cores"],
                         "kind": base["kind"], "sample": base["sample"]},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def workload_config(a):
    return {
        "workload": f"adaptive 2-D product-Gaussian KDE, pilot + evaluation: N={a.n} refs "
                    f"(bimodal mixture, weights U[0.5,1.5]), M={a.m} uniform queries on "
                    f"[-3,3]^2 per rank, h=(0.05,0.05), alpha=0.5",
        "n_ref": a.n, "n_query_per_rank": a.m, "kernel": "GaussianProductKernel2d",
        "h": [0.05, 0.05], "alpha": 0.5, "precision": "FP32C (FP32 Kahan, FP64 combine)",
        "evals_per_step_per_rank": 2 * a.n * a.m,
        "l2": "flushed between timed steps (256 MB write)",
        "parallelism": "queries sharded across ranks, refs replicated" if a.gpus > 1 else "1 GPU",
    }


def main():
    a = parse()
    world, rank, local = dist_env()
    if a.impl == "reference":
        return run_reference_arm(a, world, rank)
    if a.workload == "surrogate-grid":
        return run_surrogate_grid(a, world, rank, local)
    if a.workload == "plain-small":
        return run_plain_small(a, world, rank, local)
    if a.workload == "cv-batch":
        return run_cv_batch(a, world, rank, local)
    if a.workload == "direct1d":
        return run_direct1d(a, world, rank, local)

    import torch
    import bbrcit_kde_b200 as bk
    from bbrcit_kde_b200 import workloads as W
    from bbrcit_kde_b200.parity import error_stats

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    wl = W.config2(n=a.n, m=a.m)
    wl.queries = rank_queries(W, wl, rank, a.m)
    wn = wl.weights / wl.weights.sum()
    n, m = len(wl.refs), len(wl.queries)
    evals_per_step = 2.0 * n * m

    stream = torch.cuda.Stream()   # a real (non-null) stream shared with the library
    torch.cuda.set_stream(stream)
    ctx = bk.Context(local)
    ctx.set_stream(stream.cuda_stream)
    sm_count, _ = ctx.device_info()
    desc = bk.kernel_desc(wl.kind, 2, wl.h)
    out = torch.empty(m, dtype=torch.float64, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    # ---- device-resident timing ------------------------------------------
    ctx.upload(bk.REFERENCE, wl.refs, mass=wn, weight=wn)
    ctx.upload(bk.QUERY, wl.queries)

    def step():
        ctx.adapt_density(desc, wl.alpha, bk.FP32C, outputs=False)
        pilot_stats = ctx.last_launch_stats()
        ctx.eval_range_device(desc, 0, n - 1, 0, m - 1, out.data_ptr(), True, bk.FP32C)
        return pilot_stats, ctx.last_launch_stats()

    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    sampler = ClockSampler(local)
    sampler.start()
    launches0 = ctx.launch_count()
    step_ms, kernel_launches = [], []
    for _ in range(a.steps):
        l2_flush(torch, flush)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s1, s2 = step()
        e1.record(stream)
        torch.cuda.synchronize()
        step_ms.append(e0.elapsed_time(e1))
        kernel_launches += [s1, s2]
    launches = ctx.launch_count() - launches0
    clocks = sampler.stop()
    total_ms = max_over_ranks(dist, sum(step_ms), "cuda")
    if dist:
        dist.barrier()
    value = whole_job_rate(evals_per_step, a.steps, world, total_ms)

    # roofline of the pair-sum kernel (pilot and evaluation launches)
    ach = [p / (ms / 1e3) for ms, p, _ in kernel_launches if ms > 0]
    achieved = float(np.mean(ach))
    kernel_ms = float(np.mean([ms for ms, _, _ in kernel_launches]))
    peaks = measured_peaks()
    sm_max = float(peaks.get("sm_max_mhz") or clocks.get("sm_max_mhz") or 1965.0)
    _, variant = ctx.launch_variants()
    poly = VARIANT_POLY[variant] if 0 <= variant < len(VARIANT_POLY) else 0
    per_clk, bound = pair_sum_bound_per_clk_per_sm(poly)
    peak = sm_count * per_clk * sm_max * 1e6
    mufu_peak = sm_count * MUFU_EX2_PER_CLK_PER_SM * sm_max * 1e6
    observed = clocks.get("sm_mhz")
    roofline = {
        "bound": bound, "achieved": achieved / 1e9, "peak": peak / 1e9, "unit": "Geval/s",
        "frac": achieved / peak,
        "peak_basis": f"{sm_count} SMs x {per_clk:.2f} pairs/clk x {sm_max:.0f} MHz "
                      f"(sm_max_mhz, MEASURED_PEAKS.json); launch shape {variant} "
                      f"(FP32-pipe exp2 every {poly or 'no'} reference); MUFU alone: "
                      f"16 ex2/clk/SM",
        "frac_of_mufu_only_bound": achieved / mufu_peak,
        "frac_at_observed_clock": (achieved / (sm_count * per_clk * observed * 1e6))
        if observed else None,
        "kernel_ms_per_launch": kernel_ms,
        "pairs_per_launch": float(kernel_launches[0][1]),
        "traffic": TRAFFIC_BYTES_PER_LAUNCH,
        "hbm_gbs_peak": peaks.get("hbm_gbs"),
    }

    # ---- error vs FP64 (outside the timed region) -----------------------
    sl = slice(m // 2, m // 2 + 4096)
    ctx.adapt_density(desc, wl.alpha, bk.FP32C, outputs=False)
    f32 = ctx.eval_range(desc, 0, n - 1, sl.start, sl.stop - 1, True, bk.FP32C)
    abw64, mass64, pilot64, _ = ctx.adapt_density(desc, wl.alpha, bk.FP64)
    f64 = ctx.eval_range(desc, 0, n - 1, sl.start, sl.stop - 1, True, bk.FP64)
    err = error_stats(f32, f64)
    err_def = ("vs FP64 device path (pilot + eval in FP64) on 4096 queries; pass = "
               "approximately_equal(rel 1e-6, abs 1e-8) as FloatUtils.h:49-61")
    oracle_check = None
    if rank == 0:
        # The FP64 device path against the CPU oracle at full size: 1,024 of the
        # error-check queries (with the FP64 attributes) and 1,024 pilot rows.
        from oracle.pyoracle import Oracle
        orc = Oracle()
        want = orc.direct(wl.kind, 2, wl.h, wl.refs, mass64, wl.queries[sl][:1024], abw=abw64)
        rows = np.linspace(0, n - 1, 1024).astype(np.int64)
        pilot_want = orc.direct(wl.kind, 2, wl.h, wl.refs, wn, wl.refs[rows])
        oracle_check = {
            "queries": 1024, "eval": error_stats(f64[:1024], want, 1e-10, 0.0),
            "pilot_rows": 1024, "pilot": error_stats(pilot64[rows], pilot_want, 1e-10, 0.0)}
        oracle_check["pass_rate"] = min(oracle_check["eval"]["pass_rate"],
                                        oracle_check["pilot"]["pass_rate"])

    # ---- end to end through the C ABI with host buffers -----------------
    e2e = None
    if not a.no_e2e:
        pin = lambda arr: torch.from_numpy(np.ascontiguousarray(arr)).pin_memory().numpy()  # noqa
        h_refs, h_w, h_q = pin(wl.refs), pin(wn), pin(wl.queries)
        h_out = pin(np.empty(m))

        def e2e_step():
            ctx.upload(bk.REFERENCE, h_refs, mass=h_w, weight=h_w)
            ctx.upload(bk.QUERY, h_q)
            ctx.adapt_density(desc, wl.alpha, bk.FP32C, outputs=False)
            ctx.eval_range(desc, 0, n - 1, 0, m - 1, True, bk.FP32C, out=h_out)

        for _ in range(a.warmup):
            e2e_step()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        e2e_ms = []
        for _ in range(a.steps):
            l2_flush(torch, flush)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            e2e_step()
            e1.record(stream)
            torch.cuda.synchronize()
            e2e_ms.append(e0.elapsed_time(e1))
        tot = max_over_ranks(dist, sum(e2e_ms), "cuda")
        h2d = h_refs.nbytes + 2 * h_w.nbytes + h_q.nbytes
        d2h = h_out.nbytes
        e2e = {"value": whole_job_rate(evals_per_step, a.steps, world, tot), "unit": UNIT,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)}

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cpu = cpu_reference_rate(wl, a.cpu_seconds)

    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": total_ms / a.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded splitmix64 bimodal mixture, float32-representable)",
        "config": workload_config(a),
        "queries_per_s": value / n / 2.0,
        "e2e": e2e,
        "roofline": roofline,
        "cpu_baseline": cpu,
        "clocks": clocks,
        "gpu_launches": int(launches),
        "error_vs_fp64": {**err, "definition": err_def,
                          "fp64_vs_cpu_oracle": oracle_check},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# Surrogate-grid workload: the learned log-density surrogate on a dense grid.
# ---------------------------------------------------------------------------
GRID_METRIC_UNIT = "queries/s"


def _grid_errors(torch, x, ref):
    """Relative error of x against ref over every grid point."""
    e = ((x - ref).abs() / ref.clamp_min(1e-300)).float()
    n = e.numel()
    samp = e[torch.randint(0, n, (1 << 22,), device=e.device,
                           generator=torch.Generator(device=e.device).manual_seed(5))]
    q = torch.quantile(samp, torch.tensor([0.5, 0.999], device=e.device))
    return {"max": float(e.max()), "median": float(q[0]), "p999": float(q[1]),
            "frac_gt_1e-3": float((e > 1e-3).float().mean())}


def run_surrogate_grid(a, world, rank, local):
    """4,000,000 references from the seeded 8-component mixture, adaptive Gaussian
    KDE (pilot h = 0.05, alpha = 0.5), density on an 8192 x 8192 grid over
    [-4, 4]^2. One step = bbkde_eval_grid in anchored mode with the trained network
    in rescue mode: bicubic interpolation of the exact log-density between the
    anchors (every tile's first point), held-out probes per 16 x 16 tile judged at
    tolerance 5e-4, the probe set chosen by the library (probes = 0): the centre
    and edge midpoints while a tile spans at most 0.75 narrowest kernel widths --
    the case here (0.63), so anchors and probes are one 1025 x 1025 lattice of
    pitch 8 evaluated exactly -- and the quarter points besides on coarser grids;
    on the tiles whose probes miss, the
    network (two-term BF16 inference) + its bicubic residual, kept where its
    probes pass; exact culled fallback on the rest and on tiles below 1e-4 of the
    maximum. Comparators (timed once each): the plain direct sum over all grid
    points, the culled exact sum, the network on every point, the pipeline
    without the network, and the network alone with probes (no anchors)."""
    import torch
    import bbrcit_kde_b200 as bk
    from bbrcit_kde_b200 import workloads as W

    torch.cuda.set_device(local)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx = bk.Context(local)
    ctx.set_stream(stream.cuda_stream)
    sm_count, _ = ctx.device_info()
    info = {}

    refs = W.config5_refs(a.n_grid_ref)
    if rank > 0:   # replicas: each rank its own seeded draw of the same mixture
        rng = W.SplitMix64(W.SEED_BASE + 500 + rank)
        refs = refs[np.argsort(rng.uniform(len(refs)))]
    n = len(refs)
    w = np.full(n, 1.0 / n)
    desc = bk.kernel_desc(W.GAUSS, 2, (0.05, 0.05))
    ctx.upload(bk.REFERENCE, refs, mass=w, weight=w)
    # pilot to 1e-7 (culled self-sum): the adapted set every comparator shares
    t0 = time.perf_counter()
    abw, mass, _, _ = ctx.adapt_density_tol(desc, 0.5, rel_tol=1e-7)
    info["pilot_ms"] = 1e3 * (time.perf_counter() - t0)

    # Training set: exact log-densities at uniform and data-sampled points.
    rng = W.SplitMix64(0xB2000555)
    n_tr = 2_000_000
    uni = rng.uniform(n_tr, -4.0, 4.0).reshape(-1, 2)
    pick = np.minimum((rng.uniform(n_tr // 2) * n).astype(np.int64), n - 1)
    dat = refs[pick] + 0.05 * rng.normal(n_tr).reshape(-1, 2)
    xy = W.f32(np.concatenate([uni, dat]))
    ctx.upload(bk.QUERY, xy)
    # culled sum at the 1e-7 bound (every target within 1e-7 + FP32C of the full
    # sum); wall time of the synchronous call (query sort, sum, copy to the host)
    t0 = time.perf_counter()
    f, cst = ctx.eval_culled(desc, rel_tol=1e-7)
    info["train_targets_ms"] = 1e3 * (time.perf_counter() - t0)
    info["train_targets_pairs_frac"] = cst.pairs / cst.full_pairs
    ok = f > 0
    sur = bk.Surrogate(local, seed=1)
    t1 = time.perf_counter()
    loss = sur.train(xy[ok], np.log(f[ok]), steps=a.train_steps, batch=8192, lr=3e-3,
                     lr_final=1e-5)
    torch.cuda.synchronize()
    info.update(train_s=time.perf_counter() - t1, train_steps=a.train_steps, final_loss=loss,
                train_points=int(ok.sum()))
    sur.set_inference(True)

    G = a.grid
    grid = (G, G, -4.0, 4.0, -4.0, 4.0)
    npts = G * G
    out = torch.empty(npts, dtype=torch.float64, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    # exact parts (lattice, fallback) to 1e-5: 100x below the pipeline's 1e-3 bar;
    # every tile judged by its probes (no low-density cut); probe set and lattice
    # tile picked by the library
    main_cfg = dict(surrogate=sur, mode=bk.GRID_ANCHORED, tile=16, probes=0, rel_tol=5e-4,
                    low_frac=0.0, interp=3, cull_rel=1e-5, lattice_tile=0)

    def grid_step(dst, **kw):
        return ctx.eval_grid(desc, grid, dst.data_ptr(), **kw)

    for _ in range(a.warmup):
        grid_step(out, **main_cfg)
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    launches0 = ctx.launch_count()
    step_ms, stats = [], []
    for _ in range(a.steps):
        l2_flush(torch, flush)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st = grid_step(out, **main_cfg)
        e1.record(stream)
        torch.cuda.synchronize()
        step_ms.append(e0.elapsed_time(e1))
        stats.append(st.as_dict())
    launches = ctx.launch_count() - launches0
    clocks = sampler.stop()
    total_ms = sum(step_ms)
    value = npts * a.steps / (total_ms / 1e3)
    main_out = out.clone()

    # Comparators, each once.
    comp = {}
    for name, kw in [("culled_exact", dict(mode=bk.GRID_EXACT, tile=16)),
                     ("culled_exact_tile32", dict(mode=bk.GRID_EXACT, tile=32)),
                     # the whole grid at the pipeline's exact-part tolerance, tile 32,
                     # accumulation on the FP32 pipe and on the tcgen05 tensor cores
                     ("culled_exact_tile32_1e-5_fp32_pipe",
                      dict(mode=bk.GRID_EXACT, tile=32, cull_rel=1e-5, tensor_cores=1)),
                     ("culled_exact_tile32_1e-5_tensor_cores",
                      dict(mode=bk.GRID_EXACT, tile=32, cull_rel=1e-5, tensor_cores=2)),
                     ("culled_exact_pair_form", dict(mode=bk.GRID_EXACT, tile=16,
                                                     pair_form=True)),
                     ("network_pair_form", dict(main_cfg, pair_form=True)),
                     ("network_tensor_cores", dict(main_cfg, tensor_cores=2)),
                     ("network_everywhere", dict(main_cfg, net_scope=bk.NET_EVERYWHERE)),
                     ("anchored_without_network", dict(main_cfg, surrogate=None)),
                     ("network_bilinear", dict(main_cfg, interp=1)),
                     ("anchored_without_network_bilinear",
                      dict(main_cfg, surrogate=None, interp=1)),
                     ("network_bilinear_tile32", dict(main_cfg, tile=32, interp=1)),
                     ("anchored_without_network_bilinear_tile32",
                      dict(main_cfg, surrogate=None, tile=32, interp=1)),
                     ("network_only_probes", dict(surrogate=sur, mode=bk.GRID_SURROGATE,
                                                  tile=16, probes=0, rel_tol=5e-4,
                                                  low_frac=1e-4)),
                     ("network_tile32", dict(main_cfg, tile=32)),
                     ("anchored_without_network_tile32",
                      dict(main_cfg, surrogate=None, tile=32))]:
        dst = torch.empty(npts, dtype=torch.float64, device="cuda")
        for _ in range(2):   # the second run is reported (buffers sized, kernels loaded)
            l2_flush(torch, flush)
            torch.cuda.synchronize()
            st = grid_step(dst, **kw)
        comp[name] = (st.as_dict(), dst)

    plain = None
    if not a.no_plain:
        ctx.upload(bk.QUERY, W.grid_2d(-4.0, 4.0, G, -4.0, 4.0, G))
        plain = torch.empty(npts, dtype=torch.float64, device="cuda")
        l2_flush(torch, flush)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ctx.eval_range_device(desc, 0, n - 1, 0, npts - 1, plain.data_ptr())
        e1.record(stream)
        torch.cuda.synchronize()
        info["plain_direct_ms"] = e0.elapsed_time(e1)
    ref = plain if plain is not None else comp["culled_exact"][1]
    ref_name = "plain direct FP32C" if plain is not None else "culled exact FP32C"
    errors = {"pipeline": _grid_errors(torch, main_out, ref)}
    results = {}
    for name, (st, dst) in comp.items():
        errors[name] = _grid_errors(torch, dst, ref)
        results[name] = st
    # FP64 at 4096 grid points.
    idx = np.sort(np.random.default_rng(3).choice(npts, 4096, replace=False))
    pts = np.stack([-4.0 + (idx % G) * (8.0 / G), -4.0 + (idx // G) * (8.0 / G)], 1)
    ctx.upload(bk.QUERY, W.f32(pts))
    f64 = ctx.eval_all(desc, precision=bk.FP64)
    tidx = torch.from_numpy(idx).cuda()
    fp64 = {}
    for name, arr in [("pipeline", main_out), ("reference_grid", ref),
                      ("culled_exact", comp["culled_exact"][1])]:
        v = arr[tidx].cpu().numpy()
        e = np.abs(v - f64) / f64
        fp64[name] = {"max": float(e.max()), "median": float(np.median(e))}
    del comp

    # End to end through the C ABI: the adapted reference set from pinned host
    # memory in, the density grid to pinned host memory out.
    e2e = None
    if not a.no_e2e:
        pin = lambda arr: torch.from_numpy(np.ascontiguousarray(arr)).pin_memory()  # noqa
        h_refs, h_mass, h_abw, h_w = pin(refs), pin(mass), pin(abw), pin(w)
        h_out = torch.empty(npts, dtype=torch.float64).pin_memory()

        def e2e_step():
            ctx.upload(bk.REFERENCE, h_refs.numpy(), mass=h_mass.numpy(), abw=h_abw.numpy(),
                       weight=h_w.numpy())
            grid_step(out, **main_cfg)
            h_out.copy_(out, non_blocking=True)

        for _ in range(a.warmup):
            e2e_step()
        torch.cuda.synchronize()
        e2e_ms = []
        for _ in range(a.steps):
            l2_flush(torch, flush)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            e2e_step()
            e1.record(stream)
            torch.cuda.synchronize()
            e2e_ms.append(e0.elapsed_time(e1))
        h2d = h_refs.numel() * 8 + 3 * n * 8
        e2e = {"value": npts * a.steps / (sum(e2e_ms) / 1e3), "unit": GRID_METRIC_UNIT,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(npts * 8)}

    # Roofline of the factored culled sum at the lattice's tile edge T (the
    # pipeline's largest launch): on a T x T tile every reference costs 2T kernel
    # factors (MUFU ex2) and T^2 multiply-adds, one per pair. The FMA pipe allows
    # 128 pairs/clk/SM; MUFU 16 ex2/clk/SM = 16 T^2 / 2T = 8T pairs/clk/SM (128 at
    # T = 16, 256 at T = 32): the FMA pipe is the bound. Pairs at tile granularity
    # of the culled-exact comparator at that tile edge over its device time.
    lt = int(stats[-1]["lattice_tile_used"])
    peaks = measured_peaks()
    sm_max = float(peaks.get("sm_max_mhz") or clocks.get("sm_max_mhz") or 1965.0)
    if lt == 32:
        # At tile 32 the lattice (culled to 1e-5) runs on the tensor cores: the
        # whole-grid tensor-core comparator measures that kernel; its ceiling is the
        # factored method's MUFU bound, 2T ex2 per reference and tile = 8T pairs/clk/SM.
        ce = results["culled_exact_tile32_1e-5_tensor_cores"]
        peak = sm_count * MUFU_EX2_PER_CLK_PER_SM * (lt / 2) * sm_max * 1e6
        ach = ce["pairs"] / (ce["ms_total"] / 1e3)
        roofline = {"bound": "mufu", "kernel": "k_pair_sum_culled_sep_tc<GAUSS_ISO> (factored "
                                               "culled grid on the tcgen05 tensor cores; the "
                                               "pipeline's lattice launch)",
                    "achieved": ach / 1e9, "peak": peak / 1e9, "unit": "Gpair/s",
                    "frac": ach / peak, "traffic": None,
                    "peak_basis": f"{sm_count} SMs x 16 MUFU ex2/clk x {lt // 2} pairs per ex2 "
                                  f"(2T factors per reference on a T x T tile, T = {lt}) x "
                                  f"{sm_max:.0f} MHz; measured by the whole-grid comparator "
                                  "at 1e-5; compute-bound, DRAM traffic negligible"}
    else:
        ce = results["culled_exact"]
        peak = sm_count * FP32_FMA_PER_CLK_PER_SM * sm_max * 1e6
        ach = ce["pairs"] / (ce["ms_total"] / 1e3)
        roofline = {"bound": "fp32", "kernel": f"k_pair_sum_culled_sep<GAUSS_ISO,{lt}> "
                                               "(factored culled exact grid; the pipeline's "
                                               "lattice launch)",
                    "achieved": ach / 1e9, "peak": peak / 1e9, "unit": "Gpair/s",
                    "frac": ach / peak, "traffic": None,
                    "peak_basis": f"{sm_count} SMs x 128 FP32 FMA/clk x {sm_max:.0f} MHz "
                                  f"(MUFU allows {8 * lt} pairs/clk/SM at tile {lt}); "
                                  "compute-bound, DRAM traffic negligible"}
    cpu = None
    if rank == 0 and not a.no_cpu_baseline:
        wl = W.Workload("cfg5", W.GAUSS, 2, (0.05, 0.05), refs, w,
                        W.f32(pts[:2048]))
        r = cpu_reference_rate(wl, a.cpu_seconds)
        cpu = {"value": r["value"] / n, "unit": GRID_METRIC_UNIT, "cores": r["cores"],
               "kind": r["kind"],
               "sample": r["sample"] + "; queries/s = pair rate / 4M references "
                                       "(Gaussian kernel, fixed bandwidth: same per-pair "
                                       "cost as the adaptive sum)"}
    ctx.close()
    sur.close()
    if rank != 0:
        return 0
    speedup = {}
    if plain is not None:
        pm = info["plain_direct_ms"]
        speedup = {"pipeline_vs_plain_direct": pm / (total_ms / a.steps),
                   # one grid including the network's training data and training
                   "pipeline_with_training_vs_plain_direct":
                       pm / (total_ms / a.steps + info["train_targets_ms"] +
                             1e3 * info["train_s"])}
        for name, st in results.items():
            speedup[f"{name}_vs_plain_direct"] = pm / st["ms_total"]
    line = {
        "metric": METRIC, "value": value, "unit": GRID_METRIC_UNIT, "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": total_ms / a.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+bf16",
        "data": "synthetic (seeded splitmix64 8-component mixture, float32-representable)",
        "config": {"workload": f"surrogate grid: adaptive Gaussian KDE of {n} refs (pilot "
                               f"h=0.05, alpha=0.5) on a {G}x{G} grid over [-4,4]^2",
                   "pipeline": "bbkde_eval_grid anchored mode, bicubic residual, tile 16, "
                               f"automatic probe set ({stats[-1]['probes_used']} at this "
                               "spacing) and lattice tile "
                               f"({stats[-1]['lattice_tile_used']}), probe tolerance 5e-4, "
                               "no low-density cut, exact parts culled to 1e-5 (tile-32 "
                               "factored sums on the tcgen05 tensor cores); network in "
                               "rescue mode (two-term BF16 inference on tcgen05 on the tiles "
                               "the interpolated exact anchors miss)",
                   "l2": "flushed between timed steps (256 MB write)"},
        "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "clocks": clocks,
        "gpu_launches": int(launches), "step_stats": stats[-1], "comparators": results,
        "speedup": speedup, "errors_vs": ref_name, "errors": errors, "errors_vs_fp64_4096": fp64,
        "setup": info,
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# Smaller workloads: the reference's CPU-runnable case, batched cross-validation,
# the 1-D roofline probe.
# ---------------------------------------------------------------------------
def _device_setup(local):
    import torch
    import bbrcit_kde_b200 as bk
    torch.cuda.set_device(local)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx = bk.Context(local)
    ctx.set_stream(stream.cuda_stream)
    return torch, bk, stream, ctx


def _timed(torch, stream, fn, steps, warmup, flush=None):
    """Device time (CUDA events on `stream`) of each of `steps` calls after `warmup`."""
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    ms = []
    for _ in range(steps):
        if flush is not None:
            l2_flush(torch, flush)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    return ms


def _line(a, world, metric_unit, value, ms, config, dtype, **extra):
    d = {"metric": METRIC, "value": value, "unit": metric_unit, "n_gpus": world,
         "steps": a.steps, "warmup": a.warmup, "ms_per_step": float(np.mean(ms)),
         "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": dtype,
         "data": "synthetic (seeded splitmix64 mixtures, float32-representable)",
         "config": config}
    d.update(extra)
    print(json.dumps(d), flush=True)


def run_plain_small(a, world, rank, local):
    """10,000 references (bimodal mixture, unit weights), h = 0.1 Gaussian, 100 x 100
    grid over [-3, 3)^2: 1e8 pair evaluations per call. Launch-latency bound; the
    line reports the device time and the end-to-end latency of one call through the
    C ABI (upload queries from pinned host memory, evaluate, read back)."""
    torch, bk, stream, ctx = _device_setup(local)
    from bbrcit_kde_b200 import workloads as W
    from bbrcit_kde_b200.parity import error_stats
    wl = W.config1()
    n, m = len(wl.refs), len(wl.queries)
    w = wl.weights / wl.weights.sum()
    desc = bk.kernel_desc(wl.kind, 2, wl.h)
    ctx.upload(bk.REFERENCE, wl.refs, mass=w, weight=w)
    ctx.upload(bk.QUERY, wl.queries)
    out = torch.empty(m, dtype=torch.float64, device="cuda")
    sm_count, _ = ctx.device_info()
    kernel_ms = []

    def step():
        ctx.eval_range_device(desc, 0, n - 1, 0, m - 1, out.data_ptr())
        kernel_ms.append(ctx.last_launch_stats()[0])

    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    launches0 = ctx.launch_count()
    sampler = ClockSampler(local)
    sampler.start()
    ms = _timed(torch, stream, step, a.steps, a.warmup, flush)
    clocks = sampler.stop()
    launches = (ctx.launch_count() - launches0) * a.steps // (a.steps + a.warmup)
    _, variant = ctx.launch_variants()
    pin = lambda arr: torch.from_numpy(np.ascontiguousarray(arr)).pin_memory().numpy()  # noqa
    h_q, h_out = pin(wl.queries), pin(np.empty(m))

    def e2e_step():
        ctx.upload(bk.QUERY, h_q)
        ctx.eval_range(desc, 0, n - 1, 0, m - 1, True, bk.FP32C, out=h_out)

    e2e_ms = _timed(torch, stream, e2e_step, a.steps, a.warmup, flush)
    got = ctx.eval_all(desc)
    f64 = ctx.eval_all(desc, precision=bk.FP64)
    from oracle.pyoracle import Oracle
    want = Oracle().direct(wl.kind, 2, wl.h, wl.refs, w, wl.queries)
    cpu = cpu_reference_rate(wl, min(a.cpu_seconds, 4.0)) if not a.no_cpu_baseline else None
    ctx.close()
    pairs = float(n) * m
    peaks = measured_peaks()
    sm_max = float(peaks.get("sm_max_mhz") or clocks.get("sm_max_mhz") or 1965.0)
    poly = VARIANT_POLY[variant] if 0 <= variant < len(VARIANT_POLY) else 0
    per_clk, bound = pair_sum_bound_per_clk_per_sm(poly)
    peak = sm_count * per_clk * sm_max * 1e6
    kms = float(np.mean(kernel_ms[-a.steps:]))
    _line(a, world, UNIT, pairs * world / (np.mean(ms) / 1e3), ms,
          {"workload": "plain 2-D Gaussian, 10k bimodal refs, h=0.1, 100x100 grid on "
                       "[-3,3)^2 (1e8 evals per call)",
           "l2": "flushed between timed steps (256 MB write)"}, "f32",
          clocks=clocks,
          roofline={"bound": bound, "achieved": pairs / (kms / 1e3) / 1e9,
                    "peak": peak / 1e9, "unit": "Geval/s",
                    "frac": pairs / (kms / 1e3) / peak, "traffic": None,
                    "kernel_ms_per_launch": kms, "launch_shape": variant,
                    "note": "1e8 pairs fill the 148 SMs for ~20 us: launch and tail bound"},
          latency_us={"device": float(np.median(ms) * 1e3),
                      "e2e_c_abi": float(np.median(e2e_ms) * 1e3)},
          e2e={"value": pairs * world / (np.mean(e2e_ms) / 1e3), "unit": UNIT,
               "h2d_bytes_per_step": int(h_q.nbytes), "d2h_bytes_per_step": int(h_out.nbytes)},
          gpu_launches=int(launches),
          cpu_baseline=cpu,
          error_vs_reference_fp64=error_stats(got, want),
          fp64_path_vs_oracle_max_rel=float(np.max(np.abs(f64 - want) / want)))
    return 0


def _cv_cpu_baseline(bk, W, sets, hb, seconds):
    """The reference's likelihood_cross_validate + lsq_convolution_cross_validate
    (rel = abs = 0: its dual tree then sums every pair exactly), one bandwidth per
    call as grid_search does, on all host cores (one (hx, hy) per thread), on a
    bounded sample: the first dataset of at least 10,000 points cut to 10,000."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle.pyoracle import Reference, nthreads_default
    if not Reference.available():
        return None
    ref = Reference()
    s1 = next(s for s in sets if len(s) >= 10_000)[:10_000]
    ones = np.ones(len(s1))
    threads = nthreads_default()
    rng = np.random.default_rng(11)
    grid = [(hb[i], hb[j]) for i, j in zip(rng.integers(0, len(hb), 4096),
                                           rng.integers(0, len(hb), 4096))]

    def one(h):
        ref.likelihood_cv(bk.EPANECHNIKOV_PRODUCT_2D, 2, h, s1, ones)
        ref.lsq_conv_cv(bk.EPANECHNIKOV_PRODUCT_2D, 2, h, s1, ones)

    done, t0 = 0, time.perf_counter()
    with ThreadPoolExecutor(threads) as ex:
        while time.perf_counter() - t0 < seconds and done < len(grid):
            batch = grid[done: done + threads]
            list(ex.map(one, batch))
            done += len(batch)
    dt = time.perf_counter() - t0
    return {"value": float(len(s1)) ** 2 * 2 * done / dt,
            "unit": "(pair, bandwidth, kernel) items/s", "cores": threads, "kind": "reference",
            "sample": f"likelihood_cross_validate + lsq_convolution_cross_validate (rel = abs "
                      f"= 0) of one 10,000-point dataset at {done} random (hx, hy) of the "
                      f"64 x 64 grid, one bandwidth per call on {threads} threads, {dt:.1f} s"}


def run_cv_batch(a, world, rank, local):
    """Batched cross-validation: 16 datasets (log-uniform sizes in [1e4, 5e5], 3-component
    mixtures), Epanechnikov product kernel, 64 x 64 log-spaced (hx, hy) over [0.01, 1]^2:
    LOO likelihood and LSQ-convolution scores for every (dataset, hx, hy) in one
    persistent graph-captured launch. One step = one bbkde_cv_batch call: host
    datasets in, both score tables out. `value` is the device time of the launch
    (CUDA events around the graph), `e2e` the whole call (binning on the host,
    uploads, launch, downloads)."""
    torch, bk, stream, ctx = _device_setup(local)
    from bbrcit_kde_b200 import workloads as W
    sizes = [a.cv_size] * a.cv_sets if a.cv_size else None
    sets = W.config3_datasets(n_sets=a.cv_sets, sizes=sizes)
    if rank > 0:
        sets = [s[np.argsort(W.SplitMix64(W.SEED_BASE + 300 + rank).uniform(len(s)))]
                for s in sets]
    hb = W.config3_bandwidths()
    ds = [(s, None) for s in sets]
    sm_count, _ = ctx.device_info()
    res, dev_ms = {}, []
    launches0 = ctx.launch_count()

    def step():
        res["out"] = ctx.cv_batch(bk.EPANECHNIKOV_PRODUCT_2D, ds, hb, hb)
        dev_ms.append(ctx.last_launch_stats()[0])

    sampler = ClockSampler(local)
    sampler.start()
    ms = _timed(torch, stream, step, a.steps, a.warmup)
    clocks = sampler.stop()
    launches = (ctx.launch_count() - launches0) // (a.steps + a.warmup)
    _, pairs, _ = ctx.last_launch_stats()
    lik_pairs, conv_pairs, plan, n_plans = ctx.cv_batch_info()
    lik, lsq = res["out"]
    # Exactness: a few (dataset, hx, hy) against the per-bandwidth FP64 pair sums.
    small = int(np.argmin([len(s) for s in sets]))
    s0 = sets[small]
    w0 = np.full(len(s0), 1.0 / len(s0))
    ctx.upload(bk.REFERENCE, s0, mass=w0, weight=w0)
    checks = []
    for ia, ib in [(0, 0), (20, 45), (41, 49), (63, 63)]:
        d = bk.kernel_desc(bk.EPANECHNIKOV_PRODUCT_2D, 2, (hb[ia], hb[ib]))
        l64 = ctx.likelihood_cv(d, bk.FP64)
        q64 = ctx.lsq_conv_cv(d, bk.FP64)
        lg, qg = lik[small, ia, ib], lsq[small, ia, ib]
        checks.append({"hx": hb[ia], "hy": hb[ib],
                       "lik_rel": (abs(lg - l64) / abs(l64)) if np.isfinite(l64) else
                       (0.0 if lg == l64 else 1.0),
                       "lsq_rel": abs(qg - q64) / abs(q64)})
    cpu = None
    if rank == 0 and not a.no_cpu_baseline:
        cpu = _cv_cpu_baseline(bk, W, sets, hb, a.cpu_seconds)
    ctx.close()
    items = pairs * hb.size * hb.size * 2
    kms = float(np.mean(dev_ms[-a.steps:]))
    # Roofline: the histograms are built by 64-bit shared-memory atomic adds, 4 per
    # in-support likelihood pair and 16 per in-support convolution pair. The shared
    # pipe moves one 128-byte wavefront per clock per SM; a warp's 64-bit atomic
    # without bank conflicts is two wavefronts, i.e. 16 atomics per clock per SM.
    atomics = 4.0 * lik_pairs + 16.0 * conv_pairs
    peaks = measured_peaks()
    sm_max = float(peaks.get("sm_max_mhz") or clocks.get("sm_max_mhz") or 1965.0)
    peak = sm_count * 16 * sm_max * 1e6
    h2d = sum(s.nbytes for s in sets)
    nout = len(sets) * hb.size * hb.size
    _line(a, world, "(pair, bandwidth, kernel) items/s", items * world / (kms / 1e3), ms,
          {"workload": f"batched CV: {len(sets)} datasets (sizes {min(map(len, sets))}.."
                       f"{max(map(len, sets))}), Epanechnikov product, 64x64 (hx,hy) "
                       f"log-spaced on [0.01,1]^2, likelihood + LSQ-conv",
           "pairs": pairs, "bandwidths": int(hb.size ** 2),
           "l2": "inputs (the datasets, up to 8 MB each) are re-uploaded by every call; "
                 "the launch runs for seconds, so L2 state between steps is immaterial"},
          "fixed-point int64 + f64",
          clocks=clocks,
          e2e={"value": items * world / (np.mean(ms) / 1e3),
               "unit": "(pair, bandwidth, kernel) items/s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(2 * nout * 8)},
          roofline={"bound": "shared-memory pipe (64-bit atomic adds of the moment "
                             "histograms; 16 per clk per SM without bank conflicts)",
                    "achieved": atomics / (kms / 1e3) / 1e9, "peak": peak / 1e9,
                    "unit": "G atomics/s", "frac": atomics / (kms / 1e3) / peak,
                    "traffic": None, "lik_pairs_in_support": lik_pairs,
                    "conv_pairs_in_support": conv_pairs, "kernel_ms_per_launch": kms,
                    "work_item_plan": plan, "plans": n_plans,
                    "plan_note": "autotuned on the warm-up calls (each untried plan once)"},
          gpu_launches=int(launches), exactness_vs_fp64_per_bandwidth=checks, cpu_baseline=cpu,
          pairs_per_s=pairs * world / (kms / 1e3))
    return 0


def run_direct1d(a, world, rank, local):
    """1-D Gaussian roofline probe: 2^24 references (5-component mixture), h = 0.02,
    2^24 uniform queries on [-6, 6]; FP32-compensated direct sum."""
    torch, bk, stream, ctx = _device_setup(local)
    from bbrcit_kde_b200 import workloads as W
    from bbrcit_kde_b200.parity import error_stats
    wl = W.config4(n=a.n1d, m=a.m1d)
    if rank > 0:
        rng = W.SplitMix64(W.SEED_BASE + 400 + rank)
        wl.queries = W.f32(rng.uniform(a.m1d, -6.0, 6.0)).reshape(-1, 1)
    n, m = len(wl.refs), len(wl.queries)
    w = np.full(n, 1.0 / n)
    desc = bk.kernel_desc(wl.kind, 1, wl.h)
    ctx.upload(bk.REFERENCE, wl.refs, mass=w, weight=w)
    ctx.upload(bk.QUERY, wl.queries)
    sm_count, _ = ctx.device_info()
    out = torch.empty(m, dtype=torch.float64, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    sampler = ClockSampler(local)
    kernel_ms = []

    def step():
        ctx.eval_range_device(desc, 0, n - 1, 0, m - 1, out.data_ptr())
        kernel_ms.append(ctx.last_launch_stats()[0])

    launches0 = ctx.launch_count()
    sampler.start()
    ms = _timed(torch, stream, step, a.steps, a.warmup, flush)
    clocks = sampler.stop()
    launches = (ctx.launch_count() - launches0) * a.steps // (a.steps + a.warmup)
    pairs = float(n) * m
    # error vs FP64 on 4096 queries
    q0 = m // 2
    _, variant = ctx.launch_variants()
    f32 = ctx.eval_range(desc, 0, n - 1, q0, q0 + 4095)
    f64 = ctx.eval_range(desc, 0, n - 1, q0, q0 + 4095, True, bk.FP64)
    # end to end through the C ABI: queries in from pinned host memory, densities
    # out to pinned host memory, every step
    e2e = None
    if not a.no_e2e:
        pin = lambda arr: torch.from_numpy(np.ascontiguousarray(arr)).pin_memory().numpy()  # noqa
        h_q, h_out = pin(wl.queries), pin(np.empty(m))

        def e2e_step():
            ctx.upload(bk.QUERY, h_q)
            ctx.eval_range(desc, 0, n - 1, 0, m - 1, True, bk.FP32C, out=h_out)

        e2e_ms = _timed(torch, stream, e2e_step, a.steps, a.warmup, flush)
        e2e = {"value": pairs * world / (np.mean(e2e_ms) / 1e3), "unit": UNIT,
               "h2d_bytes_per_step": int(h_q.nbytes), "d2h_bytes_per_step": int(h_out.nbytes)}
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cpu = cpu_reference_rate(wl, a.cpu_seconds)
    ctx.close()
    peaks = measured_peaks()
    sm_max = float(peaks.get("sm_max_mhz") or clocks.get("sm_max_mhz") or 1965.0)
    poly = VARIANT_POLY[variant] if 0 <= variant < len(VARIANT_POLY) else 0
    per_clk, bound = pair_sum_bound_per_clk_per_sm(poly, fma_cycles=8.0)
    peak = sm_count * per_clk * sm_max * 1e6
    kms = float(np.mean(kernel_ms[-a.steps:]))
    _line(a, world, UNIT, pairs * world / (np.mean(ms) / 1e3), ms,
          {"workload": f"1-D Gaussian, h=0.02, {n} refs (5-component mixture), {m} uniform "
                       f"queries on [-6,6] per rank", "l2": "flushed between timed steps"},
          "f32", clocks=clocks, e2e=e2e, cpu_baseline=cpu, gpu_launches=int(launches),
          roofline={"bound": bound, "achieved": pairs / (kms / 1e3) / 1e9, "peak": peak / 1e9,
                    "unit": "Geval/s", "frac": pairs / (kms / 1e3) / peak, "traffic": None,
                    "launch_shape": variant,
                    "frac_of_mufu_only_bound": pairs / (kms / 1e3) /
                    (sm_count * MUFU_EX2_PER_CLK_PER_SM * sm_max * 1e6)},
          error_vs_fp64=error_stats(f32, f64))
    return 0


if __name__ == "__main__":
    sys.exit(main())
