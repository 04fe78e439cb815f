"""Benchmark: block-Vecchia log-likelihood evaluations per second.

Workload (the configuration the headline metric is quoted on): n = 1,000,000
locations uniform on [0,1]^2 (seed 0), Matern nu = 2.5, sigma2 = 1.0,
range = 0.05, no nugget, k-means into bc = 100,000 blocks, conditioning size
cs = 200.  Observations are one draw of the same Gaussian process by random
Fourier features (1024 features; a dense draw at n = 1M is infeasible).  One
step = one full log-likelihood evaluation.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs under torchrun, one process per GPU: every rank evaluates its
shard of the blocks and the FP64 partials are all-gathered (NCCL) and summed
in rank order (strong scaling: the evaluation is fixed, split over ranks).

--impl reference times the reference's algorithm on the host cores (the CPU
oracle: restated llh_Xvecchia_batch with OpenBLAS dense LA and OpenMP over
blocks), on a bounded sample of blocks of the same workload, extrapolated by
algorithmic FLOPs to one full evaluation.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = json.load(open(os.path.join(ROOT, "BASELINE.json")))["metric"] \
    if os.path.exists(os.path.join(ROOT, "BASELINE.json")) else \
    "loglik evals/s n=1M cs=200, mixed vs FP64 at rel err<=1e-8; serve p50/p99 ms"

WORKLOADS = {
    # The headline configuration.
    "c3": dict(name="n=1M uniform, nu=2.5 sigma2=1 range=0.05, bc=100k, cs=200",
               n=1_000_000, bc=100_000, cs=200, sigma2=1.0, range=0.05, nu=2.5, seed=0,
               kmeans_epochs=50, rff_features=1024),
    # Same kernel shape (cs = 200, blocks of ~10 points) on 4,000 blocks: the
    # case ncu captures with full sections.
    "c3-small": dict(name="n=40k uniform, nu=2.5 sigma2=1 range=0.05, bc=4k, cs=200 (profiling case)",
                     n=40_000, bc=4_000, cs=200, sigma2=1.0, range=0.05, nu=2.5, seed=0,
                     kmeans_epochs=50, rff_features=1024),
}
WORKLOAD = WORKLOADS["c3"]


# ----------------------------------------------------------------- workload

def make_locations(n, seed):
    rng = np.random.default_rng(seed)
    return rng.random(n), rng.random(n)


def rff_draw(x, y, sigma2, rng_, nu, features, seed, device=None):
    """One approximate draw of the zero-mean Matern GP (covariance
    sigma2 * c(d / range), the reference's parameterisation) by random Fourier
    features: omega ~ Z / (range * sqrt(chi2_{2 nu})), phase ~ U(0, 2 pi)."""
    g = np.random.default_rng(seed + 12345)
    Z = g.standard_normal((features, 2))
    W = g.chisquare(2 * nu, features)
    om = Z / (rng_ * np.sqrt(W))[:, None]
    ph = g.random(features) * 2 * np.pi
    amp = math.sqrt(2 * sigma2 / features)
    try:
        import torch
        if device is not None and torch.cuda.is_available():
            X = torch.as_tensor(np.stack([x, y], 1), device=device)
            O = torch.as_tensor(om.T, device=device)
            P = torch.as_tensor(ph, device=device)
            out = torch.empty(len(x), dtype=torch.float64, device=device)
            for s in range(0, len(x), 65536):
                out[s:s + 65536] = torch.cos(X[s:s + 65536] @ O + P).sum(1) * amp
            return out.cpu().numpy()
    except Exception:
        pass
    out = np.empty(len(x))
    for s in range(0, len(x), 16384):
        out[s:s + 16384] = np.cos(np.stack([x[s:s + 16384], y[s:s + 16384]], 1) @ om.T + ph).sum(1) * amp
    return out


def block_flops(batchNum, cs):
    """Algorithmic FP64 flops per block (LAPACK conventions of
    include/flops.h): potrf(cs) + trsm (cs^2 bs + cs^2) + gemm (2 bs^2 cs +
    2 bs cs) + potrf(bs) + trsm (bs^2) + norm (2 bs); block 0 unconditioned."""
    bs = batchNum.astype(np.float64)
    potrf = lambda m: m ** 3 / 3 + m ** 2 / 2 + m / 6  # noqa: E731
    f = potrf(cs) + cs * cs * bs + cs * cs + 2 * bs * bs * cs + 2 * bs * cs + potrf(bs) + bs * bs + 2 * bs
    f[0] = potrf(bs[0]) + bs[0] ** 2 + 2 * bs[0]
    f[bs == 0] = 0.0
    return f


# ------------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi samples (SM clock, throttle reasons) during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            if len(r) < 9:
                continue
            for k, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(k)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------- CPU sample

class CpuSample:
    """The CPU oracle (restated llh_Xvecchia_batch, OpenBLAS dense LA, OpenMP
    over blocks, all host threads) on a fixed contiguous sample of blocks of
    this workload; one step() times the sample and extrapolates by algorithmic
    FLOPs to evaluations/s of the full workload."""

    def __init__(self, layout, knn_fill, theta, flops, budget_s):
        from oracle import oracle as O
        O.build(ref=False)
        self.O = O
        self.theta = theta
        self.threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
        bc, cs = len(layout["batchNum"]), layout["cs"]
        self.knn = np.zeros(bc * cs, dtype=np.int32)
        mid = max(1, bc // 2)
        # Calibrate the sample size on a small range, then fix it.
        b0, b1 = mid, min(bc, mid + 4 * self.threads)
        knn_fill(self.knn, b0, b1)
        self.P = O.OracleProblem(layout["batchNum"], layout["batchNumAccum"], layout["x"],
                                 layout["y"], layout["obs"], self.knn, cs)
        t = time.perf_counter()
        O.llh_blas(self.P, theta, threads=self.threads, block_begin=b0, block_end=b1)
        dt = time.perf_counter() - t
        count = int(min(bc - mid, max(b1 - b0, (b1 - b0) * budget_s / max(dt, 1e-3))))
        self.b0, self.b1 = mid, min(bc, mid + count)
        knn_fill(self.knn, b1, self.b1)
        self.frac = float(flops[self.b0:self.b1].sum() / flops.sum())
        self.last_dt = None

    def step(self):
        t = time.perf_counter()
        self.O.llh_blas(self.P, self.theta, threads=self.threads, block_begin=self.b0,
                        block_end=self.b1)
        self.last_dt = time.perf_counter() - t
        return self.frac / self.last_dt

    def describe(self):
        bc = len(self.P.batchNum)
        return (f"blocks {self.b0}..{self.b1 - 1} of {bc} ({self.b1 - self.b0} blocks, "
                f"{self.frac * 100:.2f}% of the evaluation's flops) in {self.last_dt:.2f} s per "
                f"sample, extrapolated by flops")


def knn_fill_cpu(L):
    """Conditioning sets of a block range on the CPU (oracle, exact
    findNearestPoints semantics)."""
    from oracle import oracle as O

    def fill(knn, b0, b1):
        cs = L["cs"]
        for b in range(b0, b1):
            knn[b * cs:(b + 1) * cs] = O.knn_block_fast(L["x"], L["y"], int(L["batchNumAccum"][b]),
                                                        L["cx"][b], L["cy"][b], cs)
    return fill


def build_layout_arrays(bv_mod=None):
    """The workload's block layout (host k-means ordering, as the reference's
    driver builds it).  Uses the product's host layout code when available
    (it matches the reference's), else nothing."""
    w = WORKLOAD
    x, y = make_locations(w["n"], w["seed"])
    obs = rff_draw(x, y, w["sigma2"], w["range"], w["nu"], w["rff_features"], w["seed"],
                   device="cuda" if bv_mod is not None else None)
    import blockvecchia_b200 as bv
    L = bv.build_layout(x, y, obs, w["bc"], w["cs"], seed=w["seed"], epochs=w["kmeans_epochs"])
    return L


# ---------------------------------------------------------------- our arm

def run_ours(args):
    import torch
    import torch.distributed as dist

    import blockvecchia_b200 as bv
    from blockvecchia_b200.parallel import combine_partials

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != args.gpus:
        raise SystemExit(f"--gpus {args.gpus} but WORLD_SIZE={world}")
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    w = WORKLOAD
    theta = (w["sigma2"], w["range"], w["nu"])

    t_setup = time.perf_counter()
    L = build_layout_arrays(bv)
    L.knn_idx = bv.knn(L, device=local)
    setup_layout_s = time.perf_counter() - t_setup
    D = bv.LlhData(L, precision=args.precision, device=local, on_failure="continue",
                   shard_count=world, shard_index=rank)
    stream = torch.cuda.Stream(device=local)
    D.set_stream(stream.cuda_stream)
    flops = block_flops(L.batchNum, L.cs)
    mask = bv.shard_blocks(L.batchNum, L.cs, world, rank)
    my_flops = float(flops[mask].sum())
    # L2 flush buffer (256 MB > 126 MB L2), written between timed evaluations.
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=local)

    def step():
        with torch.cuda.stream(stream):
            flush.fill_(1.0)
        part = D(theta)
        if world > 1:
            with torch.cuda.stream(stream):
                return combine_partials(part)
        return part

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    kernel_ms = 0.0
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        v = step()
        kernel_ms += D.status()["kernel_ms"]
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    clk = clocks.stop()
    st = D.status()

    # End to end through the C ABI with host buffers: pinned inputs copied in
    # every step (locations, observations, conditioning indices), the
    # log-likelihood read back.
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    hx, hy, hobs, hknn = pin(L.x), pin(L.y), pin(L.obs), pin(L.knn_idx)
    h2d = hx.nbytes + hy.nbytes + hobs.nbytes + hknn.nbytes
    for _ in range(2):
        D.eval_host(hobs, theta, x=hx, y=hy, knn_idx=hknn)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(args.steps):
        part = D.eval_host(hobs, theta, x=hx, y=hy, knn_idx=hknn)
        if world > 1:
            with torch.cuda.stream(stream):
                combine_partials(part)
    f1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = f0.elapsed_time(f1)

    if world > 1:
        t = torch.tensor([ms, ms_e2e, kernel_ms], dtype=torch.float64, device=local)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, ms_e2e, kernel_ms = (float(a) for a in t.tolist())
    if rank != 0:
        D.close()
        if world > 1:
            dist.destroy_process_group()
        return

    # Roofline of the fused kernel: algorithmic FP64 flops / kernel time,
    # against this GPU's FP64 peak measured now (cuBLAS DGEMM through torch).
    a = torch.randn(8192, 8192, dtype=torch.float64, device=local)
    b = torch.randn_like(a)
    for _ in range(2):
        a @ b
    best = 1e30
    for _ in range(3):
        g0 = torch.cuda.Event(enable_timing=True)
        g1 = torch.cuda.Event(enable_timing=True)
        g0.record()
        a @ b
        g1.record()
        torch.cuda.synchronize()
        best = min(best, g0.elapsed_time(g1))
    peak_tf = 2 * 8192 ** 3 / (best * 1e-3) / 1e12
    del a, b
    kernel_s = kernel_ms / args.steps / 1e3
    achieved_tf = my_flops / kernel_s / 1e12

    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        layout = dict(batchNum=L.batchNum, batchNumAccum=L.batchNumAccum, x=L.x, y=L.y, obs=L.obs,
                      cs=L.cs, cx=L.cx, cy=L.cy)
        cs_ = CpuSample(layout, knn_fill_cpu(layout), theta, flops, budget_s=12.0)
        rate = cs_.step()
        cpu = {"value": rate, "unit": "evals/s", "cores": cs_.threads, "kind": "port",
               "sample": cs_.describe()}

    # Mixed precision on the same workload (the FP64 path is the reference):
    # timed like the FP64 loop, plus the range sweep's relative error and
    # fallback counts.
    mixed = None
    if world == 1 and not args.no_mixed and args.precision == "fp64":
        with bv.LlhData(L, precision="mixed", device=local, on_failure="continue") as Mx:
            Mx.set_stream(stream.cuda_stream)
            for _ in range(args.warmup):
                step_mx = Mx(theta)
            torch.cuda.synchronize()
            m0 = torch.cuda.Event(enable_timing=True)
            m1 = torch.cuda.Event(enable_timing=True)
            m0.record(stream)
            for _ in range(args.steps):
                with torch.cuda.stream(stream):
                    flush.fill_(1.0)
                vm = Mx(theta)
            m1.record(stream)
            torch.cuda.synchronize()
            ms_mx = m0.elapsed_time(m1)
            stm = Mx.status()
            sweep = []
            for rg_ in (0.02, 0.05, 0.1, 0.2, 0.3):
                th_ = (w["sigma2"], rg_, w["nu"])
                v64_ = D(th_)
                s64_ = D.status()
                vm_ = Mx(th_)
                sm_ = Mx.status()
                sweep.append({"range": rg_, "rel_err": abs(vm_ - v64_) / abs(v64_) if v64_ else None,
                              "fp32_fallback_blocks": sm_["fp32_fallback"],
                              "fp64_failed_blocks": s64_["failed"]})
            D(theta)
        mixed = {"value": args.steps / (ms_mx / 1e3), "unit": "evals/s",
                 "vs_fp64": (args.steps / (ms_mx / 1e3)) / (args.steps / (ms / 1e3)),
                 "rel_err_vs_fp64": abs(vm - v) / abs(v), "fp32_fallback_blocks": stm["fp32_fallback"],
                 "blocks": int(L.bc), "tol": 1e-8, "range_sweep": sweep,
                 "note": "FP32 factor of Sigma22 + FP64 refinement; blocks whose FP32 factor or "
                         "refinement fails are recomputed in FP64 (a probe of every 64th block "
                         "skips the FP32 pass when most would fail)"}
    serve = None
    if world == 1 and args.serve_sample > 0:
        serve = serve_workload(args.serve_sample, 4, 6.0, 2)
        serve.pop("clocks", None)

    # FP64: fused kernel + reduction; mixed: probe, decision, mixed pass,
    # FP64 fallback pass, reduction.
    launches_per_eval = 2 if args.precision == "fp64" else 5
    value = args.steps / (ms / 1e3)
    out = {
        "metric": METRIC,
        "value": value,
        "unit": "evals/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms / args.steps,
        "higher_is_better": True,
        "scaling": "strong",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (uniform locations seed 0; GP draw by 1024 random Fourier features)",
        "config": {"workload": w["name"], "n": w["n"], "bc_requested": w["bc"], "bc": int(L.bc),
                   "cs": w["cs"], "nu": w["nu"], "sigma2": w["sigma2"], "range": w["range"],
                   "precision": args.precision, "kmeans_epochs": w["kmeans_epochs"],
                   "l2": "flushed between evaluations (256 MB device write, inside the timed region)",
                   "blocks_failed_fp64": int(st["failed"]),
                   "setup_layout_knn_s": round(setup_layout_s, 2)},
        "e2e": {"value": args.steps / (ms_e2e / 1e3), "unit": "evals/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": 48},
        "roofline": {"bound": "tensor", "achieved": achieved_tf, "peak": peak_tf, "unit": "TFLOP/s",
                     "frac": achieved_tf / peak_tf, "traffic": traffic_per_launch(L),
                     "peak_source": "FP64 DGEMM 8192^3 (cuBLAS via torch) measured in this run; "
                                    "MEASURED_PEAKS.json has no FP64 figure",
                     "kernel": "llh_fp64_kernel (fused Matern + augmented Cholesky, mma.sync f64)",
                     "flops_per_launch": my_flops, "kernel_ms_per_launch": kernel_ms / args.steps},
        "cpu_baseline": cpu,
        "clocks": clk,
        "gpu_launches": launches_per_eval * args.steps,
        "llk": v,
        "mixed": mixed,
        "serve": serve,
    }
    print(json.dumps(out))
    D.close()
    if world > 1:
        dist.destroy_process_group()


def traffic_per_launch(L):
    """DRAM bytes per launch of the fused kernel from the committed ncu
    summary (profiles/llh_fp64_kernel.json: bytes per block measured on a
    smaller case), scaled by blocks; None when absent."""
    p = os.path.join(ROOT, "profiles", "llh_fp64_kernel.json")
    if not os.path.exists(p):
        return None
    try:
        d = json.load(open(p))
        return float(d["dram_bytes_per_block"]) * int(L.bc)
    except Exception:
        return None


# ---------------------------------------------------------- reference arm

def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    w = WORKLOAD
    theta = (w["sigma2"], w["range"], w["nu"])
    x, y = make_locations(w["n"], w["seed"])
    obs = rff_draw(x, y, w["sigma2"], w["range"], w["nu"], w["rff_features"], w["seed"])
    import blockvecchia_b200 as bv  # host layout code only (matches the reference's driver)
    L = bv.build_layout(x, y, obs, w["bc"], w["cs"], seed=w["seed"], epochs=w["kmeans_epochs"])
    layout = dict(batchNum=L.batchNum, batchNumAccum=L.batchNumAccum, x=L.x, y=L.y, obs=L.obs,
                  cs=L.cs, cx=L.cx, cy=L.cy)
    flops = block_flops(L.batchNum, L.cs)
    budget = max(1.0, 90.0 / max(1, args.steps + args.warmup))
    sampler = CpuSample(layout, knn_fill_cpu(layout), theta, flops, budget_s=budget)
    rates = []
    for i in range(args.warmup + args.steps):
        r = sampler.step()
        if i >= args.warmup:
            rates.append(r)
    value = statistics.median(rates)
    cores, sample = sampler.threads, sampler.describe()
    out = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": "evals/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 / value,
        "higher_is_better": True,
        "scaling": "strong",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (uniform locations seed 0; GP draw by 1024 random Fourier features)",
        "config": {"workload": w["name"], "n": w["n"], "bc": int(L.bc), "cs": w["cs"], "nu": w["nu"],
                   "sigma2": w["sigma2"], "range": w["range"], "precision": "fp64"},
        "cpu_baseline": {"value": value, "unit": "evals/s", "cores": cores, "kind": "port",
                         "sample": sample + "; the reference's own llh needs MAGMA (not installed), "
                                            "so its algorithm runs as the oracle port"},
        "e2e": {"value": value, "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))

# ------------------------------------------------------------------ serving

def serve_workload(jobs, evals, rate, inflight, seed=20241):
    """Serving workload: independent fitting jobs with Poisson arrivals.  Per
    job: n log-uniform in 5,000-500,000 locations uniform on [0,1]^2, nu from
    {0.5, 1.5, 2.5}, sigma2 uniform in 0.5-2, range uniform in 0.02-0.2, cs
    from {60, 120, 300}, bc = n/10; observations one random-Fourier-feature
    draw of the job's process.  Each job is a client that opens the job,
    issues `evals` sequential evaluations (the first at the true parameters,
    then optimizer-like probes around them, nu included, so the general-nu
    Bessel path runs too) and closes the job.  Returns throughput and request
    latency (submit to result) percentiles."""
    from concurrent.futures import ThreadPoolExecutor

    import torch

    import blockvecchia_b200 as bv

    torch.cuda.set_device(0)
    J, E = jobs, evals
    g = np.random.default_rng(seed)
    ns = np.exp(g.uniform(np.log(5_000), np.log(500_000), J)).astype(np.int64)
    nus = g.choice([0.5, 1.5, 2.5], J)
    s2 = g.uniform(0.5, 2.0, J)
    rg = g.uniform(0.02, 0.2, J)
    css = g.choice([60, 120, 300], J)
    arrivals = np.cumsum(g.exponential(1.0 / rate, J))

    t_prep = time.perf_counter()
    draws = []
    for i in range(J):
        x, y = make_locations(int(ns[i]), 1000 + i)
        obs = rff_draw(x, y, s2[i], rg[i], nus[i], 256, 1000 + i, device="cuda")
        draws.append((x, y, obs))

    def prep(i):
        x, y, obs = draws[i]
        return bv.build_layout(x, y, obs, int(ns[i]) // 10, int(css[i]), seed=i, epochs=10, threads=1)

    with ThreadPoolExecutor(max_workers=os.cpu_count() or 8) as ex:
        layouts = list(ex.map(prep, range(J)))
    del draws
    for L in layouts:
        L.knn_idx = bv.knn(L)
    prep_s = time.perf_counter() - t_prep

    srv = bv.Server(device=0, max_inflight=inflight)
    # Warm-up: closed-form and general nu, shared-memory and global-slab
    # jobs, then clear the record.
    for i in range(min(J, 6)):
        j = srv.open_job(layouts[i])
        srv.evaluate(j, (s2[i], rg[i], nus[i]))
        srv.evaluate(j, (s2[i], rg[i], nus[i] * 1.03))
        srv.close_job(j)
    srv.reset_stats()

    results = [None] * J
    t0 = time.perf_counter()

    def client(i):
        time.sleep(max(0.0, t0 + arrivals[i] - time.perf_counter()))
        r = np.random.default_rng(5000 + i)
        j = srv.open_job(layouts[i])
        th0 = np.array([s2[i], rg[i], nus[i]])
        out = []
        for e in range(E):
            th = th0 if e == 0 else th0 * np.exp(0.1 * r.standard_normal(3))
            out.append(srv.wait(srv.submit(j, th)))
        srv.close_job(j)
        results[i] = (out, time.perf_counter())

    clocks = ClockSampler(0)
    clocks.start()
    threads = [threading.Thread(target=client, args=(i,)) for i in range(J)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    wall = max(r[1] for r in results) - t0
    clk = clocks.stop()
    st = srv.stats()
    srv.close()
    lat = np.array([lt for r in results for (_, lt) in r[0]])
    bad = int(sum(1 for r in results for (v, _) in r[0] if not math.isfinite(v)))
    return {
        "evals_per_s": round(len(lat) / wall, 3),
        "p50_ms": round(float(np.percentile(lat, 50)), 2),
        "p99_ms": round(float(np.percentile(lat, 99)), 2),
        "max_ms": round(float(lat.max()), 2),
        "mean_batch": round(st["mean_batch"], 2), "batches": st["batches"],
        "evals": int(len(lat)), "nonfinite_llk": bad, "wall_s": round(wall, 2),
        "prep_s": round(prep_s, 1),
        "workload": f"{J} jobs, Poisson arrivals at {rate}/s, n log-uniform 5k-500k, "
                    f"cs in {{60,120,300}}, bc=n/10, nu in {{0.5,1.5,2.5}}, {E} sequential "
                    f"evaluations per job, {inflight} batches in flight",
        "total_points": int(ns.sum()),
        "clocks": clk,
    }


def run_serve(args):
    r = serve_workload(args.serve_jobs, args.serve_evals, args.serve_rate, args.serve_inflight)
    out = {
        "metric": "serve p50/p99 ms and evals/s, mixed-size concurrent fitting jobs",
        "value": r["evals_per_s"], "unit": "evals/s", "n_gpus": 1, "higher_is_better": True,
        "impl": "ours", "mode": "serve", "dtype": "f64", "data": "synthetic",
        "config": {"workload": r["workload"], "total_points": r["total_points"]},
        "clocks": r.pop("clocks"),
    }
    out.update({k: v for k, v in r.items() if k not in ("workload", "total_points")})
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision comparison")
    ap.add_argument("--serve-sample", type=int, default=64,
                    help="jobs in the short serving sample of the default run (0: none)")
    ap.add_argument("--serve", action="store_true",
                    help="serving workload: concurrent fitting jobs through the request loop")
    ap.add_argument("--serve-jobs", type=int, default=512)
    ap.add_argument("--serve-evals", type=int, default=6)
    ap.add_argument("--serve-rate", type=float, default=8.0, help="job arrivals per second")
    ap.add_argument("--serve-inflight", type=int, default=2)
    ap.add_argument("--case", choices=sorted(WORKLOADS), default="c3",
                    help="c3: the headline workload (default); c3-small: profiling case")
    args = ap.parse_args()
    global WORKLOAD
    WORKLOAD = WORKLOADS[args.case]
    if args.warmup < 3:
        args.warmup = 3
    if args.serve:
        run_serve(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
