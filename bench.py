"""Benchmark: block-Vecchia log-likelihood evaluations per second.

Workload (the configuration the headline metric is quoted on): n = 1,000,000
locations uniform on [0,1]^2 (seed 0), Matern nu = 2.5, sigma2 = 1.0,
range = 0.05, no nugget, k-means into bc = 100,000 blocks, conditioning size
cs = 200.  Observations are one draw of the same Gaussian process by random
Fourier features (1024 features; a dense draw at n = 1M is infeasible).  One
step = one full log-likelihood evaluation.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
    python bench.py --write-layout [--case c3]   # the shared layout file only

The workload's locations, observations and block layout are built once by
the library's host layout code (the reference driver's k-means ordering,
which that code reproduces bit for bit) and saved under bench_data/; both
arms read that file, so they evaluate the same blocks.

N > 1 runs under torchrun, one process per GPU: every rank evaluates its
shard of the blocks and the FP64 partials are all-gathered (NCCL) and summed
in rank order (strong scaling: the evaluation is fixed, split over ranks).

--impl reference times the reference's algorithm on the host cores (the CPU
oracle: restated llh_Xvecchia_batch with OpenBLAS dense LA and OpenMP over
blocks; the conditioning sets by the oracle's restated findNearestPoints).
It loads no library of this package.  Its K timed steps are K contiguous
slices of the blocks with equal algorithmic FLOPs that together make one
whole evaluation, so the value is the measured time of one evaluation.
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


def finite_json(o):
    """JSON text of o with every non-finite float written as null (strict
    JSON has no NaN or Infinity)."""
    def clean(v):
        if isinstance(v, float) and not math.isfinite(v):
            return None
        if isinstance(v, dict):
            return {k: clean(x) for k, x in v.items()}
        if isinstance(v, (list, tuple)):
            return [clean(x) for x in v]
        return v
    return json.dumps(clean(o))

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
    # The batching configuration (blocks of 3-30 points, cs = 120).
    "c2": dict(name="n=200k uniform, nu=1.5 sigma2=1 range=0.08, bc=20k, cs=120",
               n=200_000, bc=20_000, cs=120, sigma2=1.0, range=0.08, nu=1.5, seed=0,
               kmeans_epochs=50, rff_features=1024),
    # The general-nu stress configuration: 2M points from a 50-component
    # Gaussian mixture, cs = 300 (streamed path), nu = 0.8 (Bessel K_nu),
    # nugget 0.01.  The oracle checks a sample of blocks (a whole CPU
    # evaluation takes hours).
    "c5": dict(name="n=2M Gaussian mixture (50 comps), nu=0.8 sigma2=1 range=0.1 nugget=0.01, "
                    "bc=200k, cs=300",
               n=2_000_000, bc=200_000, cs=300, sigma2=1.0, range=0.1, nu=0.8, nugget=0.01,
               seed=0, kmeans_epochs=50, rff_features=1024, locations="mixture",
               oracle_sample=400),
    # The small configuration's shape (cs = 300: the streamed large-block path).
    "c1": dict(name="n=20k uniform, nu=0.5 sigma2=1.5 range=0.1, bc=1.5k, cs=300",
               n=20_000, bc=1_500, cs=300, sigma2=1.5, range=0.1, nu=0.5, seed=0,
               kmeans_epochs=50, rff_features=1024),
}
for _k, _w in WORKLOADS.items():
    _w["key"] = _k
WORKLOAD = WORKLOADS["c3"]


# ----------------------------------------------------------------- workload

def make_locations(n, seed):
    rng = np.random.default_rng(seed)
    return rng.random(n), rng.random(n)


def mixture_locations(n, seed, components=50):
    """A 2-D Gaussian mixture: component centres uniform on [0,1]^2, standard
    deviations uniform in [0.01, 0.05], equal weights (not clipped)."""
    g = np.random.default_rng(seed)
    centers = g.random((components, 2))
    stds = g.uniform(0.01, 0.05, components)
    comp = g.integers(0, components, n)
    pts = centers[comp] + g.standard_normal((n, 2)) * stds[comp, None]
    return pts[:, 0].copy(), pts[:, 1].copy()


def workload_locations(w):
    if w.get("locations") == "mixture":
        return mixture_locations(w["n"], w["seed"])
    return make_locations(w["n"], w["seed"])


def workload_theta(w):
    th = (w["sigma2"], w["range"], w["nu"])
    return th + ((w["nugget"],) if w.get("nugget") else ())


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


# ------------------------------------------------------------- layout file

DATA = os.path.join(ROOT, "bench_data")


def _recipe(w):
    keys = ("n", "bc", "cs", "sigma2", "range", "nu", "seed", "kmeans_epochs", "rff_features")
    r = {k: w[k] for k in keys}
    if w.get("locations"):
        r["locations"] = w["locations"]
    return r


def layout_path(w):
    return os.path.join(DATA, f"{w['key']}_layout.npz")


def write_layout(w):
    """Build the workload's layout with the library's host code (k-means
    ordering, first-block merge, block reordering) and save it with the
    locations and observations, block-ordered."""
    import blockvecchia_b200 as bv
    x, y = workload_locations(w)
    obs = rff_draw(x, y, w["sigma2"], w["range"], w["nu"], w["rff_features"], w["seed"])
    L = bv.build_layout(x, y, obs, w["bc"], w["cs"], seed=w["seed"], epochs=w["kmeans_epochs"])
    os.makedirs(DATA, exist_ok=True)
    path = layout_path(w)
    tmp = path + ".tmp.npz"
    np.savez(tmp, recipe=json.dumps(_recipe(w)), batchNum=L.batchNum, batchNumAccum=L.batchNumAccum,
             x=L.x, y=L.y, obs=L.obs, cx=L.cx, cy=L.cy,
             first_cluster_count=np.int64(L.first_cluster_count))
    os.replace(tmp, path)
    return path


def load_layout(w, child_build=False):
    """The saved layout as plain arrays (dict), built first if absent or made
    from another recipe.  child_build: build it in a child process, so that
    this process loads no library of the package."""
    path = layout_path(w)
    ok = False
    if os.path.exists(path):
        with np.load(path) as f:
            ok = json.loads(str(f["recipe"])) == _recipe(w)
    source = "file"
    if not ok:
        if child_build:
            subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--write-layout",
                            "--case", w["key"]], check=True)
            source = "built now by the library's host layout code (child process)"
        else:
            write_layout(w)
            source = "built now by the library's host layout code"
    with np.load(path) as f:
        d = {k: f[k] for k in f.files if k != "recipe"}
    d["cs"] = w["cs"]
    d["first_cluster_count"] = int(d["first_cluster_count"])
    d["source"] = source
    return d


def host_threads():
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)


def workload_config(w, bc):
    """The `config` object of both arms' lines (identical by construction)."""
    return {"workload": w["name"], "n": w["n"], "bc_requested": w["bc"], "bc": int(bc), "cs": w["cs"],
            "nu": w["nu"], "sigma2": w["sigma2"], "range": w["range"], "precision": "fp64",
            "kmeans_epochs": w["kmeans_epochs"],
            "l2": "GPU arm: inputs stay in HBM, a 256 MB buffer is written between evaluations "
                  "(L2 flushed, inside the timed region); CPU arm: not applicable"}


def chunk_bounds(flops, k):
    """k contiguous block ranges of about equal total FLOPs covering all blocks."""
    c = np.cumsum(flops)
    cuts = [0]
    for t in range(1, k):
        cuts.append(int(np.searchsorted(c, c[-1] * t / k)))
    cuts.append(len(flops))
    cuts = sorted(set(cuts))
    return list(zip(cuts[:-1], cuts[1:]))


def oracle_parity_sample(L, theta, dev_blocks, dev_knn, flops, count, threads, nugget=0.0):
    """For workloads too large for a whole CPU evaluation: a contiguous
    sample of blocks from the middle of the order, their conditioning sets
    recomputed by the oracle (must equal the device's bit for bit) and their
    contributions by the oracle (with the same nugget); the sample's time,
    extrapolated by algorithmic FLOPs, is the CPU baseline."""
    from oracle import oracle as O
    O.build(ref=False)
    cs, bc = L.cs, L.bc
    b0 = bc // 2
    b1 = min(bc, b0 + count)
    knn = np.array(dev_knn, copy=True)
    same = True
    for b in range(b0, b1):
        ref = O.knn_block_fast(L.x, L.y, int(L.batchNumAccum[b]), L.cx[b], L.cy[b], cs)
        same = same and np.array_equal(ref, dev_knn[b * cs:(b + 1) * cs])
        knn[b * cs:(b + 1) * cs] = ref
    P = O.OracleProblem(L.batchNum, L.batchNumAccum, L.x, L.y, L.obs, knn, cs, nugget=nugget)
    t0 = time.perf_counter()
    _, pb = O.llh_blas(P, theta[:3], threads=threads, block_begin=b0, block_end=b1, per_block=True)
    dt = time.perf_counter() - t0
    ref_blocks = O.block_llk(L.batchNum, pb)[b0:b1]
    dev = dev_blocks[b0:b1]
    ok = (pb[b0:b1, 2] == 0) & (pb[b0:b1, 3] == 0)
    rel = np.abs(dev - ref_blocks) / np.maximum(1.0, np.abs(ref_blocks))
    frac = float(flops[b0:b1].sum() / flops.sum())
    parity = {"sample_blocks": [int(b0), int(b1)], "knn_bit_exact": bool(same),
              "rel_err_sample_sum": abs(float(dev[ok].sum()) - float(ref_blocks[ok].sum())) /
              abs(float(ref_blocks[ok].sum())),
              "max_block_rel_diff": float(rel[ok].max()) if ok.any() else None,
              "blocks_over_1e-10": int((rel[ok] > 1e-10).sum()),
              "failed_blocks_oracle": int((~ok).sum()), "nugget": nugget}
    cpu = {"value": frac / dt, "unit": "evals/s", "cores": threads, "kind": "port",
           "sample": f"blocks {b0}..{b1 - 1} ({frac * 100:.2f}% of the evaluation's flops) in {dt:.1f} s, "
                     "extrapolated by flops"}
    return parity, cpu


def oracle_parity(L, theta, dev_blocks, dev_status, dev_total, threads, nugget=0.0):
    """One whole evaluation by the CPU oracle (timed: the CPU baseline) and
    its comparison with the device evaluation of the same blocks: the total,
    and per block, split into blocks where either side met a non-positive
    pivot (not comparable: the oracle's LAPACK potrf stops at the failing
    column, the device zeroes it and continues) and the rest."""
    from oracle import oracle as O
    O.build(ref=False)
    P = O.OracleProblem(L.batchNum, L.batchNumAccum, L.x, L.y, L.obs, L.knn_idx, L.cs, nugget=nugget)
    t0 = time.perf_counter()
    ref_total, pb = O.llh_blas(P, theta, threads=threads, per_block=True)
    dt = time.perf_counter() - t0
    ref_blocks = O.block_llk(L.batchNum, pb)
    failed = (pb[:, 2] != 0) | (pb[:, 3] != 0) | ((dev_status & 3) != 0)
    ok = ~failed
    rel = np.abs(dev_blocks - ref_blocks) / np.maximum(1.0, np.abs(ref_blocks))
    ref_ok = float(np.sum(ref_blocks[ok]))
    dev_ok = float(np.sum(dev_blocks[ok]))
    # The blocks furthest apart, and two others, against a 40-digit
    # evaluation of the same inputs, with the condition number of each
    # block's joint covariance.
    from oracle import hp
    eps = np.finfo(np.float64).eps
    okb = np.nonzero(ok)[0]
    worst = okb[np.argsort(-rel[okb])[:3]]
    others = np.random.default_rng(1).choice(np.setdiff1d(okb, worst), min(2, len(okb) - len(worst)),
                                             replace=False) if len(okb) > 3 else np.zeros(0, int)
    worst_rows = []
    for b in np.concatenate([worst, others]).astype(int):
        cs = L.cs
        ci = L.knn_idx[b * cs:(b + 1) * cs] if b > 0 else np.zeros(0, dtype=np.int32)
        p = np.concatenate([ci, np.arange(L.batchNumAccum[b], L.batchNumAccum[b + 1])])
        ev = np.linalg.eigvalsh(O.matern(L.x[p], L.y[p], L.x[p], L.y[p], theta))
        kap = float(ev[-1] / ev[0]) if ev[0] > 0 else None
        try:
            truth = hp.block_llk(L.x, L.y, L.obs, L.batchNumAccum, L.knn_idx, L.cs, int(b), theta)
        except ArithmeticError:
            truth = None
        worst_rows.append({"block": int(b), "bs": int(L.batchNum[b]), "rel_diff": float(rel[b]),
                           "kappa_joint_cov": kap,
                           "rel_diff_over_kappa_eps": float(rel[b] / (kap * eps)) if kap else None,
                           "hp40_value": truth,
                           "device_abs_err_vs_hp40": abs(float(dev_blocks[b]) - truth) if truth is not None else None,
                           "oracle_abs_err_vs_hp40": abs(float(ref_blocks[b]) - truth) if truth is not None else None})
    fin = lambda v: float(v) if np.isfinite(v) else None  # noqa: E731
    parity = {
        "oracle_llk": fin(ref_total),
        "rel_err_total": fin(abs(dev_total - ref_total) / abs(ref_total)),
        "blocks": int(len(ref_blocks)),
        "failed_blocks_oracle": int(((pb[:, 2] != 0) | (pb[:, 3] != 0)).sum()),
        "failed_blocks_device": int(((dev_status & 3) != 0).sum()),
        "comparable_blocks": int(ok.sum()),
        "rel_err_sum_comparable": abs(dev_ok - ref_ok) / abs(ref_ok),
        "comparable_blocks_over_1e-10": int((rel[ok] > 1e-10).sum()),
        "comparable_blocks_over_1e-8": int((rel[ok] > 1e-8).sum()),
        "max_block_rel_diff": float(rel[ok].max()) if ok.any() else None,
        "failed_blocks_over_1e-10": int((rel[failed] > 1e-10).sum()),
        "blocks_checked_at_40_digits": worst_rows,
        "tolerance": "1e-10 relative (FP64 parity bound); per block |diff| / max(1, |block|); "
                     "a block with joint-covariance condition number kappa carries ~kappa*eps "
                     "in any FP64 evaluation",
    }
    cpu = {"value": 1.0 / dt, "unit": "evals/s", "cores": threads, "kind": "port",
           "sample": f"one whole evaluation ({len(ref_blocks)} blocks) in {dt:.1f} s: the oracle "
                     "(restated llh_Xvecchia_batch, the reference's Matern with K_nu for every nu, "
                     "OpenBLAS potrf/trsm/gemm, OpenMP over blocks)"}
    return parity, cpu


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
    theta = workload_theta(w)

    t_setup = time.perf_counter()
    d = load_layout(w)
    L = bv.Layout(d["batchNum"], d["batchNumAccum"], d["x"], d["y"], d["obs"], w["cs"], d["cx"],
                  d["cy"], None, d["first_cluster_count"])
    setup_layout_s = time.perf_counter() - t_setup
    t_knn = time.perf_counter()
    L.knn_idx = bv.knn(L, device=local)
    setup_knn_s = time.perf_counter() - t_knn
    D = bv.LlhData(L, precision=args.precision, device=local, on_failure="continue",
                   nugget=bool(w.get("nugget")),
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

    # The CPU oracle over the same blocks: one whole evaluation, timed (the
    # CPU baseline), compared block by block with the device's.
    cpu = parity = None
    if world == 1 and not args.no_cpu_baseline:
        dev_blocks = D.block_llk()
        dev_status = D.block_status()
        if w.get("oracle_sample"):
            parity, cpu = oracle_parity_sample(L, theta, dev_blocks, L.knn_idx, flops,
                                               w["oracle_sample"], host_threads(),
                                               nugget=w.get("nugget", 0.0))
        else:
            parity, cpu = oracle_parity(L, theta, dev_blocks, dev_status, v, host_threads(),
                                        nugget=w.get("nugget", 0.0))

    # Mixed precision on the same workload (the FP64 path is the reference),
    # timed like the FP64 loop: the default policy (FP64 throughout) and the
    # forced FP32 pass (mixed_fp32), with the range sweep's relative error and
    # fallback counts of the forced pass.
    mixed = None
    if world == 1 and not args.no_mixed and args.precision == "fp64":
        def time_mixed(H):
            H.set_stream(stream.cuda_stream)
            for _ in range(args.warmup):
                H(theta)
            torch.cuda.synchronize()
            m0 = torch.cuda.Event(enable_timing=True)
            m1 = torch.cuda.Event(enable_timing=True)
            m0.record(stream)
            for _ in range(args.steps):
                with torch.cuda.stream(stream):
                    flush.fill_(1.0)
                vm_ = H(theta)
            m1.record(stream)
            torch.cuda.synchronize()
            return vm_, m0.elapsed_time(m1)

        nug = bool(w.get("nugget"))
        with bv.LlhData(L, precision="mixed", device=local, on_failure="continue", nugget=nug) as Mx:
            vm, ms_mx = time_mixed(Mx)
            stm = Mx.status()
        with bv.LlhData(L, precision="mixed", mixed_fp32=True, device=local, on_failure="continue",
                        nugget=nug) as Mf:
            vf, ms_mf = time_mixed(Mf)
            stf = Mf.status()
            sweep = []
            for rg_ in (0.02, 0.05, 0.1, 0.2, 0.3):
                th_ = (w["sigma2"], rg_, w["nu"]) + tuple(theta[3:])
                v64_ = D(th_)
                s64_ = D.status()
                vm_ = Mf(th_)
                sm_ = Mf.status()
                sweep.append({"range": rg_, "rel_err": abs(vm_ - v64_) / abs(v64_) if v64_ else None,
                              "fp32_fallback_blocks": sm_["fp32_fallback"],
                              "fp64_failed_blocks": s64_["failed"]})
            D(theta)
        evs = lambda t: args.steps / (t / 1e3)
        mixed = {"value": evs(ms_mx), "unit": "evals/s", "vs_fp64": evs(ms_mx) / evs(ms),
                 "rel_err_vs_fp64": abs(vm - v) / abs(v), "fp32_fallback_blocks": stm["fp32_fallback"],
                 "blocks": int(L.bc), "tol": 1e-8,
                 "fp32_forced": {"value": evs(ms_mf), "unit": "evals/s", "vs_fp64": evs(ms_mf) / evs(ms),
                                 "rel_err_vs_fp64": abs(vf - v) / abs(v),
                                 "fp32_fallback_blocks": stf["fp32_fallback"], "range_sweep": sweep},
                 "note": "default policy: every block in FP64 (the FP32 factor + FP64 refinement "
                         "kernel is slower than the FP64 path on B200); fp32_forced: FP32 factor "
                         "of Sigma22 + FP64 refinement where a probe of every 64th block accepts, "
                         "rejected blocks recomputed in FP64"}
    serve = None
    if world == 1 and args.serve_sample > 0:
        # At the server's capacity: 16 fitting jobs in flight at all times
        # (closed loop), so requests queue and batches form.
        serve = serve_workload(args.serve_sample, 6, 0.0, 2, repeats=3, concurrency=16)
        serve.pop("clocks", None)

    # FP64: fused kernel + reduction; mixed: probe, decision, mixed pass,
    # FP64 fallback pass, reduction.
    launches_per_eval = int(st["launches"])
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
        "config": workload_config(w, L.bc),
        "precision": args.precision,
        "blocks_failed_fp64": int(st["failed"]),
        "setup": {"layout": d["source"], "layout_load_s": round(setup_layout_s, 2),
                  "knn_device_s": round(setup_knn_s, 2)},
        "e2e": {"value": args.steps / (ms_e2e / 1e3), "unit": "evals/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": 48},
        "roofline": {"bound": "tensor", "achieved": achieved_tf, "peak": peak_tf, "unit": "TFLOP/s",
                     "frac": achieved_tf / peak_tf, "traffic": traffic_per_launch(st),
                     "peak_source": "FP64 DGEMM 8192^3 (cuBLAS via torch) measured in this run; "
                                    "MEASURED_PEAKS.json has no FP64 figure",
                     "kernel": kernel_name(st),
                     "flops_per_launch": my_flops, "kernel_ms_per_launch": kernel_ms / args.steps},
        "cpu_baseline": cpu,
        "parity_vs_oracle": parity,
        "clocks": clk,
        "gpu_launches": launches_per_eval * args.steps,
        "llk": v,
        "mixed": mixed,
        "serve": serve,
    }
    print(finite_json(out))
    D.close()
    if world > 1:
        dist.destroy_process_group()


def kernel_name(st):
    """The fused kernel(s) the evaluation ran, from the library's split."""
    bc = int(st["blocks"])
    lean = "llh_lean_kernel_t (multi-CTA streamed: fused Matern + augmented Cholesky, mma.sync f64)"
    pers = "llh_fp64_kernel_t (persistent: fused Matern + augmented Cholesky, mma.sync f64)"
    n = int(st.get("streamed_blocks", 0))
    if n == bc:
        return lean
    if n == 0:
        return pers
    return f"{lean} for {n} blocks + {pers} for {bc - n}"


def traffic_per_launch(st):
    """DRAM bytes per launch of the fused kernel from the committed ncu
    summary of the kernel that ran (profiles/<kernel>.json: bytes per block
    measured on a smaller case), scaled by blocks; None when absent or when
    the evaluation split its blocks over both kernels."""
    n, bc = int(st.get("streamed_blocks", 0)), int(st["blocks"])
    name = "llh_lean_kernel" if n == bc else ("llh_fp64_kernel" if n == 0 else None)
    if name is None:
        return None
    p = os.path.join(ROOT, "profiles", name + ".json")
    if not os.path.exists(p):
        return None
    try:
        d = json.load(open(p))
        return float(d["dram_bytes_per_block"]) * bc
    except Exception:
        return None


# ---------------------------------------------------------- reference arm

def run_reference(args):
    """The reference's algorithm on the host cores, on the same layout file:
    conditioning sets by the oracle's findNearestPoints restatement (setup,
    untimed), then one whole evaluation split into K timed steps of equal
    algorithmic FLOPs.  Warm-up steps evaluate the first 1% of the blocks.
    Loads only the oracle's libraries."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    w = WORKLOAD
    theta = workload_theta(w)
    d = load_layout(w, child_build=True)
    from oracle import oracle as O
    O.build(ref=False)
    threads = host_threads()
    cs = w["cs"]
    t0 = time.perf_counter()
    knn = O.knn_all_fast(d["x"], d["y"], cs, d["batchNumAccum"], d["cx"], d["cy"], threads=threads)
    knn_s = time.perf_counter() - t0
    P = O.OracleProblem(d["batchNum"], d["batchNumAccum"], d["x"], d["y"], d["obs"], knn, cs,
                        nugget=w.get("nugget", 0.0))
    bc = len(d["batchNum"])
    flops = block_flops(d["batchNum"], cs)
    chunks = chunk_bounds(flops, args.steps)
    warm_end = max(1, bc // 100)
    for _ in range(args.warmup):
        O.llh_blas(P, theta, threads=threads, block_begin=0, block_end=warm_end)
    times, llk = [], 0.0
    for b0, b1 in chunks:
        t = time.perf_counter()
        llk += O.llh_blas(P, theta, threads=threads, block_begin=b0, block_end=b1)
        times.append(time.perf_counter() - t)
    eval_s = sum(times)
    value = 1.0 / eval_s
    sample = (f"one whole evaluation ({bc} blocks) in {len(chunks)} timed steps of equal algorithmic "
              f"FLOPs, {eval_s:.1f} s in all; the reference's own llh needs MAGMA and a GPU (neither "
              f"installed), so its algorithm runs as the oracle port (restated llh_Xvecchia_batch, "
              f"the reference's Matern with K_nu for every nu, OpenBLAS potrf/trsm/gemm, OpenMP over "
              f"blocks)")
    out = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": "evals/s",
        "n_gpus": world,
        "steps": len(chunks),
        "warmup": args.warmup,
        "ms_per_step": eval_s * 1e3 / len(chunks),
        "higher_is_better": True,
        "scaling": "strong",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (uniform locations seed 0; GP draw by 1024 random Fourier features)",
        "config": workload_config(w, bc),
        "cpu_baseline": {"value": value, "unit": "evals/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        # Blocks whose LAPACK potrf fails make the OpenBLAS evaluation NaN
        # (the device path zeroes the failed pivot and goes on).
        "llk": llk if np.isfinite(llk) else None,
        "llk_note": None if np.isfinite(llk) else "not finite: some blocks' potrf failed",
        "setup": {"layout": d["source"], "knn_oracle_s": round(knn_s, 1)},
    }
    print(finite_json(out))


# ------------------------------------------------------------------ serving

def serve_workload(jobs, evals, rate, inflight, seed=20241, repeats=1, concurrency=0):
    """Serving workload: independent fitting jobs with Poisson arrivals.  Per
    job: n log-uniform in 5,000-500,000 locations uniform on [0,1]^2, nu from
    {0.5, 1.5, 2.5}, sigma2 uniform in 0.5-2, range uniform in 0.02-0.2, cs
    from {60, 120, 300}, bc = n/10; observations one random-Fourier-feature
    draw of the job's process.  Each job is a client that opens the job,
    issues `evals` sequential evaluations (the first at the true parameters,
    then optimizer-like probes around them, nu included, so the general-nu
    Bessel path runs too) and closes the job.  Returns throughput and request
    latency (submit to result) percentiles.  concurrency > 0: closed loop
    instead -- that many clients, each running one job after another (jobs
    taken in order), so the offered load is whatever the server sustains."""
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
    arrivals = np.cumsum(g.exponential(1.0 / rate, J)) if rate > 0 else np.zeros(J)

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

    def one_run():
        results = [None] * J
        srv.reset_stats()
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

        if concurrency > 0:
            nxt = [0]
            lock = threading.Lock()

            def worker():
                while True:
                    with lock:
                        i = nxt[0]
                        nxt[0] += 1
                    if i >= J:
                        return
                    arrivals[i] = time.perf_counter() - t0  # starts now
                    client(i)
            threads = [threading.Thread(target=worker) for _ in range(concurrency)]
        else:
            threads = [threading.Thread(target=client, args=(i,)) for i in range(J)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        wall = max(r[1] for r in results) - t0
        st = srv.stats()
        lat = np.array([lt for r in results for (_, lt) in r[0]])
        vals = [v for r in results for (v, _) in r[0]]
        return {"evals_per_s": round(len(lat) / wall, 3),
                "p50_ms": round(float(np.percentile(lat, 50)), 2),
                "p99_ms": round(float(np.percentile(lat, 99)), 2),
                "max_ms": round(float(lat.max()), 2),
                "mean_batch": round(st["mean_batch"], 2), "batches": st["batches"],
                "evals": int(len(lat)), "wall_s": round(wall, 2)}, vals

    clocks = ClockSampler(0)
    clocks.start()
    runs, values = [], []
    for _ in range(max(1, repeats)):
        r, v = one_run()
        runs.append(r)
        values.append(v)
    clk = clocks.stop()
    srv.close()
    same = all(np.array_equal(np.array(values[0]), np.array(v), equal_nan=True) for v in values[1:])
    bad = int(sum(1 for v in values[0] if not math.isfinite(v)))
    med = lambda k: float(np.median([r[k] for r in runs]))  # noqa: E731
    out = {
        "evals_per_s": round(med("evals_per_s"), 3),
        "p50_ms": round(med("p50_ms"), 2),
        "p99_ms": round(med("p99_ms"), 2),
        "mean_batch": round(med("mean_batch"), 2),
        "spread": {k: [min(r[k] for r in runs), max(r[k] for r in runs)]
                   for k in ("evals_per_s", "p50_ms", "p99_ms", "mean_batch")},
        "repeats": runs,
        "values_identical_across_repeats": bool(same),
        "nonfinite_llk": bad,
        "prep_s": round(prep_s, 1),
        "workload": (f"{J} jobs, " + (f"{concurrency} concurrent clients (closed loop: a client "
                                       f"starts the next job when its job ends)" if concurrency > 0
                                       else f"Poisson arrivals at {rate}/s") +
                     f", n log-uniform 5k-500k, cs in {{60,120,300}}, bc=n/10, nu in {{0.5,1.5,2.5}}, "
                     f"{E} sequential evaluations per job, {inflight} batches in flight, the same "
                     f"sample run {len(runs)} times (median and [min, max] reported)"),
        "total_points": int(ns.sum()),
        "clocks": clk,
    }
    return out


def run_serve(args):
    r = serve_workload(args.serve_jobs, args.serve_evals, args.serve_rate, args.serve_inflight,
                       repeats=args.serve_repeats, concurrency=args.serve_concurrency)
    out = {
        "metric": "serve p50/p99 ms and evals/s, mixed-size concurrent fitting jobs",
        "value": r["evals_per_s"], "unit": "evals/s", "n_gpus": 1, "higher_is_better": True,
        "impl": "ours", "mode": "serve", "dtype": "f64", "data": "synthetic",
        "config": {"workload": r["workload"], "total_points": r["total_points"]},
        "clocks": r.pop("clocks"),
    }
    out.update({k: v for k, v in r.items() if k not in ("workload", "total_points")})
    print(finite_json(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision comparison")
    ap.add_argument("--serve-sample", type=int, default=96,
                    help="jobs in the short serving sample of the default run (0: none)")
    ap.add_argument("--serve", action="store_true",
                    help="serving workload: concurrent fitting jobs through the request loop")
    ap.add_argument("--serve-jobs", type=int, default=512)
    ap.add_argument("--serve-evals", type=int, default=6)
    ap.add_argument("--serve-rate", type=float, default=8.0, help="job arrivals per second")
    ap.add_argument("--serve-inflight", type=int, default=2)
    ap.add_argument("--serve-repeats", type=int, default=1)
    ap.add_argument("--serve-concurrency", type=int, default=0,
                    help="closed loop with this many concurrent clients (0: Poisson arrivals)")
    ap.add_argument("--case", choices=sorted(WORKLOADS), default="c3",
                    help="c3: the headline workload (default); c3-small: profiling case")
    ap.add_argument("--write-layout", action="store_true",
                    help="only build and save the workload's layout file (bench_data/)")
    args = ap.parse_args()
    global WORKLOAD
    WORKLOAD = WORKLOADS[args.case]
    if args.write_layout:
        print(write_layout(WORKLOAD))
        return
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
