"""test_dvecchia_batch on the device: one --perf evaluation against the
oracle, and a fit whose optimum matches a fit of the oracle's likelihood."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu
EXE = os.path.join(ROOT, "blockvecchia_b200", "bin", "test_dvecchia_batch")


@pytest.fixture(scope="module")
def exe(bvlib):
    from blockvecchia_b200 import build
    build.build()
    return EXE


def _run(exe, args, cwd):
    r = subprocess.run([exe, *args], capture_output=True, text=True, timeout=600, cwd=cwd)
    assert r.returncode == 0, r.stdout + r.stderr
    # Per-evaluation lines ("<k>th Model Parameters ...") come first; the
    # summary line of the optimum is the last match.
    m = re.findall(r"Model Parameters \(Variance, range, smoothness\): \(([-\d.e]+), ([-\d.e]+), "
                   r"([-\d.e]+)\) -> Loglik: ([-\d.eE+]+)", r.stdout)
    assert m, r.stdout
    last = m[-1]
    return np.array([float(last[i]) for i in (0, 1, 2)]), float(last[3]), r.stdout


def test_perf_mode_matches_oracle(exe, bvlib, oracle, tmp_path):
    """--perf: GenerateXYLoc locations, zero observations, one evaluation."""
    n, bc, cs = 3000, 200, 60
    _, llk, _ = _run(exe, ["--num_loc", str(n), "--vecchia_bc", str(bc), "--vecchia_cs", str(cs),
                           "--ikernel", "1.5:0.1:0.5", "--perf", "1", "--seed", "0"], tmp_path)
    x, y = bvlib.generate_xy(n, 0)
    L = bvlib.build_layout(x, y, np.zeros(n), bc, cs, seed=0, epochs=50)
    knn = oracle.knn_all(L.x, L.y, cs, L.batchNumAccum, L.cx, L.cy)
    P = oracle.OracleProblem(L.batchNum, L.batchNumAccum, L.x, L.y, L.obs, knn, cs)
    ref = oracle.llh(P, (1.5, 0.1, 0.5))
    assert abs(llk - ref) <= 1e-10 * abs(ref)
    # The perf-mode dumps (src/test_Xvecchia_batch.cpp:405-451), in the
    # stream's default 6-significant-digit format: each block's points, then
    # each block's conditioning points (block 0: the first cs points).
    g = lambda v: f"{v:g}"
    pts = (tmp_path / "log" / "points_Random.csv").read_text().splitlines()
    assert pts[0] == "x,y,cluster" and len(pts) == n + 1
    cl = np.repeat(np.arange(len(L.batchNum)), L.batchNum)
    assert pts[1:] == [f"{g(a)},{g(b)},{c}" for a, b, c in zip(L.x, L.y, cl)]
    nbr = (tmp_path / "log" / "neighbors_Random.csv").read_text().splitlines()
    bc_eff = len(L.batchNum)
    assert nbr[0] == "x,y,cluster" and len(nbr) == bc_eff * cs + 1
    src = np.concatenate([np.arange(cs), np.asarray(knn).reshape(-1)[cs:]])
    assert nbr[1:] == [f"{g(L.x[s])},{g(L.y[s])},{t // cs}" for t, s in enumerate(src)]


@pytest.mark.parametrize("name,suffix", [("morton", "Morton"), ("kdtree", "KDtree"), ("mmd", "MMD")])
def test_perf_mode_orderings(exe, bvlib, oracle, tmp_path, name, suffix):
    """--perf with another centroid ordering: the layout of that ordering,
    the likelihood against the oracle, the dumps named for the ordering."""
    n, bc, cs = 3000, 200, 60
    _, llk, _ = _run(exe, ["--num_loc", str(n), "--vecchia_bc", str(bc), "--vecchia_cs", str(cs),
                           "--ikernel", "1.5:0.1:0.5", "--perf", "1", "--seed", "0",
                           "--permutation", name], tmp_path)
    x, y = bvlib.generate_xy(n, 0)
    L = bvlib.build_layout(x, y, np.zeros(n), bc, cs, seed=0, epochs=50, ordering=name)
    knn = oracle.knn_all(L.x, L.y, cs, L.batchNumAccum, L.cx, L.cy)
    P = oracle.OracleProblem(L.batchNum, L.batchNumAccum, L.x, L.y, L.obs, knn, cs)
    ref = oracle.llh(P, (1.5, 0.1, 0.5))
    assert abs(llk - ref) <= 1e-10 * abs(ref)
    pts = (tmp_path / "log" / f"points_{suffix}.csv").read_text().splitlines()
    assert pts[0] == "x,y,cluster" and len(pts) == n + 1
    assert (tmp_path / "log" / f"neighbors_{suffix}.csv").exists()


def test_fit_matches_oracle_fit(exe, bvlib, oracle, tmp_path):
    """A fit from 0.1:0.1:0.1 on an exact GP draw; the optimum agrees with a
    Nelder-Mead maximisation of the oracle's likelihood to the optimizer
    tolerance, and the device optimum's likelihood is at least as high."""
    scipy_opt = pytest.importorskip("scipy.optimize")
    n, bc, cs = 1500, 150, 40
    theta_true = (1.5, 0.1, 0.5)
    x, y = bvlib.generate_xy(n, 1)
    Sigma = oracle.matern(x, y, x, y, theta_true)
    z = np.linalg.cholesky(Sigma + 1e-12 * np.eye(n)) @ np.random.default_rng(1).standard_normal(n)
    np.savetxt(tmp_path / "xy.csv", np.stack([x, y], 1), delimiter=",", fmt="%.17g")
    np.savetxt(tmp_path / "z.csv", z, fmt="%.17g")
    th, llk, out = _run(exe, ["--num_loc", str(n), "--vecchia_bc", str(bc), "--vecchia_cs", str(cs),
                              "--xy_path", "xy.csv", "--obs_path", "z.csv", "--kernel_init",
                              "0.1:0.1:0.1", "--tol", "7", "--maxiter", "2000", "--seed", "0"],
                        tmp_path)
    assert "Loglik" in out and "Found maximum" in out
    L = bvlib.build_layout(x, y, z, bc, cs, seed=0, epochs=50)
    knn = oracle.knn_all(L.x, L.y, cs, L.batchNumAccum, L.cx, L.cy)
    P = oracle.OracleProblem(L.batchNum, L.batchNumAccum, L.x, L.y, L.obs, knn, cs)
    res = scipy_opt.minimize(lambda t: -oracle.llh(P, np.clip(t, 0.01, 3.0)), th, method="Nelder-Mead",
                             options=dict(xatol=1e-8, fatol=1e-10, maxiter=4000))
    ref_th = np.clip(res.x, 0.01, 3.0)
    assert np.all(np.abs(th - ref_th) <= 1e-3 * np.abs(ref_th)), (th, ref_th)
    assert llk >= -res.fun - 1e-6 * abs(res.fun)


def test_fit_c1_matches_oracle_fit(exe, bvlib, oracle, tmp_path):
    """The small configuration's fit (src/test_Xvecchia_batch.cpp:700-753):
    n = 20,000 GenerateXYLoc locations, bc = 1,500, cs = 300, from
    0.1:0.1:0.1 at tolerance 1e-4.  The golden optimum is the same
    Nelder-Mead driven by the CPU oracle's likelihood
    (tests/golden/make_fit_golden.py); the device fit must land on it within
    the optimizer tolerance (1e-3 relative per parameter, 10x the stopping
    rule's simplex spread) and reach the same maximum (1e-8 relative)."""
    g = np.load(os.path.join(ROOT, "tests", "golden", "fit_c1.npz"))
    n = 20_000
    x, y = bvlib.generate_xy(n, 0)
    np.savetxt(tmp_path / "xy.csv", np.stack([x, y], 1), delimiter=",", fmt="%.17g")
    np.savetxt(tmp_path / "z.csv", g["obs"], fmt="%.17g")
    th, llk, out = _run(exe, ["--num_loc", str(n), "--vecchia_bc", "1500", "--vecchia_cs", "300",
                              "--xy_path", "xy.csv", "--obs_path", "z.csv", "--kernel_init",
                              "0.1:0.1:0.1", "--tol", "4", "--seed", "0"], tmp_path)
    ref_th, ref_llk = g["theta"], float(g["llk"])
    print({"device": th.tolist(), "oracle": ref_th.tolist(), "llk": llk, "oracle_llk": ref_llk})
    assert np.all(np.abs(th - ref_th) <= 1e-3 * np.abs(ref_th)), (th, ref_th)
    assert abs(llk - ref_llk) <= 1e-8 * abs(ref_llk), (llk, ref_llk)


def test_earth_one_evaluation_matches_oracle(exe, bvlib, oracle, tmp_path):
    """--earth on latitude/longitude files with --dist_scale: the first
    evaluation (at --kernel_init) against the oracle's great-circle
    likelihood on the same layout and conditioning sets."""
    n, bc, cs = 4000, 300, 50
    rng = np.random.default_rng(3)
    lat, lon = rng.uniform(-50, 50, n), rng.uniform(-120, 120, n)
    z = rng.standard_normal(n)
    np.savetxt(tmp_path / "xy.csv", np.stack([lat, lon], 1), delimiter=",", fmt="%.17g")
    np.savetxt(tmp_path / "z.csv", z, fmt="%.17g")
    r = subprocess.run([exe, "--num_loc", str(n), "--vecchia_bc", str(bc), "--vecchia_cs", str(cs),
                        "--xy_path", "xy.csv", "--obs_path", "z.csv", "--kernel_init", "1.0:0.2:0.5",
                        "--dist_scale", "1000", "--earth", "--maxiter", "1", "--seed", "0"],
                       capture_output=True, text=True, timeout=600, cwd=tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    m = re.findall(r"Model Parameters \(Variance, range, smoothness\): \(([-\d.e]+), ([-\d.e]+), "
                   r"([-\d.e]+)\) -> Loglik: ([-\d.eE+]+)", r.stdout)
    assert m, r.stdout
    llk = float(m[0][3])
    L = bvlib.build_layout(lat, lon, z, bc, cs, seed=0, epochs=50)
    knn = oracle.knn_all_earth_fast(L.x, L.y, cs, L.batchNumAccum, L.cx, L.cy)
    P = oracle.OracleProblem(L.batchNum, L.batchNumAccum, L.x, L.y, L.obs, knn, cs,
                             dist_scale=1000.0, earth=True)
    ref = oracle.llh(P, (1.0, 0.2, 0.5))
    # The CLI prints the log-likelihood with 6 decimals.
    assert abs(llk - ref) <= max(1e-10 * abs(ref), 1e-6), (llk, ref)
